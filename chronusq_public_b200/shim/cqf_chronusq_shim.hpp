// ChronusQ-side binding of libcqfock.so (the C ABI of include/cqfock.h).
//
// A ChronusQ maintainer adds this header to the reference build and selects
// B200DirectTPIContraction where ChronusQ constructs GTODirectTPIContraction
// (src/cxxapi/input/singleslateropts.cxx:1340-1440).  It derives from the
// reference class, keeps the virtual twoBodyContract signature of
// TPIContractions (include/particleintegrals/twopints.hpp:219-223), and turns a
// nonzero cqf_status into CErr, the reference's error path (include/cerr.hpp).
// Compiles only inside the ChronusQ tree (it includes ChronusQ headers).
#pragma once

#include <complex>
#include <memory>
#include <type_traits>
#include <vector>

#include <cerr.hpp>
#include <particleintegrals/twopints/gtodirecttpi.hpp>

#include "cqfock.h"

namespace ChronusQ {

template <typename MatsT, typename IntsT>
class B200DirectTPIContraction : public GTODirectTPIContraction<MatsT, IntsT> {
  // one device basis per contraction object; rebuilt when the geometry moves
  mutable cqf_basis* basis_ = nullptr;
  mutable std::vector<double> alpha_, coef_;

  void ensure_basis() const {
    if (basis_) return;
    auto& tpi = *std::dynamic_pointer_cast<DirectTPI<IntsT>>(this->ints_);
    BasisSet& bs = tpi.basisSet();
    std::vector<cqf_shell> sh(bs.nShell);
    alpha_.clear();
    coef_.clear();
    for (auto& s : bs.shells) {
      alpha_.insert(alpha_.end(), s.alpha.begin(), s.alpha.end());
      coef_.insert(coef_.end(), s.contr[0].coeff.begin(), s.contr[0].coeff.end());
    }
    size_t off = 0;
    for (size_t i = 0; i < bs.nShell; i++) {
      const libint2::Shell& s = bs.shells[i];
      sh[i].l = s.contr[0].l;
      sh[i].pure = s.contr[0].pure ? 1 : 0;
      sh[i].nprim = (int)s.alpha.size();
      sh[i].alpha = alpha_.data() + off;
      sh[i].coeff = coef_.data() + off;
      for (int x = 0; x < 3; x++) sh[i].origin[x] = s.O[x];
      off += s.alpha.size();
    }
    cqf_status st = cqf_basis_create(sh.data(), (int)sh.size(), tpi.threshSchwarz(), 0, &basis_);
    if (st != CQF_OK) CErr(std::string("cqf_basis_create: ") + cqf_last_error());
  }

 public:
  using GTODirectTPIContraction<MatsT, IntsT>::GTODirectTPIContraction;

  // GTODirectTPIContraction::twoBodyContract (gtodirecttpi.hpp:199-206)
  void twoBodyContract(MPI_Comm comm, const bool screen,
                       std::vector<TwoBodyContraction<MatsT>>& list,
                       EMPerturbation& pert) const override {
    if (MPISize(comm) > 1 || this->contractSecond) {  // not offloaded
      GTODirectTPIContraction<MatsT, IntsT>::twoBodyContract(comm, screen, list, pert);
      return;
    }
    ensure_basis();
    std::vector<cqf_contraction> c(list.size());
    for (size_t i = 0; i < list.size(); i++) {
      if (list[i].contType != COULOMB && list[i].contType != EXCHANGE)
        CErr("B200DirectTPIContraction: only COULOMB / EXCHANGE");
      c[i].X = list[i].X;
      c[i].AX = list[i].AX;
      c[i].hermitian = list[i].HER ? 1 : 0;
      c[i].type = list[i].contType == COULOMB ? CQF_COULOMB : CQF_EXCHANGE;
    }
    cqf_opts o;
    cqf_opts_default(&o);
    o.is_complex = std::is_same<MatsT, std::complex<double>>::value ? 1 : 0;
    o.screen = screen ? 1 : 0;
    cqf_status st = cqf_two_body_contract(basis_, c.data(), (int)c.size(), &o, nullptr);
    if (st != CQF_OK) CErr(std::string("cqf_two_body_contract: ") + cqf_last_error());
  }

  ~B200DirectTPIContraction() override {
    if (basis_) cqf_basis_destroy(basis_);
  }
};

}  // namespace ChronusQ
