// ChronusQ-side binding of the four-component contraction of libcqfock.so.
//
// A ChronusQ maintainer selects B200DirectRelERIContraction where ChronusQ
// constructs GTODirectRelERIContraction<dcomplex,double>
// (src/cxxapi/input/singleslateropts.cxx:1340-1440).  It overrides the 4C
// twoBodyContract overload of the reference class
// (include/particleintegrals/twopints/gtodirectreleri.hpp:75-94), which
// FourCompFock::formGDDirect calls on the concrete type for BARE_COULOMB,
// LLSS and SSSS (include/fockbuilder/fourcompfock/impl.hpp:3923, :4030,
// :4177): the 17 (X, AX) entries in DIRAC_PAULI_SPINOR_COMP order go to
// cqf_rel_two_body_contract, which zeroes AX like directScaffoldLibcint
// (include/particleintegrals/contract/direct4C_libcint.hpp:313-314).  Other
// contraction types (LLLL, GAUNT, GAUGE), the spin-free / spin-dependent
// variants, approximations and MPI runs stay on the reference
// implementation.  A nonzero cqf_status becomes CErr.  Compiles only inside
// the ChronusQ tree (it includes ChronusQ headers).
#pragma once

#include <complex>
#include <string>
#include <vector>

#include <cerr.hpp>
#include <particleintegrals/twopints/gtodirectreleri.hpp>

#include "cqfock.h"

namespace ChronusQ {

template <typename MatsT, typename IntsT>
class B200DirectRelERIContraction : public GTODirectRelERIContraction<MatsT, IntsT> {
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
  using GTODirectRelERIContraction<MatsT, IntsT>::GTODirectRelERIContraction;

  void twoBodyContract(MPI_Comm comm, const bool screen,
                       std::vector<TwoBodyContraction<MatsT>>& list, EMPerturbation& pert,
                       const bool computeExchange = true,
                       const TYPE_4C type4C = TYPE_4C::All,
                       const APPROXIMATION_TYPE_4C approx = APPROXIMATION_TYPE_4C::None)
      const override {
    const auto t = list.empty() ? COULOMB : list[0].contType;
    const bool ours = MPISize(comm) == 1 && type4C == TYPE_4C::All &&
                      approx == APPROXIMATION_TYPE_4C::None && list.size() == 17 &&
                      (t == BARE_COULOMB || t == LLSS || t == SSSS);
    if (!ours) {
      GTODirectRelERIContraction<MatsT, IntsT>::twoBodyContract(comm, screen, list, pert,
                                                                computeExchange, type4C, approx);
      return;
    }
    ensure_basis();
    const void* X[CQF_REL_NMAT];
    void* AX[CQF_REL_NMAT];
    for (int m = 0; m < CQF_REL_NMAT; m++) {
      X[m] = list[m].X;
      AX[m] = list[m].AX;
    }
    cqf_opts o;
    cqf_opts_default(&o);
    o.is_complex = 1;
    o.screen = screen ? 1 : 0;
    const int type = t == BARE_COULOMB ? CQF_REL_BARE_COULOMB
                     : t == LLSS       ? CQF_REL_LLSS
                                       : CQF_REL_SSSS;
    cqf_status st = cqf_rel_two_body_contract(basis_, X, AX, type, computeExchange ? 1 : 0, &o,
                                              nullptr);
    if (st != CQF_OK) CErr(std::string("cqf_rel_two_body_contract: ") + cqf_last_error());
  }

  ~B200DirectRelERIContraction() override {
    if (basis_) cqf_basis_destroy(basis_);
  }
};

}  // namespace ChronusQ
