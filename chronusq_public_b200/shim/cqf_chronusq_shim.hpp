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

#include "cqf_chronusq_basis.hpp"
#include "cqfock.h"

namespace ChronusQ {

template <typename MatsT, typename IntsT>
class B200DirectTPIContraction : public GTODirectTPIContraction<MatsT, IntsT> {
  // the device basis of the DirectTPI's BasisSet, rebuilt whenever its
  // shells change (a geometry step moves them)
  mutable CqfBasisCache cache_;

  cqf_basis* basis() const {
    auto& tpi = *std::dynamic_pointer_cast<DirectTPI<IntsT>>(this->ints_);
    return cache_.get(tpi.basisSet(), tpi.threshSchwarz());
  }

 public:
  using GTODirectTPIContraction<MatsT, IntsT>::GTODirectTPIContraction;
  // keep the convenience overloads of TPIContractions (screen = true, no
  // EMPerturbation; twopints.hpp:225-244) callable on this type
  using GTODirectTPIContraction<MatsT, IntsT>::twoBodyContract;

  // GTODirectTPIContraction::twoBodyContract (gtodirecttpi.hpp:199-206)
  void twoBodyContract(MPI_Comm comm, const bool screen,
                       std::vector<TwoBodyContraction<MatsT>>& list,
                       EMPerturbation& pert) const override {
    if (MPISize(comm) > 1 || this->contractSecond) {  // not offloaded
      GTODirectTPIContraction<MatsT, IntsT>::twoBodyContract(comm, screen, list, pert);
      return;
    }
    cqf_basis* b = basis();
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
    cqf_status st = cqf_two_body_contract(b, c.data(), (int)c.size(), &o, nullptr);
    if (st != CQF_OK) CErr(std::string("cqf_two_body_contract: ") + cqf_last_error());
  }
};

}  // namespace ChronusQ
