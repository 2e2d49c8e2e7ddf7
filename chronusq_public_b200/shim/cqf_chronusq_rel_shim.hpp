// ChronusQ-side binding of the four-component contraction of libcqfock.so.
//
// A ChronusQ maintainer selects B200DirectRelERIContraction where ChronusQ
// constructs GTODirectRelERIContraction<dcomplex,double>
// (src/cxxapi/input/singleslateropts.cxx:1340-1440).  It overrides the 4C
// twoBodyContract overload of the reference class
// (include/particleintegrals/twopints/gtodirectreleri.hpp:75-94), which
// FourCompFock::formGDDirect calls on the concrete type for BARE_COULOMB,
// LLSS, SSSS, GAUNT and GAUGE (include/fockbuilder/fourcompfock/impl.hpp:
// 3923, :4030, :4177, :4279, :4441): the 17 (X, AX) entries in
// DIRAC_PAULI_SPINOR_COMP order (29 for GAUNT and GAUGE) go to
// cqf_rel_two_body_contract, which zeroes the AX it writes like
// directScaffoldLibcint (include/particleintegrals/contract/
// direct4C_libcint.hpp:313-314).  The other contraction type (LLLL), the
// spin-free / spin-dependent variants,
// approximations and MPI runs stay on the reference implementation.  A
// nonzero cqf_status becomes CErr.  Compiles only inside the ChronusQ tree
// (it includes ChronusQ headers).
#pragma once

#include <complex>
#include <string>
#include <vector>

#include <cerr.hpp>
#include <particleintegrals/twopints/gtodirectreleri.hpp>

#include "cqf_chronusq_basis.hpp"
#include "cqfock.h"

namespace ChronusQ {

template <typename MatsT, typename IntsT>
class B200DirectRelERIContraction : public GTODirectRelERIContraction<MatsT, IntsT> {
  // the device basis of the DirectTPI's BasisSet, rebuilt whenever its
  // shells change (a geometry step moves them)
  mutable CqfBasisCache cache_;

  cqf_basis* basis() const {
    auto& tpi = *std::dynamic_pointer_cast<DirectTPI<IntsT>>(this->ints_);
    return cache_.get(tpi.basisSet(), tpi.threshSchwarz());
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
                      approx == APPROXIMATION_TYPE_4C::None &&
                      ((list.size() == 17 && (t == BARE_COULOMB || t == LLSS || t == SSSS)) ||
                       (list.size() == 29 && (t == GAUNT || t == GAUGE)));
    if (!ours) {
      GTODirectRelERIContraction<MatsT, IntsT>::twoBodyContract(comm, screen, list, pert,
                                                                computeExchange, type4C, approx);
      return;
    }
    cqf_basis* b = basis();
    const void* X[CQF_REL_NMAT_GAUNT] = {};
    void* AX[CQF_REL_NMAT_GAUNT] = {};
    for (int m = 0; m < (int)list.size(); m++) {
      X[m] = list[m].X;
      AX[m] = list[m].AX;
    }
    cqf_opts o;
    cqf_opts_default(&o);
    o.is_complex = 1;
    o.screen = screen ? 1 : 0;
    const int type = t == BARE_COULOMB ? CQF_REL_BARE_COULOMB
                     : t == LLSS       ? CQF_REL_LLSS
                     : t == SSSS       ? CQF_REL_SSSS
                     : t == GAUNT      ? CQF_REL_GAUNT
                                       : CQF_REL_GAUGE;
    cqf_status st = cqf_rel_two_body_contract(b, X, AX, type, computeExchange ? 1 : 0, &o,
                                              nullptr);
    if (st != CQF_OK) CErr(std::string("cqf_rel_two_body_contract: ") + cqf_last_error());
  }
};

}  // namespace ChronusQ
