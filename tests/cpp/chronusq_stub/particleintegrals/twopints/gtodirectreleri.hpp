// Test stand-in for GTODirectRelERIContraction
// (include/particleintegrals/twopints/gtodirectreleri.hpp:30-100): the
// four-component twoBodyContract overload with its default arguments, and
// the TYPE_4C / APPROXIMATION_TYPE_4C switches (include/hamiltonianoptions.hpp:33-35).  The reference's libcint
// path is not here: the stub's base implementation raises CErr.
#pragma once

#include <particleintegrals/twopints/gtodirecttpi.hpp>

namespace ChronusQ {

enum class TYPE_4C { All, SpinFree, SpinDependent };
enum class APPROXIMATION_TYPE_4C { None, ThreeCenter, TwoCenter, OneCenter, AtomicMeanField };

template <typename MatsT, typename IntsT>
class GTODirectRelERIContraction : public GTODirectTPIContraction<MatsT, IntsT> {
 public:
  GTODirectRelERIContraction(std::shared_ptr<TwoPInts<IntsT>> tpi)
      : GTODirectTPIContraction<MatsT, IntsT>(tpi) {}
  virtual void twoBodyContract(MPI_Comm, const bool, std::vector<TwoBodyContraction<MatsT>>&,
                               EMPerturbation&, const bool computeExchange = true,
                               const TYPE_4C type4C = TYPE_4C::All,
                               const APPROXIMATION_TYPE_4C approximate4C =
                                   APPROXIMATION_TYPE_4C::None) const {
    CErr("reference libcint contraction is not part of this stub");
  }
};

}  // namespace ChronusQ
