// Test stand-in for the parts of ChronusQ the shims of libcqfock.so use, with
// the reference's names, members and signatures, so that
// chronusq_public_b200/shim/*.hpp compile and run outside the ChronusQ tree:
//   libint2::Shell {alpha, contr[k].{l, pure, coeff}, O}   (libint2 shell.h)
//   BasisSet {nShell, shells}                 (include/basisset.hpp)
//   TWOBODY_CONTRACTION_TYPE, TwoBodyContraction<T>
//                                             (include/particleintegrals/twopints.hpp:31-75)
//   TPIContractions<MatsT,IntsT>::twoBodyContract
//                                             (twopints.hpp:172-260)
//   DirectTPI<IntsT> {basisSet(), threshSchwarz()}
//                                             (twopints/gtodirecttpi.hpp:30-141)
//   GTODirectTPIContraction<MatsT,IntsT>      (twopints/gtodirecttpi.hpp:143-228)
// The reference's own CPU contraction is not here: the stub's base
// twoBodyContract raises CErr, so a call the shim does not offload fails.
#pragma once

#include <array>
#include <memory>
#include <vector>

#include <cerr.hpp>

typedef int MPI_Comm;
#ifndef MPI_COMM_WORLD
#define MPI_COMM_WORLD 0
#endif

namespace libint2 {
struct Shell {
  struct Contraction {
    int l;
    bool pure;
    std::vector<double> coeff;
  };
  std::vector<double> alpha;
  std::vector<Contraction> contr;
  std::array<double, 3> O;
};
}  // namespace libint2

namespace ChronusQ {

inline int MPISize(MPI_Comm) { return 1; }

struct EMPerturbation {};

struct BasisSet {
  size_t nBasis = 0;
  size_t nShell = 0;
  std::vector<libint2::Shell> shells;
};

enum TWOBODY_CONTRACTION_TYPE {
  COULOMB, EXCHANGE, PAIR, BARE_COULOMB, LLLL, LLSS, SSSS, GAUNT, GAUGE
};

enum INTEGRAL_TRANSPOSE { TRANS_NONE, TRANS_MN_TRANS_KL, TRANS_MNKL, TRANS_KL, TRANS_MN };

template <typename T>
struct TwoBodyContraction {
  T* X;
  T* AX;
  bool HER;
  TWOBODY_CONTRACTION_TYPE contType;
  double* ERI4 = nullptr;
  INTEGRAL_TRANSPOSE intTrans;
};

template <typename IntsT>
class TwoPInts {
 public:
  virtual ~TwoPInts() {}
};

template <typename IntsT>
class DirectTPI : public TwoPInts<IntsT> {
 protected:
  BasisSet& basisSet_;
  double threshSchwarz_ = 1e-12;

 public:
  DirectTPI(BasisSet& basis, double threshSchwarz)
      : basisSet_(basis), threshSchwarz_(threshSchwarz) {}
  BasisSet& basisSet() { return basisSet_; }
  const BasisSet& basisSet() const { return basisSet_; }
  double threshSchwarz() const { return threshSchwarz_; }
};

template <typename MatsT, typename IntsT>
class TPIContractions {
 protected:
  std::shared_ptr<TwoPInts<IntsT>> ints_;

 public:
  TPIContractions(std::shared_ptr<TwoPInts<IntsT>> tpi) : ints_(tpi) {}
  virtual void twoBodyContract(MPI_Comm, const bool, std::vector<TwoBodyContraction<MatsT>>&,
                               EMPerturbation&) const = 0;
  inline void twoBodyContract(MPI_Comm comm, const bool screen,
                              std::vector<TwoBodyContraction<MatsT>>& contList) const {
    EMPerturbation pert;
    twoBodyContract(comm, screen, contList, pert);
  }
  inline void twoBodyContract(MPI_Comm comm,
                              std::vector<TwoBodyContraction<MatsT>>& contList) const {
    twoBodyContract(comm, true, contList);
  }
  virtual ~TPIContractions() {}
  bool contractSecond = false;
};

template <typename MatsT, typename IntsT>
class GTODirectTPIContraction : public TPIContractions<MatsT, IntsT> {
 public:
  GTODirectTPIContraction(std::shared_ptr<TwoPInts<IntsT>> tpi)
      : TPIContractions<MatsT, IntsT>(tpi) {}
  using TPIContractions<MatsT, IntsT>::twoBodyContract;
  virtual void twoBodyContract(MPI_Comm, const bool, std::vector<TwoBodyContraction<MatsT>>&,
                               EMPerturbation&) const {
    CErr("reference CPU contraction is not part of this stub");
  }
  virtual ~GTODirectTPIContraction() {}
};

}  // namespace ChronusQ
