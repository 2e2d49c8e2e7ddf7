// cqfock.hpp -- header-only C++17 host layer over the C ABI (cqfock.h).
//
// Mirrors the C++ interface of ChronusQ's direct contraction so C++ callers
// keep the reference's names and semantics:
//   TWOBODY_CONTRACTION_TYPE, TwoBodyContraction<T>
//       include/particleintegrals/twopints.hpp:31-75
//   DirectTPI (shells + threshSchwarz, Schwarz cached per basis)
//       include/particleintegrals/twopints/gtodirecttpi.hpp:30-141
//   GTODirectTPIContraction<MatsT>::twoBodyContract(screen, list)
//       include/particleintegrals/twopints/gtodirecttpi.hpp:199-206
// Errors become std::runtime_error, as ChronusQ's CErr does (include/cerr.hpp).
#pragma once

#include <complex>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "cqfock.h"

namespace cqfock {

enum TWOBODY_CONTRACTION_TYPE { COULOMB = CQF_COULOMB, EXCHANGE = CQF_EXCHANGE };

template <typename T>
struct TwoBodyContraction {
  T* X;       // 1-body (2-index) operator to contract with (N x N, column-major)
  T* AX;      // storage of the contraction, accumulated (AX += G[X])
  bool HER;   // whether X is Hermitian
  TWOBODY_CONTRACTION_TYPE contType;
};

inline void check(cqf_status s, const char* what) {
  if (s != CQF_OK) throw std::runtime_error(std::string(what) + ": " + cqf_last_error());
}

// One contracted shell: exponents, libint-normalised coefficients, centre.
struct Shell {
  int l;
  bool pure;
  std::vector<double> alpha, coeff;
  double O[3];
};

// Device-resident basis: significant shell pairs, primitive-pair data and
// Schwarz bounds (built once per geometry).
class DirectTPI {
 public:
  DirectTPI(const std::vector<Shell>& shells, double threshSchwarz = 1e-12, int device = 0)
      : thresh_(threshSchwarz) {
    std::vector<cqf_shell> s(shells.size());
    for (size_t i = 0; i < shells.size(); i++) {
      s[i].l = shells[i].l;
      s[i].pure = shells[i].pure ? 1 : 0;
      s[i].nprim = (int)shells[i].alpha.size();
      s[i].alpha = shells[i].alpha.data();
      s[i].coeff = shells[i].coeff.data();
      for (int x = 0; x < 3; x++) s[i].origin[x] = shells[i].O[x];
    }
    cqf_basis* b = nullptr;
    check(cqf_basis_create(s.data(), (int)s.size(), threshSchwarz, device, &b),
          "cqf_basis_create");
    basis_.reset(b);
    check(cqf_basis_info(b, &nbasis_, &nshell_, &npair_), "cqf_basis_info");
  }
  int nBasis() const { return nbasis_; }
  int nShell() const { return nshell_; }
  int nSigPairs() const { return npair_; }
  double threshSchwarz() const { return thresh_; }
  cqf_basis* handle() const { return basis_.get(); }
  std::vector<double> schwarz() const {
    std::vector<double> q((size_t)nshell_ * nshell_);
    check(cqf_basis_schwarz(basis_.get(), q.data()), "cqf_basis_schwarz");
    return q;
  }

 private:
  struct Del {
    void operator()(cqf_basis* b) const { cqf_basis_destroy(b); }
  };
  std::unique_ptr<cqf_basis, Del> basis_;
  double thresh_;
  int nbasis_ = 0, nshell_ = 0, npair_ = 0;
};

// GTODirectTPIContraction<MatsT,double> on the GPU (MatsT = double or
// std::complex<double>).
template <typename MatsT>
class GTODirectTPIContraction {
  static_assert(std::is_same<MatsT, double>::value ||
                    std::is_same<MatsT, std::complex<double>>::value,
                "MatsT must be double or std::complex<double>");

 public:
  explicit GTODirectTPIContraction(std::shared_ptr<DirectTPI> tpi) : tpi_(std::move(tpi)) {}

  // AX += G[X] for every entry (directScaffoldNew semantics); host pointers.
  void twoBodyContract(const bool screen, std::vector<TwoBodyContraction<MatsT>>& list,
                       cqf_stats* stats = nullptr) const {
    std::vector<cqf_contraction> c(list.size());
    for (size_t i = 0; i < list.size(); i++) {
      c[i].X = list[i].X;
      c[i].AX = list[i].AX;
      c[i].hermitian = list[i].HER ? 1 : 0;
      c[i].type = list[i].contType;
    }
    cqf_opts o;
    cqf_opts_default(&o);
    o.is_complex = std::is_same<MatsT, std::complex<double>>::value ? 1 : 0;
    o.screen = screen ? 1 : 0;
    check(cqf_two_body_contract(tpi_->handle(), c.data(), (int)c.size(), &o, stats),
          "cqf_two_body_contract");
  }
  void twoBodyContract(std::vector<TwoBodyContraction<MatsT>>& list) const {
    twoBodyContract(true, list);
  }

 private:
  std::shared_ptr<DirectTPI> tpi_;
};

}  // namespace cqfock
