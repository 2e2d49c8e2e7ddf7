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
//   GTODirectRelERIContraction / FourCompFock (the four-component build)
//       gtodirectreleri.hpp:75-94, fockbuilder/fourcompfock/impl.hpp:3752-4636
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

// include/particleintegrals/twopints.hpp:31-41 (same order and values)
enum TWOBODY_CONTRACTION_TYPE {
  COULOMB = CQF_COULOMB,
  EXCHANGE = CQF_EXCHANGE,
  PAIR,
  BARE_COULOMB,
  LLLL,
  LLSS,
  SSSS,
  GAUNT,
  GAUGE
};

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

// GTODirectRelERIContraction<dcomplex,double>::twoBodyContract
// (include/particleintegrals/twopints/gtodirectreleri.hpp:75-94): 17 entries
// in DIRAC_PAULI_SPINOR_COMP order (29 for GAUNT and GAUGE), contType of
// entry 0 = BARE_COULOMB, LLSS, SSSS, GAUNT or GAUGE; the AX the type writes
// are overwritten (zeroed, then the contraction).
class GTODirectRelERIContraction {
 public:
  explicit GTODirectRelERIContraction(std::shared_ptr<DirectTPI> tpi) : tpi_(std::move(tpi)) {}

  void twoBodyContract(const bool screen,
                       std::vector<TwoBodyContraction<std::complex<double>>>& list,
                       const bool computeExchange = true, cqf_stats* stats = nullptr) const {
    if (list.empty()) throw std::runtime_error("GTODirectRelERIContraction: empty list");
    int type;
    switch (list[0].contType) {
      case BARE_COULOMB: type = CQF_REL_BARE_COULOMB; break;
      case LLSS: type = CQF_REL_LLSS; break;
      case SSSS: type = CQF_REL_SSSS; break;
      case GAUNT: type = CQF_REL_GAUNT; break;
      case GAUGE: type = CQF_REL_GAUGE; break;
      default: throw std::runtime_error("GTODirectRelERIContraction: unsupported contraction type");
    }
    const int n = type >= CQF_REL_GAUNT ? CQF_REL_NMAT_GAUNT : CQF_REL_NMAT;
    if ((int)list.size() != n)
      throw std::runtime_error("GTODirectRelERIContraction: the 4C list has 17 entries (29 for "
                               "GAUNT and GAUGE)");
    const void* X[CQF_REL_NMAT_GAUNT] = {};
    void* AX[CQF_REL_NMAT_GAUNT] = {};
    for (int m = 0; m < n; m++) {
      X[m] = list[m].X;
      AX[m] = list[m].AX;
    }
    cqf_opts o;
    cqf_opts_default(&o);
    o.is_complex = 1;
    o.screen = screen ? 1 : 0;
    check(cqf_rel_two_body_contract(tpi_->handle(), X, AX, type, computeExchange ? 1 : 0, &o,
                                    stats),
          "cqf_rel_two_body_contract");
  }

 private:
  std::shared_ptr<DirectTPI> tpi_;
};

// FourCompFock<dcomplex,double>::formGDDirect
// (include/fockbuilder/fourcompfock/impl.hpp:3752-4636) with the
// HamiltonianOptions switches BareCoulomb, DiracCoulomb, DiracCoulombSSSS,
// Libcint, Gaunt and Gauge.  D and G: the four Pauli components (scalar, MX, MY,
// MZ) of the 2N x 2N complex 4C matrices, column-major, LL block first.
class FourCompFock {
 public:
  explicit FourCompFock(std::shared_ptr<DirectTPI> tpi, bool BareCoulomb = true,
                        bool DiracCoulomb = true, bool DiracCoulombSSSS = true,
                        bool Libcint = true, bool Gaunt = false, bool Gauge = false)
      : tpi_(std::move(tpi)) {
    cqf_dc_opts_default(&dc_);
    dc_.bare_coulomb = BareCoulomb;
    dc_.dirac_coulomb = DiracCoulomb;
    dc_.dirac_coulomb_ssss = DiracCoulombSSSS;
    dc_.libcint = Libcint;
    dc_.gaunt = Gaunt;
    dc_.gauge = Gauge;
  }

  void formGD(const std::complex<double>* const D[4], std::complex<double>* const G[4],
              double xHFX = 1.0, cqf_stats* stats = nullptr) const {
    cqf_dc_opts dc = dc_;
    dc.xHFX = xHFX;
    const void* d[4] = {D[0], D[1], D[2], D[3]};
    void* g[4] = {G[0], G[1], G[2], G[3]};
    cqf_opts o;
    cqf_opts_default(&o);
    o.is_complex = 1;
    check(cqf_four_comp_gd(tpi_->handle(), d, g, &dc, &o, stats), "cqf_four_comp_gd");
  }

 private:
  std::shared_ptr<DirectTPI> tpi_;
  cqf_dc_opts dc_;
};

// DirectGradContraction<double,double>::gradTwoBodyContract
// (include/particleintegrals/gradints.hpp:278-283): cList[3 atom + xyz][m],
// every component with the same X / HER / contType and its own AX (added
// into); shellAtom: ChronusQ's mapSh2Cen.
class DirectGradContraction {
 public:
  explicit DirectGradContraction(std::shared_ptr<DirectTPI> tpi) : tpi_(std::move(tpi)) {}

  void gradTwoBodyContract(std::vector<std::vector<TwoBodyContraction<double>>>& cList,
                           const std::vector<int>& shellAtom, cqf_stats* stats = nullptr) const {
    if (cList.empty() || cList.size() % 3)
      throw std::runtime_error("DirectGradContraction: 3 components per atom");
    const int nMat = (int)cList[0].size();
    std::vector<cqf_contraction> list(nMat);
    for (int m = 0; m < nMat; m++)
      list[m] = {cList[0][m].X, nullptr, cList[0][m].HER ? 1 : 0, (int)cList[0][m].contType};
    std::vector<void*> AX;
    for (auto& comp : cList) {
      if ((int)comp.size() != nMat)
        throw std::runtime_error("DirectGradContraction: ragged contraction list");
      for (auto& c : comp) AX.push_back(c.AX);
    }
    cqf_opts o;
    cqf_opts_default(&o);
    check(cqf_grad_two_body_contract(tpi_->handle(), shellAtom.data(), (int)cList.size() / 3,
                                     list.data(), nMat, AX.data(), &o, stats),
          "cqf_grad_two_body_contract");
  }

 private:
  std::shared_ptr<DirectTPI> tpi_;
};

}  // namespace cqfock
