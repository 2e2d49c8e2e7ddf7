// Device basis of a ChronusQ BasisSet for the shims of libcqfock.so.
//
// The reference keeps its Schwarz table on the DirectTPI object and
// recomputes it whenever the integrals are recomputed for a new geometry
// (include/particleintegrals/twopints/gtodirecttpi.hpp:39-41; the basis'
// shells move with the nuclei, src/basisset/basisset.cxx:98-191).  This cache
// holds one cqf_basis and compares the BasisSet's shells (angular momentum,
// pure flag, exponents, contraction coefficients and centres) with the copy
// it was built from on every call: any change -- a geometry step, a new basis
// -- destroys the device basis and builds it again, so a contraction never
// runs against stale shells or Schwarz bounds.
// Compiles only inside the ChronusQ tree (it includes ChronusQ headers).
#pragma once

#include <string>
#include <vector>

#include <cerr.hpp>

#include "cqfock.h"

namespace ChronusQ {

class CqfBasisCache {
  cqf_basis* basis_ = nullptr;
  double thresh_ = 0.0;
  // flattened copy of the shells the device basis was built from:
  // per shell {l, pure, nprim, x, y, z, alpha..., coeff...}
  std::vector<double> key_;
  std::vector<double> alpha_, coef_;

  template <class Shells>
  static std::vector<double> snapshot(const Shells& shells) {
    std::vector<double> k;
    for (const auto& s : shells) {
      k.push_back(s.contr[0].l);
      k.push_back(s.contr[0].pure ? 1.0 : 0.0);
      k.push_back((double)s.alpha.size());
      for (int x = 0; x < 3; x++) k.push_back(s.O[x]);
      k.insert(k.end(), s.alpha.begin(), s.alpha.end());
      k.insert(k.end(), s.contr[0].coeff.begin(), s.contr[0].coeff.end());
    }
    return k;
  }

 public:
  CqfBasisCache() = default;
  CqfBasisCache(const CqfBasisCache&) = delete;
  CqfBasisCache& operator=(const CqfBasisCache&) = delete;
  ~CqfBasisCache() { reset(); }

  void reset() {
    if (basis_) cqf_basis_destroy(basis_);
    basis_ = nullptr;
    key_.clear();
  }

  // The device basis of `bs`, rebuilt when its shells or the Schwarz
  // threshold differ from those of the current one.
  template <class BasisSetT>
  cqf_basis* get(const BasisSetT& bs, double threshSchwarz) {
    std::vector<double> k = snapshot(bs.shells);
    if (basis_ && k == key_ && threshSchwarz == thresh_) return basis_;
    reset();
    std::vector<cqf_shell> sh(bs.shells.size());
    alpha_.clear();
    coef_.clear();
    for (const auto& s : bs.shells) {
      alpha_.insert(alpha_.end(), s.alpha.begin(), s.alpha.end());
      coef_.insert(coef_.end(), s.contr[0].coeff.begin(), s.contr[0].coeff.end());
    }
    size_t off = 0;
    for (size_t i = 0; i < bs.shells.size(); i++) {
      const auto& s = bs.shells[i];
      sh[i].l = s.contr[0].l;
      sh[i].pure = s.contr[0].pure ? 1 : 0;
      sh[i].nprim = (int)s.alpha.size();
      sh[i].alpha = alpha_.data() + off;
      sh[i].coeff = coef_.data() + off;
      for (int x = 0; x < 3; x++) sh[i].origin[x] = s.O[x];
      off += s.alpha.size();
    }
    cqf_basis* b = nullptr;
    cqf_status st = cqf_basis_create(sh.data(), (int)sh.size(), threshSchwarz, 0, &b);
    if (st != CQF_OK) CErr(std::string("cqf_basis_create: ") + cqf_last_error());
    basis_ = b;
    key_.swap(k);
    thresh_ = threshSchwarz;
    return basis_;
  }
};

}  // namespace ChronusQ
