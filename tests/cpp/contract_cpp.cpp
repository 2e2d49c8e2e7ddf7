// C++ caller of the library through include/cqfock.hpp: reads a basis and a
// matrix from raw files, runs one twoBodyContract, writes AX.
//   contract_cpp <dir> <her> <type> <complex>
// With <type> = 4: the four-component FourCompFock::formGD on D0..D3.bin
// (<her> is then the libcint switch).
// <dir>/shells.txt: nshell, then per shell "l pure nprim x y z" + alpha + coeff
// <dir>/X.bin: N*N doubles (x2 if complex), column-major; writes <dir>/AX.bin
#include <complex>
#include <cstdio>
#include <fstream>
#include <iostream>
#include <memory>
#include <vector>

#include "cqfock.hpp"

template <typename T>
int run(const std::string& dir, const std::vector<cqfock::Shell>& sh, bool her, int type) {
  auto tpi = std::make_shared<cqfock::DirectTPI>(sh);
  const size_t N = tpi->nBasis();
  std::vector<T> X(N * N), AX(N * N, T(0));
  std::ifstream fx(dir + "/X.bin", std::ios::binary);
  fx.read(reinterpret_cast<char*>(X.data()), X.size() * sizeof(T));
  cqfock::GTODirectTPIContraction<T> con(tpi);
  std::vector<cqfock::TwoBodyContraction<T>> list = {
      {X.data(), AX.data(), her, type ? cqfock::EXCHANGE : cqfock::COULOMB}};
  con.twoBodyContract(true, list);
  std::ofstream fo(dir + "/AX.bin", std::ios::binary);
  fo.write(reinterpret_cast<const char*>(AX.data()), AX.size() * sizeof(T));
  return 0;
}

// 4C mode: <dir>/D0..D3.bin (2N x 2N complex each) -> <dir>/G0..G3.bin
int run4c(const std::string& dir, const std::vector<cqfock::Shell>& sh, bool libcint) {
  using Z = std::complex<double>;
  auto tpi = std::make_shared<cqfock::DirectTPI>(sh);
  const size_t N2 = 2 * (size_t)tpi->nBasis();
  std::vector<Z> D[4], G[4];
  const Z* dp[4];
  Z* gp[4];
  for (int c = 0; c < 4; c++) {
    D[c].resize(N2 * N2);
    G[c].resize(N2 * N2);
    std::ifstream fd(dir + "/D" + std::to_string(c) + ".bin", std::ios::binary);
    fd.read(reinterpret_cast<char*>(D[c].data()), D[c].size() * sizeof(Z));
    dp[c] = D[c].data();
    gp[c] = G[c].data();
  }
  cqfock::FourCompFock fock(tpi, true, true, true, libcint);
  fock.formGD(dp, gp);
  for (int c = 0; c < 4; c++) {
    std::ofstream fo(dir + "/G" + std::to_string(c) + ".bin", std::ios::binary);
    fo.write(reinterpret_cast<const char*>(G[c].data()), G[c].size() * sizeof(Z));
  }
  return 0;
}

int main(int argc, char** argv) {
  if (argc < 5) return 2;
  std::string dir = argv[1];
  bool her = std::atoi(argv[2]) != 0, cplx = std::atoi(argv[4]) != 0;
  int type = std::atoi(argv[3]);
  std::ifstream fs(dir + "/shells.txt");
  int ns;
  fs >> ns;
  std::vector<cqfock::Shell> sh(ns);
  for (auto& s : sh) {
    int pure, np;
    fs >> s.l >> pure >> np >> s.O[0] >> s.O[1] >> s.O[2];
    s.pure = pure != 0;
    s.alpha.resize(np);
    s.coeff.resize(np);
    for (auto& a : s.alpha) fs >> a;
    for (auto& c : s.coeff) fs >> c;
  }
  try {
    if (type == 4) return run4c(dir, sh, her);  // her: libcint switch in this mode
    return cplx ? run<std::complex<double>>(dir, sh, her, type) : run<double>(dir, sh, her, type);
  } catch (const std::exception& e) {
    std::cerr << e.what() << "\n";
    return 1;
  }
}
