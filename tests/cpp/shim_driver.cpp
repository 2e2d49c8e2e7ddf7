// Runs the ChronusQ-side shims (chronusq_public_b200/shim/) against the test
// stand-ins of ChronusQ's classes (tests/cpp/chronusq_stub/): one BasisSet,
// one DirectTPI and one contraction object, as ChronusQ holds them across an
// SCF or a geometry optimisation.  The shells move between calls, and each
// call must see the current geometry.
//   shim_driver <dir> 1c : J and K of the real density D.bin (N x N) at the
//                          geometries of shells0.txt, shells1.txt, shells1.txt
//                          -> JK0.bin, JK1.bin, JK2.bin (J then K, column-major)
//   shim_driver <dir> 4c : BARE_COULOMB on the complex Hermitian matrices
//                          R0..R4.bin (N x N each: CLLMS, XLLMS, XLLMX, XLLMY,
//                          XLLMZ) at the same three geometries -> REL0..2.bin
//                          (the five outputs)
//   shim_driver <dir> gaunt|gauge : GAUNT / GAUGE on the 4C density blocks
//                          G0..G15.bin (LL, SS, LS, SL x scalar, MX, MY, MZ)
//                          at the geometry of shells0.txt -> gaunt.bin /
//                          gauge.bin (XLLM*, XSSM*, XLSM*, CLSM*)
// shells<k>.txt: nshell, then per shell "l pure nprim x y z" + alpha + coeff
#include <complex>
#include <fstream>
#include <iostream>
#include <memory>
#include <string>
#include <vector>

#include <particleintegrals/twopints/gtodirecttpi.hpp>
#include <particleintegrals/twopints/gtodirectreleri.hpp>

#include "cqf_chronusq_rel_shim.hpp"
#include "cqf_chronusq_shim.hpp"

using namespace ChronusQ;

static std::vector<libint2::Shell> read_shells(const std::string& path, size_t& nbasis) {
  std::ifstream f(path);
  int n = 0;
  f >> n;
  std::vector<libint2::Shell> sh(n);
  nbasis = 0;
  for (auto& s : sh) {
    int l, pure, np;
    f >> l >> pure >> np >> s.O[0] >> s.O[1] >> s.O[2];
    s.alpha.resize(np);
    s.contr.resize(1);
    s.contr[0].l = l;
    s.contr[0].pure = pure != 0;
    s.contr[0].coeff.resize(np);
    for (auto& a : s.alpha) f >> a;
    for (auto& c : s.contr[0].coeff) f >> c;
    nbasis += pure ? 2 * l + 1 : (l + 1) * (l + 2) / 2;
  }
  return sh;
}

template <typename T>
static std::vector<T> read_bin(const std::string& path, size_t n) {
  std::vector<T> v(n);
  std::ifstream f(path, std::ios::binary);
  f.read(reinterpret_cast<char*>(v.data()), n * sizeof(T));
  if (!f) CErr("short read: " + path);
  return v;
}

template <typename T>
static void write_bin(const std::string& path, const std::vector<T>& v) {
  std::ofstream f(path, std::ios::binary);
  f.write(reinterpret_cast<const char*>(v.data()), v.size() * sizeof(T));
}

int main(int argc, char** argv) {
  if (argc < 3) {
    std::cerr << "usage: shim_driver <dir> 1c|4c|gaunt|gauge" << std::endl;
    return 2;
  }
  const std::string dir = argv[1], mode = argv[2];
  try {
    BasisSet bs;
    bs.shells = read_shells(dir + "/shells0.txt", bs.nBasis);
    bs.nShell = bs.shells.size();
    const size_t N = bs.nBasis;
    auto tpi = std::make_shared<DirectTPI<double>>(bs, 1e-12);
    const char* geo[3] = {"shells0.txt", "shells1.txt", "shells1.txt"};
    if (mode == "1c") {
      B200DirectTPIContraction<double, double> con(tpi);
      std::vector<double> D = read_bin<double>(dir + "/D.bin", N * N);
      for (int g = 0; g < 3; g++) {
        size_t nb = 0;
        bs.shells = read_shells(dir + "/" + geo[g], nb);  // the nuclei moved
        std::vector<double> JK(2 * N * N, 0.0);
        std::vector<TwoBodyContraction<double>> list = {
            {D.data(), JK.data(), true, COULOMB}, {D.data(), JK.data() + N * N, true, EXCHANGE}};
        con.twoBodyContract(MPI_COMM_WORLD, list);
        write_bin(dir + "/JK" + std::to_string(g) + ".bin", JK);
      }
    } else if (mode == "4c") {
      using Z = std::complex<double>;
      B200DirectRelERIContraction<Z, double> con(tpi);
      std::vector<std::vector<Z>> R(17, std::vector<Z>(N * N, Z(0)));
      for (int k = 0; k < 5; k++) R[k] = read_bin<Z>(dir + "/R" + std::to_string(k) + ".bin", N * N);
      for (int g = 0; g < 3; g++) {
        size_t nb = 0;
        bs.shells = read_shells(dir + "/" + geo[g], nb);
        std::vector<std::vector<Z>> out(17, std::vector<Z>(N * N, Z(1.0)));  // zeroed by the call
        std::vector<TwoBodyContraction<Z>> list(17);
        for (int k = 0; k < 17; k++)
          list[k] = {R[k].data(), out[k].data(), true, k == 0 ? BARE_COULOMB : EXCHANGE};
        EMPerturbation pert;
        con.twoBodyContract(MPI_COMM_WORLD, true, list, pert);
        std::vector<Z> o;
        for (int k = 0; k < 5; k++) o.insert(o.end(), out[k].begin(), out[k].end());
        write_bin(dir + "/REL" + std::to_string(g) + ".bin", o);
      }
    } else if (mode == "gaunt" || mode == "gauge") {
      // the reference's GAUNT list (fourcompfock/impl.hpp:4237-4274): 29
      // entries, the CSLM* / XSLM* AX pointed at the CLSM* / XLSM* outputs
      using Z = std::complex<double>;
      B200DirectRelERIContraction<Z, double> con(tpi);
      std::vector<std::vector<Z>> G(16);  // LL, SS, LS, SL x (S, X, Y, Z)
      for (int k = 0; k < 16; k++) G[k] = read_bin<Z>(dir + "/G" + std::to_string(k) + ".bin", N * N);
      std::vector<std::vector<Z>> out(29, std::vector<Z>(N * N, Z(1.0)));
      std::vector<TwoBodyContraction<Z>> list(29);
      for (int c = 0; c < 4; c++) {
        list[1 + c] = {G[c].data(), out[1 + c].data(), true, EXCHANGE};         // XLLM*
        list[5 + c] = {G[4 + c].data(), out[5 + c].data(), true, EXCHANGE};     // CSSM*
        list[9 + c] = {G[4 + c].data(), out[9 + c].data(), true, EXCHANGE};     // XSSM*
        list[13 + c] = {G[8 + c].data(), out[13 + c].data(), true, EXCHANGE};   // XLSM*
        list[17 + c] = {G[8 + c].data(), out[17 + c].data(), true, EXCHANGE};   // CLSM*
        list[21 + c] = {G[12 + c].data(), out[17 + c].data(), true, EXCHANGE};  // CSLM*
        list[25 + c] = {G[12 + c].data(), out[13 + c].data(), true, EXCHANGE};  // XSLM*
      }
      list[0] = {G[0].data(), out[0].data(), true, mode == "gaunt" ? GAUNT : GAUGE};
      EMPerturbation pert;
      con.twoBodyContract(MPI_COMM_WORLD, true, list, pert);
      std::vector<Z> o;
      for (int base : {1, 9, 13, 17})
        for (int c = 0; c < 4; c++) o.insert(o.end(), out[base + c].begin(), out[base + c].end());
      write_bin(dir + "/" + mode + ".bin", o);
    } else {
      std::cerr << "unknown mode " << mode << std::endl;
      return 2;
    }
  } catch (const std::exception& e) {
    std::cerr << "shim_driver: " << e.what() << std::endl;
    return 1;
  }
  return 0;
}
