"""Four-component two-electron terms rebuilt from kinetically balanced
2-spinors with numpy -- test infrastructure, independent of the oracle's and
the library's four-component code.

Basis: large-component spinors chi_mu |s> and small-component spinors
(sigma.p) chi_mu |s> / (2c), p = -i grad.  With a 4-spinor basis the
two-electron matrix is G = J - K over spin-orbital indices,
J_PQ = sum_RS (PQ|RS) D_SR and K_PQ = sum_RS (PS|RQ) D_SR, and the
reference stores every 2N x 2N block as Pauli components S = aa + bb,
X = ab + ba, Y = i (ab - ba), Z = aa - bb (the same convention for D and G).

* Dirac-Coulomb: charge densities Phi_P^+ Phi_Q of equal type --
  LL: chi_mu chi_nu delta_ss', SS: (1 / 4c^2) sum_ij (sigma_i sigma_j)_ss'
  d_i chi_mu d_j chi_nu (sigma_i sigma_j = delta_ij + i eps_ijk sigma_k).
* Gaunt, -alpha_1 . alpha_2 / r_12 with alpha_k = [[0, sigma_k],
  [sigma_k, 0]]: charge densities Phi_P^+ alpha_k Phi_Q of mixed type --
  LS: (-i / 2c) sum_j (sigma_k sigma_j)_ss' chi_mu d_j chi_nu,
  SL: (i / 2c) sum_j (sigma_j sigma_k)_ss' d_j chi_mu chi_nu --
  and (PQ|RS)_Gaunt = -sum_k (rho^k_PQ | rho^k_RS).

* Breit gauge part, -(alpha_1 . r)(alpha_2 . r) / r^3 (r = r1 - r2): the
  same densities with the kernel K_ii' = -r_i r_i' / r^3 between rho^i and
  rho^i' in place of Gaunt's -delta_ii' / r.  Since
  r_i r_i' / r^3 = delta_ii' / r - d_i d_i' r, it is Gaunt plus the kernel
  d_i d_i' r12, whose integrals are the oracle's r12 integrals with the
  Hermite index shifted (checked against the Coulomb ones through
  sum_i d_i d_i r = 2 / r in test_gaunt_golden.py).

Derivative ERIs (d/dr of the orbitals) come from the oracle's
eri_deriv_quartet, checked against finite differences in
test_oracle_deriv.py.
"""
import numpy as np

import oracle as O
from chronusq_public_b200.workloads import SPEED_OF_LIGHT

SIG = np.array([[[0, 1], [1, 0]], [[0, -1j], [1j, 0]], [[1, 0], [0, -1]]], dtype=complex)
# sigma_i sigma_j, (3, 3, 2, 2)
SS = np.einsum("iab,jbc->ijac", SIG, SIG)
C2 = 1.0 / (4.0 * SPEED_OF_LIGHT ** 2)


def deriv_tensor(basis, dmask):
    """(3,)*nd + (N, N, N, N) derivative ERI tensor, derivatives on the
    centres in dmask (bit 0..3 = function 1..4)."""
    ob = O.OracleBasis(basis)
    N = basis.nbasis
    nd = bin(dmask).count("1")
    out = np.zeros((3 ** nd, N, N, N, N))
    off, sz = basis.offsets, basis.sizes
    ns = basis.nshell
    for a in range(ns):
        for b in range(ns):
            for c in range(ns):
                for d in range(ns):
                    blk = ob.eri_deriv_quartet(a, b, c, d, dmask)
                    out[:, off[a]:off[a] + sz[a], off[b]:off[b] + sz[b],
                        off[c]:off[c] + sz[c], off[d]:off[d] + sz[d]] = blk
    return out.reshape((3,) * nd + (N, N, N, N))


def spin_blocks(M, N):
    """Pauli components [S, X, Y, Z] (2N x 2N, LL first) -> the spatial
    blocks LL, LS, SL, SS as spin-orbital arrays [mu, s, nu, s']."""
    S, X, Y, Z = M
    out = {}
    for name, (r, c) in {"LL": (0, 0), "LS": (0, 1), "SL": (1, 0), "SS": (1, 1)}.items():
        sl = (slice(r * N, (r + 1) * N), slice(c * N, (c + 1) * N))
        b = np.zeros((N, 2, N, 2), dtype=complex)
        b[:, 0, :, 0] = (S[sl] + Z[sl]) / 2
        b[:, 1, :, 1] = (S[sl] - Z[sl]) / 2
        b[:, 0, :, 1] = (X[sl] - 1j * Y[sl]) / 2
        b[:, 1, :, 0] = (X[sl] + 1j * Y[sl]) / 2
        out[name] = b
    return out


def pauli(b):
    """Spin-orbital block [mu, s, nu, s'] -> Pauli components [S, X, Y, Z]."""
    aa, bb, ab, ba = b[:, 0, :, 0], b[:, 1, :, 1], b[:, 0, :, 1], b[:, 1, :, 0]
    return [aa + bb, ab + ba, 1j * (ab - ba), aa - bb]


def assemble(blocks, N):
    """Spin-orbital blocks {LL, LS, SL, SS} -> 4 Pauli components, 2N x 2N."""
    G = [np.zeros((2 * N, 2 * N), dtype=complex) for _ in range(4)]
    for name, (r, c) in {"LL": (0, 0), "LS": (0, 1), "SL": (1, 0), "SS": (1, 1)}.items():
        if name not in blocks:
            continue
        for k, m in enumerate(pauli(blocks[name])):
            G[k][r * N:(r + 1) * N, c * N:(c + 1) * N] = m
    return G


def gaunt(basis, D):
    """The Gaunt two-electron matrix G = J - K (4 Pauli components) of the
    4C density D (4 Pauli components, 2N x 2N)."""
    N = basis.nbasis
    Db = spin_blocks(D, N)
    T = deriv_tensor(basis, 10)  # (a d_j b | c d_l d), T[j, l, a, b, c, d]
    k4 = C2  # (1/2c)^2
    # spin factors of the four type pairs, sum over k included, with the
    # Gaunt sign: M[j, l, s, s', t, t']
    M_LSLS = k4 * np.einsum("kjab,klcd->jlabcd", SS, SS)
    M_LSSL = -k4 * np.einsum("kjab,lkcd->jlabcd", SS, SS)
    M_SLLS = -k4 * np.einsum("jkab,klcd->jlabcd", SS, SS)
    M_SLSL = k4 * np.einsum("jkab,lkcd->jlabcd", SS, SS)
    o = dict(optimize=True)
    # Coulomb-type: LS and SL blocks from the LS / SL densities
    JLS = (np.einsum("jlxytu,jlabcd,duct->axby", M_LSLS, T, Db["SL"], **o)
           + np.einsum("jlxytu,jlabcd,cudt->axby", M_LSSL, T, Db["LS"], **o))
    JSL = (np.einsum("jlxytu,jlabcd,duct->bxay", M_SLLS, T, Db["SL"], **o)
           + np.einsum("jlxytu,jlabcd,cudt->bxay", M_SLSL, T, Db["LS"], **o))
    # exchange-type: LL from SS, SS from LL, LS from SL, SL from LS
    KLL = np.einsum("jlxuty,jlabcd,budt->axcy", M_LSSL, T, Db["SS"], **o)
    KSS = np.einsum("jlxuty,jlabcd,auct->bxdy", M_SLLS, T, Db["LL"], **o)
    KLS = np.einsum("jlxuty,jlabcd,buct->axdy", M_LSLS, T, Db["SL"], **o)
    KSL = np.einsum("jlxuty,jlabcd,audt->bxcy", M_SLSL, T, Db["LS"], **o)
    return assemble({"LL": -KLL, "SS": -KSS, "LS": JLS - KLS, "SL": JSL - KSL}, N)


def r12_tensor(basis):
    """U[i, i', j, l, a, b, c, d] = (a d_j b | d_i d_i' r12 | c d_l d)."""
    ob = O.OracleBasis(basis)
    N = basis.nbasis
    off, sz = basis.offsets, basis.sizes
    ns = basis.nshell
    U = np.zeros((3, 3, 3, 3, N, N, N, N))
    for i in range(3):
        for ip in range(i, 3):
            for a in range(ns):
                for b in range(ns):
                    for c in range(ns):
                        for d in range(ns):
                            blk = ob.r12_deriv_quartet(a, b, c, d, 10, i, ip)
                            U[i, ip, :, :, off[a]:off[a] + sz[a], off[b]:off[b] + sz[b],
                              off[c]:off[c] + sz[c], off[d]:off[d] + sz[d]] = \
                                blk.reshape(3, 3, sz[a], sz[b], sz[c], sz[d])
            U[ip, i] = U[i, ip]
    return U


def kernel_term(basis, D, V):
    """G = J - K of the two-electron operator sum_ii' alpha_1i K_ii' alpha_2i'
    with V[i, i', j, l, a, b, c, d] = (a d_j b | K_ii' | c d_l d) (4 Pauli
    components); V = -delta_ii' T is the Gaunt term."""
    N = basis.nbasis
    Db = spin_blocks(D, N)
    k4 = C2
    o = dict(optimize=True)
    A = {"LSLS": -k4 * np.einsum("ijxy,kltu,ikjlabcd->xytuabcd", SS, SS, V, **o),
         "LSSL": k4 * np.einsum("ijxy,lktu,ikjlabcd->xytuabcd", SS, SS, V, **o),
         "SLLS": k4 * np.einsum("jixy,kltu,ikjlabcd->xytuabcd", SS, SS, V, **o),
         "SLSL": -k4 * np.einsum("jixy,lktu,ikjlabcd->xytuabcd", SS, SS, V, **o)}
    JLS = (np.einsum("xytuabcd,duct->axby", A["LSLS"], Db["SL"], **o)
           + np.einsum("xytuabcd,cudt->axby", A["LSSL"], Db["LS"], **o))
    JSL = (np.einsum("xytuabcd,duct->bxay", A["SLLS"], Db["SL"], **o)
           + np.einsum("xytuabcd,cudt->bxay", A["SLSL"], Db["LS"], **o))
    KLL = np.einsum("xutyabcd,budt->axcy", A["LSSL"], Db["SS"], **o)
    KSS = np.einsum("xutyabcd,auct->bxdy", A["SLLS"], Db["LL"], **o)
    KLS = np.einsum("xutyabcd,buct->axdy", A["LSLS"], Db["SL"], **o)
    KSL = np.einsum("xutyabcd,audt->bxcy", A["SLSL"], Db["LS"], **o)
    return assemble({"LL": -KLL, "SS": -KSS, "LS": JLS - KLS, "SL": JSL - KSL}, N)


def gauge(basis, D):
    """The gauge term -(alpha_1 . r)(alpha_2 . r) / r^3 at the Gaunt term's
    weight (the Breit build takes half of each)."""
    T = deriv_tensor(basis, 10)
    V = r12_tensor(basis)
    for i in range(3):
        V[i, i] -= T
    return kernel_term(basis, D, V)
