"""The index and Pauli-algebra identities the four-component kernels rely on
(csrc/cqf_common.cuh, csrc/cqf_deriv.cuh, csrc/cqf_rel.cu), checked on the
host against their definitions: closed-form Cartesian exponents against the
enumeration of the component order, the multiply-high division against
integer division over the index ranges the kernels use, the incremental
Hermite index step against the compact index, and the specialised Pauli
products against 2 x 2 matrix products."""
import numpy as np


def nherm(L):
    return (L + 1) * (L + 2) * (L + 3) // 6 if L >= 0 else 0


def hidx(t, u, v):
    return nherm(t + u + v - 1) + (u + v) * (u + v + 1) // 2 + v


def cart_row(i):  # cqf_common.cuh
    return sum(i >= tri for tri in (1, 3, 6, 10, 15, 21, 28, 36))


def test_cartesian_exponents_closed_form():
    for l in range(9):
        i = 0
        for a in range(l + 1):
            for b in range(a + 1):  # the libint / CCA component order
                r = cart_row(i)
                lz = i - r * (r + 1) // 2
                assert (l - r, r - lz, lz) == (l - a, a - b, b)
                i += 1


def test_fastdiv_multiply_high():
    # FastDiv (cqf_rel.cu): m = floor((2^32 - 1) / d) + 1, q = (x m) >> 32
    rng = np.random.default_rng(7)
    for d in list(range(2, 300)) + [1024, 4096]:
        m = (0xFFFFFFFF // d + 1) & 0xFFFFFFFF
        xs = np.concatenate([np.arange(0, 4096), rng.integers(0, 1 << 20, 4096)])
        for x in xs.tolist():
            assert (x * m) >> 32 == x // d, (x, d)


def test_incremental_hermite_index():
    # hdot_v (cqf_deriv.cuh): hidx(t, u, v + k) by steps
    for t in range(9):
        for u in range(9):
            for v in range(9):
                s = t + u + v
                idx, inc = hidx(t, u, v), (s + 1) * (s + 2) // 2 + (u + v) + 2
                for k in range(9):
                    assert idx == hidx(t, u, v + k)
                    idx += inc
                    inc += s + k + 3


_SIG = [np.eye(2), np.array([[0, 1], [1, 0]]), np.array([[0, -1j], [1j, 0]]),
        np.diag([1.0, -1.0])]


def _mat(q):
    return sum(c * s for c, s in zip(q, _SIG))


def _dec(M):
    return np.array([np.trace(M @ s) / 2 for s in _SIG])


def test_pauli_right_sigma_and_real_imaginary_product():
    rng = np.random.default_rng(3)
    for _ in range(20):
        t = rng.standard_normal(4) + 1j * rng.standard_normal(4)
        s, x, y, z = t
        # qsig: t sigma_k
        want = [_dec(_mat(t) @ _SIG[k]) for k in (1, 2, 3)]
        got = [np.array([x, s, 1j * z, -1j * y]), np.array([y, -1j * z, s, 1j * x]),
               np.array([z, 1j * y, -1j * x, s])]
        for w, g in zip(want, got):
            assert np.allclose(w, g)
        # qmul_ri: p (m0 + i w.sigma), m0 and w real
        m0, w = rng.standard_normal(), rng.standard_normal(3)
        ref = _dec(_mat(t) @ _mat(np.array([m0, 1j * w[0], 1j * w[1], 1j * w[2]])))
        ps, pv = t[0], t[1:]
        got = np.concatenate([[m0 * ps + 1j * (pv @ w)], 1j * ps * w + m0 * pv - np.cross(pv, w)])
        assert np.allclose(ref, got)
