"""Basis sets and molecules on the host side of the direct Fock build.

This mirrors the input layer ChronusQ feeds into its direct J/K contraction:

* ``.gbs`` (Gaussian94) parsing as in ``src/basisset/reference.cxx:126-300``:
  ``SP`` shells split into an S and a P shell, S and P shells are Cartesian and
  l >= 2 shells are spherical (``reference.cxx:267-272``), shells are placed on
  atoms in atom order (``reference.cxx:302-330``).
* Contraction coefficients are renormalised the way ``libint2::Shell`` does it
  (the object ChronusQ builds for every shell): every primitive carries the
  normalisation of its x^l Cartesian component and the contracted x^l function
  has unit norm.  Spherical functions built from those Cartesians with the
  real-solid-harmonic coefficients of Helgaker, Jorgensen & Olsen (eq. 6.4.47)
  are then unit-normalised.
* AO order: shells in order, Cartesian components in lexicographic order
  (x^l first), spherical components m = -l..l.
* Coordinates in Angstrom are converted with ``AngPerBohr = 0.52917721092``
  (``src/cxxapi/input/molopts.cxx:179-182``, ``include/physcon.hpp:32``).
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field
from typing import Dict, List, Sequence, Tuple

import numpy as np

ANG_PER_BOHR = 0.52917721092
L_OF = {"S": 0, "P": 1, "D": 2, "F": 3, "G": 4, "H": 5, "I": 6, "K": 7}
BASIS_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "basis")

_SYMBOLS = (
    "X H He Li Be B C N O F Ne Na Mg Al Si P S Cl Ar K Ca Sc Ti V Cr Mn Fe Co "
    "Ni Cu Zn Ga Ge As Se Br Kr Rb Sr Y Zr Nb Mo Tc Ru Rh Pd Ag Cd In Sn Sb Te "
    "I Xe Cs Ba La Ce Pr Nd Pm Sm Eu Gd Tb Dy Ho Er Tm Yb Lu Hf Ta W Re Os Ir "
    "Pt Au Hg Tl Pb Bi Po At Rn Fr Ra Ac Th Pa U Np Pu Am Cm Bk Cf Es Fm Md No "
    "Lr Rf Db Sg Bh Hs Mt Ds Rg Cn Nh Fl Mc Lv Ts Og").split()
Z_OF = {s.upper(): z for z, s in enumerate(_SYMBOLS)}


def atomic_number(sym: str) -> int:
    return Z_OF[sym.strip().upper()]


# Mass number of each element's default isotope (the most abundant stable
# one, as the reference's defaultIsotope map in include/atom.hpp), Z = 1..54
# without Tc; used for the finite-nucleus charge radius.
_MASS_NUMBER = dict(zip(range(1, 55), (
    1, 4, 7, 9, 11, 12, 14, 16, 19, 20, 23, 24, 27, 28, 31, 32, 35, 40, 39, 40,
    45, 48, 51, 52, 55, 56, 59, 58, 63, 64, 69, 74, 75, 80, 79, 84, 85, 88, 89,
    90, 93, 98, None, 102, 103, 106, 107, 114, 115, 120, 121, 130, 127, 132)))


def finite_nucleus_exponent(mass_number: int) -> float:
    """Exponent zeta of the Gaussian nuclear charge Z (zeta/pi)^{3/2}
    exp(-zeta r^2) with root-mean-square radius 0.836 A^{1/3} + 0.570 fm:
    zeta = 3 / (2 r^2), r in Bohr (Molecule::computeCDist,
    src/molecule/molecule.cxx:197-226)."""
    r = (0.836 * mass_number ** (1.0 / 3.0) + 0.570) * 1e-5 / ANG_PER_BOHR
    return 1.5 / (r * r)


def n_cart(l: int) -> int:
    return (l + 1) * (l + 2) // 2


def n_sph(l: int) -> int:
    return 2 * l + 1


def cart_list(l: int) -> List[Tuple[int, int, int]]:
    """Cartesian exponents (lx, ly, lz) of a shell in libint/CCA order."""
    out = []
    for i in range(l + 1):
        lx = l - i
        for j in range(i + 1):
            out.append((lx, i - j, j))
    return out


def _dfact(n: int) -> float:
    """(n)!! with (-1)!! = 0!! = 1."""
    r = 1.0
    while n > 1:
        r *= n
        n -= 2
    return r


def normalize_contraction(l: int, alpha: Sequence[float],
                          coef: Sequence[float]) -> np.ndarray:
    """libint2-convention normalised coefficients of one contracted shell.

    Primitive factor N(a) = sqrt((2a/pi)^(3/2) (4a)^l / (2l-1)!!), followed by
    a rescale that makes the contracted x^l function unit-normalised.
    """
    a = np.asarray(alpha, dtype=np.float64)
    c = np.asarray(coef, dtype=np.float64)
    df = _dfact(2 * l - 1)
    prim = np.sqrt((2.0 * a / math.pi) ** 1.5 * (4.0 * a) ** l / df)
    c = c * prim
    ab = a[:, None] + a[None, :]
    s = df / (2.0 * ab) ** l * (math.pi / ab) ** 1.5
    norm = float(c @ s @ c)
    return c / math.sqrt(norm)


def solid_harmonic_matrix(l: int) -> np.ndarray:
    """T[i_cart, m] mapping Cartesian components to real solid harmonics.

    Helgaker, Jorgensen & Olsen, *Molecular Electronic-Structure Theory*,
    eqs. 6.4.47-6.4.50; columns ordered m = -l..l.
    """
    carts = cart_list(l)
    idx = {c: i for i, c in enumerate(carts)}
    T = np.zeros((len(carts), 2 * l + 1))
    for m in range(-l, l + 1):
        am = abs(m)
        vm = 0.0 if m >= 0 else 0.5
        N = 1.0 / (2 ** am * math.factorial(l)) * math.sqrt(
            2.0 * math.factorial(l + am) * math.factorial(l - am)
            / (2.0 if m == 0 else 1.0))
        for t in range((l - am) // 2 + 1):
            for u in range(t + 1):
                v = vm
                vmax = math.floor(am / 2.0 - vm) + vm
                while v <= vmax + 1e-9:
                    C = ((-1) ** int(round(t + v - vm)) * 0.25 ** t
                         * math.comb(l, t) * math.comb(l - t, am + t)
                         * math.comb(t, u) * math.comb(am, int(round(2 * v))))
                    lx = int(round(2 * t + am - 2 * (u + v)))
                    ly = int(round(2 * (u + v)))
                    lz = l - 2 * t - am
                    T[idx[(lx, ly, lz)], m + l] += N * C
                    v += 1.0
    return T


@dataclass
class Shell:
    l: int
    pure: bool
    alpha: np.ndarray
    coef_raw: np.ndarray          # coefficients as written in the .gbs file
    origin: np.ndarray            # Bohr
    atom: int = -1
    coef: np.ndarray = field(init=False)

    def __post_init__(self):
        self.alpha = np.asarray(self.alpha, dtype=np.float64)
        self.coef_raw = np.asarray(self.coef_raw, dtype=np.float64)
        self.origin = np.asarray(self.origin, dtype=np.float64)
        self.coef = normalize_contraction(self.l, self.alpha, self.coef_raw)

    @property
    def size(self) -> int:
        return n_sph(self.l) if self.pure else n_cart(self.l)

    @property
    def ncart(self) -> int:
        return n_cart(self.l)

    @property
    def nprim(self) -> int:
        return len(self.alpha)


def parse_gbs(text: str, force_cart: bool = False
              ) -> Dict[int, List[Tuple[int, bool, List[float], List[float]]]]:
    """Parse a Gaussian94 basis file into {Z: [(l, pure, exps, coefs), ...]}."""
    lines = text.splitlines()
    out: Dict[int, list] = {}
    i = 0
    cur = None
    n = len(lines)
    while i < n:
        s = lines[i].strip()
        i += 1
        if not s or s.startswith("!"):
            continue
        if s == "****":
            cur = None
            continue
        toks = s.split()
        if cur is None:
            try:
                z = atomic_number(toks[0])
            except KeyError:
                continue
            cur = out.setdefault(z, [])
            out[z] = cur = []
            continue
        sym = toks[0].upper()
        nprim = int(toks[1])
        exps, c1, c2 = [], [], []
        for _ in range(nprim):
            pt = lines[i].replace("D", "E").replace("d", "e").split()
            i += 1
            exps.append(float(pt[0]))
            c1.append(float(pt[1]))
            if sym == "SP":
                c2.append(float(pt[2]))
        if sym == "SP":
            cur.append((0, False, exps, c1))
            cur.append((1, False, exps, c2))
        else:
            l = L_OF[sym]
            pure = (l > 1) and not force_cart
            cur.append((l, pure, exps, c1))
    return out


def load_gbs(name: str, force_cart: bool = False):
    path = name if os.path.exists(name) else os.path.join(
        BASIS_DIR, name.lower() + ".gbs")
    with open(path) as f:
        return parse_gbs(f.read(), force_cart)


@dataclass
class Molecule:
    Z: np.ndarray          # (natom,) int
    xyz: np.ndarray        # (natom, 3) Bohr

    @classmethod
    def from_angstrom(cls, atoms: Sequence[Tuple[str, float, float, float]]):
        Z = np.array([atomic_number(a[0]) for a in atoms], dtype=np.int64)
        xyz = np.array([[a[1], a[2], a[3]] for a in atoms],
                       dtype=np.float64) / ANG_PER_BOHR
        return cls(Z, xyz)

    @property
    def natom(self) -> int:
        return len(self.Z)

    def nuclei(self, finite: bool = False, mass_numbers=None) -> np.ndarray:
        """(natom, 5) rows {Z, x, y, z (Bohr), zeta}: zeta = 0 for point
        charges, else the Gaussian finite-nucleus exponent of each atom's
        default isotope (or of ``mass_numbers``)."""
        out = np.zeros((self.natom, 5))
        out[:, 0] = self.Z
        out[:, 1:4] = self.xyz
        if finite:
            for i, z in enumerate(self.Z):
                A = mass_numbers[i] if mass_numbers is not None else _MASS_NUMBER.get(int(z))
                if A is None:
                    raise KeyError("no default isotope for Z = %d; pass mass_numbers" % z)
                out[i, 4] = finite_nucleus_exponent(A)
        return out

    def nuclear_repulsion(self) -> float:
        e = 0.0
        for i in range(self.natom):
            for j in range(i):
                e += self.Z[i] * self.Z[j] / np.linalg.norm(
                    self.xyz[i] - self.xyz[j])
        return float(e)


class BasisSet:
    """Ordered list of shells for a molecule (``BasisSet::update``,
    ``src/basisset/basisset.cxx:98-191``)."""

    def __init__(self, shells: List[Shell]):
        self.shells = shells
        self.nshell = len(shells)
        self.sizes = np.array([s.size for s in shells], dtype=np.int64)
        self.offsets = np.concatenate([[0], np.cumsum(self.sizes)[:-1]]
                                      ).astype(np.int64)
        self.nbasis = int(self.sizes.sum())
        self.ncart_sizes = np.array([s.ncart for s in shells], dtype=np.int64)
        self.cart_offsets = np.concatenate(
            [[0], np.cumsum(self.ncart_sizes)[:-1]]).astype(np.int64)
        self.ncart = int(self.ncart_sizes.sum())
        self.max_l = max(s.l for s in shells)
        self.max_prim = max(s.nprim for s in shells)

    @classmethod
    def build(cls, mol: Molecule, name, force_cart: bool = False,
              uncontract: bool = False) -> "BasisSet":
        """Shells for ``mol`` from a named basis (or a pre-parsed dict)."""
        ref = load_gbs(name, force_cart) if isinstance(name, str) else name
        shells = []
        for ia in range(mol.natom):
            z = int(mol.Z[ia])
            if z not in ref:
                raise ValueError("Cannot find Z=%d in basis definition" % z)
            recs = ref[z]
            if uncontract:
                recs = _uncontract(recs)
            for (l, pure, exps, coefs) in recs:
                shells.append(Shell(l, pure, exps, coefs, mol.xyz[ia], ia))
        return cls(shells)

    def cart_to_sph(self) -> np.ndarray:
        """Block-diagonal (ncart x nbasis) transform from Cartesian AOs."""
        T = np.zeros((self.ncart, self.nbasis))
        for s, sh in enumerate(self.shells):
            c0, f0 = self.cart_offsets[s], self.offsets[s]
            if sh.pure:
                T[c0:c0 + sh.ncart, f0:f0 + sh.size] = solid_harmonic_matrix(
                    sh.l)
            else:
                T[c0:c0 + sh.ncart, f0:f0 + sh.size] = np.eye(sh.ncart)
        return T

    # flat arrays consumed by the C ABI and by the oracle
    def flat(self):
        l = np.array([s.l for s in self.shells], dtype=np.int32)
        pure = np.array([1 if s.pure else 0 for s in self.shells],
                        dtype=np.int32)
        nprim = np.array([s.nprim for s in self.shells], dtype=np.int32)
        alpha = np.concatenate([s.alpha for s in self.shells])
        coef = np.concatenate([s.coef for s in self.shells])
        coef_raw = np.concatenate([s.coef_raw for s in self.shells])
        origin = np.stack([s.origin for s in self.shells]).astype(np.float64)
        return dict(l=l, pure=pure, nprim=nprim, alpha=alpha, coef=coef,
                    coef_raw=coef_raw, origin=np.ascontiguousarray(origin))


def _uncontract(recs):
    """Unique primitives per angular momentum, as ``BasisSet::uncontractBasis``
    (``src/basisset/basisset.cxx:323-343``) produces them: one primitive shell
    per distinct exponent, in order of first appearance within each l."""
    out = []
    seen = {}
    for (l, pure, exps, _c) in recs:
        for e in exps:
            key = (l, e)
            if key in seen:
                continue
            seen[key] = True
            out.append((l, pure, [e], [1.0]))
    return out
