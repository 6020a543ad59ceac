"""Gaussian basis sets with the reference's parsing and normalisation conventions.

Conventions restated from the reference (paths within the ChronusQ tree):

* ``.gbs`` records: ``!`` comment lines and empty lines skipped, records separated by
  ``****``; the first line of a record names the element; each shell line is
  ``<sym> <nprim> <scale>`` followed by ``nprim`` lines ``exponent coef [coefP]``; the
  scale column is ignored; ``SP`` shells become an S shell followed by a P shell
  (src/basisset/basisset_read.cpp:200-262).
* Numbers are read with ``std::stod``, which stops at the first character that cannot
  continue a decimal literal, so a Fortran ``0.45D-03`` reads as ``0.45``
  (basisset_read.cpp:231-234).  :func:`_stod` reproduces that.
* Shells with L > 1 are spherical (real solid harmonics, m = -l..l) unless
  ``force_cart``; s and p are Cartesian (basisset_read.cpp:250-251).
* Cartesian component order x^l, x^(l-1)y, x^(l-1)z, ... (include/basisset.h:79-86).
* Contraction coefficients are normalised as a Libint2 ``Shell`` does (primitive
  normalisation of the axis-aligned x^l component, then unit self-overlap of the
  contracted function) and again by ``renormShells`` (src/basisset/basisset_misc.cpp:
  95-111), which divides by the square root of the first component's self-overlap.
* Shells are placed atom by atom in input order, in record order within an element
  (src/basisset/basisset_gen.cpp:30-79); ``mapSh2Bf`` is the running offset
  (src/basisset/basisset_map.cpp:29-40).
"""
from __future__ import annotations

import math
import os
import re
from dataclasses import dataclass, field
from typing import Dict, List, Sequence, Tuple

import numpy as np

ELEMENTS = ["X", "H", "He", "Li", "Be", "B", "C", "N", "O", "F", "Ne",
            "Na", "Mg", "Al", "Si", "P", "S", "Cl", "Ar"]
SYMBOL_TO_Z = {s.upper(): z for z, s in enumerate(ELEMENTS) if z > 0}
L_SYMBOLS = {"S": 0, "P": 1, "D": 2, "F": 3, "G": 4, "H": 5, "I": 6}

BASIS_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "basis_data")
BASIS_ALIASES = {
    "sto-3g": "sto3g.gbs", "sto3g": "sto3g.gbs",
    "6-31g": "6-31g.gbs",
    "6-31g*": "6-31g*.gbs", "6-31g(d)": "6-31g*.gbs",
    "cc-pvdz": "cc-pvdz.gbs", "cc-pvtz": "cc-pvtz.gbs",
}

_STOD_RE = re.compile(r"\s*[+-]?(\d+\.?\d*([eE][+-]?\d+)?|\.\d+([eE][+-]?\d+)?)")


def _stod(tok: str) -> float:
    """Longest decimal prefix of ``tok`` as a float, like C++ ``std::stod``."""
    m = _STOD_RE.match(tok)
    if not m:
        raise ValueError("not a number: %r" % tok)
    return float(m.group(0))


def ncart(l: int) -> int:
    return (l + 1) * (l + 2) // 2


def nsph(l: int) -> int:
    return 2 * l + 1


def cart_list(l: int) -> List[Tuple[int, int, int]]:
    """Cartesian exponents of angular momentum ``l`` in the reference order."""
    out = []
    for i in range(l + 1):
        lx = l - i
        for j in range(i + 1):
            out.append((lx, i - j, j))
    return out


def _dfact(n: int) -> float:
    """(n)!! with (-1)!! = 1."""
    r = 1.0
    while n > 1:
        r *= n
        n -= 2
    return r


def solid_harmonic_matrix(l: int) -> np.ndarray:
    """Coefficients C[m+l, k] of unit-normalised real solid harmonics in Cartesians.

    Column k runs over :func:`cart_list` (each Cartesian carrying the x^l primitive
    normalisation).  Rows are m = -l..l.  The polynomial is the real regular solid
    harmonic of Helgaker, Jorgensen & Olsen, *Molecular Electronic-Structure Theory*
    eqs. (6.4.47)-(6.4.50) (no Condon-Shortley phase); each row is then scaled to unit
    self-overlap using Gaussian moment ratios (2i-1)!!(2j-1)!!(2k-1)!!/(2l-1)!!.
    """
    carts = cart_list(l)
    idx = {c: k for k, c in enumerate(carts)}
    mat = np.zeros((2 * l + 1, len(carts)))
    for m in range(-l, l + 1):
        am = abs(m)
        vm = 0.0 if m >= 0 else 0.5
        row = np.zeros(len(carts))
        for t in range((l - am) // 2 + 1):
            for u in range(t + 1):
                nv = int(math.floor(am / 2.0 - vm))
                for iv in range(nv + 1):
                    v = iv + vm
                    two_v = int(round(2 * v))
                    sign = (-1.0) ** int(round(t + v - vm))
                    c = (sign * 0.25 ** t * math.comb(l, t) * math.comb(l - t, am + t)
                         * math.comb(t, u) * math.comb(am, two_v))
                    px = 2 * t + am - 2 * u - two_v
                    py = 2 * u + two_v
                    pz = l - 2 * t - am
                    row[idx[(px, py, pz)]] += c
        # normalise: overlap of monomials relative to x^l, x^l
        gram = np.zeros((len(carts), len(carts)))
        for a, (ax, ay, az) in enumerate(carts):
            for b, (bx, by, bz) in enumerate(carts):
                sx, sy, sz = ax + bx, ay + by, az + bz
                if sx % 2 or sy % 2 or sz % 2:
                    continue
                gram[a, b] = (_dfact(sx - 1) * _dfact(sy - 1) * _dfact(sz - 1)
                              / _dfact(2 * l - 1))
        nrm = float(row @ gram @ row)
        mat[m + l] = row / math.sqrt(nrm)
    return mat


@dataclass
class Shell:
    """One contracted shell: angular momentum, exponents, normalised coefficients."""
    l: int
    pure: bool
    alpha: np.ndarray
    coef: np.ndarray          # normalised contraction coefficients (Libint convention)
    raw_coef: np.ndarray      # as read from the file
    origin: np.ndarray = field(default_factory=lambda: np.zeros(3))
    atom: int = -1

    @property
    def size(self) -> int:
        return nsph(self.l) if self.pure else ncart(self.l)

    @property
    def nprim(self) -> int:
        return len(self.alpha)


def normalize_contraction(l: int, alpha: Sequence[float], coef: Sequence[float]) -> np.ndarray:
    """Libint2 ``Shell::renorm`` followed by ChronusQ ``renormShells``.

    Primitive factor sqrt(2^l (2a)^(l+3/2) / (pi^(3/2) (2l-1)!!)) for the axis-aligned
    component, then one overall factor making the contracted x^l (or m=-l solid
    harmonic, which has the same self-overlap) function unit-normalised.  The
    ``renormShells`` step (basisset_misc.cpp:95-111) divides by the square root of
    that same self-overlap once more; in exact arithmetic it is 1, and it is applied
    here in the same floating-point order.
    """
    alpha = np.asarray(alpha, dtype=np.float64)
    c = np.asarray(coef, dtype=np.float64).copy()
    pi32 = math.pi ** 1.5
    df = _dfact(2 * l - 1)
    for p in range(len(alpha)):
        if alpha[p] != 0:
            ta = 2.0 * alpha[p]
            c[p] *= math.sqrt((2.0 ** l) * (ta ** (l + 1)) * math.sqrt(ta) / (pi32 * df))

    def self_overlap(cc):
        s = 0.0
        for p in range(len(alpha)):
            for q in range(p + 1):
                g = alpha[p] + alpha[q]
                s += ((1.0 if p == q else 2.0) * df * pi32 * cc[p] * cc[q]
                      / ((2.0 ** l) * (g ** (l + 1)) * math.sqrt(g)))
        return s

    c *= 1.0 / math.sqrt(self_overlap(c))
    c /= math.sqrt(self_overlap(c))
    return c


def parse_gbs(path: str, force_cart: bool = False) -> Dict[int, List[Shell]]:
    """Parse a .gbs file into {Z: [Shell (origin unset), ...]} (reference semantics)."""
    with open(path) as f:
        text = f.read().splitlines()
    records: List[List[str]] = []
    for line in text:
        if len(line) == 0:
            continue
        if line[0] == "!":
            continue
        if line == "****" or line.strip() == "****":
            records.append([])
            continue
        if not records:
            records.append([])
        records[-1].append(line)
    out: Dict[int, List[Shell]] = {}
    for rec in records:
        if not rec or not rec[0].split():
            continue
        z = SYMBOL_TO_Z[rec[0].split()[0].upper()]
        shells: List[Shell] = []
        i = 1
        while i < len(rec):
            toks = rec[i].split()
            if not toks:
                i += 1
                continue
            sym, nprim = toks[0].upper(), int(toks[1])
            exps, c1, c2 = [], [], []
            for k in range(nprim):
                t2 = rec[i + 1 + k].split()
                exps.append(_stod(t2[0]))
                c1.append(_stod(t2[1]))
                if sym == "SP":
                    c2.append(_stod(t2[2]))
            i += 1 + nprim
            if sym == "SP":
                for l, cc in ((0, c1), (1, c2)):
                    shells.append(Shell(l, False, np.array(exps), normalize_contraction(l, exps, cc),
                                        np.array(cc)))
            else:
                l = L_SYMBOLS[sym]
                pure = (l > 1) and not force_cart
                shells.append(Shell(l, pure, np.array(exps), normalize_contraction(l, exps, c1),
                                    np.array(c1)))
        out[z] = shells
    return out


def basis_path(name: str) -> str:
    if os.path.isfile(name):
        return name
    key = name.lower()
    if key in BASIS_ALIASES:
        return os.path.join(BASIS_DIR, BASIS_ALIASES[key])
    cand = os.path.join(BASIS_DIR, key if key.endswith(".gbs") else key + ".gbs")
    if os.path.isfile(cand):
        return cand
    raise FileNotFoundError("basis set %r not found" % name)


class BasisSet:
    """Shells placed on a molecule, with the reference's metadata."""

    def __init__(self, name: str, atoms: Sequence[int], coords_bohr: np.ndarray,
                 force_cart: bool = False):
        lib = parse_gbs(basis_path(name), force_cart=force_cart)
        self.name = name
        self.shells: List[Shell] = []
        coords = np.asarray(coords_bohr, dtype=np.float64).reshape(-1, 3)
        for a, z in enumerate(atoms):
            if z not in lib:
                raise ValueError("Atomic Number %d not found in current Basis Set" % z)
            for s in lib[z]:
                self.shells.append(Shell(s.l, s.pure, s.alpha.copy(), s.coef.copy(),
                                         s.raw_coef.copy(), coords[a].copy(), a))
        self.map_sh2bf = []
        n = 0
        for s in self.shells:
            self.map_sh2bf.append(n)
            n += s.size
        self.nbasis = n
        self.map_sh2bf = np.array(self.map_sh2bf, dtype=np.int64)

    @property
    def nshell(self) -> int:
        return len(self.shells)

    @property
    def max_l(self) -> int:
        return max(s.l for s in self.shells)

    @property
    def max_prim(self) -> int:
        return max(s.nprim for s in self.shells)

    def flat(self):
        """Flat arrays describing the shells (the layout the C-ABI takes)."""
        L = np.array([s.l for s in self.shells], dtype=np.int32)
        pure = np.array([1 if s.pure else 0 for s in self.shells], dtype=np.int32)
        nprim = np.array([s.nprim for s in self.shells], dtype=np.int32)
        alpha = np.concatenate([s.alpha for s in self.shells]).astype(np.float64)
        coef = np.concatenate([s.coef for s in self.shells]).astype(np.float64)
        centers = np.array([s.origin for s in self.shells], dtype=np.float64).reshape(-1, 3)
        return L, pure, nprim, alpha, coef, centers
