"""ctypes front end of the C oracle, plus an independent solid-harmonic construction.

TEST INFRASTRUCTURE ONLY: imported by tests, the smoke check and the CPU-baseline leg of
the benchmark, as the checker.  Nothing in the product imports it.

Functions mirror the reference entry points they restate:

* :func:`twoe_contract_direct`  -- AOIntegrals::newTwoEContractDirect
  (include/aointegrals/aointegrals_contract.h:24-194)
* :func:`schwarz`               -- AOIntegrals::computeSchwartz
  (src/aointegrals/aointegrals_builders.cpp:469-517)
* :func:`shblk_norm`            -- BasisSet::computeShBlkNorm (include/basisset.h:495-509)
* :func:`one_e`                 -- S, T, V from OneEDriver (builders.cpp:27-133)
* :func:`form_pt`               -- SingleSlater::formPT list construction
  (include/singleslater/singleslater_fock.h:31-93)
"""
from __future__ import annotations

import ctypes
import math
import os
import subprocess
from typing import List, Sequence

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libcqoracle.so")
_lib = None

COULOMB, EXCHANGE = 0, 1


def build():
    subprocess.check_call(["make", "-s", "-C", _HERE])


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = ctypes.CDLL(_LIB_PATH)
        d = ctypes.POINTER(ctypes.c_double)
        i = ctypes.POINTER(ctypes.c_int)
        pp = ctypes.POINTER(ctypes.c_void_p)
        _lib.oracle_boys.argtypes = [ctypes.c_int, ctypes.c_double, d]
        _lib.oracle_eri_quartet.argtypes = [ctypes.c_int, i, i, i, d, d, d, pp,
                                            ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, d]
        _lib.oracle_eri_full.argtypes = [ctypes.c_int, i, i, i, d, d, d, pp, d]
        _lib.oracle_schwarz.argtypes = [ctypes.c_int, i, i, i, d, d, d, pp, d]
        _lib.oracle_shblk_norm.argtypes = [ctypes.c_int, i, i, d, ctypes.c_int, d]
        _lib.oracle_twoe_contract_direct.argtypes = [
            ctypes.c_int, i, i, i, d, d, d, pp, d, ctypes.c_double,
            ctypes.c_int, pp, pp, i, d, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_longlong),
            ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        _lib.oracle_twoe_contract_direct.restype = ctypes.c_longlong
        _lib.oracle_one_e.argtypes = [ctypes.c_int, i, i, i, d, d, d, pp, ctypes.c_int, d, d, d, d, d]
        _lib.oracle_dipole.argtypes = [ctypes.c_int, i, i, i, d, d, d, pp, d, d, d, d]
    return _lib


# ---------------------------------------------------------------- solid harmonics ---
def _cart_list(l):
    out = []
    for i in range(l + 1):
        for j in range(i + 1):
            out.append((l - i, i - j, j))
    return out


def _dfact(n):
    r = 1.0
    while n > 1:
        r *= n
        n -= 2
    return r


def oracle_solid_harmonics(l: int) -> np.ndarray:
    """Unit-normalised real solid harmonics in x^l-normalised Cartesians, rows m=-l..l.

    Built independently of the package: r^l * P_l^|m|(cos t) * {cos, sin}(|m| phi) with
    the associated Legendre function taken WITHOUT the Condon-Shortley phase, sampled at
    random points and fitted to the Cartesian monomials by least squares, then scaled to
    unit self-overlap with Gaussian moment ratios.
    """
    from scipy.special import lpmv
    carts = _cart_list(l)
    rng = np.random.default_rng(1234 + l)
    npts = 8 * len(carts) + 16
    xyz = rng.normal(size=(npts, 3))
    r = np.linalg.norm(xyz, axis=1)
    ct = xyz[:, 2] / r
    phi = np.arctan2(xyz[:, 1], xyz[:, 0])
    A = np.stack([xyz[:, 0] ** a * xyz[:, 1] ** b * xyz[:, 2] ** c for (a, b, c) in carts], axis=1)
    gram = np.zeros((len(carts), len(carts)))
    for i, (ax, ay, az) in enumerate(carts):
        for j, (bx, by, bz) in enumerate(carts):
            sx, sy, sz = ax + bx, ay + by, az + bz
            if sx % 2 == 0 and sy % 2 == 0 and sz % 2 == 0:
                gram[i, j] = _dfact(sx - 1) * _dfact(sy - 1) * _dfact(sz - 1) / _dfact(2 * l - 1)
    out = np.zeros((2 * l + 1, len(carts)))
    for m in range(-l, l + 1):
        am = abs(m)
        plm = lpmv(am, l, ct) * (-1.0) ** am      # remove Condon-Shortley phase
        ang = np.cos(am * phi) if m >= 0 else np.sin(am * phi)
        y = r ** l * plm * ang
        c, *_ = np.linalg.lstsq(A, y, rcond=None)
        c[np.abs(c) < 1e-12 * np.abs(c).max()] = 0.0
        c /= math.sqrt(c @ gram @ c)
        out[m + l] = c
    return out


class OracleBasis:
    """Flat shell arrays + solid-harmonic matrices kept alive for ctypes calls."""

    def __init__(self, L, pure, nprim, alpha, coef, centers):
        self.L = np.ascontiguousarray(L, dtype=np.int32)
        self.pure = np.ascontiguousarray(pure, dtype=np.int32)
        self.nprim = np.ascontiguousarray(nprim, dtype=np.int32)
        self.alpha = np.ascontiguousarray(alpha, dtype=np.float64)
        self.coef = np.ascontiguousarray(coef, dtype=np.float64)
        self.centers = np.ascontiguousarray(centers, dtype=np.float64).reshape(-1, 3)
        self.nshell = len(self.L)
        self.sizes = np.array([2 * l + 1 if p else (l + 1) * (l + 2) // 2
                               for l, p in zip(self.L, self.pure)], dtype=np.int64)
        self.offsets = np.concatenate([[0], np.cumsum(self.sizes)[:-1]]).astype(np.int64)
        self.nbf = int(self.sizes.sum())
        self._sph = [np.ascontiguousarray(oracle_solid_harmonics(l)) for l in range(5)]
        self._sph_ptrs = (ctypes.c_void_p * 5)(*[s.ctypes.data for s in self._sph])

    @classmethod
    def from_basis(cls, bs):
        return cls(*bs.flat())

    def args(self):
        d = ctypes.POINTER(ctypes.c_double)
        i = ctypes.POINTER(ctypes.c_int)
        return (self.nshell, self.L.ctypes.data_as(i), self.pure.ctypes.data_as(i),
                self.nprim.ctypes.data_as(i), self.alpha.ctypes.data_as(d),
                self.coef.ctypes.data_as(d), self.centers.ctypes.data_as(d),
                ctypes.cast(self._sph_ptrs, ctypes.POINTER(ctypes.c_void_p)))


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def boys(mmax: int, T: float) -> np.ndarray:
    out = np.zeros(mmax + 1)
    lib().oracle_boys(mmax, T, _dp(out))
    return out


def eri_quartet(ob: OracleBasis, s1, s2, s3, s4) -> np.ndarray:
    n = [int(ob.sizes[s]) for s in (s1, s2, s3, s4)]
    out = np.zeros(int(np.prod(n)))
    rc = lib().oracle_eri_quartet(*ob.args(), s1, s2, s3, s4, _dp(out))
    if rc != 0:
        raise ValueError("oracle_eri_quartet failed")
    return out.reshape(n)


def eri_full(ob: OracleBasis) -> np.ndarray:
    n = ob.nbf
    out = np.zeros(n ** 4)
    lib().oracle_eri_full(*ob.args(), _dp(out))
    return out.reshape(n, n, n, n)


def schwarz(ob: OracleBasis) -> np.ndarray:
    Q = np.zeros((ob.nshell, ob.nshell), order="F")
    lib().oracle_schwarz(*ob.args(), _dp(Q))
    return Q


def shblk_norm(ob: OracleBasis, X: np.ndarray) -> np.ndarray:
    Xf = np.asfortranarray(X, dtype=np.float64)
    out = np.zeros((ob.nshell, ob.nshell), order="F")
    i = ctypes.POINTER(ctypes.c_int)
    lib().oracle_shblk_norm(ob.nshell, ob.L.ctypes.data_as(i), ob.pure.ctypes.data_as(i),
                            _dp(Xf), Xf.shape[0], _dp(out))
    return out


def twoe_contract_direct(ob: OracleBasis, X: Sequence[np.ndarray], AX: List[np.ndarray],
                         types: Sequence[int], scale: Sequence[float], thresh: float = 1e-14,
                         Q: np.ndarray = None, nthreads: int = 0, per_class: bool = False,
                         s1_range=(-1, -1), s1_residue=(1, 0)):
    """AX[i] += 0.5*scale[i]*G_i (in place, Fortran-ordered arrays).  Returns the number of
    screened quartets (and the per-(la,lb,lc,ld) histogram when ``per_class``).
    ``s1_range`` restricts the outermost shell index to [lo, hi); ``s1_residue = (m, r)``
    keeps only s1 with s1 % m == r (the m residue classes partition the loop)."""
    if Q is None:
        Q = schwarz(ob)
    Q = np.asfortranarray(Q)
    nmat = len(X)
    Xs = [np.asfortranarray(x, dtype=np.float64) for x in X]
    for a in AX:
        if not (a.flags.f_contiguous and a.dtype == np.float64):
            raise ValueError("AX must be Fortran-ordered float64 (accumulated in place)")
    xp = (ctypes.c_void_p * nmat)(*[x.ctypes.data for x in Xs])
    ap = (ctypes.c_void_p * nmat)(*[a.ctypes.data for a in AX])
    t = np.ascontiguousarray(types, dtype=np.int32)
    s = np.ascontiguousarray(scale, dtype=np.float64)
    hist = np.zeros(625, dtype=np.int64)
    n = lib().oracle_twoe_contract_direct(
        *ob.args(), _dp(Q), float(thresh), nmat,
        ctypes.cast(xp, ctypes.POINTER(ctypes.c_void_p)), ctypes.cast(ap, ctypes.POINTER(ctypes.c_void_p)),
        t.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), _dp(s), Xs[0].shape[0], int(nthreads),
        hist.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong)) if per_class else None,
        int(s1_range[0]), int(s1_range[1]), int(s1_residue[0]), int(s1_residue[1]))
    if per_class:
        return int(n), hist.reshape(5, 5, 5, 5)
    return int(n)


def one_e(ob: OracleBasis, charges: Sequence[float], coords: np.ndarray):
    n = ob.nbf
    S = np.zeros((n, n), order="F")
    T = np.zeros((n, n), order="F")
    V = np.zeros((n, n), order="F")
    Z = np.ascontiguousarray(charges, dtype=np.float64)
    R = np.ascontiguousarray(coords, dtype=np.float64).reshape(-1, 3)
    lib().oracle_one_e(*ob.args(), len(Z), _dp(Z), _dp(R), _dp(S), _dp(T), _dp(V))
    return S, T, V


def dipole(ob: OracleBasis, origin=(0.0, 0.0, 0.0)):
    """Electric dipole integrals <a| r - origin |b> (x, y, z), each nbf x nbf."""
    n = ob.nbf
    D = [np.zeros((n, n), order="F") for _ in range(3)]
    O_ = np.ascontiguousarray(origin, dtype=np.float64)
    lib().oracle_dipole(*ob.args(), _dp(O_), *[_dp(d) for d in D])
    return D


def form_pt(ob: OracleBasis, Ps: np.ndarray, Pz: np.ndarray = None, xHF: float = -0.5,
            thresh: float = 1e-14, Q: np.ndarray = None, nthreads: int = 0):
    """SingleSlater::formPT (singleslater_fock.h:31-93): RHF lists [(Ps,COULOMB,1),
    (Ps,EXCHANGE,xHF)] into PTs; UHF adds (Pz,EXCHANGE,xHF) into PTz.  PT zeroed first."""
    n = ob.nbf
    PTs = np.zeros((n, n), order="F")
    if Pz is None:
        cnt = twoe_contract_direct(ob, [Ps, Ps], [PTs, PTs], [COULOMB, EXCHANGE], [1.0, xHF],
                                   thresh, Q, nthreads)
        return PTs, None, cnt
    PTz = np.zeros((n, n), order="F")
    cnt = twoe_contract_direct(ob, [Ps, Ps, Pz], [PTs, PTs, PTz], [COULOMB, EXCHANGE, EXCHANGE],
                               [1.0, xHF, xHF], thresh, Q, nthreads)
    return PTs, PTz, cnt
