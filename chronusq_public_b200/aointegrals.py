"""Python mirror of the reference's ``AOIntegrals`` two-electron interface, on the GPU engine.

Names, argument meaning and error behaviour follow the reference:

* ``newTwoEContractDirect(X, AX, contractionList, scalingFactors)`` --
  include/aointegrals/aointegrals_contract.h:24-194 (declared include/aointegrals.h:474-480):
  ``AX[i] += 0.5*scale[i]*G_i`` with ``G = 4J[X]`` (COULOMB) or ``4K[X]`` (EXCHANGE).
  Mismatched list lengths raise ``AssertionError`` like the reference's ``assert``
  (contract.h:31-33).
* ``newTwoEContract`` -- the dispatcher (aointegrals.h:489-502); only the DIRECT
  algorithm exists here.
* ``computeSchwartz`` -- src/aointegrals/aointegrals_builders.cpp:469-517, evaluated on
  the device when the basis is uploaded.
* ``formPT`` -- SingleSlater<double>::formPT (include/singleslater/singleslater_fock.h:31-93).

Matrices are real, symmetric, nbf x nbf FP64.  They may be numpy arrays (host; the call
copies to and from the device) or CUDA torch tensors (device; the call only enqueues work on
the current torch stream).  Because X and the result are symmetric, row- and column-major
storage are interchangeable; arrays must be contiguous in one of the two.
"""
from __future__ import annotations

import ctypes
from enum import IntEnum
from typing import List, Optional, Sequence

import numpy as np

from . import _lib
from .basis import BasisSet


class ERI_CONTRACTION_TYPE(IntEnum):
    COULOMB = 0
    EXCHANGE = 1


COULOMB = ERI_CONTRACTION_TYPE.COULOMB
EXCHANGE = ERI_CONTRACTION_TYPE.EXCHANGE

PREC_FP64 = 0
PREC_MIXED = 1


def _is_torch(x):
    return type(x).__module__.startswith("torch")


def _ptr_ld(x, n):
    """(pointer, leading dimension, on_device) of a symmetric n x n matrix."""
    if _is_torch(x):
        if x.dtype.__repr__() != "torch.float64":
            raise TypeError("matrices must be float64")
        if tuple(x.shape) != (n, n):
            raise ValueError("matrix shape %s != (%d, %d)" % (tuple(x.shape), n, n))
        st = x.stride()
        if st == (n, 1):
            ld = n
        elif st == (1, n):
            ld = n
        elif st[1] == 1 and st[0] >= n:
            ld = st[0]
        elif st[0] == 1 and st[1] >= n:
            ld = st[1]
        else:
            raise ValueError("matrix must be contiguous in rows or columns")
        return x.data_ptr(), ld, 1 if x.is_cuda else -1
    a = x
    if not isinstance(a, np.ndarray) or a.dtype != np.float64:
        raise TypeError("matrices must be float64 numpy arrays or torch tensors")
    if a.shape != (n, n):
        raise ValueError("matrix shape %s != (%d, %d)" % (a.shape, n, n))
    if not (a.flags.c_contiguous or a.flags.f_contiguous):
        raise ValueError("matrix must be contiguous")
    return a.ctypes.data, n, 0


class AOIntegrals:
    """Direct two-electron contraction engine bound to one basis on one GPU."""

    def __init__(self, basis: BasisSet, device: int = 0, thresholdSchwartz: float = 1e-14):
        L = _lib.lib()
        self._L = L
        self.basisSet = basis
        self.nBasis = basis.nbasis
        ctx = ctypes.c_void_p()
        _lib.check(L.cqg_create(ctypes.byref(ctx), int(device)))
        self._ctx = ctx
        self.device = device
        Ls, pure, nprim, alpha, coef, centers = basis.flat()
        self._keep = [np.ascontiguousarray(a) for a in (Ls, pure, nprim, alpha, coef, centers)]
        i = ctypes.POINTER(ctypes.c_int)
        d = ctypes.POINTER(ctypes.c_double)
        k = self._keep
        _lib.check(L.cqg_set_basis(ctx, len(Ls), k[0].ctypes.data_as(i), k[1].ctypes.data_as(i),
                                   k[2].ctypes.data_as(i), k[3].ctypes.data_as(d), k[4].ctypes.data_as(d),
                                   k[5].ctypes.data_as(d)), ctx)
        self.thresholdSchwartz = thresholdSchwartz
        self.haveSchwartz = True

    # ------------------------------------------------------------------ settings ---
    @property
    def thresholdSchwartz(self) -> float:
        return self._thresh

    @thresholdSchwartz.setter
    def thresholdSchwartz(self, v: float):
        _lib.check(self._L.cqg_set_threshold(self._ctx, float(v)), self._ctx)
        self._thresh = float(v)

    def setPrecision(self, policy: int, fp32_cutoff: float = 0.0):
        _lib.check(self._L.cqg_set_precision(self._ctx, int(policy), float(fp32_cutoff)), self._ctx)

    def setListBudget(self, quartets: int):
        """Largest number of quartets held in the device list at once (chunking above)."""
        _lib.check(self._L.cqg_set_list_budget(self._ctx, int(quartets)), self._ctx)

    def setTiming(self, on: bool):
        _lib.check(self._L.cqg_set_timing(self._ctx, 1 if on else 0), self._ctx)

    def autotune_next(self):
        """The next contraction times every candidate launch shape of each quartet-class
        work list and keeps the fastest for the later calls of this context."""
        _lib.check(self._L.cqg_autotune_next(self._ctx), self._ctx)

    def launch_shapes(self):
        """(CTAs per SM, warps per CTA) chosen per class work list (0 = default)."""
        sch = self.schedule()
        return sch["cta_per_sm"], sch["warps_per_cta"]

    def schedule(self):
        """Per work list (lists named by ``_lib.schedule_lists()``: FP64 lists then FP32
        lists, each the quartet classes then the sibling-group lists): CTAs per SM, warps per
        CTA and quartets claimed per warp (0 = default), and the kernel form (1 =
        warp-cooperative, 0 = one quartet per thread)."""
        n = int(self._L.cqg_schedule_lists())
        out = [(ctypes.c_int * n)() for _ in range(4)]
        _lib.check(self._L.cqg_get_schedule(self._ctx, *out), self._ctx)
        return {k: list(v) for k, v in zip(("cta_per_sm", "warps_per_cta", "quartets_per_warp", "warp_form"), out)}

    def setFusion(self, tier: int):
        """0: one launch per class list; 1 / 2: the light / all per-thread classes up to
        (dd|dd) in one class-fused persistent kernel fed by a device work queue."""
        _lib.check(self._L.cqg_set_fusion(self._ctx, int(tier)), self._ctx)

    def fusion(self):
        """(tier in use, the autotuner's times in ms of tiers 0, 1, 2; zeros before tuning)."""
        t = ctypes.c_int()
        ms = (ctypes.c_double * 3)()
        _lib.check(self._L.cqg_get_fusion(self._ctx, ctypes.byref(t), ms), self._ctx)
        return int(t.value), list(ms)

    def setSiblings(self, on: bool):
        """Sibling groups on / off (default): (ss|ss), (ps|ss), (ps|ps), (pp|ss) and (ds|ss)
        get lists of entries of sibling shell pairs (same centres, angular momenta and
        exponents), evaluated from one pass over their shared primitive pairs.  The quartets,
        their count and the result are those of the pair-level lists."""
        _lib.check(self._L.cqg_set_siblings(self._ctx, 1 if on else 0), self._ctx)

    def setSiblingMin(self, cls: str, min_members: int):
        """Sibling class `cls` ("(ss|ss)"): a pair of sibling groups becomes one sibling entry
        when it holds at least `min_members` member quartets; smaller ones run as pair
        quartets."""
        k = _lib.class_names().index(cls)
        _lib.check(self._L.cqg_set_sibling_min(self._ctx, k, int(min_members)), self._ctx)

    def siblings(self) -> bool:
        v = ctypes.c_int()
        _lib.check(self._L.cqg_get_siblings(self._ctx, ctypes.byref(v)), self._ctx)
        return bool(v.value)

    def setSchedule(self, cta_per_sm=None, warps_per_cta=None, quartets_per_warp=None, warp_form=None):
        """Set the per-list schedule (sequences as :meth:`schedule` returns them, or one int
        for every list; None leaves that part unchanged)."""
        n = int(self._L.cqg_schedule_lists())

        def arr(v):
            if v is None:
                return None
            v = [int(v)] * n if isinstance(v, (int, np.integer)) else [int(x) for x in v]
            if len(v) != n:
                raise ValueError("a schedule has %d entries (FP64 lists, then FP32 lists)" % n)
            return (ctypes.c_int * n)(*v)
        _lib.check(self._L.cqg_set_schedule(self._ctx, arr(cta_per_sm), arr(warps_per_cta), arr(quartets_per_warp),
                                            arr(warp_form)), self._ctx)

    # ------------------------------------------------------------------ queries ---
    def computeSchwartz(self) -> np.ndarray:
        ns = self.basisSet.nshell
        Q = np.zeros((ns, ns), order="F")
        _lib.check(self._L.cqg_get_schwarz(self._ctx, Q.ctypes.data_as(ctypes.POINTER(ctypes.c_double))),
                   self._ctx)
        return Q

    def stats(self) -> dict:
        s = _lib.CqgStats()
        _lib.check(self._L.cqg_get_stats(self._ctx, ctypes.byref(s)), self._ctx)
        names = _lib.class_names()
        return {
            "quartets": int(s.quartets), "quartets_fp32": int(s.quartets_fp32),
            "prim_quartets": int(s.prim_quartets), "model_flops": float(s.model_flops),
            "model_flops_fp32": float(s.model_flops_fp32),
            "ms_screen": s.ms_screen, "ms_eri": s.ms_eri, "ms_total": s.ms_total,
            "launches": int(s.launches), "chunks": int(s.chunks),
            "class_quartets": {names[k]: int(s.class_quartets[k]) for k in range(len(names))},
            "class_ms": {names[k]: float(s.class_ms[k]) for k in range(len(names))},
            "ms_fused": float(s.ms_fused), "fused_tier": int(s.fused_tier),
            "list_entries": int(s.list_entries),
            "sibling_classes": [names[k] for k in range(len(names)) if (int(s.sibling_classes) >> k) & 1],
        }

    # ------------------------------------------------------------------ contraction ---
    def _stream(self, on_device):
        if on_device == 1:
            import torch
            return ctypes.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)
        return ctypes.c_void_p(0)

    def newTwoEContractDirect(self, X: Sequence, AX: List, contractionList: Sequence[int],
                              scalingFactors: Sequence[float]):
        assert len(X) == len(AX)
        assert len(X) == len(contractionList)
        assert len(X) == len(scalingFactors)
        n = self.nBasis
        nmat = len(X)
        xs = [_ptr_ld(x, n) for x in X]
        axs = [_ptr_ld(a, n) for a in AX]
        modes = {m for (_, _, m) in xs + axs}
        if -1 in modes:
            raise ValueError("torch tensors must live on the GPU")
        if len(modes) != 1:
            raise ValueError("mixing host and device matrices in one call is not supported")
        on_device = modes.pop()
        lds = {ld for (_, ld, _) in xs + axs}
        if len(lds) != 1:
            raise ValueError("all matrices in one call must share a leading dimension")
        ld = lds.pop()
        if on_device == 0:
            for a in AX:
                if not a.flags.writeable:
                    raise ValueError("AX must be writeable")
        Xp = (ctypes.c_void_p * nmat)(*[p for (p, _, _) in xs])
        Ap = (ctypes.c_void_p * nmat)(*[p for (p, _, _) in axs])
        t = (ctypes.c_int * nmat)(*[int(c) for c in contractionList])
        s = (ctypes.c_double * nmat)(*[float(v) for v in scalingFactors])
        st = self._L.cqg_twoe_contract_direct(self._ctx, nmat, Xp, Ap, t, s, ld, on_device,
                                              self._stream(on_device))
        _lib.check(st, self._ctx)

    def newTwoEContract(self, X, AX, contractionList, scalingFactors):
        self.newTwoEContractDirect(X, AX, contractionList, scalingFactors)

    def formPT(self, Ps, Pz=None, xHF: float = -0.5, PTs=None, PTz=None):
        """SingleSlater::formPT: returns (PTs, PTz); RHF when ``Pz`` is None."""
        n = self.nBasis
        is_rhf = Pz is None
        if PTs is None:
            PTs = self._like(Ps)
        if not is_rhf and PTz is None:
            PTz = self._like(Pz)
        ps, ld, mode = _ptr_ld(Ps, n)
        pts, _, _ = _ptr_ld(PTs, n)
        pz = ptz = None
        if not is_rhf:
            pz, _, _ = _ptr_ld(Pz, n)
            ptz, _, _ = _ptr_ld(PTz, n)
        st = self._L.cqg_form_pt(self._ctx, 1 if is_rhf else 0, float(xHF), ps, pz, pts, ptz, ld, mode,
                                 self._stream(mode))
        _lib.check(st, self._ctx)
        return PTs, (None if is_rhf else PTz)

    def computeAOOneE(self, charges, coords_bohr, device_out: bool = False):
        """Overlap, kinetic and nuclear-attraction matrices (AOIntegrals::computeAOOneE,
        src/aointegrals/aointegrals_builders.cpp:337-467), evaluated on the GPU.
        Returns (S, T, V) as CUDA torch tensors when ``device_out`` else numpy arrays."""
        n = self.nBasis
        Z = np.ascontiguousarray(charges, dtype=np.float64)
        R = np.ascontiguousarray(coords_bohr, dtype=np.float64).reshape(-1, 3)
        d = ctypes.POINTER(ctypes.c_double)
        if device_out:
            import torch
            S, T, V = (torch.zeros((n, n), dtype=torch.float64, device="cuda:%d" % self.device) for _ in range(3))
            ptrs = [ctypes.c_void_p(x.data_ptr()) for x in (S, T, V)]
            mode = 1
        else:
            S, T, V = (np.zeros((n, n), order="F") for _ in range(3))
            ptrs = [ctypes.c_void_p(x.ctypes.data) for x in (S, T, V)]
            mode = 0
        st = self._L.cqg_one_e(self._ctx, len(Z), Z.ctypes.data_as(d), R.ctypes.data_as(d), ptrs[0], ptrs[1],
                               ptrs[2], n, mode, self._stream(mode))
        _lib.check(st, self._ctx)
        return S, T, V

    def computeDipole(self, origin=(0.0, 0.0, 0.0), device_out: bool = False):
        """Electric dipole integrals <mu| r_k - origin_k |nu>, k = x, y, z (the first
        electric multipoles of AOIntegrals::computeAOOneE, split per component in
        AOIntegrals::breakUpMultipole, src/aointegrals/aointegrals_builders.cpp:640-650),
        evaluated on the GPU.  Returns a (3, n, n) CUDA torch tensor when ``device_out``,
        else a numpy array; each matrix is symmetric."""
        n = self.nBasis
        O_ = np.ascontiguousarray(origin, dtype=np.float64)
        if device_out:
            import torch
            D = torch.zeros((3, n, n), dtype=torch.float64, device="cuda:%d" % self.device)
            ptr, mode = ctypes.c_void_p(D.data_ptr()), 1
        else:
            D = np.zeros((3, n, n))
            ptr, mode = ctypes.c_void_p(D.ctypes.data), 0
        st = self._L.cqg_dipole(self._ctx, O_.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), ptr, n, mode,
                                self._stream(mode))
        _lib.check(st, self._ctx)
        return D

    @staticmethod
    def _like(x):
        if _is_torch(x):
            import torch
            return torch.zeros_like(x)
        return np.zeros(x.shape, order="F")

    def close(self):
        if getattr(self, "_ctx", None):
            self._L.cqg_destroy(self._ctx)
            self._ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def probe_fma_peak(fp64: bool = True, ms: float = 50.0, device: int = 0) -> float:
    out = ctypes.c_double()
    _lib.check(_lib.lib().cqg_probe_fma_peak(device, 1 if fp64 else 0, ms, ctypes.byref(out)))
    return out.value
