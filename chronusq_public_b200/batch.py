"""Many independent molecules of uneven size in one engine context.

A batch context holds the shells of every molecule; one batched contraction evaluates
the screened quartets of all active molecules in the same per-class kernels (one work
list per quartet class holds the quartets of every molecule).  Matrices are packed on
the device: molecule m's nbf_m x nbf_m matrix occupies ``offsets[m] : offsets[m] +
nbf_m**2`` of one flat FP64 tensor.  The contraction semantics per molecule are those of
newTwoEContractDirect (include/aointegrals/aointegrals_contract.h:24-194).
"""
from __future__ import annotations

import ctypes
from typing import List, Optional, Sequence

import numpy as np

from . import _lib
from .basis import BasisSet


class BatchAOIntegrals:
    def __init__(self, basis_sets: Sequence[BasisSet], device: int = 0, thresholdSchwartz: float = 1e-14):
        import torch
        self.torch = torch
        L = _lib.lib()
        self._L = L
        self.device = device
        self.basis_sets = list(basis_sets)
        ctx = ctypes.c_void_p()
        _lib.check(L.cqg_create(ctypes.byref(ctx), int(device)))
        self._ctx = ctx
        flats = [bs.flat() for bs in basis_sets]
        nsh = np.array([len(f[0]) for f in flats], dtype=np.int32)
        cat = [np.ascontiguousarray(np.concatenate([f[k] for f in flats])) for k in range(6)]
        self._keep = [nsh] + cat
        i = ctypes.POINTER(ctypes.c_int)
        d = ctypes.POINTER(ctypes.c_double)
        _lib.check(L.cqg_set_basis_batch(ctx, len(basis_sets), nsh.ctypes.data_as(i), cat[0].ctypes.data_as(i),
                                         cat[1].ctypes.data_as(i), cat[2].ctypes.data_as(i),
                                         cat[3].ctypes.data_as(d), cat[4].ctypes.data_as(d),
                                         cat[5].ctypes.data_as(d)), ctx)
        self.nmol = len(basis_sets)
        nbf = np.zeros(self.nmol, dtype=np.int32)
        off = np.zeros(self.nmol, dtype=np.int64)
        packed = ctypes.c_longlong()
        _lib.check(L.cqg_get_batch_layout(ctx, nbf.ctypes.data_as(i), off.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong)),
                                          ctypes.byref(packed)), ctx)
        self.nbf = nbf.tolist()
        self.offsets = off.tolist()
        self.packed = int(packed.value)
        _lib.check(L.cqg_set_threshold(ctx, float(thresholdSchwartz)), ctx)

    # ------------------------------------------------------------------ layout ---
    def zeros(self):
        return self.torch.zeros(self.packed, dtype=self.torch.float64, device="cuda:%d" % self.device)

    def view(self, packed, m):
        n, o = self.nbf[m], self.offsets[m]
        return packed[o:o + n * n].view(n, n)

    def pack(self, mats: Sequence, out=None):
        out = self.zeros() if out is None else out
        for m, a in enumerate(mats):
            self.view(out, m).copy_(self.torch.as_tensor(a, dtype=self.torch.float64))
        return out

    def _stream(self):
        return ctypes.c_void_p(self.torch.cuda.current_stream(self.device).cuda_stream)

    # ------------------------------------------------------------------ integrals ---
    def computeAOOneE(self, molecules):
        S, T, V = self.zeros(), self.zeros(), self.zeros()
        Z = np.ascontiguousarray(np.concatenate([np.asarray(m.atoms, dtype=np.float64) for m in molecules]))
        R = np.ascontiguousarray(np.concatenate([np.asarray(m.coords, dtype=np.float64).reshape(-1, 3)
                                                 for m in molecules]))
        nc = np.array([m.natoms for m in molecules], dtype=np.int32)
        d = ctypes.POINTER(ctypes.c_double)
        _lib.check(self._L.cqg_one_e_batch(self._ctx, nc.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                           Z.ctypes.data_as(d), R.ctypes.data_as(d), ctypes.c_void_p(S.data_ptr()),
                                           ctypes.c_void_p(T.data_ptr()), ctypes.c_void_p(V.data_ptr()),
                                           self._stream()), self._ctx)
        return S, T, V

    def newTwoEContractDirect(self, X, AX, contractionList, scalingFactors, active=None):
        assert len(X) == len(AX) == len(contractionList) == len(scalingFactors)
        nmat = len(X)
        Xp = (ctypes.c_void_p * nmat)(*[x.data_ptr() for x in X])
        Ap = (ctypes.c_void_p * nmat)(*[a.data_ptr() for a in AX])
        t = (ctypes.c_int * nmat)(*[int(c) for c in contractionList])
        s = (ctypes.c_double * nmat)(*[float(v) for v in scalingFactors])
        act = None if active is None else bytes(bytearray(1 if a else 0 for a in active))
        _lib.check(self._L.cqg_twoe_contract_direct_batch(self._ctx, nmat, Xp, Ap, t, s, act, self._stream()),
                   self._ctx)

    def formPT(self, Ps, xHF: float = -0.5, active=None, PTs=None):
        """RHF formPT for every active molecule: PTs = 2J[Ps] + 2 xHF K[Ps] (packed)."""
        PTs = self.zeros() if PTs is None else PTs.zero_()
        self.newTwoEContractDirect([Ps, Ps], [PTs, PTs], [0, 1], [1.0, xHF], active)
        return PTs

    # ------------------------------------------------------------------ graphs / tuning ---
    def set_active(self, active=None):
        act = None if active is None else bytes(bytearray(1 if a else 0 for a in active))
        _lib.check(self._L.cqg_set_active(self._ctx, act), self._ctx)

    def enable_graph(self, capacity: int, max_groups: int = 1):
        """Sync-free contractions with a quartet list of `capacity` entries (0: off)."""
        _lib.check(self._L.cqg_set_graph_mode(self._ctx, int(capacity), int(max_groups)), self._ctx)

    def graph_status(self):
        q = ctypes.c_longlong()
        o, nf, asym = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _lib.check(self._L.cqg_graph_status(self._ctx, ctypes.byref(q), ctypes.byref(o), ctypes.byref(nf),
                                            ctypes.byref(asym)), self._ctx)
        return {"quartets": int(q.value), "overflow": bool(o.value), "nonfinite": bool(nf.value),
                "asymmetric": bool(asym.value)}

    def autotune_next(self):
        _lib.check(self._L.cqg_autotune_next(self._ctx), self._ctx)

    def launch_shapes(self):
        n = int(self._L.cqg_schedule_lists())
        cta = np.zeros(n, dtype=np.int32)
        wpb = np.zeros(n, dtype=np.int32)
        i = ctypes.POINTER(ctypes.c_int)
        _lib.check(self._L.cqg_get_launch_shapes(self._ctx, cta.ctypes.data_as(i), wpb.ctypes.data_as(i)), self._ctx)
        return cta, wpb

    def capture_formPT(self, P_static, PT_static, xHF: float = -0.5, warm: bool = True):
        """CUDA graph of one batched RHF Fock build reading P_static, writing PT_static.
        Graph mode must be on.  With `warm`, the call is first run once uncaptured, which
        sets the kernels' attributes; a context that has already run a contraction of the
        same molecules can skip it."""
        torch = self.torch
        if warm:
            self.formPT(P_static, xHF=xHF, PTs=PT_static)
        torch.cuda.synchronize(self.device)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self.formPT(P_static, xHF=xHF, PTs=PT_static)
        return g

    def stats(self):
        s = _lib.CqgStats()
        _lib.check(self._L.cqg_get_stats(self._ctx, ctypes.byref(s)), self._ctx)
        return {"quartets": int(s.quartets), "launches": int(s.launches), "model_flops": float(s.model_flops),
                "ms_total": s.ms_total}

    def close(self):
        if getattr(self, "_ctx", None):
            self._L.cqg_destroy(self._ctx)
            self._ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
