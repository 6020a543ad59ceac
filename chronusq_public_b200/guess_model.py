"""Learned initial density: an MLP on atom pairs, equivariant by construction.

For every atom pair (A, B) closer than ``rcut`` (and every atom with itself) the network
predicts the density block P_AB expressed in a local frame fixed by the geometry:

* A != B: e_z along R_B - R_A; e_x from the atom nearest the pair midpoint (other than A
  and B), projected perpendicular to e_z; e_y = e_z x e_x.
* A == B: e_z towards the nearest atom, e_x from the next nearest.

The network sees only rotation- and translation-invariant inputs (element one-hots, the
pair distance, and the local-frame coordinates, distances and elements of the KNEIGH atoms
nearest the pair midpoint), so what it predicts is a local-frame block.  The block is
carried to the molecular frame by the exact rotation matrices of the basis functions
(1 for s, the frame matrix for Cartesian p, the real-solid-harmonic rotation for pure d
and f), which makes the assembled density equivariant under rotations and translations by
construction.  Pairs are ordered heavier element first; one network whose maxf x maxf
output (maxf: the largest function count of one atom in the basis, head_size) is masked
per pair type serves every pair type of the basis.

Training and inference run through the library's kernels (csrc/mlp.cu: BF16 tensor-core
GEMM with fused bias and SiLU, SiLU backward, bias reduction, masked MSE, Adam); torch only
holds device memory.  The SCF starts its iterations from the natural-orbital projection of
a prediction, so the guess can change the iteration count but not the converged answer.
"""
from __future__ import annotations

import ctypes
import itertools
import math
import os
from typing import Dict, List, Sequence, Tuple

import numpy as np

from . import _lib
from .basis import BasisSet, cart_list, solid_harmonic_matrix

ELEMS = (1, 8)                 # element vocabulary (H, O)
KNEIGH = 8                     # environment atoms per pair
NFEAT = 2 * len(ELEMS) + 4 + KNEIGH * (4 + len(ELEMS)) + 1
MAXF = 14                      # default head: largest per-atom function count (O in 6-31G(d) and cc-pVDZ)


# ---------------------------------------------------------------- rotations ---
def _monomial_tables(l: int):
    """For degree l: per Cartesian component its axis multiset, and for every index tuple
    (i_1..i_l) the Cartesian component of prod_m r_{i_m}."""
    carts = cart_list(l)
    pos = {c: k for k, c in enumerate(carts)}
    axes = [[0] * c[0] + [1] * c[1] + [2] * c[2] for c in carts]
    tuples = []
    for idx in itertools.product(range(3), repeat=l):
        e = [0, 0, 0]
        for i in idx:
            e[i] += 1
        tuples.append((idx, pos[tuple(e)]))
    return axes, tuples


_SH = {l: (solid_harmonic_matrix(l), np.linalg.pinv(solid_harmonic_matrix(l))) for l in (2, 3)}
_MONO = {l: _monomial_tables(l) for l in (2, 3)}


def pure_rotation(l: int, F: np.ndarray) -> np.ndarray:
    """W (P, 2l+1, 2l+1) with phi_local = phi_global @ W for pure shells of degree l; F
    (P, 3, 3) holds the frames (columns = local axes in molecular coordinates).

    With mono(F^T r) = M mono(r) for the degree-l monomials and S = C mono the solid
    harmonics, S(F^T r) = C M C^+ S(r), so W = (C M C^+)^T."""
    axes, tuples = _MONO[l]
    nc = len(axes)
    M = np.zeros((F.shape[0], nc, nc))
    for k, ax in enumerate(axes):
        for idx, target in tuples:
            term = F[:, idx[0], ax[0]]
            for m in range(1, l):
                term = term * F[:, idx[m], ax[m]]
            M[:, k, target] += term
    C, Cp = _SH[l]
    D = np.einsum("ij,pjk,kl->pil", C, M, Cp)
    return np.transpose(D, (0, 2, 1))


def atom_rotations(shells: Sequence[Tuple[int, bool]], F: np.ndarray) -> np.ndarray:
    """Block-diagonal W (P, nf, nf) for an atom carrying `shells` ((l, pure) pairs)."""
    sizes = [(2 * l + 1) if (pure or l < 2) else (l + 1) * (l + 2) // 2 for l, pure in shells]
    nf = sum(sizes)
    W = np.zeros((F.shape[0], nf, nf))
    o = 0
    for (l, pure), k in zip(shells, sizes):
        if l == 0:
            W[:, o, o] = 1.0
        elif l == 1:
            W[:, o:o + 3, o:o + 3] = F
        elif pure:
            W[:, o:o + k, o:o + k] = pure_rotation(l, F)
        else:
            raise NotImplementedError("Cartesian shells with l > 1")
        o += k
    return W


class AtomLayout:
    """Per atom of a molecule: element, first basis function and function count; per
    element its (l, pure) shell list (the same for every atom of an element in a basis)."""

    def __init__(self, Z: Sequence[int], bs: BasisSet, maxf: int = MAXF):
        self.maxf = int(maxf)
        self.Z = np.asarray(Z, dtype=np.int64)
        n = len(self.Z)
        self.off = np.full(n, -1, dtype=np.int64)
        self.nf = np.zeros(n, dtype=np.int64)
        per_atom: Dict[int, List[Tuple[int, bool]]] = {a: [] for a in range(n)}
        for s, o in zip(bs.shells, bs.map_sh2bf):
            if self.off[s.atom] < 0:
                self.off[s.atom] = o
            self.nf[s.atom] += s.size
            per_atom[s.atom].append((s.l, s.pure))
        self.shells: Dict[int, List[Tuple[int, bool]]] = {}
        for a in range(n):
            z = int(self.Z[a])
            if z not in ELEMS:
                raise ValueError("element %d is outside the model's vocabulary" % z)
            if z in self.shells and self.shells[z] != per_atom[a]:
                raise ValueError("atoms of one element carry different shells")
            self.shells[z] = per_atom[a]
        if int(self.nf.max()) > self.maxf:
            raise ValueError("an atom has %d functions; the model handles at most %d" % (self.nf.max(), self.maxf))


# ---------------------------------------------------------------- pairs, frames, features ---
def _unit(v):
    return v / np.maximum(np.linalg.norm(v, axis=-1, keepdims=True), 1e-12)


def canonical_pairs(Z: np.ndarray, R: np.ndarray, rcut: float) -> np.ndarray:
    """(P, 2) atom pairs (a, b): every atom with itself and every distinct pair closer
    than rcut, heavier element first (index order within one element)."""
    n = len(Z)
    D = np.linalg.norm(R[:, None, :] - R[None, :, :], axis=-1)
    ia, ib = np.triu_indices(n)
    keep = (ia == ib) | (D[ia, ib] <= rcut)
    ia, ib = ia[keep], ib[keep]
    swap = Z[ib] > Z[ia]
    return np.stack([np.where(swap, ib, ia), np.where(swap, ia, ib)], axis=1)


def frames_and_features(Z: np.ndarray, R: np.ndarray, pairs: np.ndarray):
    """Local frames F (P, 3, 3) and invariant features X (P, NFEAT) of every pair."""
    n = len(Z)
    a, b = pairs[:, 0], pairs[:, 1]
    same = a == b
    P = len(a)
    rows = np.arange(P)
    mid = 0.5 * (R[a] + R[b])
    dm = np.linalg.norm(R[None, :, :] - mid[:, None, :], axis=-1)           # (P, n)
    dm[rows, a] = np.inf
    dm[rows, b] = np.inf
    order = np.argsort(dm, axis=1, kind="stable")                            # other atoms, nearest first
    nother = n - 1 - (~same).astype(np.int64)
    ez = np.empty((P, 3))
    ez[~same] = _unit(R[b[~same]] - R[a[~same]])
    if same.any():
        has = nother[same] > 0
        v = np.where(has[:, None], R[order[same, 0]] - mid[same], np.array([0.0, 0.0, 1.0]))
        ez[same] = _unit(v)
    # e_x: the first remaining other atom off the e_z axis
    ex = np.full((P, 3), np.nan)
    start = np.where(same, 1, 0)
    for k in range(n):
        valid = (start + k) < nother
        if not valid.any():
            break
        col = np.minimum(start + k, n - 1)
        cand = R[order[rows, col]] - mid
        cand = cand - np.sum(cand * ez, axis=1, keepdims=True) * ez
        ok = valid & np.isnan(ex[:, 0]) & (np.linalg.norm(cand, axis=1) > 1e-6)
        ex[ok] = _unit(cand[ok])
        if not np.isnan(ex[:, 0]).any():
            break
    miss = np.isnan(ex[:, 0])
    if miss.any():
        t = np.where(np.abs(ez[miss, 0:1]) < 0.9, np.array([1.0, 0.0, 0.0]), np.array([0.0, 1.0, 0.0]))
        ex[miss] = _unit(t - np.sum(t * ez[miss], axis=1, keepdims=True) * ez[miss])
    F = np.stack([ex, np.cross(ez, ex), ez], axis=2)
    onehot = np.stack([(Z == e).astype(np.float64) for e in ELEMS], axis=1)
    dab = np.linalg.norm(R[b] - R[a], axis=1)
    cols = [onehot[a], onehot[b], dab[:, None], (1.0 / (1.0 + dab))[:, None], np.exp(-dab)[:, None],
            same[:, None].astype(np.float64)]
    for k in range(KNEIGH):
        valid = (k < nother)[:, None].astype(np.float64)
        j = order[:, min(k, n - 1)]
        loc = np.einsum("pij,pi->pj", F, R[j] - mid)
        r = np.linalg.norm(loc, axis=1, keepdims=True)
        cols += [loc * valid, r * valid, onehot[j] * valid]
    cols.append(np.ones((P, 1)))
    X = np.concatenate(cols, axis=1)
    return F, X


def pair_type_groups(layout: AtomLayout, pairs: np.ndarray):
    """Indices of the pairs of each (Z_a, Z_b) type."""
    za, zb = layout.Z[pairs[:, 0]], layout.Z[pairs[:, 1]]
    return {key: np.nonzero((za == key[0]) & (zb == key[1]))[0]
            for key in sorted(set(zip(za.tolist(), zb.tolist())))}


def _block_index(layout, pairs, idx, na, nb):
    ra = layout.off[pairs[idx, 0]][:, None] + np.arange(na)[None, :]
    rb = layout.off[pairs[idx, 1]][:, None] + np.arange(nb)[None, :]
    return ra[:, :, None], rb[:, None, :]


def local_blocks(layout: AtomLayout, pairs, F, P: np.ndarray):
    """Targets Wa^T P_ab Wb in the pair frames and their masks, padded to maxf x maxf."""
    npair = len(pairs)
    mf = layout.maxf
    T = np.zeros((npair, mf, mf))
    M = np.zeros((npair, mf, mf), dtype=np.float32)
    for (za, zb), idx in pair_type_groups(layout, pairs).items():
        Wa, Wb = atom_rotations(layout.shells[za], F[idx]), atom_rotations(layout.shells[zb], F[idx])
        na, nb = Wa.shape[1], Wb.shape[1]
        ra, rb = _block_index(layout, pairs, idx, na, nb)
        T[idx, :na, :nb] = np.matmul(np.matmul(np.transpose(Wa, (0, 2, 1)), P[ra, rb]), Wb)
        M[idx, :na, :nb] = 1.0
    return T.reshape(npair, -1), M.reshape(npair, -1)


def assemble_density(layout: AtomLayout, pairs, F, blocks: np.ndarray, nbf: int) -> np.ndarray:
    """Molecular-frame density from local-frame blocks (P, maxf*maxf); pairs not listed
    (farther apart than the cut-off) stay zero."""
    B = np.asarray(blocks).reshape(-1, layout.maxf, layout.maxf)
    D = np.zeros((nbf, nbf))
    for (za, zb), idx in pair_type_groups(layout, pairs).items():
        Wa, Wb = atom_rotations(layout.shells[za], F[idx]), atom_rotations(layout.shells[zb], F[idx])
        na, nb = Wa.shape[1], Wb.shape[1]
        blk = np.matmul(np.matmul(Wa, B[idx, :na, :nb]), np.transpose(Wb, (0, 2, 1)))
        same = pairs[idx, 0] == pairs[idx, 1]
        if same.any():
            blk[same] = 0.5 * (blk[same] + np.transpose(blk[same], (0, 2, 1)))
        ra, rb = _block_index(layout, pairs, idx, na, nb)
        D[ra, rb] = blk
        D[np.swapaxes(rb, 1, 2), np.swapaxes(ra, 1, 2)] = np.transpose(blk, (0, 2, 1))
    return D


def molecule_samples(mol, bs: BasisSet, rcut: float, P: np.ndarray = None, maxf: int = MAXF):
    """(layout, pairs, frames, features) of one molecule, plus (targets, masks) when the
    density P is given; blocks are padded to the head size `maxf`."""
    Z = np.asarray(mol.atoms, dtype=np.int64)
    R = np.asarray(mol.coords, dtype=np.float64).reshape(-1, 3)
    layout = AtomLayout(Z, bs, maxf)
    pairs = canonical_pairs(Z, R, rcut)
    F, X = frames_and_features(Z, R, pairs)
    if P is None:
        return layout, pairs, F, X
    T, M = local_blocks(layout, pairs, F, np.asarray(P))
    return layout, pairs, F, X, T, M


# ---------------------------------------------------------------- the network ---
class PairMLP:
    """NFEAT -> width (x `layers` hidden layers, SiLU) -> maxf*maxf; BF16 operands and
    activations, FP32 accumulation, FP32 master weights updated by Adam.  `maxf` is the
    head's per-atom block size: the largest function count of one atom in the basis the
    model predicts in (14 for O in 6-31G(d) and cc-pVDZ, 30 in cc-pVTZ; head_size)."""

    def __init__(self, width: int = 256, layers: int = 4, seed: int = 0, device: int = 0, rcut: float = 8.0,
                 maxf: int = MAXF):
        import torch
        self.torch = torch
        self.L = _lib.lib()
        self.dev = torch.device("cuda", device)
        self.rcut = float(rcut)
        self.maxf = int(maxf)
        rng = np.random.default_rng(seed)
        self.dims = [NFEAT] + [width] * layers + [self.maxf * self.maxf]
        W, b = [], []
        for i in range(len(self.dims) - 1):
            w = rng.normal(0.0, 1.0 / math.sqrt(self.dims[i]), size=(self.dims[i + 1], self.dims[i]))
            if i == len(self.dims) - 2:
                w *= 0.1
            W.append(w)
            b.append(np.zeros(self.dims[i + 1]))
        self.set_weights(W, b)
        self.xmean = np.zeros(NFEAT)
        self.xstd = np.ones(NFEAT)
        self.ymean = np.zeros(self.maxf * self.maxf)
        self.ystd = 1.0

    def set_weights(self, W, b):
        t = self.torch
        self.W = [t.tensor(np.asarray(w), dtype=t.float32, device=self.dev).contiguous() for w in W]
        self.b = [t.tensor(np.asarray(x), dtype=t.float32, device=self.dev).contiguous() for x in b]
        self.Wbf = [w.to(t.bfloat16) for w in self.W]
        self.mW = [t.zeros_like(w) for w in self.W]
        self.vW = [t.zeros_like(w) for w in self.W]
        self.mb = [t.zeros_like(x) for x in self.b]
        self.vb = [t.zeros_like(x) for x in self.b]
        self.step = 0

    def _stream(self):
        return ctypes.c_void_p(self.torch.cuda.current_stream(self.dev).cuda_stream)

    @staticmethod
    def _p(x):
        return ctypes.c_void_p(x.data_ptr()) if x is not None else None

    # ------------------------------------------------------------------ passes ---
    def forward(self, Xbf, keep: bool = False):
        """Xbf (M, NFEAT) BF16 -> FP32 output (M, maxf*maxf).  keep: also return, per
        layer, its BF16 input and FP32 pre-activation for the backward pass."""
        t = self.torch
        M = Xbf.shape[0]
        h, cache, nl = Xbf, [], len(self.W)
        out = None
        for i in range(nl):
            N, K = self.dims[i + 1], self.dims[i]
            Z = t.empty((M, N), dtype=t.float32, device=self.dev)
            last = i == nl - 1
            Y = None if last else t.empty((M, N), dtype=t.bfloat16, device=self.dev)
            _lib.check(self.L.cqg_mlp_gemm_bf16(self._p(h), K, 1, self._p(self.Wbf[i]), K, 1, self._p(Z), N, M, N,
                                                K, self._p(self.b[i]), self._p(Y), N, 0 if last else 1, 0,
                                                self._stream()))
            if keep:
                cache.append((h, Z))
            h, out = Y, Z
        return out, cache

    def backward(self, dout, cache):
        """dout (M, maxf*maxf) FP32 = dLoss/dOutput -> FP32 weight and bias gradients."""
        t = self.torch
        nl = len(self.W)
        gW, gb = [None] * nl, [None] * nl
        dY = dout
        for i in range(nl - 1, -1, -1):
            h, Z = cache[i]
            M, N, K = h.shape[0], self.dims[i + 1], self.dims[i]
            dZ = t.empty((M, N), dtype=t.bfloat16, device=self.dev)
            if i == nl - 1:
                _lib.check(self.L.cqg_mlp_to_bf16(self._p(dY), self._p(dZ), M * N, self._stream()))
            else:
                _lib.check(self.L.cqg_mlp_silu_bwd(self._p(dY), self._p(Z), self._p(dZ), M * N, self._stream()))
            gW[i] = t.empty((N, K), dtype=t.float32, device=self.dev)          # dW[n][k] = sum_m dZ[m][n] h[m][k]
            _lib.check(self.L.cqg_mlp_gemm_bf16(self._p(dZ), 1, N, self._p(h), 1, K, self._p(gW[i]), K, N, K, M,
                                                None, None, 0, 0, 0, self._stream()))
            gb[i] = t.empty(N, dtype=t.float32, device=self.dev)
            _lib.check(self.L.cqg_mlp_colsum(self._p(dZ), M, N, self._p(gb[i]), self._stream()))
            if i > 0:                                                           # dX[m][k] = sum_n dZ[m][n] W[n][k]
                dX = t.empty((M, K), dtype=t.float32, device=self.dev)
                _lib.check(self.L.cqg_mlp_gemm_bf16(self._p(dZ), N, 1, self._p(self.Wbf[i]), 1, K, self._p(dX), K,
                                                    M, K, N, None, None, 0, 0, 0, self._stream()))
                dY = dX
        return gW, gb

    def loss_grad(self, out, target, mask, inv_count: float):
        """Masked squared error sum * inv_count and its gradient."""
        t = self.torch
        dout = t.empty_like(out)
        loss = t.zeros(1, dtype=t.float32, device=self.dev)
        _lib.check(self.L.cqg_mlp_mse(self._p(out), self._p(target), self._p(mask), out.numel(), inv_count,
                                      self._p(dout), self._p(loss), self._stream()))
        return loss, dout

    def adam(self, gW, gb, lr: float, wd: float = 0.0):
        self.step += 1
        for i in range(len(self.W)):
            _lib.check(self.L.cqg_mlp_adam(self._p(self.W[i]), self._p(gW[i]), self._p(self.mW[i]),
                                           self._p(self.vW[i]), self.W[i].numel(), lr, 0.9, 0.999, 1e-8, self.step,
                                           wd, self._p(self.Wbf[i]), self._stream()))
            _lib.check(self.L.cqg_mlp_adam(self._p(self.b[i]), self._p(gb[i]), self._p(self.mb[i]),
                                           self._p(self.vb[i]), self.b[i].numel(), lr, 0.9, 0.999, 1e-8, self.step,
                                           0.0, None, self._stream()))

    # ------------------------------------------------------------------ training ---
    def normalise_inputs(self, X: np.ndarray):
        t = self.torch
        Xn = (np.asarray(X) - self.xmean) / self.xstd
        return t.tensor(Xn, dtype=t.float32, device=self.dev).to(t.bfloat16).contiguous()

    def adam_dev(self, gW, gb, hyper, wd: float = 0.0):
        """Adam step with {lr, 1 - b1^step, 1 - b2^step} read from the device tensor `hyper`
        (capturable in a CUDA graph); the host step counter advances as in :meth:`adam`."""
        self.step += 1
        for i in range(len(self.W)):
            _lib.check(self.L.cqg_mlp_adam_dev(self._p(self.W[i]), self._p(gW[i]), self._p(self.mW[i]),
                                               self._p(self.vW[i]), self.W[i].numel(), self._p(hyper), 0.9, 0.999,
                                               1e-8, wd, self._p(self.Wbf[i]), self._stream()))
            _lib.check(self.L.cqg_mlp_adam_dev(self._p(self.b[i]), self._p(gb[i]), self._p(self.mb[i]),
                                               self._p(self.vb[i]), self.b[i].numel(), self._p(hyper), 0.9, 0.999,
                                               1e-8, 0.0, None, self._stream()))

    def fit(self, X, T, M, epochs: int = 40, batch: int = 2048, lr: float = 2e-3, seed: int = 0, log=None,
            graph: bool = True):
        """Masked-MSE training on (features, local-frame targets, masks).  Inputs are
        standardised per feature, targets by their masked mean per output and one global
        scale.  Returns the per-epoch mean training loss (standardised units).

        With `graph`, one full-batch training step (batch gather, forward, loss, backward,
        Adam with the step's learning rate and bias corrections taken from device memory)
        is captured once as a CUDA graph and replayed for every later full batch; the
        partial last batch of an epoch runs uncaptured.  The arithmetic is the same as the
        uncaptured loop's."""
        t = self.torch
        X = np.asarray(X)
        T = np.asarray(T)
        Mf = np.asarray(M, dtype=np.float32)
        self.xmean = X.mean(0)
        self.xstd = X.std(0) + 1e-6
        self.xmean[-1], self.xstd[-1] = 0.0, 1.0                     # the constant input stays 1
        cnt = np.maximum(Mf.sum(0), 1.0)
        self.ymean = (T * Mf).sum(0) / cnt
        self.ystd = float(np.sqrt((((T - self.ymean) * Mf) ** 2).sum() / max(Mf.sum(), 1.0)))
        Xd = self.normalise_inputs(X)
        Td = t.tensor((T - self.ymean) / self.ystd, dtype=t.float32, device=self.dev)
        Md = t.tensor(Mf, dtype=t.float32, device=self.dev)
        n = Xd.shape[0]
        g = t.Generator(device=self.dev)
        g.manual_seed(seed)
        hist = []
        per_epoch = (n + batch - 1) // batch
        steps = max(1, epochs * per_epoch)

        def lr_at(k):
            warm = min(1.0, (k + 1) / 100.0)
            return lr * warm * 0.5 * (1.0 + math.cos(math.pi * k / steps))

        # {lr, 1 - b1^step, 1 - b2^step} of every step, on the device
        sched = np.array([[lr_at(k), 1.0 - 0.9 ** (self.step + k + 1), 1.0 - 0.999 ** (self.step + k + 1)]
                          for k in range(steps)], dtype=np.float32)
        sched_d = t.tensor(sched, device=self.dev)
        hyper = t.zeros(3, dtype=t.float32, device=self.dev)
        idx_s = t.zeros(batch, dtype=t.int64, device=self.dev)
        tot = t.zeros(1, dtype=t.float32, device=self.dev)
        use_graph = graph and n >= 2 * batch
        stream = t.cuda.Stream(device=self.dev) if use_graph else None
        cuda_graph = None

        def step_body(idx, nb):
            out, cache = self.forward(Xd.index_select(0, idx), keep=True)
            loss, dout = self.loss_grad(out, Td.index_select(0, idx), Md.index_select(0, idx), 1.0 / float(nb))
            gW, gb = self.backward(dout, cache)
            self.adam_dev(gW, gb, hyper)
            tot.add_(loss * nb)

        k = 0
        for ep in range(epochs):
            perm = t.randperm(n, device=self.dev, generator=g)
            tot.zero_()
            for s in range(0, n, batch):
                idx = perm[s:s + batch]
                nb = int(idx.numel())
                hyper.copy_(sched_d[k])
                if nb == batch and cuda_graph is not None:
                    idx_s.copy_(idx)
                    cuda_graph.replay()
                    self.step += 1                    # the captured Adam's step, on the host
                else:
                    step_body(idx, nb)
                    if use_graph and cuda_graph is None and nb == batch:
                        # capture the full-batch step once (after this eager one warmed it up)
                        t.cuda.synchronize(self.dev)
                        cuda_graph = t.cuda.CUDAGraph()
                        stream.wait_stream(t.cuda.current_stream(self.dev))
                        step0 = self.step
                        with t.cuda.stream(stream):
                            with t.cuda.graph(cuda_graph, stream=stream):
                                step_body(idx_s, batch)
                        t.cuda.current_stream(self.dev).wait_stream(stream)
                        self.step = step0                 # capture enqueued nothing
                k += 1
            hist.append(float(tot) / n)
            if log:
                log(ep, hist[-1])
        return hist

    def predict(self, X: np.ndarray) -> np.ndarray:
        if len(X) == 0:
            return np.zeros((0, self.maxf * self.maxf))
        out, _ = self.forward(self.normalise_inputs(X))
        return out.double().cpu().numpy() * self.ystd + self.ymean

    # ------------------------------------------------------------------ persistence ---
    def state(self) -> Dict[str, np.ndarray]:
        d = {"dims": np.array(self.dims), "rcut": np.array(self.rcut), "xmean": self.xmean, "xstd": self.xstd,
             "ymean": self.ymean, "ystd": np.array(self.ystd), "kneigh": np.array(KNEIGH)}
        for i, (w, b) in enumerate(zip(self.W, self.b)):
            d["W%d" % i] = w.cpu().numpy()
            d["b%d" % i] = b.cpu().numpy()
        return d

    def save(self, path: str):
        np.savez_compressed(path, **self.state())

    @classmethod
    def load(cls, path: str, device: int = 0) -> "PairMLP":
        d = np.load(path)
        dims = [int(x) for x in d["dims"]]
        maxf = int(round(math.sqrt(dims[-1])))
        if dims[0] != NFEAT or maxf * maxf != dims[-1] or int(d["kneigh"]) != KNEIGH:
            raise ValueError("weights were made for another feature layout")
        m = cls(width=dims[1], layers=len(dims) - 2, device=device, rcut=float(d["rcut"]), maxf=maxf)
        nl = len(dims) - 1
        m.set_weights([d["W%d" % i] for i in range(nl)], [d["b%d" % i] for i in range(nl)])
        m.xmean, m.xstd = d["xmean"], d["xstd"]
        m.ymean, m.ystd = d["ymean"], float(d["ystd"])
        return m


WEIGHTS_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "guess_weights")


def default_weights(basis: str):
    """Path of the shipped weights for water clusters in `basis`, or None."""
    path = os.path.join(WEIGHTS_DIR, "h2o_%s.npz" % basis.lower().replace("*", "d"))
    return path if os.path.exists(path) else None


def head_size(basis: str) -> int:
    """Head block size a network needs for `basis`: the largest function count of one atom
    of the model's elements in that basis."""
    return max(BasisSet(basis, [z], np.zeros((1, 3))).nbasis for z in ELEMS)


def predict_densities(model: PairMLP, mols, bss) -> List[np.ndarray]:
    """Molecular densities assembled from the network's local-frame pair blocks; the
    pairs of all molecules go through one forward pass."""
    samples = [molecule_samples(m, bs, model.rcut, maxf=model.maxf) for m, bs in zip(mols, bss)]
    Y = model.predict(np.concatenate([s[3] for s in samples]))
    out, o = [], 0
    for (layout, pairs, F, X), bs in zip(samples, bss):
        out.append(assemble_density(layout, pairs, F, Y[o:o + len(X)], bs.nbasis))
        o += len(X)
    return out


def predict_density(model: PairMLP, mol, bs: BasisSet) -> np.ndarray:
    return predict_densities(model, [mol], [bs])[0]


def project_density(P_src, bs_src: BasisSet, bs_tgt: BasisSet, device: int = 0):
    """Carry a density from basis `bs_src` into `bs_tgt` on the same molecule by the
    overlap projection P_tgt = S_tt^-1 S_ts P_src S_st S_tt^-1 (the density of the
    projected orbitals; torch tensors on the device).  The overlaps come from the
    library's one-electron kernel run on the union of the two bases."""
    import copy
    import torch
    from .aointegrals import AOIntegrals
    u = copy.copy(bs_tgt)
    u.shells = list(bs_tgt.shells) + list(bs_src.shells)
    u.map_sh2bf = np.cumsum([0] + [s.size for s in u.shells[:-1]]).astype(np.int64)
    u.nbasis = bs_tgt.nbasis + bs_src.nbasis
    u.name = "%s+%s" % (bs_tgt.name, bs_src.name)
    ints = AOIntegrals(u, device=device, thresholdSchwartz=1e-12)
    try:
        S, _, _ = ints.computeAOOneE([], np.zeros((0, 3)), device_out=True)
    finally:
        ints.close()
    nt = bs_tgt.nbasis
    Ps = torch.as_tensor(P_src, dtype=torch.float64, device=S.device)
    M = torch.linalg.solve(S[:nt, :nt], S[:nt, nt:])         # S_tt^-1 S_ts
    return M @ Ps @ M.T
