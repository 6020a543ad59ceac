"""Lock-step RHF SCF for a batch of independent molecules on one GPU.

Every SCF iteration makes ONE batched Fock build for all still-active molecules
(:class:`~chronusq_public_b200.batch.BatchAOIntegrals`, one work list per quartet class
shared by all molecules), and does the per-molecule linear algebra in stacks of equally
sized molecules (batched cuBLAS GEMMs and cuSOLVER ``syevd`` through torch).  The
iteration itself follows :mod:`chronusq_public_b200.scf` (SAD guess, commutator DIIS,
damping, the reference's convergence tests), with the energy evaluated for the density the
Fock matrix was built from, E = Tr(P h) + 1/4 Tr(P PT[P]) + E_nuc.
"""
from __future__ import annotations

import math
import time
from typing import List, Optional, Sequence

import numpy as np

from .basis import BasisSet
from .batch import BatchAOIntegrals
from .molecule import Molecule


def occupied_projector(F, nocc: int, max_iter: int = 100, check: int = 4, finish: int = 3):
    """Projector on the `nocc` lowest eigenvectors of each symmetric matrix of the stack F
    (..., n, n), by trace-correcting purification (A. M. N. Niklasson, Phys. Rev. B 66,
    155115 (2002)): the Gershgorin interval [lo, hi] of each matrix is mapped onto [0, 1],
    X0 = (hi I - F) / (hi - lo), so the lowest orbitals sit nearest 1; each step replaces X
    by X^2 or by 2X - X^2, whichever brings the trace nearer nocc, which drives every
    eigenvalue to 0 or 1 with the trace held at nocc.  Once every matrix has
    tr X - tr X^2 < 1e-6 (each eigenvalue within about 1e-6 of 0 or 1) and its trace within
    1e-3 of nocc, `finish` more steps take the deviations, which square at every step, to
    the rounding floor.  The convergence is read back every `check` steps.  Returns None
    when that is not reached in `max_iter` steps (no gap at the Fermi level): the caller
    diagonalises.  Everything is batched FP64 matrix products on the device."""
    import torch as t
    n = F.shape[-1]
    diag = F.diagonal(dim1=-2, dim2=-1)
    rad = F.abs().sum(-1) - diag.abs()
    lo = (diag - rad).amin(-1)
    hi = (diag + rad).amax(-1)
    eye = t.eye(n, dtype=F.dtype, device=F.device)
    X = (hi[..., None, None] * eye - F) / (hi - lo).clamp_min(1e-300)[..., None, None]
    left = None
    for it in range(1, max_iter + 1):
        X2 = X @ X
        tr1 = X.diagonal(dim1=-2, dim2=-1).sum(-1)
        tr2 = X2.diagonal(dim1=-2, dim2=-1).sum(-1)
        square = (tr2 - nocc).abs() <= (2.0 * tr1 - tr2 - nocc).abs()
        X = t.where(square[..., None, None], X2, 2.0 * X - X2)
        if left is not None:
            left -= 1
            if left == 0:
                return 0.5 * (X + X.transpose(-1, -2))
        elif it % check == 0:
            if float((tr1 - tr2).abs().max()) < 1e-6 and float((tr1 - nocc).abs().max()) < 1e-3:
                left = finish
    return None


class BatchSCF:
    def __init__(self, molecules: Sequence[Molecule], basis: str, device: int = 0,
                 thresholdSchwartz: float = 1e-12, ndiis: int = 6):
        import torch
        self.torch = torch
        self.mols = list(molecules)
        self.bss = [BasisSet(basis, m.atoms, m.coords) for m in self.mols]
        self.basis_name = basis
        self.dev = torch.device("cuda", device)
        self.B = BatchAOIntegrals(self.bss, device=device, thresholdSchwartz=thresholdSchwartz)
        self.thresh = thresholdSchwartz
        self.density_method = "purify"     # or "eigh": see _density
        self.nmol = len(self.mols)
        self.nocc = []
        for m in self.mols:
            if m.nelectrons % 2 or m.mult != 1:
                raise ValueError("batched SCF is RHF only")
            self.nocc.append(m.nelectrons // 2)
        self.ndiis = ndiis
        self.eneTol = 1e-10
        self.denTol = 1e-8
        self.maxSCFIter = 128
        self.dampParam = 0.1
        self.Enuc = torch.tensor([m.nuclear_repulsion() for m in self.mols], dtype=torch.float64, device=self.dev)
        # stacks of equally sized molecules
        sizes = {}
        for i, n in enumerate(self.B.nbf):
            sizes.setdefault(n, []).append(i)
        self.groups = []
        for n, members in sorted(sizes.items()):
            idx = torch.tensor(members, dtype=torch.long, device=self.dev)
            flat = torch.stack([torch.arange(self.B.offsets[m], self.B.offsets[m] + n * n, device=self.dev)
                                for m in members])
            nocc = self.nocc[members[0]]
            if any(self.nocc[m] != nocc for m in members):
                raise ValueError("molecules of one size must have the same electron count")
            self.groups.append({"n": n, "members": members, "idx": idx, "flat": flat, "nocc": nocc})
        S, T, V = self.B.computeAOOneE(self.mols)
        self.S, self.H = S, T + V
        for g in self.groups:
            Sg = self.gather(S, g)
            w, U = torch.linalg.eigh(Sg)
            g["X"] = (U * w.rsqrt().unsqueeze(-2)) @ U.transpose(-1, -2)
            g["H"] = self.gather(self.H, g)
            g["S"] = Sg

    # ------------------------------------------------------------------ packing ---
    def gather(self, packed, g):
        return packed[g["flat"]].view(-1, g["n"], g["n"])

    def scatter(self, stacked, g, packed):
        packed[g["flat"].reshape(-1)] = stacked.reshape(-1)

    # ------------------------------------------------------------------ pieces ---
    def _density(self, FO, g):
        """AO density 2 X Q X^T of a stack of orthonormal Fock matrices, Q the projector on the
        nocc lowest orbitals: by purification (`density_method` "purify", batched GEMMs) or
        by eigenvectors ("eigh"); the same aufbau density when the HOMO-LUMO gap is open."""
        t = self.torch
        Q = None
        if self.density_method == "purify":
            Q = occupied_projector(FO, g["nocc"])
        if Q is None:
            _, C = t.linalg.eigh(0.5 * FO)
            Co = C[..., : g["nocc"]]
            Q = Co @ Co.transpose(-1, -2)
        return g["X"] @ (2.0 * Q) @ g["X"].transpose(-1, -2)

    def sad_density(self):
        from .scf import atomic_density
        P = self.B.zeros()
        cache = {}
        for m, (mol, bs) in enumerate(zip(self.mols, self.bss)):
            view = self.B.view(P, m)
            off = {}
            o = 0
            for s in bs.shells:
                off.setdefault(s.atom, [o, 0])
                off[s.atom][1] += s.size
                o += s.size
            for a, z in enumerate(mol.atoms):
                if z not in cache:
                    cache[z] = atomic_density(z, self.basis_name, self.dev.index, self.thresh)[0]
                b0, nb = off[a]
                view[b0:b0 + nb, b0:b0 + nb] = cache[z]
        return P

    def learned_density(self, model):
        """Packed densities predicted by `model` (guess_model.PairMLP, one forward pass for
        all molecules), each projected on its natural orbitals (the nocc most occupied
        eigenvectors of the orthonormal-basis density are occupied).  A molecule whose
        prediction is not finite or whose Tr(PS) is more than 10 % off the electron count
        takes the SAD superposition instead (projected the same way).  Returns the packed
        density and the per-molecule flag of a usable prediction."""
        from .guess_model import predict_densities
        t = self.torch
        t0 = time.perf_counter()
        P = self.B.zeros()
        preds = predict_densities(model, self.mols, self.bss)
        for m, Pm in enumerate(preds):
            self.B.view(P, m).copy_(t.as_tensor(Pm, dtype=t.float64, device=self.dev))
        t.cuda.synchronize(self.dev)
        self.predict_seconds = time.perf_counter() - t0
        ok = np.zeros(self.nmol, dtype=bool)
        sad = None
        for g in self.groups:
            Pg = self.gather(P, g)
            ne = (Pg * g["S"]).sum((-1, -2)).cpu().numpy()
            nel = np.array([self.mols[m].nelectrons for m in g["members"]], dtype=float)
            good = np.isfinite(ne) & (np.abs(ne - nel) <= 0.1 * nel)
            ok[g["members"]] = good
            if not good.all():
                sad = self.sad_density() if sad is None else sad
                keep = t.as_tensor(good, device=self.dev)[:, None, None]
                Pg = t.where(keep, Pg, self.gather(sad, g))
            Xi = g["S"] @ g["X"]                  # X^-1 = S^(1/2) for the Loewdin X
            DO = Xi.transpose(-1, -2) @ Pg @ Xi
            self.scatter(self._density(-DO, g), g, P)   # most occupied natural orbitals
        return P, ok

    # ------------------------------------------------------------------ SCF ---
    def run(self, density=None, use_graph: bool = False, autotune: bool = False, model=None):
        """Converge every molecule; returns the per-molecule energies (numpy).

        The guess density is the SAD superposition, or `density` (packed), or the one
        `model` (guess_model.PairMLP) predicts, made inside the timed region.
        use_graph: the batched Fock build of every iteration is one CUDA-graph replay
        (captured once, after the first iteration's build).  autotune: the first build from
        a full (not block-diagonal) density picks the launch shape of every class work list:
        the first iteration's build after a SAD guess, the guess build itself for a learned
        or given density, so both guesses tune on the same kind of work lists.
        `guess_seconds` records the time until the first iterate exists."""
        t = self.torch
        t.cuda.synchronize(self.dev)
        t0 = time.perf_counter()
        # guess density -> one batched Fock build -> diagonalise; a learned guess is the
        # first iterate itself, and its build is the first iteration's
        first_PT = None
        self.guess_fallbacks = 0
        sad = model is None and density is None
        if model is not None:
            P, ok = self.learned_density(model)
            self.guess_fallbacks = int((~ok).sum())
        else:
            P = self.sad_density() if density is None else density.clone()
        if autotune and not sad:
            self.B.autotune_next()
        PT = self.B.formPT(P)
        tune_first_iteration = autotune and sad
        graph = None
        self.graph_replays = 0
        self.graph_captures = 0
        if use_graph:
            # the graph is captured after the first iteration's build, which is run
            # uncaptured: its screened count sizes the list capacity (the guess build's
            # count, from a block-diagonal density, is far smaller)
            free, _ = t.cuda.mem_get_info(self.dev)
            self.graph_memory_limit = 0.4 * free
            P_static, PT_static = None, self.B.zeros()
        if model is not None:
            first_PT = PT
        else:
            for g in self.groups:
                F = 2.0 * g["H"] + self.gather(PT, g)
                self.scatter(self._density(g["X"].transpose(-1, -2) @ F @ g["X"], g), g, P)
        t.cuda.synchronize(self.dev)
        self.guess_seconds = time.perf_counter() - t0
        active = np.ones(self.nmol, dtype=bool)
        Eold = t.zeros(self.nmol, dtype=t.float64, device=self.dev)
        energies = t.zeros(self.nmol, dtype=t.float64, device=self.dev)
        for g in self.groups:
            g["hist_F"], g["hist_E"] = [], []
            g["damp"] = t.full((len(g["members"]),), self.dampParam, dtype=t.float64, device=self.dev)
            g["FO_prev"] = None
        self.iterations = np.zeros(self.nmol, dtype=int)
        self.fock_builds = 0
        self.fock_seconds = 0.0           # wall time of the Fock builds (device-synchronised)
        self.log = []
        for it in range(self.maxSCFIter):
            t.cuda.synchronize(self.dev)
            tf = time.perf_counter()
            if first_PT is not None:
                PT, first_PT = first_PT, None
            elif it == 0 and (use_graph or tune_first_iteration):
                if tune_first_iteration:
                    self.B.autotune_next()
                PT = self.B.formPT(P, active=active.tolist())
            elif graph is not None:
                self.B.set_active(active.tolist())
                P_static.copy_(P)
                graph.replay()
                st = self.B.graph_status()
                if st["overflow"]:
                    # more quartets than the capture's list capacity: rebuild this iteration
                    # without the graph, then recapture with room for this density's quartets
                    self.B.enable_graph(0)
                    self.B.set_active(None)
                    PT = self.B.formPT(P, active=active.tolist())
                    need = int(1.25 * self.B.stats()["quartets"]) + 4096
                    graph = None
                    if need * 8 <= self.graph_memory_limit:
                        self.B.set_active(None)
                        self.B.enable_graph(need, 1)
                        P_static.copy_(P)
                        graph = self.B.capture_formPT(P_static, PT_static, warm=False)
                        self.graph_captures += 1
                else:
                    PT = PT_static
                    self.graph_replays += 1
            else:
                PT = self.B.formPT(P, active=active.tolist())
            self.fock_builds += 1
            t.cuda.synchronize(self.dev)
            self.fock_seconds += time.perf_counter() - tf
            if use_graph and graph is None and P_static is None:
                need = int(1.25 * self.B.stats()["quartets"]) + 4096
                P_static = P.clone()
                if need * 8 <= self.graph_memory_limit:
                    self.B.set_active(None)
                    self.B.enable_graph(need, 1)
                    graph = self.B.capture_formPT(P_static, PT_static, warm=False)
                    self.graph_captures = 1
            Pnew = P.clone()
            active_d = t.as_tensor(active, device=self.dev)
            conv_d = t.zeros(self.nmol, dtype=t.bool, device=self.dev)
            for mi in np.nonzero(active)[0]:
                self.iterations[mi] = it + 1
            # the group loop only enqueues device work; convergence flags come back once below
            for g in self.groups:
                gidx = g["idx"]
                if not active[g["members"]].any():
                    continue
                act = active_d[gidx]
                Pg = self.gather(P, g)
                PTg = self.gather(PT, g)
                E = (Pg * g["H"]).sum((-1, -2)) + 0.25 * (Pg * PTg).sum((-1, -2)) + self.Enuc[gidx]
                energies[gidx] = t.where(act, E, energies[gidx])
                F = 2.0 * g["H"] + PTg
                X = g["X"]
                FO = X.transpose(-1, -2) @ F @ X
                Xi = g["S"] @ X          # X^-1 = S^(1/2) = S X for the Loewdin X
                DO = Xi.transpose(-1, -2) @ Pg @ Xi
                err = FO @ DO
                err = err - err.transpose(-1, -2)
                g["hist_F"].append(F)
                g["hist_E"].append(err)
                if len(g["hist_F"]) > self.ndiis:
                    g["hist_F"].pop(0)
                    g["hist_E"].pop(0)
                m = len(g["hist_F"])
                if m > 1:
                    Es = t.stack(g["hist_E"], 1).flatten(2)          # (G, m, n^2)
                    Bm = Es @ Es.transpose(-1, -2)
                    sc = Bm.diagonal(dim1=-2, dim2=-1).amax(-1).clamp_min(1e-300)
                    A = t.zeros((Bm.shape[0], m + 1, m + 1), dtype=t.float64, device=self.dev)
                    A[:, :m, :m] = Bm / sc[:, None, None]
                    A[:, m, :m] = -1.0
                    A[:, :m, m] = -1.0
                    rhs = t.zeros((Bm.shape[0], m + 1), dtype=t.float64, device=self.dev)
                    rhs[:, m] = -1.0
                    # solve_ex: no host round trip for an error check; a singular system
                    # gives non-finite c, caught by `ok` below
                    c = t.linalg.solve_ex(A + 1e-14 * t.eye(m + 1, dtype=t.float64, device=self.dev), rhs)[0][:, :m]
                    ok = t.isfinite(c).all(-1) & (c.abs().amax(-1) < 1e6)
                    Fx = (c[:, :, None, None] * t.stack(g["hist_F"], 1)).sum(1)
                    F = t.where(ok[:, None, None], Fx, F)
                    FO = X.transpose(-1, -2) @ F @ X
                damp = g["damp"]
                if g["FO_prev"] is not None:
                    FO = (1.0 - damp)[:, None, None] * FO + damp[:, None, None] * g["FO_prev"]
                g["FO_prev"] = FO
                Pn = self._density(FO, g)
                dE = E - Eold[gidx]
                dP = (Pn - Pg).flatten(1).norm(dim=-1)
                Eold[gidx] = t.where(act, E, Eold[gidx])
                g["damp"] = t.where(dE.abs() < 1e-6, t.zeros_like(damp),
                                    t.where(damp <= 0.0, t.full_like(damp, self.dampParam), damp))
                conv_d[gidx] = (dE.abs() < self.eneTol) & (dP < self.denTol) & act
                Pn = t.where(act[:, None, None], Pn, Pg)
                self.scatter(Pn, g, Pnew)
            active &= ~conv_d.cpu().numpy()
            P = Pnew
            t.cuda.synchronize(self.dev)
            self.log.append((it, int(active.sum()), time.perf_counter() - t0))
            if not active.any():
                break
        if use_graph:
            self.B.enable_graph(0)
            self.B.set_active(None)
        self.seconds = time.perf_counter() - t0
        self.converged = not active.any()
        self.energies = energies.cpu().numpy()
        self.P = P
        return self.energies

    def close(self):
        self.B.close()
