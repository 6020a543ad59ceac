"""Training data, training and evaluation of the learned initial density.

* :func:`converged_densities` -- converged RHF densities of seeded water clusters, made by
  this engine's batched SCF (one batched Fock build per iteration, CUDA-graph replays).
* :func:`training_arrays` -- pair features, local-frame targets and masks
  (:mod:`~chronusq_public_b200.guess_model`) of a list of molecules.
* :func:`train` -- trains a :class:`~chronusq_public_b200.guess_model.PairMLP` on the GPU
  with the library's BF16 kernels, and saves the weights (``.npz``).
* :func:`evaluate` -- held-out molecules converged from the SAD guess and from the learned
  guess (batched, and one at a time on a subset): SCF iterations, wall time and the
  converged-energy difference.

Run as ``python -m chronusq_public_b200.learned_guess --basis 6-31g* --train 4000
--heldout 500 --out weights.npz`` to regenerate a weight file from scratch.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import time
from typing import Dict, List, Sequence

import numpy as np

from .basis import BasisSet
from .guess_model import PairMLP, head_size, molecule_samples
from .molecule import Molecule, single_water, water_cluster


def cluster_set(count: int, nmin: int, nmax: int, seed: int) -> List[Molecule]:
    """`count` seeded water clusters (H2O)_n with n uniform in [nmin, nmax]."""
    rng = np.random.Generator(np.random.PCG64(seed))
    sizes = rng.integers(nmin, nmax + 1, size=count)
    return [single_water(seed * 1000003 + i) if n == 1 else water_cluster(int(n), seed * 1000003 + i)
            for i, n in enumerate(sizes)]


def converged_densities(mols: Sequence[Molecule], basis: str, chunk: int = 512, thresh: float = 1e-12,
                        eneTol: float = 1e-8, denTol: float = 1e-6, model=None):
    """Converged RHF densities (numpy, one per molecule), energies and iteration counts
    from the batched SCF, `chunk` molecules per batch."""
    from .batch_scf import BatchSCF
    P_out, E_out, it_out, secs = [], [], [], 0.0
    for s in range(0, len(mols), chunk):
        part = list(mols[s:s + chunk])
        b = BatchSCF(part, basis, thresholdSchwartz=thresh)
        b.eneTol, b.denTol = eneTol, denTol
        E = b.run(use_graph=True, autotune=True, model=model)
        secs += b.seconds
        for m in range(len(part)):
            P_out.append(b.B.view(b.P, m).cpu().numpy())
        E_out.extend(E.tolist())
        it_out.extend(b.iterations.tolist())
        b.close()
    return P_out, np.array(E_out), np.array(it_out), secs


def training_arrays(mols: Sequence[Molecule], basis: str, densities, rcut: float, maxf: int = None):
    """Features, local-frame targets and masks of every pair of `mols`, blocks padded to the
    head size `maxf` (default: the basis's, head_size)."""
    maxf = head_size(basis) if maxf is None else maxf
    X, T, M = [], [], []
    for mol, P in zip(mols, densities):
        _, _, _, x, t, m = molecule_samples(mol, BasisSet(basis, mol.atoms, mol.coords), rcut, P, maxf)
        X.append(x)
        T.append(t)
        M.append(m)
    return np.concatenate(X), np.concatenate(T), np.concatenate(M)


def train(basis: str = "6-31g*", ntrain: int = 4000, nmin: int = 2, nmax: int = 16, seed: int = 7,
          epochs: int = 40, width: int = 256, layers: int = 4, rcut: float = 8.0, out: str = None,
          lr: float = 2e-3, log=print) -> Dict:
    """Generate converged densities for `ntrain` seeded clusters, train the pair network on
    them, and save it to `out`.  Returns a report (timings, losses)."""
    t0 = time.perf_counter()
    mols = cluster_set(ntrain, nmin, nmax, seed)
    P, E, its, scf_s = converged_densities(mols, basis)
    t1 = time.perf_counter()
    maxf = head_size(basis)
    X, T, M = training_arrays(mols, basis, P, rcut, maxf)
    t2 = time.perf_counter()
    model = PairMLP(width=width, layers=layers, seed=seed, rcut=rcut, maxf=maxf)
    hist = model.fit(X, T, M, epochs=epochs, lr=lr, log=(lambda e, l: log("epoch %d loss %.3e" % (e, l))) if log else None)
    model.torch.cuda.synchronize()
    t3 = time.perf_counter()
    if out:
        model.save(out)
    return {"basis": basis, "train_molecules": ntrain, "cluster_sizes": [nmin, nmax], "seed": seed,
            "pairs": int(len(X)), "data_seconds": t1 - t0, "batched_scf_seconds": scf_s,
            "feature_seconds": t2 - t1, "train_seconds": t3 - t2, "epochs": epochs, "loss_first": hist[0],
            "loss_last": hist[-1], "mean_scf_iterations_sad": float(its.mean()), "model": model}


def training_throughput(pairs: int = 692570, epochs: int = 2, width: int = 256, layers: int = 4,
                        batch: int = 2048, seed: int = 0) -> Dict:
    """Speed of the network's training on the GPU with the library's kernels, on random
    inputs of the shipped training set's shape (`pairs` rows): seconds per epoch (epochs
    after the first, which also captures the training-step graph) and the
    GEMM FLOPs per epoch over that time (forward, weight gradients, input gradients of
    every layer but the first), plus one large forward GEMM (all rows, width x width) timed
    alone, each against the measured dense BF16 peak when known."""
    import torch
    from .guess_model import NFEAT, MAXF
    from . import _lib
    rng = np.random.default_rng(seed)
    X = rng.normal(size=(pairs, NFEAT)).astype(np.float32)
    X[:, -1] = 1.0
    T = rng.normal(size=(pairs, MAXF * MAXF)).astype(np.float32)
    M = np.ones_like(T)
    model = PairMLP(width=width, layers=layers, seed=seed)
    model.fit(X[:batch * 4], T[:batch * 4], M[:batch * 4], epochs=1, batch=batch)     # warm-up
    torch.cuda.synchronize()
    # epoch times from the training log (each epoch ends with a device synchronisation);
    # the first epoch also captures the step graph, the host set-up before it is excluded
    stamps = []
    model.fit(X, T, M, epochs=epochs + 1, batch=batch, log=lambda e, l: stamps.append(time.perf_counter()))
    sec = (stamps[-1] - stamps[0]) / epochs
    kn = [a * b for a, b in zip(model.dims[:-1], model.dims[1:])]
    flops = 2.0 * pairs * (2 * sum(kn) + sum(kn[1:]))
    # one forward GEMM over all rows, width -> width, alone
    A = torch.randn((pairs, width), device="cuda").to(torch.bfloat16)
    B = torch.randn((width, width), device="cuda").to(torch.bfloat16)
    C = torch.empty((pairs, width), device="cuda")
    L = _lib.lib()
    args = [ctypes.c_void_p(A.data_ptr()), width, 1, ctypes.c_void_p(B.data_ptr()), width, 1,
            ctypes.c_void_p(C.data_ptr()), width, pairs, width, width, None, None, 0, 0, 0, None]
    for _ in range(3):
        _lib.check(L.cqg_mlp_gemm_bf16(*args))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(10):
        _lib.check(L.cqg_mlp_gemm_bf16(*args))
    e1.record()
    torch.cuda.synchronize()
    gemm_s = e0.elapsed_time(e1) / 10 * 1e-3
    gemm_tf = 2.0 * pairs * width * width / gemm_s / 1e12
    peak = None
    try:
        import json as _json
        import os as _os
        pp = _os.path.join(_os.path.dirname(_os.path.dirname(_os.path.abspath(__file__))), "MEASURED_PEAKS.json")
        peak = float(_json.load(open(pp))["bf16_tflops"])
    except (OSError, ValueError, KeyError):
        peak = None
    out = {"pairs": pairs, "batch": batch, "dims": model.dims, "seconds_per_epoch": sec,
           "gemm_tflop_per_epoch": flops / 1e12, "training_tflops": flops / sec / 1e12,
           "gemm_alone": {"shape": [pairs, width, width], "ms": gemm_s * 1e3, "tflops": gemm_tf},
           "bf16_peak_tflops": peak}
    if peak:
        out["training_frac_of_peak"] = out["training_tflops"] / peak
        out["gemm_alone"]["frac_of_peak"] = gemm_tf / peak
    return out


def evaluate(model: PairMLP, basis: str = "6-31g*", nheld: int = 500, nmin: int = 2, nmax: int = 16,
             seed: int = 8, single: int = 32, thresh: float = 1e-12) -> Dict:
    """Held-out clusters (a seed disjoint from training) converged to the reference's
    thresholds from the SAD guess and from the learned guess."""
    from .batch_scf import BatchSCF
    from .scf import SingleSlater, atomic_density
    mols = cluster_set(nheld, nmin, nmax, seed)
    for z in (1, 8):
        atomic_density(z, basis, 0, thresh)
    res = {"heldout_molecules": nheld}
    E = {}
    for name, mdl in (("sad", None), ("learned", model)):
        b = BatchSCF(mols, basis, thresholdSchwartz=thresh)
        E[name] = b.run(use_graph=True, autotune=True, model=mdl)
        res["batched_%s_seconds" % name] = b.seconds
        res["batched_%s_mean_iterations" % name] = float(b.iterations.mean())
        res["batched_%s_max_iterations" % name] = int(b.iterations.max())
        res["batched_%s_converged" % name] = bool(b.converged)
        res["batched_%s_guess_seconds" % name] = b.guess_seconds
        res["batched_%s_fock_seconds" % name] = b.fock_seconds
        if mdl is not None:
            res["batched_learned_fallbacks"] = int(b.guess_fallbacks)
            res["batched_learned_predict_seconds"] = b.predict_seconds
        else:
            # guess quality: distance of the starting densities from the converged ones
            P0, _ = b.learned_density(model)
            Ps = b.sad_density()
            rel = {"learned": [], "sad": []}
            for m in range(nheld):
                Pc = b.B.view(b.P, m)
                nc = float(Pc.norm())
                rel["learned"].append(float((b.B.view(P0, m) - Pc).norm()) / nc)
                rel["sad"].append(float((b.B.view(Ps, m) - Pc).norm()) / nc)
            res["guess_rel_density_error_learned"] = float(np.mean(rel["learned"]))
            res["guess_rel_density_error_sad"] = float(np.mean(rel["sad"]))
        b.close()
    res["batched_max_abs_dE"] = float(np.abs(E["sad"] - E["learned"]).max())
    # one at a time on a subset
    k = min(single, nheld)
    its = {"SAD": [], "LEARNED": []}
    secs = {"SAD": 0.0, "LEARNED": 0.0}
    dmax = 0.0
    for mol in mols[:k]:
        bs = BasisSet(basis, mol.atoms, mol.coords)
        Es = {}
        for g in ("SAD", "LEARNED"):
            hf = SingleSlater(mol, bs, thresholdSchwartz=thresh)
            hf.guess = g
            hf.guess_model = model
            Es[g] = hf.SCF3()
            its[g].append(len(hf.log))
            secs[g] += hf.scf_seconds
            hf.close()
        dmax = max(dmax, abs(Es["SAD"] - Es["LEARNED"]))
    res.update({"single_molecules": k, "single_sad_mean_iterations": float(np.mean(its["SAD"])),
                "single_learned_mean_iterations": float(np.mean(its["LEARNED"])),
                "single_sad_seconds": secs["SAD"], "single_learned_seconds": secs["LEARNED"],
                "single_max_abs_dE": dmax})
    return res


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--basis", default="6-31g*")
    ap.add_argument("--train", type=int, default=4000)
    ap.add_argument("--heldout", type=int, default=500)
    ap.add_argument("--nmin", type=int, default=2)
    ap.add_argument("--nmax", type=int, default=16)
    ap.add_argument("--epochs", type=int, default=40)
    ap.add_argument("--single", type=int, default=32)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--seed", type=int, default=7)
    ap.add_argument("--out", required=True)
    ap.add_argument("--report", default=None)
    a = ap.parse_args(argv)
    rep = train(a.basis, a.train, a.nmin, a.nmax, seed=a.seed, epochs=a.epochs, lr=a.lr, out=a.out)
    model = rep.pop("model")
    rep.update(evaluate(model, a.basis, a.heldout, a.nmin, a.nmax, seed=a.seed + 1, single=a.single))
    print(json.dumps(rep))
    if a.report:
        with open(a.report, "w") as f:
            json.dump(rep, f, indent=1)


if __name__ == "__main__":
    main()
