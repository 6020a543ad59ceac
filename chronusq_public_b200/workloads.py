"""Seeded synthetic workloads of the engine's benchmark configurations.

* :func:`cluster_batch` -- independent water clusters (H2O)_n, n uniform in [nmin, nmax],
  each generated by :func:`~chronusq_public_b200.molecule.water_cluster` from its own seed
  (batched-SCF configuration).
* :func:`batch_scf_comparison` -- molecules per second to convergence of the lock-step
  batched SCF (one batched Fock build per iteration, replayed as a CUDA graph, launch shapes
  autotuned) against the same molecules converged one at a time with the one-molecule SCF.
  The one-at-a-time time of the whole batch is estimated from a sample stratified by
  cluster size: `per_size` molecules of every size n present, each size's mean time
  weighted by how many molecules of that size the batch holds.
"""
from __future__ import annotations

import time
from typing import List

import numpy as np

from .basis import BasisSet
from .molecule import Molecule, single_water, water_cluster


def cluster_batch(count: int, nmin: int = 1, nmax: int = 24, seed: int = 0) -> List[Molecule]:
    rng = np.random.Generator(np.random.PCG64(seed))
    sizes = rng.integers(nmin, nmax + 1, size=count)
    out = []
    for i, n in enumerate(sizes):
        s = seed * 100003 + i
        out.append(single_water(s) if n == 1 else water_cluster(int(n), s))
    return out


def batch_scf_comparison(count: int = 512, per_size: int = 2, basis: str = "6-31g*", seed: int = 0,
                         thresh: float = 1e-12):
    import torch
    from .batch_scf import BatchSCF
    from .scf import SingleSlater, atomic_density
    mols = cluster_batch(count, seed=seed)
    for z in (1, 8):                               # atomic SAD densities, cached for both
        atomic_density(z, basis, 0, thresh)
    b = BatchSCF(mols, basis, thresholdSchwartz=thresh)
    E = b.run(use_graph=True, autotune=True)
    sizes = [int(m.natoms // 3) for m in mols]
    res = {"molecules": count, "sizes_first": sizes[:8], "nbasis_total": int(sum(b.B.nbf)),
           "batched_seconds": b.seconds, "batched_fock_seconds": b.fock_seconds,
           "batched_guess_seconds": b.guess_seconds, "batched_molecules_per_s": count / b.seconds,
           "batched_iterations_max": int(b.iterations.max()), "batched_fock_builds": b.fock_builds,
           "graph_replays": b.graph_replays, "graph_captures": b.graph_captures, "converged": bool(b.converged)}
    b.close()
    # one at a time: the first `per_size` molecules of every cluster size, each its own
    # context and SCF; the batch's one-at-a-time time is the size-weighted sum of the means
    by_size = {}
    for i, n in enumerate(sizes):
        by_size.setdefault(n, []).append(i)
    secs_by_size, dmax, sample = {}, 0.0, 0
    for n in sorted(by_size):
        ts = []
        for i in by_size[n][:per_size]:
            m = mols[i]
            hf = SingleSlater(m, BasisSet(basis, m.atoms, m.coords), thresholdSchwartz=thresh)
            torch.cuda.synchronize()
            hf.SCF3()
            ts.append(hf.scf_seconds)
            dmax = max(dmax, abs(hf.totalEnergy - E[i]))
            hf.close()
            sample += 1
        secs_by_size[n] = sum(ts) / len(ts)
    est = sum(secs_by_size[n] * len(idx) for n, idx in by_size.items())
    res.update({"one_at_a_time_sample": "%d molecules: the first %d of every cluster size (%d sizes)"
                % (sample, per_size, len(by_size)),
                "one_at_a_time_seconds_estimated": est,
                "one_at_a_time_molecules_per_s": count / est,
                "one_at_a_time_seconds_by_size": {str(n): secs_by_size[n] for n in sorted(secs_by_size)},
                "max_abs_dE_batched_vs_single": dmax})
    res["speedup"] = res["batched_molecules_per_s"] / res["one_at_a_time_molecules_per_s"]
    return res
