#!/usr/bin/env python
"""Fock-build throughput of the direct two-electron contraction on B200.

Workload (default): RHF Fock build G[D] = 2J[D] - K[D] (``formPT``, reference
include/singleslater/singleslater_fock.h:31-93 -> newTwoEContractDirect) for a seeded
(H2O)_32 cluster at liquid density in cc-pVDZ (768 basis functions, quartet classes up to
(dd|dd)), Schwarz threshold 1e-14 (the reference default, include/aointegrals.h:334), on
the SAD-guess density.  One step = one Fock build over one density.  Metric: screened
unique shell quartets per second (the reference's loop unit, contract.h:96-131).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

The ``value`` leg times the device path (inputs resident in HBM, CUDA events on the
launching stream, L2 flushed between steps).  ``e2e`` times the same build through the C
ABI with host buffers (host->device and device->host copies inside the timed region).
On one GPU the line also carries, untimed by the contract:

* ``scf``: time to a converged SCF (|dE| <= 1 uEh) of (H2O)_32 cc-pVDZ for the plain FP64
  build (median of repeats), the mixed-precision incremental build with the FP32 cutoff
  swept 1e-10..1e-6, and the learned-guess arms, each with |dE| and max|dG| against FP64;
* ``scf_headline``: the same arms on (H2O)_64 cc-pVDZ, with the speed-ups with and without
  the relaxed mixed-phase screen;
* ``batch_scf``: 512 clusters (H2O)_n, n in 1..24, 6-31G(d), batched (CUDA graph, one
  launch per class and iteration) against one-at-a-time SCFs (stratified sample);
* ``cpu_baseline``: the oracle on the host cores, one residue class of the outer loop.

``--impl reference`` times the CPU restatement of the reference loop (the oracle; the
reference itself needs Libint and cannot be built here) on all host cores, with its input
density computed on the host as well: the timed steps are residue classes of the outer
shell index that together make up one whole Fock build.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    "h2o32-ccpvdz": dict(nwater=32, basis="cc-pvdz", seed=1, thresh=1e-14),
    "h2o8-ccpvdz": dict(nwater=8, basis="cc-pvdz", seed=1, thresh=1e-14),
    "h2o1-631gd": dict(nwater=1, basis="6-31g*", seed=0, thresh=1e-12),
    "h2o64-ccpvtz": dict(nwater=64, basis="cc-pvtz", seed=1, thresh=1e-14),
    "h2o64-ccpvdz": dict(nwater=64, basis="cc-pvdz", seed=1, thresh=1e-14),
}


def synthetic_density(bs, seed):
    """Seeded symmetric density with the distance decay of a molecular density matrix:
    D_mn = u_mn exp(-0.5 R_mn) (+1 on the diagonal), u uniform in [-1, 1], R_mn the
    distance in bohr between the centres of functions m and n."""
    rng = np.random.default_rng(seed)
    cent = np.concatenate([np.repeat(s.origin[None, :], s.size, axis=0) for s in bs.shells])
    R = np.linalg.norm(cent[:, None, :] - cent[None, :, :], axis=-1)
    u = rng.uniform(-1, 1, (bs.nbasis, bs.nbasis))
    D = 0.5 * (u + u.T) * np.exp(-0.5 * R)
    D[np.diag_indices_from(D)] += 1.0
    return np.ascontiguousarray(D)


def workload_geometry(name):
    """Molecule and basis of a named workload (host-only: no GPU code is loaded)."""
    from chronusq_public_b200.basis import BasisSet
    from chronusq_public_b200.molecule import water_cluster, single_water
    w = WORKLOADS[name]
    mol = single_water(w["seed"]) if w["nwater"] == 1 else water_cluster(w["nwater"], w["seed"])
    return w, mol, BasisSet(w["basis"], mol.atoms, mol.coords)


def build_workload(name, density="sad"):
    """Molecule, basis and the density of the benchmarked Fock build: the SAD-guess
    density of the SCF (atomic UHF densities, one Fock build, diagonalised; computed on
    the GPU) or, with density="synthetic", a seeded distance-decaying matrix."""
    w, mol, bs = workload_geometry(name)
    if density == "synthetic":
        D = synthetic_density(bs, 1234)
    else:
        from chronusq_public_b200.scf import SingleSlater
        hf = SingleSlater(mol, bs, thresholdSchwartz=w["thresh"])
        Ps, _, _, _ = hf.formGuess()
        D = np.ascontiguousarray(Ps.cpu().numpy())
        D = 0.5 * (D + D.T)
        hf.close()
    return w, mol, bs, D


def reference_workload(name, density="sad"):
    """The same workload built on the host alone for the reference arm: the SAD-guess
    density comes from the oracle's restatement of SingleSlater::formGuess (atomic UHF
    densities, one Fock build with the oracle's contraction, Loewdin diagonalisation), so
    the arm never loads the GPU library."""
    w, mol, bs = workload_geometry(name)
    if density == "synthetic":
        return w, mol, bs, synthetic_density(bs, 1234)
    from oracle import scf_ref
    return w, mol, bs, scf_ref.sad_guess_density(mol, bs, w["thresh"], nthreads=os.cpu_count())


def gpu_library_loaded():
    """Whether this process has mapped the engine's CUDA library (read from /proc)."""
    try:
        with open("/proc/self/maps") as f:
            return any("libcqgpu" in line for line in f)
    except OSError:
        return None


class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.lines = []
        if self.proc is not None:
            time.sleep(0.3)
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in getattr(self, "lines", []):
            f = [x.strip() for x in l.split(",")]
            try:
                sm.append(float(f[0]))
                mx = float(f[1])
            except (ValueError, IndexError):
                continue
            for n, v in zip(names, f[2:]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def max_over_ranks(x: float, pg=None, device="cuda") -> float:
    """The largest of every rank's `x` (a time: the job ends with its slowest replica);
    `x` itself on one rank.  `pg` is torch.distributed once initialised, else None."""
    if pg is None:
        return x
    import torch
    t = torch.tensor([x], device=device, dtype=torch.float64)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def oracle_build_part(ob, Q, D, thresh, modulus, residue, threads):
    """One residue class of the oracle's Fock build (RHF formPT lists: COULOMB 1, EXCHANGE
    -0.5): the quartets whose outermost shell index s1 satisfies s1 % modulus == residue.
    The `modulus` classes together are the whole loop of contract.h:96-193.  Returns
    (quartets, seconds)."""
    from oracle import oracle as O
    G = np.zeros_like(D, order="F")
    t0 = time.perf_counter()
    n = O.twoe_contract_direct(ob, [D, D], [G, G], [0, 1], [1.0, -0.5], thresh=thresh, Q=Q,
                               nthreads=threads, s1_residue=(modulus, residue))
    return n, time.perf_counter() - t0


_PRIMES = (5, 7, 11, 13, 17, 19, 23, 29, 31, 37, 41, 43, 47, 53, 59, 61)


def cpu_baseline(bs, D, thresh, target_s=15.0, nthreads=0):
    """Time the oracle (CPU restatement of the reference loop) on a bounded sample of the
    same workload: one residue class of the outermost shell index (s1 % K == 1).  K is a
    prime above 3, so that it shares no factor with the shells per molecule (12 for water
    in cc-pVDZ): the class then holds every shell type of every part of the cluster in
    equal measure.  K is chosen from a first class of 61 so that the sample takes about
    `target_s` seconds."""
    from oracle import oracle as O
    ob = O.OracleBasis.from_basis(bs)
    Q = O.schwarz(ob)
    Dm = np.asfortranarray(D)
    threads = nthreads or os.cpu_count()
    n0, t0 = oracle_build_part(ob, Q, Dm, thresh, 61, 0, threads)
    want = 61 * t0 / max(target_s, 1e-3)
    K = min(_PRIMES, key=lambda p: abs(p - want))
    n, dt = oracle_build_part(ob, Q, Dm, thresh, K, 1, threads)
    return {"value": n / dt, "unit": "quartets/s", "cores": threads, "kind": "port",
            "sample": "oracle restatement of newTwoEContractDirect (FP64 Obara-Saika/HGP, OpenMP), "
                      "quartets with s1 %% %d == 1 (one of %d residue classes of the outermost shell index; "
                      "%d is prime, so the class spans every shell type across the whole cluster): "
                      "%d quartets in %.2f s" % (K, K, K, n, dt),
            "quartets": n, "seconds": dt, "residue_classes": K}


def run_reference(args, ws, rank):
    """Reference arm: the CPU restatement of the reference loop (the reference needs Libint,
    which cannot be built here), on all host cores, with no GPU code loaded.  The timed
    steps split one full Fock build into `steps` residue classes of the outermost shell
    index (step k: s1 % steps == k), so together they are exactly one whole build; the
    warm-up steps run classes of 4 x steps."""
    if rank != 0:
        return
    from oracle import oracle as O
    w, mol, bs, D = reference_workload(args.workload, args.density)
    ob = O.OracleBasis.from_basis(bs)
    Q = O.schwarz(ob)
    Dm = np.asfortranarray(D)
    threads = os.cpu_count()
    K = max(1, args.steps)
    for j in range(args.warmup):
        oracle_build_part(ob, Q, Dm, w["thresh"], 4 * K, j % (4 * K), threads)
    times, counts = [], []
    for k in range(args.steps):
        n, dt = oracle_build_part(ob, Q, Dm, w["thresh"], K, k, threads)
        times.append(dt)
        counts.append(n)
    v = sum(counts) / sum(times)
    cfg = config_of(args, w, bs)
    cfg["density"] = ("SAD guess density, computed on the host by the oracle's restatement of "
                      "formGuess" if args.density == "sad" else cfg["density"])
    line = {"impl": "reference", "metric": "fock_build_quartets_per_s", "value": v, "unit": "quartets/s",
            "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * sum(times) / len(times), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": cfg,
            "quartets_per_build": sum(counts), "seconds_per_build": sum(times),
            "cpu_baseline": {"value": v, "unit": "quartets/s", "cores": threads, "kind": "port",
                             "sample": "oracle restatement of newTwoEContractDirect (no Libint here); timed step "
                                       "k runs the quartets with s1 %% %d == k, so the %d timed steps together "
                                       "are one whole Fock build (%d quartets)" % (K, args.steps, sum(counts))},
            "gpu_library_loaded": gpu_library_loaded(),
            "e2e": {"value": v, "unit": "quartets/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


FUSED_TIER1 = {"(ss|ss)", "(ps|ss)"}
WARP_TO_DD = {"(dp|pp)", "(dp|dp)", "(dd|pp)", "(dd|ds)", "(dd|dp)", "(dd|dd)"}   # warp-only classes to (dd|dd)


def schedule_summary(ints, st):
    """The autotuned schedule of the lists that had work: per class, the kernel form (one
    quartet per thread, warp-cooperative, or inside the class-fused kernel), CTAs per SM,
    warps per CTA, quartets claimed per warp and the class kernel's time; plus the fusion
    tier in use, the fused kernel's time and the autotuner's times of the three tiers."""
    sch = ints.schedule()
    tier, tuned = ints.fusion()
    out = {"fusion": {"tier": tier, "fused_kernel_ms": round(st.get("ms_fused", 0.0), 4),
                      "tuned_ms_tier0_1_2": [round(x, 4) for x in tuned]}}
    from chronusq_public_b200 import _lib
    lists = _lib.schedule_lists()
    sib = set(st.get("sibling_classes", []))
    for k, (name, nq) in enumerate(st["class_quartets"].items()):
        if nq <= 0:
            continue
        fused = (tier == 1 and name in FUSED_TIER1) or (tier == 2 and name not in WARP_TO_DD and "f" not in name)
        form = "fused" if fused else ("warp" if sch["warp_form"][k] else "thread")
        out[name] = {"form": form, "cta_per_sm": sch["cta_per_sm"][k], "warps_per_cta": sch["warps_per_cta"][k],
                     "quartets_per_warp": sch["quartets_per_warp"][k], "ms": round(st["class_ms"][name], 4)}
        if name in sib:   # the class's sibling-group list (its time is in the class's ms)
            b = lists.index(name + " siblings")
            out[name]["siblings"] = {"cta_per_sm": sch["cta_per_sm"][b], "quartets_per_warp": sch["quartets_per_warp"][b]}
    return out


def config_of(args, w, bs):
    return {"workload": args.workload, "molecule": "(H2O)_%d" % w["nwater"], "basis": w["basis"],
            "nbasis": bs.nbasis, "nshell": bs.nshell, "schwarz_threshold": w["thresh"],
            "density": ("SAD guess density (GPU SCF guess path)" if args.density == "sad"
                        else "seeded synthetic, distance-decaying"),
            "geometry": "seeded water cluster at 1.0 g/cm^3 (Poisson-disk O centres, min O-O 2.6 A)",
            "l2": "flushed between steps (256 MiB write)",
            "precision": "fp64", "parallelism": "replicas" if args.gpus > 1 else "single",
            "sibling_groups": getattr(args, "siblings", "off"),
            "launch_shapes": ("from %s" % os.path.basename(args.schedule_in) if getattr(args, "schedule_in", None)
                              else "default" if args.no_autotune else "autotuned in the first warm-up build")}


SCF_ARMS = ("plain", "mixed", "learned", "mixed_learned", "mixed_learned_context")


def max_dG_vs_fp64(ints, densities, mixed, cutoff, threshold, base_thresh):
    """max over `densities` of max|PT_arm[D] - PT_fp64[D]| (RHF formPT, 2J - K): the arm's
    builds (FP32 below `cutoff` when `mixed`, screened at `threshold`) against the all-FP64
    build at the context's threshold `base_thresh`.  The context is left in FP64 at
    `base_thresh`."""
    from chronusq_public_b200.aointegrals import PREC_FP64, PREC_MIXED
    worst = 0.0
    for D in densities:
        ints.setPrecision(PREC_FP64, 0.0)
        ints.thresholdSchwartz = base_thresh
        ref, _ = ints.formPT(D)
        if mixed:
            ints.setPrecision(PREC_MIXED, cutoff)
        ints.thresholdSchwartz = threshold
        got, _ = ints.formPT(D)
        worst = max(worst, float((got - ref).abs().max()))
    ints.setPrecision(PREC_FP64, 0.0)
    ints.thresholdSchwartz = base_thresh
    return worst


def scf_compare(mol, bs, thresh, cutoff, sweep=(), autotune=True, arms=SCF_ARMS, plain_repeats=1):
    """Time to converged SCF: plain FP64 GPU build vs mixed precision + incremental build,
    each with the SAD and the learned guess.  Times include the guess (atomic SCFs cached
    beforehand) and every iteration.  The plain arm runs `plain_repeats` times and its
    median time to 1 uEh is the reference of the speed-ups (its DIIS path varies from run
    to run).  Every arm reports |dE| against the FP64 energy and max|dG|: the largest
    element of PT_arm[D] - PT_fp64[D] over the SAD-guess density and the converged FP64
    density, with the arm's precision, FP32 cutoff and screening threshold.  `arms` picks a
    subset; without the plain arm, each arm's time to 1 uEh is measured against its own
    converged energy (the final phase of every arm is FP64 at the context's threshold)."""
    import torch
    from chronusq_public_b200.scf import SingleSlater
    warm = SingleSlater(mol, bs, thresholdSchwartz=thresh)
    Pg, Pzg, _, _ = warm.formGuess()      # atomic SAD densities cached, kernels warm
    if autotune:
        warm.ints.autotune_next()         # launch shapes tuned on one full build, shared by every arm
        warm.formPT(Pg, Pzg)
    ints = warm.ints
    out, E64, dens = {}, None, [Pg]
    if "plain" in arms:
        runs = []
        for _ in range(max(1, plain_repeats)):
            plain = SingleSlater(mol, bs, ints=ints)
            E = plain.SCF3()
            runs.append({"energy": E, "iterations": plain.nSCFIter, "seconds": plain.scf_seconds,
                         "seconds_to_1uEh": plain.time_to(E, 1e-6), "fock_builds": plain.fock_builds,
                         "fock_seconds": plain.fock_seconds})
            if E64 is None:
                E64 = E
                dens.append(plain.onePDMScalar.clone())
        t1 = [r["seconds_to_1uEh"] for r in runs]
        out["plain_fp64"] = dict(runs[0])
        out["plain_fp64"].update({"repeats": len(runs), "seconds_to_1uEh": statistics.median(t1),
                                  "seconds_to_1uEh_each": t1, "energy_spread": max(r["energy"] for r in runs) -
                                  min(r["energy"] for r in runs)})
    else:
        out["reference_energy"] = "each arm's own converged energy (no plain FP64 arm run)"

    def record(hf, E, extra, mixed, c, mthr):
        ref = E if E64 is None else E64
        r = {"energy": E, "iterations": hf.nSCFIter, "seconds": hf.scf_seconds,
             "seconds_to_1uEh": hf.time_to(ref, 1e-6)}
        if E64 is not None:
            r["abs_dE_vs_fp64"] = abs(E - E64)
        thr = thresh if (mthr is None or not mixed) else max(thresh, mthr)
        r["max_abs_dG_vs_fp64"] = max_dG_vs_fp64(ints, dens, mixed, c, thr, thresh)
        r["mixed_phase_threshold"] = thr if mixed else None
        r.update(extra)
        return r

    if "mixed" in arms:
        runs = {}
        for c in sorted(set([cutoff] + list(sweep))):
            mx = SingleSlater(mol, bs, ints=ints)
            mx.precision, mx.fp32_cutoff, mx.incremental = "mixed", c, True
            E = mx.SCF3()
            runs["%.0e" % c] = record(mx, E, {"fp32_quartets": mx.fp32_quartets,
                                              "fp64_switch_iteration": mx.phase_switch_iter,
                                              "fp32_cutoff": c}, True, c, mx.mixed_threshold)
            runs["%.0e" % c]["max_abs_dG_fp32_only"] = max_dG_vs_fp64(ints, dens, True, c, thresh, thresh)
        out["mixed_incremental"] = runs["%.0e" % cutoff]
        if sweep:
            out["cutoff_sweep"] = runs
    # learned initial density (network trained on this engine's converged cluster densities)
    from chronusq_public_b200.guess_model import PairMLP, default_weights
    wpath, source = default_weights(bs.name), None
    if wpath is None and default_weights("cc-pvdz"):
        # no network for this basis: predict in cc-pVDZ and project the density
        wpath, source = default_weights("cc-pvdz"), "cc-pvdz"
    if wpath:
        net = PairMLP.load(wpath)
        # the last arm keeps the context's threshold in the mixed phase too: what the relaxed
        # mixed-phase screening contributes
        for arm, key, mixed, mthr in (("learned", "learned_fp64", False, None),
                                      ("mixed_learned", "mixed_incremental_learned", True, 1e-11),
                                      ("mixed_learned_context", "mixed_incremental_learned_context_threshold",
                                       True, None)):
            if arm not in arms:
                continue
            lg = SingleSlater(mol, bs, ints=ints)
            lg.guess, lg.guess_model, lg.guess_source_basis = "LEARNED", net, source
            if mixed:
                lg.precision, lg.fp32_cutoff, lg.incremental, lg.mixed_threshold = "mixed", cutoff, True, mthr
            E = lg.SCF3()
            out[key] = record(lg, E, {"guess_used": lg.guess_used, "weights": os.path.basename(wpath),
                                      "guess_projected_from": source}, mixed, cutoff, mthr)
    t_plain = out.get("plain_fp64", {}).get("seconds_to_1uEh")
    for key, name in (("mixed_incremental", "speedup_time_to_1uEh_mixed"),
                      ("learned_fp64", "speedup_time_to_1uEh_learned"),
                      ("mixed_incremental_learned", "speedup_time_to_1uEh_mixed_learned"),
                      ("mixed_incremental_learned_context_threshold",
                       "speedup_time_to_1uEh_mixed_learned_without_relaxed_screen")):
        t = out.get(key, {}).get("seconds_to_1uEh")
        if t_plain and t:
            out[name] = t_plain / t
    out["speedup_reference"] = "median of the plain FP64 arm's repeats"
    warm.close()
    torch.cuda.synchronize()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="h2o32-ccpvdz", choices=sorted(WORKLOADS))
    ap.add_argument("--ref-seconds", type=float, default=12.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--class-table", action="store_true", help="print per-class times to stderr")
    ap.add_argument("--density", default="sad", choices=["sad", "synthetic"])
    ap.add_argument("--no-scf", action="store_true", help="skip the time-to-converged-SCF comparison")
    ap.add_argument("--fp32-cutoff", type=float, default=1e-8)
    ap.add_argument("--no-sweep", action="store_true", help="skip the FP32 cutoff sweep 1e-10..1e-6")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer end-to-end leg")
    ap.add_argument("--no-autotune", action="store_true", help="default launch shapes instead of autotuned ones")
    ap.add_argument("--siblings", default="off", choices=["on", "off"],
                    help="sibling-group lists for the segmented shells of one general contraction")
    ap.add_argument("--sibling-min", default="",
                    help="per sibling class, the member quartets a sibling entry holds at least, e.g. '(ss|ss)=8,(ps|ss)=4'")
    ap.add_argument("--fusion", default="auto", choices=["auto", "0", "1", "2"],
                    help="class-fusion tier of the benchmarked builds (auto: the autotuner's choice)")
    ap.add_argument("--schedule-out", default=None, help="write the autotuned per-list schedule to this JSON file")
    ap.add_argument("--schedule-in", default=None,
                    help="use the per-list schedule in this JSON file (from --schedule-out) instead of autotuning")
    ap.add_argument("--scf-arms", default=",".join(SCF_ARMS),
                    help="comma-separated SCF arms to run (%s)" % ", ".join(SCF_ARMS))
    ap.add_argument("--plain-repeats", type=int, default=3, help="runs of the plain FP64 SCF arm (median)")
    ap.add_argument("--headline", default="h2o64-ccpvdz", choices=sorted(WORKLOADS) + ["none"],
                    help="workload of the headline SCF comparison (all arms), 'none' to skip")
    ap.add_argument("--batch", type=int, default=512,
                    help="molecules of the batched-SCF comparison ((H2O)_n, n in 1..24, 6-31G(d)); 0 skips it")
    ap.add_argument("--batch-per-size", type=int, default=2,
                    help="molecules per cluster size converged one at a time (stratified sample)")
    args = ap.parse_args()
    bad = [a for a in args.scf_arms.split(",") if a not in SCF_ARMS]
    if bad:
        ap.error("unknown SCF arm(s): %s" % ", ".join(bad))
    ws, rank, local = dist_setup()
    if args.impl == "reference":
        return run_reference(args, ws, rank)

    import torch
    torch.cuda.set_device(local)
    pg = None
    if ws > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
        pg = dist
    from chronusq_public_b200.aointegrals import AOIntegrals, probe_fma_peak
    from chronusq_public_b200 import _lib

    w, mol, bs, D = build_workload(args.workload, args.density)
    n = bs.nbasis
    ints = AOIntegrals(bs, device=local, thresholdSchwartz=w["thresh"])
    ints.setSiblings(args.siblings == "on")
    for item in filter(None, args.sibling_min.split(",")):
        cls, m = item.split("=")
        ints.setSiblingMin(cls.strip(), int(m))
    Dd = torch.from_numpy(D).cuda()
    PT = torch.zeros_like(Dd)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream()

    if args.schedule_in:
        sch = json.load(open(args.schedule_in))
        ints.setSchedule(**{k: sch[k] for k in ("cta_per_sm", "warps_per_cta", "quartets_per_warp", "warp_form")})
        ints.setFusion(int(sch.get("fusion_tier", 0)))
    elif not args.no_autotune:
        ints.autotune_next()              # the first warm-up build picks every class's launch shape
    for i in range(args.warmup):
        ints.formPT(Dd, PTs=PT)
        if i == 0 and args.fusion != "auto":
            ints.setFusion(int(args.fusion))
    torch.cuda.synchronize()
    if args.schedule_out and rank == 0:
        with open(args.schedule_out, "w") as f:
            json.dump(dict(ints.schedule(), fusion_tier=ints.fusion()[0]), f)
    ints.setTiming(True)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    step_ms, eri_ms, quartets, mflops, launches, class_ms, screen_ms = [], [], [], [], 0, {}, []
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        torch.cuda.nvtx.range_push("timed")      # lets a profiler keep only the timed steps
        for k in range(args.steps):
            flush.zero_()
            ev[k][0].record(stream)
            ints.formPT(Dd, PTs=PT)
            ev[k][1].record(stream)
            st = ints.stats()
            quartets.append(st["quartets"])
            mflops.append(st["model_flops"])
            eri_ms.append(st["ms_eri"])
            screen_ms.append(st["ms_screen"])
            launches += st["launches"]
            for c, v in st["class_ms"].items():
                class_ms[c] = class_ms.get(c, 0.0) + v / args.steps
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_pop()
    if pg:
        pg.barrier()
    ints.setTiming(False)
    step_ms = [a.elapsed_time(b) for a, b in ev]
    tot_ms = max_over_ranks(sum(step_ms), pg)
    value = ws * sum(quartets) / (tot_ms * 1e-3)      # replicas: every rank builds the same workload
    st_last = ints.stats()

    # end to end through the C ABI with pinned host buffers
    Dh = torch.from_numpy(D).pin_memory()
    PTh = torch.zeros_like(Dh).pin_memory()
    L = _lib.lib()
    e2e_t = []
    for k in range(0 if args.no_e2e else args.warmup + args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        rc = L.cqg_form_pt(ints._ctx, 1, -0.5, ctypes.c_void_p(Dh.data_ptr()), None,
                           ctypes.c_void_p(PTh.data_ptr()), None, n, 0, ctypes.c_void_p(stream.cuda_stream))
        _lib.check(rc, ints._ctx)
        t1 = time.perf_counter()
        if k >= args.warmup:
            e2e_t.append(t1 - t0)
    e2e_val = ws * quartets[0] * len(e2e_t) / max_over_ranks(sum(e2e_t), pg) if e2e_t else None
    err = float(np.abs(PTh.numpy() - PT.cpu().numpy()).max()) if e2e_t else None

    if rank == 0:
        peak64 = probe_fma_peak(True, 100.0, local)
        eri_s = sum(eri_ms) / len(eri_ms) * 1e-3
        achieved = (sum(mflops) / len(mflops)) / eri_s / 1e12
        # DRAM bytes per build of the ERI kernels: the per-quartet figure of an ncu capture of
        # this workload (SAD density, autotuned schedule; profiles/traffic.json) times this
        # step's quartets; null for a workload or density that was not captured
        traffic, traffic_src = None, "no ncu capture of this workload"
        tj = os.path.join(ROOT, "profiles", "traffic.json")
        if os.path.exists(tj) and args.density == "sad":
            try:
                tr = json.load(open(tj)).get(args.workload)
                if tr:
                    traffic = tr["bytes_per_quartet"] * quartets[0]
                    traffic_src = tr.get("source", "profiles/traffic.json")
            except (ValueError, KeyError):
                traffic = None
        line = {
            "metric": "fock_build_quartets_per_s", "value": value, "unit": "quartets/s", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": tot_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": config_of(args, w, bs),
            "quartets_per_step": quartets[0], "fock_builds_per_s": 1e3 * args.steps / tot_ms,
            "screen_ms_per_step": sum(screen_ms) / len(screen_ms),
            "list_entries_per_step": st_last["list_entries"],
            "e2e": {"value": e2e_val, "unit": "quartets/s", "h2d_bytes_per_step": 2 * n * n * 8,
                    "d2h_bytes_per_step": n * n * 8, "max_abs_diff_vs_device_path": err},
            "roofline": {"bound": "fp64", "kernel": "k_eri_jk (all quartet classes, ERI + J/K digest)",
                         "achieved": achieved, "peak": peak64, "unit": "TFLOP/s", "frac": achieved / peak64,
                         "peak_source": "measured: FP64 FMA-chain probe (cqg_probe_fma_peak) on this GPU",
                         "flop_model": "MD-v1 (model FLOPs of the screened quartets)",
                         "model_flops_per_step": mflops[0], "eri_ms_per_step": eri_s * 1e3,
                         "traffic": traffic, "traffic_source": traffic_src},
            "gpu_launches": launches,
            "clocks": clk.summary(),
            "schedule": schedule_summary(ints, st_last),
        }
        extras = ws == 1                   # replicas (N > 1) report the Fock-build line only
        if extras and not args.no_scf:
            line["scf"] = scf_compare(mol, bs, w["thresh"], args.fp32_cutoff,
                                      sweep=() if args.no_sweep else (1e-10, 1e-9, 1e-8, 1e-7, 1e-6),
                                      autotune=not args.no_autotune, arms=args.scf_arms.split(","),
                                      plain_repeats=args.plain_repeats)
            if args.headline != "none" and args.headline != args.workload:
                hw, hmol, hbs = workload_geometry(args.headline)
                line["scf_headline"] = {"workload": args.headline, "nbasis": hbs.nbasis}
                line["scf_headline"].update(scf_compare(hmol, hbs, hw["thresh"], args.fp32_cutoff,
                                                        autotune=not args.no_autotune,
                                                        arms=args.scf_arms.split(","),
                                                        plain_repeats=args.plain_repeats))
        if extras and not args.no_scf:
            from chronusq_public_b200.learned_guess import training_throughput
            line["guess_training"] = training_throughput(epochs=2)
        if extras and args.batch > 0:
            from chronusq_public_b200.workloads import batch_scf_comparison
            line["batch_scf"] = batch_scf_comparison(args.batch, args.batch_per_size)
        if extras and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(bs, D, w["thresh"], target_s=args.ref_seconds)
        print(json.dumps(line), flush=True)
        if args.class_table:
            for c, v in sorted(class_ms.items(), key=lambda kv: -kv[1]):
                if v > 0:
                    print("%-8s %9.3f ms  %12d quartets" % (c, v, st_last["class_quartets"][c]), file=sys.stderr)
    ints.close()
    if pg:
        pg.barrier()
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
