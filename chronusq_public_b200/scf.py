"""Device-resident Hartree-Fock SCF around the two-electron engine.

Restates the reference's ``SingleSlater<double>`` SCF (include/singleslater/*.h) with
every matrix on the GPU (torch FP64 tensors: cuBLAS GEMMs, cuSOLVER ``syevd``) and the
Fock builds through :class:`~chronusq_public_b200.aointegrals.AOIntegrals`:

* Fock assembly (singleslater_fock.h:100-274): F_s = 2h + PTs, F_z = PTz; PT from formPT
  (fock.h:31-93).
* Orthonormal basis: Loewdin X = S^-1/2 (AOIntegrals::computeLowdin,
  src/aointegrals/aointegrals_builders.cpp:736-769); FO = X^T F X (orthoFock3,
  scfutils.h:149-168); D = X DO X^T (unOrthoDen3).
* Diagonalisation of 0.5 (FO_s +- FO_z) (populateMO4Diag / diagFock2,
  src/singleslater/singleslater_real_scf.cpp:71-108); densities P_sigma = C_occ C_occ^T,
  Ps = Pa + Pb, Pz = Pa - Pb (formDensity, misc.h:28-55).
* Commutator DIIS on [FO, DO] (genDIISCom / CDIIS4, diis.h:35-157; DIIS::extrapolate,
  extrapolate.h:26-141), extrapolating both F and PT, falling back to a plain step when
  the DIIS system is singular; SCF declared converged when the commutator norm drops
  below 5e eps (diis.h:103-157).
* Fock damping with parameter 0.1 against the previous orthonormal Fock, switched off
  once |dE| < 1e-6 and back on if |dE| grows above it (fockDamping / evalConver3,
  scfutils.h:262-355, 1065-1111).
* Convergence: |dE| < eneTol (1e-10) and ||dPs|| (and ||dPz||) < denTol (1e-8)
  (evalConver3, defaults singleslater.h:445-495).
* Energy: E = Tr(Ps h) + 1/4 [Tr(Ps PTs) + Tr(Pz PTz)] + E_nuc
  (singleslater_properties.h:26-110).
* Guesses: SAD -- an atomic UHF per unique element (core guess, no DIIS), densities
  placed block-diagonally, spin-averaged, one molecular Fock build, diagonalised
  (singleslater_guess.h:100-264); CORE -- the core Hamiltonian diagonalised; or an
  explicit density (the READ guess, guess.h:320-329).  LEARNED (no reference
  counterpart) starts the iterations from the density predicted by guess_model.PairMLP,
  projected on its natural orbitals, falling back to SAD when the prediction is
  unphysical; the converged energy does not depend on the guess.

* Static electric field (setField; singleslater_fock.h:215, aointegrals.h:505-510,
  singleslater_properties.h:95-101): h + F.<r> and E_nuc - F.mu_nuc, origin 0.
* Mixed precision (no reference counterpart): FP32 quartets below ``fp32_cutoff``,
  incremental Delta-D builds and a looser screen (``mixed_threshold``) until the DIIS
  error falls below ``fp64_switch``; then FP64 at the context's threshold, from a full
  rebuild, so the converged energy is the FP64 one.

The per-iteration HDF5 traffic of the reference (writeSCFFiles, scfutils.h:1114-1188) has
no counterpart: all state stays in device memory.
"""
from __future__ import annotations

import math
import time
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

from .aointegrals import AOIntegrals
from .basis import BasisSet
from .molecule import Molecule

# ChronusQ element default multiplicities (atomic SAD references), H..Ne
DEFAULT_MULT = {1: 2, 2: 1, 3: 2, 4: 1, 5: 2, 6: 3, 7: 4, 8: 3, 9: 2, 10: 1}


@dataclass
class SCFIteration:
    iteration: int
    energy: float
    delta_e: float
    ps_rms: float
    pz_rms: float
    t: float           # seconds since the SCF (guess included) started, device-synchronised


class SingleSlater:
    """RHF / UHF SCF on one GPU (reference names kept where they exist)."""

    def __init__(self, mol: Molecule, basis: BasisSet, ref: str = "RHF", device: int = 0,
                 thresholdSchwartz: float = 1e-14, ints: Optional[AOIntegrals] = None, field=None):
        import torch
        self.torch = torch
        self.mol = mol
        self.basis = basis
        self.ref = ref.upper()
        if self.ref not in ("RHF", "UHF"):
            raise ValueError("reference must be RHF or UHF")
        self.isClosedShell = self.ref == "RHF"
        self.dev = torch.device("cuda", device)
        self.ints = ints if ints is not None else AOIntegrals(basis, device=device, thresholdSchwartz=thresholdSchwartz)
        ne = mol.nelectrons
        if self.isClosedShell:
            if ne % 2 or mol.mult != 1:
                raise ValueError("RHF needs a closed-shell singlet")
            self.nOA = self.nOB = ne // 2
        else:
            self.nOA = (ne + mol.mult - 1) // 2
            self.nOB = ne - self.nOA
        # settings (SingleSlater defaults, singleslater.h:445-495; nDIISExtrap set for DIIS(6))
        self.denTol = 1e-8
        self.eneTol = 1e-10
        self.maxSCFIter = 256
        self.doDIIS = True
        self.nDIISExtrap = 6
        self.doDamp = True
        self.dampParam = 0.1
        self.xHF = -0.5
        self.guess = "SAD"             # "SAD", "CORE" or "LEARNED" (needs guess_model)
        self.guess_model = None
        self.guess_source_basis = None   # basis the guess network predicts in (None: this one)
        self.guess_used = None
        # mixed precision + incremental (Delta D) Fock build
        self.precision = "fp64"        # "fp64" or "mixed"
        self.fp32_cutoff = 1e-8        # density-weighted Schwarz bound below which a quartet runs in FP32
        self.incremental = False       # build PT_k = PT_{k-1} + G[D_k - D_{k-1}]
        self.nIncFock = 20             # full rebuild period of the incremental build (singleslater.h:468)
        self.fp64_switch = 1e-5        # DIIS error below which the builds return to FP64 at the
                                       # context's threshold (a full FP64 build follows, at the
                                       # switch or at convergence: see SCF3)
        self.mixed_threshold = 1e-11   # density-weighted Schwarz threshold of the mixed-phase
                                       # builds (never tighter than the context's; None: the
                                       # context's threshold throughout)
        self._base_threshold = None    # the context's own threshold while an SCF runs
        self.n = basis.nbasis
        self.log: List[SCFIteration] = []
        self.fock_builds = 0
        self.fock_seconds = 0.0
        self.elecField = None          # static electric field (a.u.), None: no field
        self._one_e()
        if field is not None:
            self.setField(field)

    # ------------------------------------------------------------------ setup ---
    def _one_e(self):
        t = self.torch
        S, T, V = self.ints.computeAOOneE(self.mol.atoms, self.mol.coords, device_out=True)
        self.overlap = S
        self._H0 = T + V
        self.coreH = self._H0
        w, U = t.linalg.eigh(S)
        self.X = (U * w.rsqrt()) @ U.T          # Loewdin S^-1/2 (symmetric)
        self.Enuc = self.mol.nuclear_repulsion()

    def setField(self, field):
        """Static electric field F (a.u., origin 0) for the SCF (SingleSlater::setField,
        singleslater.h:633-637).  The one-electron Hamiltonian becomes h + F.<r> and the
        energy gains -F.mu_nuc: the reference subtracts F times its dipole integrals, which
        carry the electron's charge, from the Fock matrix (AOIntegrals::subElecDipole,
        aointegrals.h:505-510) and adds F.mu to the energy (singleslater_properties.h:95-101).
        A zero field is no field, as in the reference.  The SAD atoms see no field (the
        reference's setField call for them is commented out, singleslater_guess.h:185)."""
        F = None if field is None else [float(x) for x in field]
        if F is not None and len(F) != 3:
            raise ValueError("the field has three components")
        if F is not None and not any(F):
            F = None
        self.elecField = F
        self.coreH = self._H0
        self.Enuc = self.mol.nuclear_repulsion()
        if F is not None:
            D = self.ints.computeDipole(device_out=True)
            self.coreH = self._H0 + F[0] * D[0] + F[1] * D[1] + F[2] * D[2]
            self.Enuc -= float(np.dot(F, self._nuclear_dipole()))

    def _nuclear_dipole(self) -> np.ndarray:
        Z = np.asarray(self.mol.atoms, dtype=np.float64)
        return Z @ np.asarray(self.mol.coords, dtype=np.float64).reshape(-1, 3)

    def dipoleMoment(self) -> np.ndarray:
        """Dipole moment (a.u., origin 0) of the current density: sum_A Z_A R_A - Tr(Ps <r>)
        (SingleSlater::computeMultipole, singleslater_properties.h:115-130)."""
        D = self.ints.computeDipole(device_out=True)
        Ps = self.onePDMScalar
        el = [float(self.torch.sum(Ps * D[k])) for k in range(3)]
        return self._nuclear_dipole() - np.asarray(el)

    # ------------------------------------------------------------------ pieces ---
    def _mixed_threshold_active(self) -> bool:
        """True when the mixed phase screens at a looser threshold than the context's."""
        base = self.ints.thresholdSchwartz if self._base_threshold is None else self._base_threshold
        return self.mixed_threshold is not None and self.mixed_threshold > base

    def _set_precision(self, mixed: bool):
        from .aointegrals import PREC_FP64, PREC_MIXED
        if self._base_threshold is None:
            self._base_threshold = self.ints.thresholdSchwartz
        if mixed:
            self.ints.setPrecision(PREC_MIXED, self.fp32_cutoff)
            if self._mixed_threshold_active():
                self.ints.thresholdSchwartz = self.mixed_threshold
        else:
            self.ints.setPrecision(PREC_FP64, 0.0)
            self.ints.thresholdSchwartz = self._base_threshold

    def formPT(self, Ps, Pz=None):
        t0 = time.perf_counter()
        PTs, PTz = self.ints.formPT(Ps, None if self.isClosedShell else Pz, xHF=self.xHF)
        self.torch.cuda.synchronize(self.dev)
        self.fock_seconds += time.perf_counter() - t0
        self.fock_builds += 1
        if PTz is None:
            PTz = self.torch.zeros_like(PTs)
        return PTs, PTz

    def formFock(self, Ps, Pz):
        PTs, PTz = self.formPT(Ps, Pz)
        Fs = 2.0 * self.coreH + PTs
        Fz = PTz.clone()
        return Fs, Fz, PTs, PTz

    def computeEnergy(self, Ps, Pz, PTs, PTz) -> float:
        t = self.torch
        e1 = t.sum(Ps * self.coreH)
        e2 = 0.25 * (t.sum(Ps * PTs) + t.sum(Pz * PTz))
        return float(e1 + e2) + self.Enuc

    def _ortho(self, F):
        return self.X.T @ F @ self.X

    def _unortho(self, DO):
        return self.X @ DO @ self.X.T

    def _diag_density(self, FOs, FOz):
        """diagFock2 + formDensity in the orthonormal basis: returns (DOs, DOz)."""
        t = self.torch
        if self.isClosedShell:
            _, C = t.linalg.eigh(0.5 * FOs)
            Co = C[:, :self.nOA]
            DOa = Co @ Co.T
            return 2.0 * DOa, t.zeros_like(DOa)
        _, Ca = t.linalg.eigh(0.5 * (FOs + FOz))
        _, Cb = t.linalg.eigh(0.5 * (FOs - FOz))
        DOa = Ca[:, :self.nOA] @ Ca[:, :self.nOA].T
        DOb = Cb[:, :self.nOB] @ Cb[:, :self.nOB].T
        return DOa + DOb, DOa - DOb

    # ------------------------------------------------------------------ guesses ---
    def _core_guess(self):
        FOs = self._ortho(2.0 * self.coreH)
        DOs, DOz = self._diag_density(FOs, self.torch.zeros_like(FOs))
        return self._unortho(DOs), self._unortho(DOz), FOs, self.torch.zeros_like(FOs)

    def _sad_density(self):
        """Block-diagonal superposition of atomic UHF densities (SADGuess, guess.h:100-222)."""
        t = self.torch
        Ps = t.zeros((self.n, self.n), dtype=t.float64, device=self.dev)
        Pz = t.zeros_like(Ps)
        offs = {}
        off = 0
        for s in self.basis.shells:
            offs.setdefault(s.atom, [off, 0])
            offs[s.atom][1] += s.size
            off += s.size
        cache = {}
        for a, z in enumerate(self.mol.atoms):
            if z not in cache:
                cache[z] = atomic_density(z, self.basis.name, self.dev.index, self.ints.thresholdSchwartz)
            b0, nb = offs[a]
            Ps[b0:b0 + nb, b0:b0 + nb] = cache[z][0]
            Pz[b0:b0 + nb, b0:b0 + nb] = cache[z][1]
        if not self.isClosedShell:   # spinAverage (guess.h:287-292)
            Pz = (self.nOA - self.nOB) / (self.nOA + self.nOB) * Ps
        return Ps, Pz

    def _learned_density(self):
        """Density predicted by ``self.guess_model`` (a guess_model.PairMLP), projected on
        its natural orbitals: the nOA (and nOB) eigenvectors of largest occupation of the
        orthonormal-basis density are occupied, which gives the idempotent density with
        the right electron counts nearest the prediction.  None when the prediction is not
        finite or its Tr(PS) is more than 10 % off the electron count."""
        from .guess_model import predict_density, project_density
        t = self.torch
        src = self.guess_source_basis
        if src and src.lower() != self.basis.name.lower():
            # the network was trained in another basis: predict there, project here
            bs_src = BasisSet(src, self.mol.atoms, self.mol.coords)
            P = project_density(predict_density(self.guess_model, self.mol, bs_src), bs_src, self.basis,
                                self.dev.index)
        else:
            P = t.as_tensor(predict_density(self.guess_model, self.mol, self.basis), dtype=t.float64,
                            device=self.dev)
        ne = float(t.sum(P * self.overlap))
        nel = self.mol.nelectrons
        if not math.isfinite(ne) or abs(ne - nel) > 0.1 * nel:
            return None
        DO = self.X.T @ self.overlap @ P @ self.overlap @ self.X
        DOs, DOz = self._diag_density(-DO, t.zeros_like(DO))
        return self._unortho(DOs), self._unortho(DOz)

    def formGuess(self, density=None):
        """Returns (Ps, Pz, FOs, FOz): the starting density and the orthonormal Fock it
        came from (the damping reference of the first iteration)."""
        t = self.torch
        if density is not None:                           # READ guess
            Ps, Pz = density
            Ps = t.as_tensor(Ps, dtype=t.float64, device=self.dev)
            Pz = t.zeros_like(Ps) if Pz is None else t.as_tensor(Pz, dtype=t.float64, device=self.dev)
            Fs, Fz, _, _ = self.formFock(Ps, Pz)
        elif self.guess == "CORE" or self.mol.natoms <= 1:
            return self._core_guess()
        elif self.guess == "SAD":
            Ps, Pz = self._sad_density()
            Fs, Fz, _, _ = self.formFock(Ps, Pz)
        elif self.guess == "LEARNED":
            # the projected prediction is the first iterate itself: no guess Fock build,
            # and no damping reference for the first iteration
            pred = self._learned_density()
            self.guess_used = "SAD" if pred is None else "LEARNED"
            if pred is not None:
                return pred[0], pred[1], None, None
            Ps, Pz = self._sad_density()
            Fs, Fz, _, _ = self.formFock(Ps, Pz)
        else:
            raise ValueError("unknown guess %r" % self.guess)
        FOs, FOz = self._ortho(Fs), self._ortho(Fz)
        DOs, DOz = self._diag_density(FOs, FOz)
        return self._unortho(DOs), self._unortho(DOz), FOs, FOz

    # ------------------------------------------------------------------ SCF ---
    def SCF3(self, density=None, on_iteration=None):
        """Run the SCF; returns the converged total energy (Eh)."""
        t = self.torch
        t.cuda.synchronize(self.dev)
        t0 = time.perf_counter()
        self.log = []
        self._set_precision(self.precision == "mixed")
        Ps, Pz, FOs_prev, FOz_prev = self.formGuess(density)
        Eold = 0.0
        self.converged = False
        hist_F, hist_PT, hist_E = [], [], []
        diis_on = self.doDIIS
        damp = self.dampParam if self.doDamp else 0.0
        xsmall = np.finfo(float).eps * 10 * 5
        mixed_phase = self.precision == "mixed"
        self._set_precision(mixed_phase)
        built = None            # (Ps, Pz, PTs, PTz) of the last build, for Delta D
        since_full = 0
        self.phase_switch_iter = None
        rebuild_pending = False
        reset_diis_next = False
        self.fp32_quartets = 0
        for it in range(self.maxSCFIter):
            if self.incremental and built is not None and since_full < self.nIncFock:
                dPs, dPz = Ps - built[0], Pz - built[1]
                dPTs, dPTz = self.formPT(dPs, dPz)
                PTs, PTz = built[2] + dPTs, built[3] + dPTz
                since_full += 1
            else:
                PTs, PTz = self.formPT(Ps, Pz)
                since_full = 0
            if mixed_phase:
                self.fp32_quartets += self.ints.stats()["quartets_fp32"]
            built = (Ps, Pz, PTs, PTz)
            if reset_diis_next:
                hist_F, hist_PT, hist_E = [], [], []
                reset_diis_next = False
            Fs = 2.0 * self.coreH + PTs
            Fz = PTz.clone()
            FOs, FOz = self._ortho(Fs), self._ortho(Fz)
            DOs = self.X.T @ self.overlap @ Ps @ self.overlap @ self.X   # orthonormal density
            DOz = self.X.T @ self.overlap @ Pz @ self.overlap @ self.X
            if self.isClosedShell:
                es = FOs @ DOs
                errs = [es - es.T]
            else:   # [F_a, P_a] and [F_b, P_b] with F_a,b = (Fs +- Fz)/2, P_a,b = (Ps +- Pz)/2
                ea = 0.25 * (FOs + FOz) @ (DOs + DOz)
                eb = 0.25 * (FOs - FOz) @ (DOs - DOz)
                errs = [ea - ea.T, eb - eb.T]
            cnorm = max(float(t.linalg.norm(e)) for e in errs)
            fp_converged = cnorm < xsmall
            if mixed_phase and cnorm < self.fp64_switch:
                # last iterations in FP64 at the context's threshold.  When the mixed phase
                # screened at a looser threshold, its PT carries the skipped quartets (about
                # 1e-7 Eh in the energy at 1e-11): the next build is a full FP64 one and DIIS
                # restarts from it, so no loose Fock matrix is extrapolated with the exact ones.
                # Otherwise (FP32 rounding only) incremental builds continue in FP64 from the
                # current PT, and the converged density is confirmed on one full FP64 build
                # (convergence is tested again on it), so the exact rebuild is not paid while
                # the SCF is still converging.
                loose = self._mixed_threshold_active()
                mixed_phase = False
                self._set_precision(False)
                self.phase_switch_iter = it
                if self.incremental and not loose:
                    rebuild_pending = True
                else:
                    built = None
                reset_diis_next = loose
            if diis_on:
                hist_F.append((Fs, Fz))
                hist_PT.append((PTs, PTz))
                hist_E.append(errs)
                if len(hist_F) > self.nDIISExtrap:
                    hist_F.pop(0)
                    hist_PT.pop(0)
                    hist_E.pop(0)
                m = len(hist_F)
                if it > 0 and m > 1 and not fp_converged:
                    c = self._diis_coefficients(hist_E)
                    if c is not None:
                        k0 = len(hist_F) - len(c)
                        Fs = sum(c[i] * hist_F[k0 + i][0] for i in range(len(c)))
                        Fz = sum(c[i] * hist_F[k0 + i][1] for i in range(len(c)))
                        PTs = sum(c[i] * hist_PT[k0 + i][0] for i in range(len(c)))
                        PTz = sum(c[i] * hist_PT[k0 + i][1] for i in range(len(c)))
                        FOs, FOz = self._ortho(Fs), self._ortho(Fz)
            if fp_converged:
                diis_on = False
            if damp > 0.0 and FOs_prev is not None:
                FOs = (1.0 - damp) * FOs + damp * FOs_prev
                if not self.isClosedShell:
                    FOz = (1.0 - damp) * FOz + damp * FOz_prev
            FOs_prev, FOz_prev = FOs, FOz
            DOs_n, DOz_n = self._diag_density(FOs, FOz)
            Ps_n, Pz_n = self._unortho(DOs_n), self._unortho(DOz_n)
            # evalConver3: energy with the new density and the PT of this iteration
            E = self.computeEnergy(Ps_n, Pz_n, PTs, PTz)
            dE = E - Eold
            if self.doDamp:
                if abs(dE) < 1e-6:
                    damp = 0.0
                elif damp <= 0.0:
                    damp = 0.1
            ps_rms = float(t.linalg.norm(Ps_n - Ps))
            pz_rms = float(t.linalg.norm(Pz_n - Pz)) if not self.isClosedShell else 0.0
            Ps, Pz = Ps_n, Pz_n
            t.cuda.synchronize(self.dev)
            rec = SCFIteration(it, E, dE, ps_rms, pz_rms, time.perf_counter() - t0)
            self.log.append(rec)
            if on_iteration is not None:
                on_iteration(self, rec)
            conv = fp_converged or (abs(dE) < self.eneTol and ps_rms < self.denTol and
                                    (self.isClosedShell or pz_rms < self.denTol))
            Eold = E
            if conv and rebuild_pending:
                rebuild_pending = False
                built = None
                continue
            if conv:
                self.converged = True
                break
        self._set_precision(False)          # the context's own threshold and FP64 again
        self._base_threshold = None
        self.onePDMScalar, self.onePDMMz = Ps, Pz
        self.totalEnergy = Eold
        self.nSCFIter = len(self.log)
        self.scf_seconds = time.perf_counter() - t0
        if not self.converged:
            raise RuntimeError("SCF Failed to converge within MAXITER iterations")
        return self.totalEnergy

    SCF = SCF3

    def _diis_coefficients(self, hist_E):
        """Pulay coefficients (DIIS::extrapolate, extrapolate.h:63-141) of the newest
        vectors.  B is scaled by its largest diagonal element, and when the system is
        numerically singular (the error vectors have become linearly dependent near
        convergence) the oldest vectors are dropped; None means a plain SCF step."""
        t = self.torch
        m = len(hist_E)
        G = t.zeros((m, m), dtype=t.float64, device=self.dev)
        for i in range(m):
            for j in range(i + 1):
                v = sum(t.sum(a * b) for a, b in zip(hist_E[i], hist_E[j]))
                G[i, j] = v
                G[j, i] = v
        Gh = G.cpu()
        for k0 in range(m - 1):
            sub = Gh[k0:, k0:]
            mm = sub.shape[0]
            sc = float(sub.diagonal().max())
            if not sc > 0.0:
                return None
            B = t.zeros((mm + 1, mm + 1), dtype=t.float64)
            B[:mm, :mm] = sub / sc
            B[mm, :mm] = -1.0
            B[:mm, mm] = -1.0
            if float(t.linalg.cond(B)) > 1e12:
                continue
            rhs = t.zeros(mm + 1, dtype=t.float64)
            rhs[mm] = -1.0
            try:
                c = t.linalg.solve(B, rhs)[:mm]
            except RuntimeError:
                continue
            if bool(t.isfinite(c).all()):
                return [float(x) for x in c]
        return None

    def time_to(self, E_ref: float, tol: float = 1e-6) -> Optional[float]:
        """Seconds until the first iteration whose energy is within ``tol`` of ``E_ref``."""
        for r in self.log:
            if abs(r.energy - E_ref) <= tol:
                return r.t
        return None

    def close(self):
        self.ints.close()


_ATOM_CACHE = {}


def atomic_density(z: int, basis_name: str, device: int = 0, thresh: float = 1e-14):
    """Atomic UHF (core guess, no DIIS) densities (Ps, Pz) for the SAD guess, cached."""
    key = (z, basis_name.lower(), device)
    if key in _ATOM_CACHE:
        return _ATOM_CACHE[key]
    mol = Molecule(atoms=[z], coords=np.zeros((1, 3)), charge=0, mult=DEFAULT_MULT.get(z, 1))
    bs = BasisSet(basis_name, mol.atoms, mol.coords)
    hf = SingleSlater(mol, bs, ref="UHF", device=device, thresholdSchwartz=thresh)
    hf.guess = "CORE"
    hf.doDIIS = False
    hf.maxSCFIter = 512
    hf.SCF3()
    out = (hf.onePDMScalar.clone(), hf.onePDMMz.clone())
    hf.close()
    _ATOM_CACHE[key] = out
    return out
