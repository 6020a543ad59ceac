"""Plain numpy SCF on top of the oracle's G[D] (TEST INFRASTRUCTURE ONLY).

Used to pin the oracle end to end: converged RHF/UHF energies of the reference's legacy
test molecules (water, Li, O2) are compared with the values the reference recorded.
The Fock assembly and energy follow the reference's conventions:

* F_s = 2h + PTs, F_z = PTz; the orbital Fock matrices are 0.5(F_s +- F_z)
  (include/singleslater/singleslater_fock.h:202-258, scfutils.h:567-581).
* E = Tr(Ps h) + 1/4 [Tr(Ps PTs) + Tr(Pz PTz)] + E_nuc (include/singleslater/
  singleslater_properties.h:54-105).
* Ps = Pa + Pb, Pz = Pa - Pb with P_sigma = C_occ C_occ^T (misc.h:28-55).

The iteration itself (core guess, Loewdin orthogonalisation, commutator DIIS) only
needs to reach the same stationary point; the converged energy does not depend on it.
"""
from __future__ import annotations

import numpy as np


def lowdin(S):
    w, U = np.linalg.eigh(S)
    return (U / np.sqrt(w)) @ U.T


def scf(S, H, Enuc, nalpha, nbeta, build_pt, uhf=False, maxiter=200, etol=1e-11, dtol=1e-9,
        ndiis=8, D0=None):
    """Returns (E, Pa, Pb, niter).  ``build_pt(Ps, Pz)`` returns (PTs, PTz)."""
    X = lowdin(S)
    n = S.shape[0]

    def diag(F, nocc):
        Fo = X.T @ F @ X
        e, C = np.linalg.eigh(Fo)
        C = X @ C
        return C[:, :nocc] @ C[:, :nocc].T

    if D0 is None:
        Pa = diag(H, nalpha)
        Pb = diag(H, nbeta)
    else:
        Pa, Pb = D0
    Eold = 0.0
    hist_f, hist_e = [], []
    for it in range(1, maxiter + 1):
        Ps, Pz = Pa + Pb, Pa - Pb
        PTs, PTz = build_pt(Ps, Pz if uhf else None)
        if PTz is None:
            PTz = np.zeros_like(PTs)
        E = float(np.sum(Ps * H) + 0.25 * (np.sum(Ps * PTs) + np.sum(Pz * PTz))) + Enuc
        Fa = H + 0.5 * (PTs + PTz)
        Fb = H + 0.5 * (PTs - PTz)
        err = np.concatenate([(Fa @ Pa @ S - S @ Pa @ Fa).ravel(), (Fb @ Pb @ S - S @ Pb @ Fb).ravel()])
        hist_f.append((Fa, Fb))
        hist_e.append(err)
        if len(hist_f) > ndiis:
            hist_f.pop(0)
            hist_e.pop(0)
        m = len(hist_f)
        if m > 1:
            B = -np.ones((m + 1, m + 1))
            B[m, m] = 0
            for i in range(m):
                for j in range(m):
                    B[i, j] = hist_e[i] @ hist_e[j]
            rhs = np.zeros(m + 1)
            rhs[m] = -1
            try:
                c = np.linalg.solve(B, rhs)[:m]
                Fa = sum(ci * f[0] for ci, f in zip(c, hist_f))
                Fb = sum(ci * f[1] for ci, f in zip(c, hist_f))
            except np.linalg.LinAlgError:
                pass
        Pa_new = diag(Fa, nalpha)
        Pb_new = diag(Fb, nbeta) if uhf else Pa_new
        dP = max(np.abs(Pa_new - Pa).max(), np.abs(Pb_new - Pb).max())
        Pa, Pb = Pa_new, Pb_new
        if abs(E - Eold) < etol and dP < dtol:
            return E, Pa, Pb, it
        Eold = E
    raise RuntimeError("SCF did not converge")


# ---------------------------------------------------------------- SAD guess density ---
# Element default multiplicities of the reference's atomic SAD references, H..Ne
# (the atomic UHF calculations of SADGuess, include/singleslater/singleslater_guess.h:100-222).
_SAD_MULT = {1: 2, 2: 1, 3: 2, 4: 1, 5: 2, 6: 3, 7: 4, 8: 3, 9: 2, 10: 1}


def _diag_uhf(X, FOs, FOz, na, nb):
    """Orthonormal Fock -> orthonormal (DOs, DOz) with aufbau occupations."""
    _, Ca = np.linalg.eigh(0.5 * (FOs + FOz))
    _, Cb = np.linalg.eigh(0.5 * (FOs - FOz))
    DOa = Ca[:, :na] @ Ca[:, :na].T
    DOb = Cb[:, :nb] @ Cb[:, :nb].T
    return DOa + DOb, DOa - DOb


def atomic_uhf_density(z, basis_name, thresh=1e-14, maxiter=512):
    """(Ps, Pz) of the atomic UHF of element z: core guess, no DIIS, Fock damping 0.1
    against the previous orthonormal Fock matrix, switched off once |dE| < 1e-6 and back
    on above it; converged when |dE| < 1e-10 and ||dPs||, ||dPz|| < 1e-8
    (singleslater_guess.h:100-222 with the SCF defaults of singleslater.h:445-495 and
    scfutils.h:262-355, 1065-1111).  G[P] from the oracle's contraction."""
    from chronusq_public_b200.basis import BasisSet
    from . import oracle as O
    bs = BasisSet(basis_name, [z], np.zeros((1, 3)))
    ob = O.OracleBasis.from_basis(bs)
    S, T, V = O.one_e(ob, [float(z)], np.zeros((1, 3)))
    h = T + V
    Q = O.schwarz(ob)
    mult = _SAD_MULT.get(z, 1)
    na = (z + mult - 1) // 2
    nb = z - na
    X = lowdin(S)
    FOs = X.T @ (2.0 * h) @ X
    FOz = np.zeros_like(FOs)
    DOs, DOz = _diag_uhf(X, FOs, FOz, na, nb)
    Ps, Pz = X @ DOs @ X.T, X @ DOz @ X.T
    FOs_prev, FOz_prev = FOs, FOz
    damp, Eold = 0.1, 0.0
    for _ in range(maxiter):
        PTs, PTz, _ = O.form_pt(ob, Ps, Pz, thresh=thresh, Q=Q, nthreads=1)
        FOs = X.T @ (2.0 * h + PTs) @ X
        FOz = X.T @ PTz @ X
        if damp > 0.0:
            FOs = (1.0 - damp) * FOs + damp * FOs_prev
            FOz = (1.0 - damp) * FOz + damp * FOz_prev
        FOs_prev, FOz_prev = FOs, FOz
        DOs, DOz = _diag_uhf(X, FOs, FOz, na, nb)
        Ps_n, Pz_n = X @ DOs @ X.T, X @ DOz @ X.T
        E = float(np.sum(Ps_n * h) + 0.25 * (np.sum(Ps_n * PTs) + np.sum(Pz_n * PTz)))
        dE = E - Eold
        if abs(dE) < 1e-6:
            damp = 0.0
        elif damp <= 0.0:
            damp = 0.1
        dps, dpz = np.linalg.norm(Ps_n - Ps), np.linalg.norm(Pz_n - Pz)
        Ps, Pz, Eold = Ps_n, Pz_n, E
        if abs(dE) < 1e-10 and dps < 1e-8 and dpz < 1e-8:
            return Ps, Pz
    raise RuntimeError("atomic UHF did not converge")


def sad_guess_density(mol, bs, thresh=1e-14, nthreads=0):
    """RHF SAD-guess density of SingleSlater::formGuess (singleslater_guess.h:100-264): the
    atomic UHF densities placed block-diagonally, one molecular Fock build F = 2h + PT[Ps]
    with the oracle's contraction at `thresh`, diagonalised in the Loewdin basis, the
    lowest nelec/2 orbitals doubly occupied.  Returns the symmetric density (nbf x nbf,
    Fortran order).  Everything runs on the host: no GPU code is loaded."""
    from . import oracle as O
    n = bs.nbasis
    offs, off = {}, 0
    for s in bs.shells:
        offs.setdefault(s.atom, [off, 0])
        offs[s.atom][1] += s.size
        off += s.size
    Ps = np.zeros((n, n))
    cache = {}
    for a, z in enumerate(mol.atoms):
        if z not in cache:
            cache[z] = atomic_uhf_density(int(z), bs.name, thresh)[0]
        b0, nb = offs[a]
        Ps[b0:b0 + nb, b0:b0 + nb] = cache[z]
    ob = O.OracleBasis.from_basis(bs)
    S, T, V = O.one_e(ob, np.asarray(mol.atoms, dtype=np.float64), np.asarray(mol.coords).reshape(-1, 3))
    PTs, _, _ = O.form_pt(ob, np.asfortranarray(Ps), thresh=thresh, nthreads=nthreads)
    X = lowdin(S)
    FOs = X.T @ (2.0 * (T + V) + PTs) @ X
    _, C = np.linalg.eigh(0.5 * FOs)
    nocc = int(sum(mol.atoms) - mol.charge) // 2
    D = X @ (2.0 * C[:, :nocc] @ C[:, :nocc].T) @ X.T
    return np.asfortranarray(0.5 * (D + D.T))
