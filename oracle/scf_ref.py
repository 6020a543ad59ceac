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
