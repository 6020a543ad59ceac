"""Pins and known-answer tests of the CPU oracle (no GPU).

The oracle is pinned end to end against the reference's recorded SCF energies
(tests/golden/legacy_pins.json, extracted from the reference's oldTests.tgz by
tests/golden/make_pins.py), and piecewise against closed forms and the in-core
contraction semantics (include/aointegrals/aointegrals_contract.h:197-262).
"""
import json
import math
import os
from decimal import Decimal, getcontext

import numpy as np
import pytest

from chronusq_public_b200.basis import BasisSet
from chronusq_public_b200.molecule import Molecule, reference_water, single_water
from oracle import oracle as O
from oracle.scf_ref import scf

HERE = os.path.dirname(os.path.abspath(__file__))
PINS = json.load(open(os.path.join(HERE, "golden", "legacy_pins.json")))


def _run_scf(pin, D0=None):
    mol = Molecule.from_angstrom([g[0] for g in pin["geom_angstrom"]], [g[1:] for g in pin["geom_angstrom"]],
                                 charge=pin["charge"], mult=pin["mult"])
    bs = BasisSet(pin["basis"], mol.atoms, mol.coords)
    ob = O.OracleBasis.from_basis(bs)
    S, T, V = O.one_e(ob, mol.atoms, mol.coords)
    Q = O.schwarz(ob)
    ne = mol.nelectrons
    na = (ne + mol.mult - 1) // 2
    nb = ne - na
    uhf = "UHF" in pin["reference"]

    def bpt(Ps, Pz):
        a, b, _ = O.form_pt(ob, Ps, Pz, Q=Q)
        return a, b
    E, *_ = scf(S, T + V, mol.nuclear_repulsion(), na, nb, bpt, uhf=uhf, D0=D0)
    return E


# O2/STO-3G UHF has a lower, symmetry-broken solution that a core guess finds; the pinned
# value is the symmetric state the reference's SAD guess leads to, checked separately.
@pytest.mark.parametrize("pin", [p for p in PINS if p["test"] != "test0010"], ids=lambda p: p["test"])
def test_legacy_energy_pins(pin):
    E = _run_scf(pin)
    assert abs(E - pin["energy"]) < 1e-8, (E, pin["energy"])


FIELD_PINS = json.load(open(os.path.join(HERE, "golden", "legacy_field_pins.json")))
DEBYE = 0.393430307      # e bohr per Debye (the reference's phys.debye, include/global.h:224)


# test0052 (O2/STO-3G UHF in a field): a core guess lands on another UHF solution, 0.25 Eh
# above the recorded one, which the reference reached from its SAD guess (as for test0010).
@pytest.mark.parametrize("pin", [p for p in FIELD_PINS if p["test"] != "test0052"], ids=lambda p: p["test"])
def test_field_energy_and_dipole_pins(pin):
    """SCF in a static field F: h + F.<r> (origin 0; Fock assembly singleslater_fock.h:215,
    aointegrals.h:505-510) and E_nuc - F.mu_nuc (energy singleslater_properties.h:95-101),
    against the reference's recorded energies and dipole moments (Debye).  Measured: energies
    within 8e-11 Eh; dipoles within 2e-6 relative for water and O2 and 3e-5 for lithium, whose
    recorded dipoles differ from this oracle's by more than the oracle's own convergence
    moves them."""
    mol = Molecule.from_angstrom([g[0] for g in pin["geom_angstrom"]], [g[1:] for g in pin["geom_angstrom"]],
                                 charge=pin["charge"], mult=pin["mult"])
    bs = BasisSet(pin["basis"], mol.atoms, mol.coords)
    ob = O.OracleBasis.from_basis(bs)
    S, T, V = O.one_e(ob, mol.atoms, mol.coords)
    D = O.dipole(ob)
    Q = O.schwarz(ob)
    F = np.asarray(pin["field"])
    Z = np.asarray(mol.atoms, dtype=float)
    mu_nuc = Z @ np.asarray(mol.coords).reshape(-1, 3)
    ne = mol.nelectrons
    na = (ne + mol.mult - 1) // 2

    def bpt(Ps, Pz):
        a, b, _ = O.form_pt(ob, Ps, Pz, Q=Q)
        return a, b
    H = T + V + sum(F[k] * D[k] for k in range(3))
    E, Pa, Pb, _ = scf(S, H, mol.nuclear_repulsion() - F @ mu_nuc, na, ne - na, bpt, uhf="UHF" in pin["reference"])
    assert abs(E - pin["energy"]) < 1e-9, (E, pin["energy"])
    mu = mu_nuc - np.array([np.sum((Pa + Pb) * D[k]) for k in range(3)])
    ref = np.asarray(pin["dipole_debye"])
    assert np.abs(mu / DEBYE - ref).max() < 5e-5 * max(1.0, np.abs(ref).max()), (mu / DEBYE, ref)


def test_boys_against_high_precision_series():
    getcontext().prec = 60
    for T in [0.0, 1e-8, 0.37, 2.5, 11.0, 29.9, 35.5, 36.5, 59.0, 61.0, 120.0]:
        F = O.boys(12, T)
        for m in (0, 1, 5, 12):
            t = Decimal(T)
            term = Decimal(1) / (2 * m + 1)
            s = term
            k = 1
            while True:
                term = term * 2 * t / (2 * m + 2 * k + 1)
                s += term
                k += 1
                if term < s * Decimal(10) ** -40:
                    break
            ref = float((-t).exp() * s)
            assert abs(F[m] - ref) <= 2e-15 * ref, (T, m, F[m], ref)


def test_ssss_closed_form():
    a, b, c, d = 1.3, 0.4, 2.2, 0.7
    A, B, C, D = (np.array(x, float) for x in ([0, 0, 0], [0.5, 0.1, -0.3], [1.2, -0.4, 0.2], [-0.3, 0.9, 0.6]))
    ob = O.OracleBasis([0, 0, 0, 0], [0, 0, 0, 0], [1, 1, 1, 1], [a, b, c, d], [1, 1, 1, 1],
                       np.array([A, B, C, D]))
    v = O.eri_quartet(ob, 0, 1, 2, 3).ravel()[0]
    p, q = a + b, c + d
    P, Qc = (a * A + b * B) / p, (c * C + d * D) / q
    rho = p * q / (p + q)
    T = rho * np.sum((P - Qc) ** 2)
    F0 = 0.5 * math.sqrt(math.pi / T) * math.erf(math.sqrt(T))
    ref = (2 * math.pi ** 2.5 / (p * q * math.sqrt(p + q)) * math.exp(-a * b / p * np.sum((A - B) ** 2))
           * math.exp(-c * d / q * np.sum((C - D) ** 2)) * F0)
    assert abs(v - ref) < 1e-14 * abs(ref)


def test_eri_permutational_symmetry():
    mol = single_water(0)
    bs = BasisSet("6-31g*", mol.atoms, mol.coords)
    ob = O.OracleBasis.from_basis(bs)
    rng = np.random.default_rng(0)
    for _ in range(20):
        s = rng.integers(0, bs.nshell, 4)
        v = O.eri_quartet(ob, *s)
        assert np.allclose(v, O.eri_quartet(ob, s[1], s[0], s[2], s[3]).transpose(1, 0, 2, 3), atol=1e-13)
        assert np.allclose(v, O.eri_quartet(ob, s[0], s[1], s[3], s[2]).transpose(0, 1, 3, 2), atol=1e-13)
        assert np.allclose(v, O.eri_quartet(ob, s[2], s[3], s[0], s[1]).transpose(2, 3, 0, 1), atol=1e-13)


def test_schwarz_bounds_every_shell_quartet():
    """Q(a,b) = sqrt(max_ij |(ij|ij)|) over the functions of shell pair (a,b)
    (builders.cpp:469-517), and the Cauchy-Schwarz inequality |(ab|cd)| <= Q_ab Q_cd that
    the screen relies on, over every shell quartet of a water molecule."""
    mol = single_water(3)
    bs = BasisSet("6-31g*", mol.atoms, mol.coords)
    ob = O.OracleBasis.from_basis(bs)
    Q = O.schwarz(ob)
    eri = O.eri_full(ob)
    off, sz = ob.offsets, ob.sizes
    sl = [slice(int(o), int(o + z)) for o, z in zip(off, sz)]
    assert np.allclose(Q, Q.T, rtol=0, atol=0)
    for a in range(bs.nshell):
        for b in range(bs.nshell):
            blk = eri[sl[a], sl[b], sl[a], sl[b]]
            diag = np.array([blk[i, j, i, j] for i in range(sz[a]) for j in range(sz[b])])
            assert abs(Q[a, b] - math.sqrt(np.abs(diag).max())) <= 1e-14 * max(1.0, Q[a, b])
    for a in range(bs.nshell):
        for b in range(bs.nshell):
            for c in range(bs.nshell):
                m = np.abs(eri[sl[a], sl[b], sl[c], :]).reshape(sz[a] * sz[b] * sz[c], -1)
                for d in range(bs.nshell):
                    assert m[:, sl[d]].max() <= Q[a, b] * Q[c, d] * (1 + 1e-12) + 1e-15


def test_direct_equals_incore_contraction():
    """newTwoEContractDirect with no screening equals the in-core N^4 contraction
    (contract.h:239-259: COULOMB {i,j,k,l}X{l,k}, EXCHANGE {i,l,k,j}X{l,k}, times 2)."""
    mol = single_water(5)
    bs = BasisSet("6-31g*", mol.atoms, mol.coords)
    ob = O.OracleBasis.from_basis(bs)
    eri = O.eri_full(ob)
    rng = np.random.default_rng(1)
    X = rng.uniform(-1, 1, (bs.nbasis,) * 2)
    X = np.asfortranarray(X + X.T)
    for typ, s in ((0, 1.0), (1, -0.5)):
        AX = np.zeros_like(X, order="F")
        n = O.twoe_contract_direct(ob, [X], [AX], [typ], [s], thresh=0.0)
        assert n == 1540  # 55 shell pairs -> 55*56/2 unique quartets
        ref = 2 * s * (np.einsum("ijkl,lk->ij", eri, X) if typ == 0 else np.einsum("ilkj,lk->ij", eri, X))
        assert np.abs(AX - ref).max() < 1e-11


def test_uhf_with_zero_spin_density_matches_rhf():
    mol = single_water(6)
    bs = BasisSet("cc-pvdz", mol.atoms, mol.coords)
    ob = O.OracleBasis.from_basis(bs)
    rng = np.random.default_rng(2)
    P = rng.uniform(-1, 1, (bs.nbasis,) * 2)
    P = np.asfortranarray(P + P.T)
    PTs_r, _, n_r = O.form_pt(ob, P)
    PTs_u, PTz_u, n_u = O.form_pt(ob, P, np.zeros_like(P, order="F"))
    assert n_r == n_u
    assert np.abs(PTs_r - PTs_u).max() < 1e-13
    assert np.abs(PTz_u).max() == 0.0


def test_threading_does_not_change_result():
    mol = single_water(7)
    bs = BasisSet("6-31g*", mol.atoms, mol.coords)
    ob = O.OracleBasis.from_basis(bs)
    rng = np.random.default_rng(3)
    P = rng.uniform(-1, 1, (bs.nbasis,) * 2)
    P = np.asfortranarray(P + P.T)
    a, _, na = O.form_pt(ob, P, nthreads=1)
    b, _, nb = O.form_pt(ob, P, nthreads=4)
    assert na == nb
    assert np.abs(a - b).max() < 1e-12
