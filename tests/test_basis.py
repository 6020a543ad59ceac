"""Basis-set parsing and normalisation conventions (no GPU)."""
import os

import numpy as np
import pytest

from chronusq_public_b200 import basis as B
from chronusq_public_b200.molecule import reference_water, single_water, water_cluster
from oracle import oracle as O


def test_stod_prefix_semantics():
    assert B._stod("0.458878D-03") == 0.458878
    assert B._stod("1.5E-02") == 0.015
    assert B._stod("-.25") == -0.25


def test_sp_split_and_pure_flags():
    lib = B.parse_gbs(B.basis_path("6-31g*"))
    o = lib[8]
    assert [s.l for s in o] == [0, 0, 1, 0, 1, 2]   # S6, SP3 -> S,P, SP1 -> S,P, D1
    assert [s.pure for s in o] == [False, False, False, False, False, True]
    lib_c = B.parse_gbs(B.basis_path("6-31g*"), force_cart=True)
    assert lib_c[8][-1].pure is False


@pytest.mark.parametrize("name,nbf,nsh", [("sto-3g", 7, 5), ("6-31g", 13, 9), ("6-31g*", 18, 10),
                                          ("cc-pvdz", 24, 12), ("cc-pvtz", 58, 22)])
def test_water_sizes(name, nbf, nsh):
    m = reference_water()
    bs = B.BasisSet(name, m.atoms, m.coords)
    assert (bs.nbasis, bs.nshell) == (nbf, nsh)


def test_cluster_sizes_match_workloads():
    m = water_cluster(32, 1)
    assert B.BasisSet("cc-pvdz", m.atoms, m.coords).nbasis == 768


def test_unit_normalisation_of_every_function():
    m = single_water(0)
    for name in ("6-31g*", "cc-pvdz", "cc-pvtz"):
        bs = B.BasisSet(name, m.atoms, m.coords)
        ob = O.OracleBasis.from_basis(bs)
        S, _, _ = O.one_e(ob, [], np.zeros((0, 3)))
        d = np.diag(S)
        for s, off in zip(bs.shells, bs.map_sh2bf):
            if s.pure or s.l <= 1:
                assert np.allclose(d[off:off + s.size], 1.0, atol=1e-12), (name, s.l)


def test_solid_harmonics_agree_with_independent_construction():
    for l in range(5):
        assert np.abs(B.solid_harmonic_matrix(l) - O.oracle_solid_harmonics(l)).max() < 1e-12


def test_cartesian_order():
    assert B.cart_list(2) == [(2, 0, 0), (1, 1, 0), (1, 0, 1), (0, 2, 0), (0, 1, 1), (0, 0, 2)]


def test_missing_element_raises():
    with pytest.raises(ValueError):
        B.BasisSet("6-31g*", [17], np.zeros((1, 3)))
