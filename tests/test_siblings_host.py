"""Host rules of the sibling groups (chronusq_public_b200/csrc/siblings.h), compiled for
the CPU by g++: shell families and the sibling groups of each pair class, on the cc-pVDZ
and 6-31G(d) water clusters the GPU tests use."""
import ctypes
import os
import shutil
import subprocess
from collections import defaultdict

import numpy as np
import pytest

from chronusq_public_b200.basis import BasisSet
from chronusq_public_b200.molecule import water_cluster
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "chronusq_public_b200", "csrc")
CAP = {(0, 0): 4, (1, 0): 2, (2, 0): 2}   # member caps (engine_impl.cuh, sibling_cap)


@pytest.fixture(scope="module")
def shim(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("no C++ compiler")
    so = tmp_path_factory.mktemp("sib") / "sib.so"
    subprocess.run(["g++", "-std=c++17", "-O1", "-shared", "-fPIC", "-I", CSRC,
                    os.path.join(ROOT, "tests", "siblings_host_shim.cpp"), "-o", str(so)], check=True)
    return ctypes.CDLL(str(so))


def _ip(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _families(shim, ob):
    ns = ob.nshell
    L = np.ascontiguousarray(ob.L, dtype=np.int32)
    npr = np.ascontiguousarray(ob.nprim, dtype=np.int32)
    poff = np.ascontiguousarray(np.concatenate([[0], np.cumsum(npr)[:-1]]), dtype=np.int32)
    alpha = np.ascontiguousarray(ob.alpha, dtype=np.float64)
    cen = np.ascontiguousarray(ob.centers, dtype=np.float64).ravel()
    mol = np.zeros(ns, dtype=np.int32)
    fam = np.zeros(ns, dtype=np.int32)
    nf = shim.sib_families(ns, _ip(L), _ip(npr), _ip(poff), _dp(alpha), _dp(cen), _ip(mol), _ip(fam))
    return L, fam, nf


def _groups(shim, L, fam, pairs, cap):
    a = np.ascontiguousarray([p[0] for p in pairs], dtype=np.int32)
    b = np.ascontiguousarray([p[1] for p in pairs], dtype=np.int32)
    gid = np.zeros(len(pairs), dtype=np.int32)
    rank = np.zeros(len(pairs), dtype=np.int32)
    ng = shim.sib_pair_groups(len(pairs), _ip(a), _ip(b), _ip(L), len(L), _ip(fam), cap, _ip(gid), _ip(rank))
    return ng, gid, rank


def _class_pairs(L, la, lb):
    """Pairs of one class in the engine's orientation (L_a >= L_b, a >= b for equal L)."""
    out = []
    for a in range(len(L)):
        for b in range(a + 1):
            x, y = (a, b) if L[a] >= L[b] else (b, a)
            if (L[x], L[y]) == (la, lb):
                out.append((x, y))
    return out


def test_cc_pvdz_oxygen_1s_2s_are_one_family(shim):
    mol = water_cluster(3, 11)
    ob = O.OracleBasis.from_basis(BasisSet("cc-pvdz", mol.atoms, mol.coords))
    L, fam, nf = _families(shim, ob)
    # per water: O 1s/2s share a family; every other shell (O 3s, p, d; H s, p) is its own
    assert nf == ob.nshell - 3
    off = np.concatenate([[0], np.cumsum(ob.nprim)])
    for s in range(ob.nshell):
        for t in range(s):
            same = (L[s] == L[t] and ob.nprim[s] == ob.nprim[t] and np.array_equal(ob.centers[s], ob.centers[t])
                    and np.array_equal(ob.alpha[off[s]:off[s + 1]], ob.alpha[off[t]:off[t + 1]]))
            assert (fam[s] == fam[t]) == same, (s, t)


@pytest.mark.parametrize("basis", ["cc-pvdz", "6-31g*"])
def test_pair_groups_partition_each_class(shim, basis):
    """Every pair is in exactly one group; the members of a group share their two families
    (unordered for s-s pairs); no group is larger than its class's cap; groups are numbered
    by their first pair and members ranked in pair order."""
    mol = water_cluster(3, 11)
    ob = O.OracleBasis.from_basis(BasisSet(basis, mol.atoms, mol.coords))
    L, fam, _ = _families(shim, ob)
    sizes_seen = defaultdict(int)
    for (la, lb), cap in list(CAP.items()) + [((1, 1), 1), ((2, 1), 1)]:
        pairs = _class_pairs(L, la, lb)
        ng, gid, rank = _groups(shim, L, fam, pairs, cap)
        members = defaultdict(list)
        for k, g in enumerate(gid):
            members[int(g)].append(k)
        assert sorted(members) == list(range(ng))
        first = [members[g][0] for g in range(ng)]
        assert first == sorted(first)
        for g, ks in members.items():
            assert 1 <= len(ks) <= cap
            assert [int(rank[k]) for k in ks] == list(range(len(ks)))
            key = {tuple(sorted((int(fam[pairs[k][0]]), int(fam[pairs[k][1]])))) if la == lb
                   else (int(fam[pairs[k][0]]), int(fam[pairs[k][1]])) for k in ks}
            assert len(key) == 1
            sizes_seen[(la, lb, len(ks))] += 1
    if basis == "cc-pvdz":
        # O 1s/2s: s-s groups of 4 (two oxygens), 3 (one oxygen), 2 (oxygen with another s)
        assert sizes_seen[(0, 0, 4)] > 0 and sizes_seen[(0, 0, 3)] == 3 and sizes_seen[(0, 0, 2)] > 0
        assert sizes_seen[(1, 0, 2)] > 0 and sizes_seen[(2, 0, 2)] > 0
    else:
        # 6-31G(d) shares exponents only between shells of different angular momentum
        assert all(n == 1 for (_, _, n) in sizes_seen)
