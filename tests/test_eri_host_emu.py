"""The generated per-thread ERI code (csrc/gen_eri.py), compiled for the host by g++
(tests/eri_host_emu.cpp), against the oracle's integrals (oracle/cq_oracle.c) on the CPU.

The GPU parity tests check the same code end to end through the Fock build; this test
isolates the integral arithmetic of every per-thread class, f shells included, so that a
change to the generator can be checked without a GPU."""
import ctypes
import importlib.util
import os
import shutil
import subprocess
import sys

import numpy as np
import pytest

from chronusq_public_b200.basis import BasisSet
from chronusq_public_b200.molecule import water_cluster
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "chronusq_public_b200", "csrc")


def _gen_module():
    spec = importlib.util.spec_from_file_location("gen_eri_for_test", os.path.join(CSRC, "gen_eri.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


@pytest.fixture(scope="module")
def emu(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("no C++ compiler")
    d = tmp_path_factory.mktemp("eri_emu")
    (d / "_gen").mkdir()
    (d / "stub").mkdir()
    (d / "stub" / "cuda_runtime.h").write_text("// host emulation of the generated code: empty\n")
    shutil.copy(os.path.join(CSRC, "eri_common.cuh"), d / "eri_common.cuh")
    shutil.copy(os.path.join(CSRC, "one_e.cuh"), d / "one_e.cuh")
    subprocess.run([sys.executable, os.path.join(CSRC, "gen_eri.py"), str(d / "_gen" / "eri_classes.cuh"), "3"],
                   check=True)
    so = d / "emu.so"
    subprocess.run(["g++", "-std=c++17", "-O1", "-shared", "-fPIC", "-Wno-unknown-pragmas",
                    "-I", str(d / "stub"), "-I", str(d / "_gen"), "-I", str(d),
                    os.path.join(ROOT, "tests", "eri_host_emu.cpp"),
                    "-o", str(so)], check=True)
    lib = ctypes.CDLL(str(so))
    dp = ctypes.POINTER(ctypes.c_double)
    ip = ctypes.POINTER(ctypes.c_int)
    lib.emu_eri.argtypes = [ctypes.c_int] * 4 + [ip, dp, dp, dp, ctypes.c_int, dp]
    lib.emu_eri.restype = ctypes.c_int
    return lib


def _run(lib, ob, shells, fp32=False):
    L = [int(ob.L[s]) for s in shells]
    off = np.concatenate([[0], np.cumsum(ob.nprim)])
    nprim = np.array([ob.nprim[s] for s in shells], dtype=np.int32)
    alpha = np.concatenate([ob.alpha[off[s]:off[s + 1]] for s in shells])
    coef = np.concatenate([ob.coef[off[s]:off[s + 1]] for s in shells])
    cen = np.ascontiguousarray(np.concatenate([ob.centers[s] for s in shells]))
    out = np.zeros(int(np.prod([ob.sizes[s] for s in shells])))
    dp = ctypes.POINTER(ctypes.c_double)
    n = lib.emu_eri(*L, nprim.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), alpha.ctypes.data_as(dp),
                    coef.ctypes.data_as(dp), cen.ctypes.data_as(dp), 1 if fp32 else 0, out.ctypes.data_as(dp))
    assert n == out.size, (L, n, out.size)
    return out


def _classes():
    g = _gen_module()
    return [q for q in g.quartet_classes(3) if q not in g.WARP_CLASSES]


def _pick(ob, rng, q):
    """Random shells of angular momenta q (engine orientation), spread over the atoms."""
    out = []
    for l in q:
        cand = np.flatnonzero(ob.L == l)
        out.append(int(rng.choice(cand)))
    return out


@pytest.fixture(scope="module")
def tz():
    mol = water_cluster(2, 5)
    return O.OracleBasis.from_basis(BasisSet("cc-pvtz", mol.atoms, mol.coords))


@pytest.mark.parametrize("q", _classes(), ids=lambda q: "%d%d%d%d" % q)
def test_generated_class_matches_oracle(emu, tz, q):
    rng = np.random.default_rng(sum(10 ** i * l for i, l in enumerate(q)))
    for _ in range(3):
        shells = _pick(tz, rng, q)
        ref = O.eri_quartet(tz, *shells).ravel()
        got = _run(emu, tz, shells)
        assert np.abs(got - ref).max() <= 1e-12 * max(1.0, np.abs(ref).max()), (q, shells)


@pytest.mark.parametrize("q", [(0, 0, 0, 0), (1, 0, 1, 0), (2, 0, 1, 1), (1, 1, 1, 1)],
                         ids=lambda q: "%d%d%d%d" % q)
def test_generated_class_fp32_instantiation(emu, tz, q):
    rng = np.random.default_rng(7)
    for _ in range(3):
        shells = _pick(tz, rng, q)
        ref = O.eri_quartet(tz, *shells).ravel()
        got = _run(emu, tz, shells, fp32=True)
        assert np.abs(got - ref).max() <= 2e-5 * max(1e-3, np.abs(ref).max()), (q, shells)


def test_every_per_thread_class_is_covered(emu, tz):
    """Warp classes are not in the generated code; every other class is."""
    g = _gen_module()
    assert len(_classes()) + len(g.WARP_CLASSES) == len(g.quartet_classes(3))
    for q in g.WARP_CLASSES:
        dp = ctypes.POINTER(ctypes.c_double)
        z = np.zeros(1)
        n = emu.emu_eri(*q, np.array([1, 1, 1, 1], dtype=np.int32).ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                        np.ones(4).ctypes.data_as(dp), np.ones(4).ctypes.data_as(dp),
                        np.zeros(12).ctypes.data_as(dp), 0, z.ctypes.data_as(dp))
        assert n == -1, q


# sibling-member variants (gen_eri.members_header): one set of primitive integrals serves
# mb bra and mk ket pairs that share exponents and differ in contraction coefficients
MEMBER_SPECS = [(0, 0, 0, 0, 3, 3), (0, 0, 0, 0, 2, 4), (1, 0, 0, 0, 2, 3), (1, 0, 1, 0, 2, 2),
                (1, 1, 0, 0, 3, 1), (2, 0, 0, 0, 1, 2), (2, 0, 1, 1, 2, 2)]


@pytest.fixture(scope="module")
def emu_members(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("no C++ compiler")
    d = tmp_path_factory.mktemp("eri_emu_members")
    (d / "_gen").mkdir()
    (d / "stub").mkdir()
    (d / "stub" / "cuda_runtime.h").write_text("// host emulation of the generated code: empty\n")
    shutil.copy(os.path.join(CSRC, "eri_common.cuh"), d / "eri_common.cuh")
    shutil.copy(os.path.join(CSRC, "one_e.cuh"), d / "one_e.cuh")
    subprocess.run([sys.executable, os.path.join(CSRC, "gen_eri.py"), str(d / "_gen" / "eri_classes.cuh"), "3"],
                   check=True)
    (d / "_gen" / "eri_gc_classes.cuh").write_text(_gen_module().members_header(MEMBER_SPECS))
    so = d / "emu_members.so"
    subprocess.run(["g++", "-std=c++17", "-O1", "-shared", "-fPIC", "-Wno-unknown-pragmas", "-DEMU_MEMBERS",
                    "-I", str(d / "stub"), "-I", str(d / "_gen"), "-I", str(d),
                    os.path.join(ROOT, "tests", "eri_host_emu.cpp"),
                    "-o", str(so)], check=True)
    lib = ctypes.CDLL(str(so))
    dp = ctypes.POINTER(ctypes.c_double)
    lib.emu_eri_members.argtypes = [ctypes.c_int] * 6 + [ctypes.POINTER(ctypes.c_int), dp, dp, dp, dp]
    lib.emu_eri_members.restype = ctypes.c_int
    return lib


@pytest.mark.parametrize("spec", MEMBER_SPECS, ids=lambda q: "%d%d%d%d_%dx%d" % q)
def test_sibling_members_match_separate_quartets(emu_members, tz, spec):
    """Each member quartet of a sibling evaluation equals the oracle's integral over the
    contracted functions with that member's coefficients."""
    la, lb, lc, ld, mb, mk = spec
    rng = np.random.default_rng(sum(spec))
    a, b, c, d = _pick(tz, rng, (la, lb, lc, ld))
    off = np.concatenate([[0], np.cumsum(tz.nprim)])
    exps = [tz.alpha[off[s]:off[s + 1]] for s in (a, b, c, d)]
    base = [tz.coef[off[s]:off[s + 1]] for s in (a, b, c, d)]
    # member 0: the basis' own coefficients; the others: perturbed copies
    sets = [[base[k] * (1.0 if m == 0 else 1.0 + 0.3 * rng.standard_normal(base[k].size))
             for m in range(mb if k < 2 else mk)] for k in range(4)]
    shells_L, shells_n, shells_a, shells_c, shells_R = [], [], [], [], []
    index = {}
    for k, s in enumerate((a, b, c, d)):
        for m, cf in enumerate(sets[k]):
            index[(k, m)] = len(shells_L)
            shells_L.append(tz.L[s])
            shells_n.append(tz.nprim[s])
            shells_a.append(exps[k])
            shells_c.append(cf)
            shells_R.append(tz.centers[s])
    ob = O.OracleBasis(shells_L, [l > 1 for l in shells_L], shells_n, np.concatenate(shells_a),
                       np.concatenate(shells_c), np.array(shells_R))
    nprim = np.array([tz.nprim[s] for s in (a, b, c, d)], dtype=np.int32)
    coef = np.concatenate([np.concatenate(sets[k]) for k in range(4)])
    cen = np.ascontiguousarray(np.concatenate([tz.centers[s] for s in (a, b, c, d)]))
    n = int(np.prod([tz.sizes[s] for s in (a, b, c, d)]))
    out = np.zeros(n * mb * mk)
    dp = ctypes.POINTER(ctypes.c_double)
    got = emu_members.emu_eri_members(la, lb, lc, ld, mb, mk, nprim.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                      np.concatenate(exps).ctypes.data_as(dp), coef.ctypes.data_as(dp),
                                      cen.ctypes.data_as(dp), out.ctypes.data_as(dp))
    assert got == out.size
    for i in range(mb):
        for j in range(mk):
            ref = O.eri_quartet(ob, index[(0, i)], index[(1, i)], index[(2, j)], index[(3, j)]).ravel()
            val = out[(i * mk + j) * n:(i * mk + j + 1) * n]
            assert np.abs(val - ref).max() <= 1e-12 * max(1.0, np.abs(ref).max()), (spec, i, j)


@pytest.mark.parametrize("sm", [1, 0, 2], ids=["shared_rows", "global_table", "runtime_L"])
def test_device_boys_against_high_precision(emu, sm):
    """The device Boys evaluations (Taylor table below T = 36 with e^-T from the degree-9
    polynomial, asymptotic form and upward recursion above) against the oracle's long-double
    series, for every total angular momentum to (ff|ff) and T across both branches."""
    dp = ctypes.POINTER(ctypes.c_double)
    emu.emu_boys.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_int, dp]
    emu.emu_boys.restype = ctypes.c_int
    Ts = np.concatenate([[0.0, 1e-12, 0.049999, 0.05, 0.05000001, 35.95, 35.999999, 36.0, 36.5, 80.0, 700.0],
                         np.random.default_rng(3).uniform(0, 40, 300)])
    worst = 0.0
    for L in range(13):
        F = np.zeros(L + 1)
        for T in Ts:
            assert emu.emu_boys(L, float(T), sm, F.ctypes.data_as(dp)) == L + 1
            ref = O.boys(L, float(T))
            worst = max(worst, float(np.max(np.abs(F - ref) / np.abs(ref))))
    assert worst < 1e-14, worst        # measured: 2.2e-15


@pytest.mark.parametrize("basis", ["6-31g*", "cc-pvtz"])
def test_device_dipole_integrals_match_oracle(emu, basis):
    """The dipole device code of one_e.cuh (k_dipole's per-pair work) against the oracle's
    dipole integrals, about the origin and about a shifted origin."""
    mol = water_cluster(2, 5)
    ob = O.OracleBasis.from_basis(BasisSet(basis, mol.atoms, mol.coords))
    n = ob.nbf
    poff = np.concatenate([[0], np.cumsum(ob.nprim)[:-1]]).astype(np.int32)
    bf = np.asarray(ob.offsets, dtype=np.int32)
    ip = ctypes.POINTER(ctypes.c_int)
    dp = ctypes.POINTER(ctypes.c_double)
    emu.emu_dipole.argtypes = [ctypes.c_int, ip, ip, ip, ip, dp, dp, dp, dp, ctypes.c_int, dp]
    emu.emu_dipole.restype = None
    for origin in ((0.0, 0.0, 0.0), (0.4, -1.1, 2.3)):
        o = np.asarray(origin)
        D = np.zeros(3 * n * n)
        emu.emu_dipole(ob.nshell, ob.L.ctypes.data_as(ip), ob.nprim.ctypes.data_as(ip), poff.ctypes.data_as(ip),
                       bf.ctypes.data_as(ip), ob.alpha.ctypes.data_as(dp), ob.coef.ctypes.data_as(dp),
                       np.ascontiguousarray(ob.centers).ctypes.data_as(dp), o.ctypes.data_as(dp), n,
                       D.ctypes.data_as(dp))
        ref = O.dipole(ob, origin)
        for k in range(3):
            got = D[k * n * n:(k + 1) * n * n].reshape(n, n, order="F")
            assert np.abs(got - ref[k]).max() < 1e-12, (basis, origin, k)


@pytest.mark.parametrize("basis", ["6-31g*", "cc-pvtz"])
def test_one_electron_kernel_body_matches_oracle(emu, basis):
    """k_one_e's per-pair work (S, T, V by McMurchie-Davidson) against the oracle's
    Obara-Saika one-electron integrals, with the nuclei and extra point charges."""
    mol = water_cluster(2, 5)
    ob = O.OracleBasis.from_basis(BasisSet(basis, mol.atoms, mol.coords))
    n = ob.nbf
    rng = np.random.default_rng(4)
    R = np.asarray(mol.coords, dtype=np.float64).reshape(-1, 3)
    Z = np.concatenate([np.asarray(mol.atoms, dtype=np.float64), rng.uniform(-1, 1, 5)])
    R = np.ascontiguousarray(np.concatenate([R, rng.uniform(-3, 3, (5, 3))]))
    poff = np.concatenate([[0], np.cumsum(ob.nprim)[:-1]]).astype(np.int32)
    bf = np.asarray(ob.offsets, dtype=np.int32)
    ip = ctypes.POINTER(ctypes.c_int)
    dp = ctypes.POINTER(ctypes.c_double)
    emu.emu_one_e.argtypes = [ctypes.c_int, ip, ip, ip, ip, dp, dp, dp, ctypes.c_int, dp, dp, ctypes.c_int, dp, dp, dp]
    emu.emu_one_e.restype = None
    out = [np.zeros((n, n), order="F") for _ in range(3)]
    emu.emu_one_e(ob.nshell, ob.L.ctypes.data_as(ip), ob.nprim.ctypes.data_as(ip), poff.ctypes.data_as(ip),
                  bf.ctypes.data_as(ip), ob.alpha.ctypes.data_as(dp), ob.coef.ctypes.data_as(dp),
                  np.ascontiguousarray(ob.centers).ctypes.data_as(dp), len(Z), Z.ctypes.data_as(dp),
                  R.ctypes.data_as(dp), n, *[x.ctypes.data_as(dp) for x in out])
    ref = O.one_e(ob, Z, R)
    for name, got, want in zip("STV", out, ref):
        assert np.abs(got - want).max() < 1e-11 * max(1.0, np.abs(want).max()), (basis, name)
