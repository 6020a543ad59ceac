"""Mixed-precision (FP32 quartets below a Schwarz-bound cutoff, FP64 accumulation) and
incremental Delta-D Fock builds against the all-FP64 GPU build."""
import numpy as np
import pytest

from chronusq_public_b200.basis import BasisSet
from chronusq_public_b200.molecule import water_cluster

pytestmark = pytest.mark.gpu


def _rand_density(n, seed):
    rng = np.random.default_rng(seed)
    a = rng.uniform(-1, 1, (n, n))
    return np.asfortranarray(0.5 * (a + a.T))


@pytest.mark.parametrize("cutoff,warp_form,tier", [(1e-10, 0, 0), (1e-8, 0, 0), (1e-6, 0, 0), (1e-6, 1, 0),
                                                   (1e-6, 0, 2)])
def test_mixed_G_close_to_fp64(cutoff, warp_form, tier):
    """warp_form = 1: the classes with both kernel forms run their FP64 and FP32 lists in
    the warp-cooperative form; tier 2: the per-thread classes' FP64 and FP32 lists go
    through the class-fused kernel."""
    from chronusq_public_b200.aointegrals import AOIntegrals, PREC_MIXED, PREC_FP64
    mol = water_cluster(4, 21)
    bs = BasisSet("cc-pvdz", mol.atoms, mol.coords)
    ints = AOIntegrals(bs)
    ints.setSchedule(warp_form=warp_form)
    ints.setFusion(tier)
    D = _rand_density(bs.nbasis, 4)
    G64, _ = ints.formPT(D)
    n64 = ints.stats()["quartets"]
    ints.setPrecision(PREC_MIXED, cutoff)
    G32, _ = ints.formPT(D)
    st = ints.stats()
    assert st["quartets"] == n64                 # same quartet set, split by precision
    assert st["quartets_fp32"] > 0
    err = np.abs(G32 - G64).max()
    assert err < 50 * cutoff, err               # FP32 quartets are bounded by the cutoff
    ints.setPrecision(PREC_FP64, 0.0)
    G64b, _ = ints.formPT(D)
    assert np.abs(G64b - G64).max() < 1e-12


def test_mixed_incremental_scf_energy_within_1uEh():
    from chronusq_public_b200.scf import SingleSlater
    mol = water_cluster(3, 2)
    bs = BasisSet("cc-pvdz", mol.atoms, mol.coords)
    ref = SingleSlater(mol, bs)
    E64 = ref.SCF3()
    mx = SingleSlater(mol, bs, ints=ref.ints)
    mx.precision = "mixed"
    mx.fp32_cutoff = 1e-7
    mx.incremental = True
    E = mx.SCF3()
    assert mx.fp32_quartets > 0
    assert abs(E - E64) < 1e-6, (E, E64)
    assert mx.time_to(E64, 1e-6) is not None
    ref.close()


def test_mixed_phase_threshold_is_loosened_then_restored():
    """The mixed phase screens at mixed_threshold (1e-11 here, looser than the context's
    1e-14); from the FP64 switch on, the builds use the context's threshold again, start
    from a full rebuild, and the converged energy matches the FP64 one within 1e-8 Eh."""
    from chronusq_public_b200.scf import SingleSlater
    mol = water_cluster(3, 2)
    bs = BasisSet("cc-pvdz", mol.atoms, mol.coords)
    ref = SingleSlater(mol, bs)
    E64 = ref.SCF3()
    seen = []
    mx = SingleSlater(mol, bs, ints=ref.ints)
    mx.precision, mx.fp32_cutoff, mx.incremental = "mixed", 1e-8, True
    assert mx.mixed_threshold == 1e-11
    E = mx.SCF3(on_iteration=lambda s, rec: seen.append((s.ints.thresholdSchwartz, s.ints.stats()["quartets"])))
    k = mx.phase_switch_iter
    assert k is not None and 0 < k < len(seen) - 1
    assert all(th == 1e-11 for th, _ in seen[:k]) and all(th == 1e-14 for th, _ in seen[k:])
    assert ref.ints.thresholdSchwartz == 1e-14
    assert abs(E - E64) < 1e-8, (E, E64)
    # the switch is decided after iteration k's (mixed) build; iteration k + 1 builds the full
    # FP64 PT: more quartets than any incremental build before it
    assert seen[k + 1][1] > max(q for _, q in seen[1:k + 1])
    # with the context's threshold throughout (mixed_threshold None) the result is the same
    tight = SingleSlater(mol, bs, ints=ref.ints)
    tight.precision, tight.fp32_cutoff, tight.incremental, tight.mixed_threshold = "mixed", 1e-8, True, None
    assert abs(tight.SCF3() - E64) < 1e-8
    ref.close()


def test_mixed_sibling_lists_match_pair_lists():
    """FP32 sibling-group lists: the same FP32 quartet set as the pair-level lists, and the
    same bound on the difference from the FP64 build."""
    from chronusq_public_b200.aointegrals import AOIntegrals, PREC_MIXED
    mol = water_cluster(4, 21)
    bs = BasisSet("cc-pvdz", mol.atoms, mol.coords)
    ints = AOIntegrals(bs)
    ints.setSiblings(True)
    D = _rand_density(bs.nbasis, 5)
    G64, _ = ints.formPT(D)
    cutoff = 1e-7
    ints.setPrecision(PREC_MIXED, cutoff)
    Gon, _ = ints.formPT(D)
    st_on = ints.stats()
    ints.setSiblings(False)
    Goff, _ = ints.formPT(D)
    st_off = ints.stats()
    assert st_on["quartets_fp32"] == st_off["quartets_fp32"] > 0
    assert st_on["quartets"] == st_off["quartets"]
    assert "(ss|ss)" in st_on["sibling_classes"]
    assert np.abs(Gon - G64).max() < 50 * cutoff
    assert np.abs(Goff - G64).max() < 50 * cutoff
