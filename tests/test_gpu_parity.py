"""GPU parity of the direct two-electron contraction against the CPU oracle.

Bar (stated in the engine's spec): max|G_gpu - G_oracle| <= 1e-10 for the FP64 path, and
the screened quartet count (the unit of work) equal to the oracle's.
"""
import numpy as np
import pytest

from chronusq_public_b200.basis import BasisSet
from chronusq_public_b200.molecule import single_water, water_cluster, reference_water, Molecule
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL_G = 1e-10


def _aoi():
    from chronusq_public_b200.aointegrals import AOIntegrals
    return AOIntegrals


def rand_sym(n, seed, scale=1.0):
    rng = np.random.default_rng(seed)
    a = rng.uniform(-scale, scale, (n, n))
    return np.asfortranarray(0.5 * (a + a.T))


def oracle_G(ob, X, types, scale, thresh):
    out = np.zeros_like(X[0], order="F")
    n = O.twoe_contract_direct(ob, X, [out] * len(X), types, scale, thresh=thresh)
    return out, n


@pytest.mark.parametrize("basis", ["sto-3g", "6-31g", "6-31g*", "cc-pvdz", "cc-pvtz"])
def test_water_rhf_G(basis):
    mol = single_water(1)
    bs = BasisSet(basis, mol.atoms, mol.coords)
    D = rand_sym(bs.nbasis, 3)
    ints = _aoi()(bs, thresholdSchwartz=1e-12)
    G = np.zeros_like(D, order="F")
    ints.newTwoEContractDirect([D, D], [G, G], [0, 1], [1.0, -0.5])
    nq = ints.stats()["quartets"]
    Gr, nr = oracle_G(O.OracleBasis.from_basis(bs), [D, D], [0, 1], [1.0, -0.5], 1e-12)
    assert nq == nr
    assert np.abs(G - Gr).max() <= TOL_G


def test_coulomb_and_exchange_separately():
    mol = water_cluster(2, 5)
    bs = BasisSet("cc-pvdz", mol.atoms, mol.coords)
    ob = O.OracleBasis.from_basis(bs)
    D = rand_sym(bs.nbasis, 7)
    ints = _aoi()(bs)
    for t, s in ((0, 1.0), (1, 1.0), (1, -0.37)):
        G = np.zeros_like(D, order="F")
        ints.newTwoEContractDirect([D], [G], [t], [s])
        Gr, _ = oracle_G(ob, [D], [t], [s], 1e-14)
        assert np.abs(G - Gr).max() <= TOL_G, (t, s)


def test_cluster_all_classes_formpt_uhf():
    mol = water_cluster(3, 11)
    bs = BasisSet("cc-pvdz", mol.atoms, mol.coords)
    ob = O.OracleBasis.from_basis(bs)
    Ps = rand_sym(bs.nbasis, 1)
    Pz = rand_sym(bs.nbasis, 2, 0.3)
    ints = _aoi()(bs)
    PTs, PTz = ints.formPT(Ps, Pz)
    st = ints.stats()
    PTs_r, PTz_r, nr = O.form_pt(ob, Ps, Pz)
    assert st["quartets"] == nr
    assert np.abs(PTs - PTs_r).max() <= TOL_G
    assert np.abs(PTz - PTz_r).max() <= TOL_G
    # every class up to (dd|dd) was exercised (the first 21 of the 55 classes)
    assert all(v > 0 for v in list(st["class_quartets"].values())[:21])


def test_device_pointers_match_host():
    torch = pytest.importorskip("torch")
    mol = water_cluster(2, 3)
    bs = BasisSet("6-31g*", mol.atoms, mol.coords)
    Ps = rand_sym(bs.nbasis, 9)
    ints = _aoi()(bs)
    PTs_h, _ = ints.formPT(Ps)
    Pd = torch.from_numpy(np.ascontiguousarray(Ps)).cuda()
    PTs_d, _ = ints.formPT(Pd)
    torch.cuda.synchronize()
    assert np.abs(PTs_d.cpu().numpy() - PTs_h).max() <= 1e-12


def test_schwarz_matches_oracle():
    mol = water_cluster(2, 4)
    bs = BasisSet("cc-pvdz", mol.atoms, mol.coords)
    Q = _aoi()(bs).computeSchwartz()
    Qr = O.schwarz(O.OracleBasis.from_basis(bs))
    assert np.allclose(Q, Qr, rtol=1e-12, atol=1e-14)


def test_accumulate_and_zero_scale():
    mol = single_water(2)
    bs = BasisSet("6-31g*", mol.atoms, mol.coords)
    D = rand_sym(bs.nbasis, 5)
    ints = _aoi()(bs)
    G1 = np.zeros_like(D, order="F")
    ints.newTwoEContractDirect([D, D], [G1, G1], [0, 1], [1.0, -0.5])
    G2 = G1.copy(order="F")
    ints.newTwoEContractDirect([D, D], [G2, G2], [0, 1], [1.0, -0.5])
    assert np.abs(G2 - 2 * G1).max() <= 1e-12
    G3 = np.zeros_like(D, order="F")
    ints.newTwoEContractDirect([D, D], [G3, G3], [0, 1], [0.0, 0.0])
    assert np.abs(G3).max() == 0.0


def test_threshold_screens_everything():
    mol = single_water(3)
    bs = BasisSet("6-31g*", mol.atoms, mol.coords)
    D = rand_sym(bs.nbasis, 5)
    ints = _aoi()(bs, thresholdSchwartz=1e30)
    G = np.full_like(D, 1.25, order="F")
    ints.newTwoEContractDirect([D], [G], [0], [1.0])
    assert ints.stats()["quartets"] == 0
    assert np.all(G == 1.25)


def test_bad_inputs_fail_loudly():
    from chronusq_public_b200._lib import CqgError
    mol = single_water(4)
    bs = BasisSet("6-31g*", mol.atoms, mol.coords)
    ints = _aoi()(bs)
    D = rand_sym(bs.nbasis, 5)
    G = np.zeros_like(D, order="F")
    Dn = D.copy(order="F")
    Dn[3, 4] = np.nan
    Dn[4, 3] = np.nan
    with pytest.raises(CqgError) as e:
        ints.newTwoEContractDirect([Dn], [G], [0], [1.0])
    assert e.value.status == 5
    Da = D.copy(order="F")
    Da[0, 1] += 0.1
    with pytest.raises(CqgError) as e:
        ints.newTwoEContractDirect([Da], [G], [0], [1.0])
    assert e.value.status == 7
    with pytest.raises(AssertionError):
        ints.newTwoEContractDirect([D, D], [G], [0, 1], [1.0, 1.0])


def test_single_atom_and_diffuse_pair():
    li = Molecule.from_angstrom(["Li"], [[0, 0, 0]], mult=2)
    bs = BasisSet("cc-pvdz", li.atoms, li.coords)
    D = rand_sym(bs.nbasis, 8)
    ints = _aoi()(bs)
    G = np.zeros_like(D, order="F")
    ints.newTwoEContractDirect([D, D], [G, G], [0, 1], [1.0, -0.5])
    Gr, nr = oracle_G(O.OracleBasis.from_basis(bs), [D, D], [0, 1], [1.0, -0.5], 1e-14)
    assert ints.stats()["quartets"] == nr
    assert np.abs(G - Gr).max() <= TOL_G


def test_f_shell_classes_cc_pvtz_pair():
    """Two waters in cc-pVTZ: every quartet class up to (ff|ff) (55 classes), UHF lists."""
    mol = water_cluster(2, 17)
    bs = BasisSet("cc-pvtz", mol.atoms, mol.coords)
    ob = O.OracleBasis.from_basis(bs)
    Ps = rand_sym(bs.nbasis, 31)
    Pz = rand_sym(bs.nbasis, 32, 0.2)
    ints = _aoi()(bs)
    PTs, PTz = ints.formPT(Ps, Pz)
    st = ints.stats()
    PTs_r, PTz_r, nr = O.form_pt(ob, Ps, Pz)
    assert st["quartets"] == nr
    assert np.abs(PTs - PTs_r).max() <= TOL_G
    assert np.abs(PTz - PTz_r).max() <= TOL_G
    assert len(st["class_quartets"]) == 55 and st["class_quartets"]["(ff|ff)"] > 0
    # Schwarz values of remote f pairs are square roots of tiny, cancellation-prone
    # integrals: compare with a relative bar on the large ones and an absolute floor
    Q = ints.computeSchwartz()
    assert np.allclose(Q, O.schwarz(ob), rtol=1e-9, atol=1e-12)


def test_chunked_quartet_list_matches_single_pass():
    """A quartet-list budget far below the screened count forces many fill/evaluate
    chunks; the result must be identical to the one-pass build."""
    mol = water_cluster(3, 7)
    bs = BasisSet("cc-pvdz", mol.atoms, mol.coords)
    D = rand_sym(bs.nbasis, 13)
    ints = _aoi()(bs)
    G1, _ = ints.formPT(D)
    n1 = ints.stats()["quartets"]
    ints.setListBudget(100000)
    G2, _ = ints.formPT(D)
    st = ints.stats()
    assert st["chunks"] > 1 and st["quartets"] == n1
    assert np.abs(G2 - G1).max() <= 1e-12


def test_form_pt_rejects_short_leading_dimension_before_writing():
    import ctypes
    mol = single_water(4)
    bs = BasisSet("6-31g*", mol.atoms, mol.coords)
    ints = _aoi()(bs)
    n = bs.nbasis
    D = rand_sym(n, 6)
    PT = np.full((n, n), 7.0, order="F")
    d = ctypes.c_void_p
    st = ints._L.cqg_form_pt(ints._ctx, 1, -0.5, d(D.ctypes.data), None, d(PT.ctypes.data), None, n - 1, 0, None)
    assert st == 1                                   # CQG_ERR_BAD_ARG
    assert b"leading dimension" in ints._L.cqg_last_error(ints._ctx)
    assert (PT == 7.0).all()                          # PT not zeroed on the rejected call
    ints.close()


@pytest.mark.parametrize("basis,nwater,seed", [("cc-pvdz", 3, 11), ("cc-pvtz", 2, 17)])
@pytest.mark.parametrize("form,qpw", [(1, 4), (0, 8)])
def test_forced_schedule_matches_oracle(basis, nwater, seed, form, qpw):
    """Every list run with a forced schedule -- the warp-cooperative form for the classes
    that have both forms (or the per-thread form), and several quartets claimed per warp
    from the work queue -- gives the oracle's G and quartet count (UHF lists)."""
    mol = water_cluster(nwater, seed)
    bs = BasisSet(basis, mol.atoms, mol.coords)
    ob = O.OracleBasis.from_basis(bs)
    Ps = rand_sym(bs.nbasis, 41)
    Pz = rand_sym(bs.nbasis, 42, 0.2)
    ints = _aoi()(bs)
    ints.setSchedule(cta_per_sm=8, warps_per_cta=2, quartets_per_warp=qpw, warp_form=form)
    sch = ints.schedule()
    assert set(sch["quartets_per_warp"]) == {qpw}
    PTs, PTz = ints.formPT(Ps, Pz)
    st = ints.stats()
    PTs_r, PTz_r, nr = O.form_pt(ob, Ps, Pz)
    assert st["quartets"] == nr
    assert np.abs(PTs - PTs_r).max() <= TOL_G
    assert np.abs(PTz - PTz_r).max() <= TOL_G
    ints.close()


def test_set_schedule_rejects_out_of_range_entries():
    from chronusq_public_b200._lib import CqgError
    mol = single_water(4)
    bs = BasisSet("6-31g*", mol.atoms, mol.coords)
    ints = _aoi()(bs)
    before = ints.schedule()
    with pytest.raises(CqgError) as e:
        ints.setSchedule(cta_per_sm=8, warp_form=2)
    assert e.value.status == 1
    assert ints.schedule() == before
    ints.close()


@pytest.mark.parametrize("tier", [1, 2])
def test_class_fused_kernel_matches_oracle(tier):
    """The class-fused persistent kernel (one launch, one device work queue over the lists
    of the tier's classes) gives the oracle's G and quartet count, RHF and UHF lists."""
    mol = water_cluster(3, 11)
    bs = BasisSet("cc-pvdz", mol.atoms, mol.coords)
    ob = O.OracleBasis.from_basis(bs)
    Ps = rand_sym(bs.nbasis, 51)
    Pz = rand_sym(bs.nbasis, 52, 0.2)
    ints = _aoi()(bs)
    ints.setFusion(tier)
    ints.setTiming(True)
    PTs, PTz = ints.formPT(Ps, Pz)
    st = ints.stats()
    assert st["fused_tier"] == tier and st["ms_fused"] > 0.0
    PTs_r, PTz_r, nr = O.form_pt(ob, Ps, Pz)
    assert st["quartets"] == nr
    assert np.abs(PTs - PTs_r).max() <= TOL_G
    assert np.abs(PTz - PTz_r).max() <= TOL_G
    G, _ = ints.formPT(Ps)
    G_r, _, _ = O.form_pt(ob, Ps)
    assert np.abs(G - G_r).max() <= TOL_G
    ints.close()


def test_autotuner_picks_a_fusion_tier_and_keeps_parity():
    mol = water_cluster(3, 12)
    bs = BasisSet("cc-pvdz", mol.atoms, mol.coords)
    ob = O.OracleBasis.from_basis(bs)
    D = rand_sym(bs.nbasis, 53)
    ints = _aoi()(bs)
    ints.autotune_next()
    G1, _ = ints.formPT(D)
    tier, ms = ints.fusion()
    assert tier in (0, 1, 2) and all(t > 0.0 for t in ms)
    G2, _ = ints.formPT(D)
    Gr, _, _ = O.form_pt(ob, D)
    assert np.abs(G1 - Gr).max() <= TOL_G and np.abs(G2 - Gr).max() <= TOL_G
    ints.close()


@pytest.mark.parametrize("basis,nwater,seed", [("cc-pvdz", 3, 11), ("cc-pvtz", 2, 17), ("6-31g*", 3, 5)])
def test_sibling_groups_match_pair_lists_and_oracle(basis, nwater, seed):
    """Sibling-group lists (pairs of the segmented shells of one general contraction share
    their primitive pairs) give the oracle's G and quartet count and the pair-level lists'
    per-class counts (RHF and UHF lists).  cc-pVXZ oxygen's 1s and 2s shells are siblings,
    so fewer list entries and fewer primitive quartets are evaluated; 6-31G(d) has no
    siblings of one angular momentum, so its sibling lists stay empty."""
    mol = water_cluster(nwater, seed)
    bs = BasisSet(basis, mol.atoms, mol.coords)
    ob = O.OracleBasis.from_basis(bs)
    Ps = rand_sym(bs.nbasis, 61)
    Pz = rand_sym(bs.nbasis, 62, 0.2)
    ints = _aoi()(bs)
    ints.setSiblings(True)
    assert ints.siblings()
    on = ints.formPT(Ps, Pz)
    st_on = ints.stats()
    ints.setSiblings(False)
    assert not ints.siblings()
    off = ints.formPT(Ps, Pz)
    st_off = ints.stats()
    PTs_r, PTz_r, nr = O.form_pt(ob, Ps, Pz)
    assert st_on["quartets"] == st_off["quartets"] == nr
    assert st_on["class_quartets"] == st_off["class_quartets"]
    for (PTs, PTz) in (on, off):
        assert np.abs(PTs - PTs_r).max() <= TOL_G
        assert np.abs(PTz - PTz_r).max() <= TOL_G
    assert np.abs(on[0] - off[0]).max() <= 1e-12 and np.abs(on[1] - off[1]).max() <= 1e-12
    assert st_off["sibling_classes"] == [] and st_off["list_entries"] == st_off["quartets"]
    if basis == "6-31g*":
        assert st_on["sibling_classes"] == [] and st_on["list_entries"] == st_on["quartets"]
    else:
        assert "(ss|ss)" in st_on["sibling_classes"] and "(ps|ss)" in st_on["sibling_classes"]
        assert st_on["list_entries"] < st_off["list_entries"]
        assert st_on["prim_quartets"] < st_off["prim_quartets"]
        assert st_on["model_flops"] == pytest.approx(st_off["model_flops"], rel=1e-12)
    ints.close()


def test_sibling_groups_under_forced_schedules_chunks_and_fusion():
    """The sibling lists through several quartets claimed per warp, a list budget that
    forces chunked fill/evaluate passes, and the class-fused kernel beside them."""
    mol = water_cluster(3, 7)
    bs = BasisSet("cc-pvdz", mol.atoms, mol.coords)
    ob = O.OracleBasis.from_basis(bs)
    D = rand_sym(bs.nbasis, 63)
    Gr, _, nr = O.form_pt(ob, D)
    ints = _aoi()(bs)
    ints.setSiblings(True)
    ints.setSchedule(cta_per_sm=8, quartets_per_warp=4)
    G1, _ = ints.formPT(D)
    assert ints.stats()["quartets"] == nr and np.abs(G1 - Gr).max() <= TOL_G
    ints.setListBudget(20000)
    G2, _ = ints.formPT(D)
    st = ints.stats()
    assert st["chunks"] > 1 and st["quartets"] == nr and np.abs(G2 - Gr).max() <= TOL_G
    ints.setListBudget(1 << 32)
    for tier in (1, 2):
        ints.setFusion(tier)
        G3, _ = ints.formPT(D)
        assert ints.stats()["quartets"] == nr and np.abs(G3 - Gr).max() <= TOL_G, tier
    ints.close()
