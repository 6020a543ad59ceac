"""Batched contexts (many molecules of uneven size) against one-molecule contexts."""
import numpy as np
import pytest

from chronusq_public_b200.basis import BasisSet
from chronusq_public_b200.molecule import water_cluster, single_water

pytestmark = pytest.mark.gpu


def _mols():
    out = [single_water(3), water_cluster(2, 4), water_cluster(3, 5), single_water(8), water_cluster(4, 6)]
    return out


def test_batch_formpt_and_one_e_match_single_contexts():
    import torch
    from chronusq_public_b200.aointegrals import AOIntegrals
    from chronusq_public_b200.batch import BatchAOIntegrals
    mols = _mols()
    bss = [BasisSet("6-31g*", m.atoms, m.coords) for m in mols]
    B = BatchAOIntegrals(bss)
    rng = np.random.default_rng(0)
    Ds = []
    for bs in bss:
        a = rng.uniform(-1, 1, (bs.nbasis, bs.nbasis))
        Ds.append(0.5 * (a + a.T))
    P = B.pack(Ds)
    PT = B.formPT(P)
    S, T, V = B.computeAOOneE(mols)
    torch.cuda.synchronize()
    total = 0
    for m, (bs, D) in enumerate(zip(bss, Ds)):
        ints = AOIntegrals(bs)
        PTr, _ = ints.formPT(np.asfortranarray(D))
        total += ints.stats()["quartets"]
        assert np.abs(B.view(PT, m).cpu().numpy() - PTr).max() < 1e-11
        Sr, Tr, Vr = ints.computeAOOneE(mols[m].atoms, mols[m].coords)
        assert np.abs(B.view(S, m).cpu().numpy() - Sr).max() < 1e-12
        assert np.abs(B.view(V, m).cpu().numpy() - Vr).max() < 1e-11
        ints.close()
    assert B.stats()["quartets"] == total
    # inactive molecules are left untouched
    PT2 = B.formPT(P, active=[1, 0, 1, 0, 1])
    torch.cuda.synchronize()
    assert float(B.view(PT2, 1).abs().max()) == 0.0
    assert np.abs(B.view(PT2, 2).cpu().numpy() - B.view(PT, 2).cpu().numpy()).max() < 1e-12
    B.close()


def test_batched_scf_matches_one_at_a_time():
    """Lock-step batched RHF (one batched Fock build per iteration) converges every
    molecule to the energy of its own one-molecule SCF (C3 procedure, small)."""
    from chronusq_public_b200.batch_scf import BatchSCF
    from chronusq_public_b200.scf import SingleSlater
    mols = [single_water(21), water_cluster(2, 22), water_cluster(3, 23), water_cluster(2, 24)]
    bscf = BatchSCF(mols, "6-31g*")
    E = bscf.run()
    assert bscf.converged
    for m, mol in enumerate(mols):
        hf = SingleSlater(mol, BasisSet("6-31g*", mol.atoms, mol.coords), thresholdSchwartz=1e-12)
        Er = hf.SCF3()
        hf.close()
        assert abs(E[m] - Er) < 1e-8, (m, E[m], Er)
    bscf.close()


def test_batched_scf_graph_and_autotune_give_same_energies():
    from chronusq_public_b200.batch_scf import BatchSCF
    mols = [single_water(31), water_cluster(2, 32), water_cluster(3, 33), single_water(34)]
    a = BatchSCF(mols, "6-31g*")
    Ea = a.run()
    a.close()
    b = BatchSCF(mols, "6-31g*")
    Eb = b.run(use_graph=True, autotune=True)
    assert b.converged and b.graph_replays > 0
    cta, wpb = b.B.launch_shapes()
    assert (cta > 0).any()
    b.close()
    assert np.abs(Ea - Eb).max() < 1e-9
