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
