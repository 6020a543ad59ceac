"""G[X] parity at the benchmarked configurations, on the SCF's own SAD-guess densities.

* (H2O)_32 in cc-pVDZ (N = 768, quartet classes to (dd|dd)), Schwarz threshold 1e-14, the
  SAD-guess density of the SCF guess path: the exact input of the Fock-build benchmark.
  The oracle restatement of newTwoEContractDirect
  (include/aointegrals/aointegrals_contract.h:96-193) runs on every host core (about a
  minute on 16 cores).
* A single water in 6-31G(d) at Schwarz threshold 1e-12, on its SAD-guess density (the
  random-density check of the same system is in test_gpu_parity.py).

Bar: the screened quartet count equal to the oracle's and max|G_gpu - G_oracle| <= 1e-10.
"""
import os

import numpy as np
import pytest

from chronusq_public_b200.basis import BasisSet
from chronusq_public_b200.molecule import single_water, water_cluster
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL_G = 1e-10


def _sad_density(mol, bs, thresh):
    from chronusq_public_b200.scf import SingleSlater
    hf = SingleSlater(mol, bs, thresholdSchwartz=thresh)
    Ps, _, _, _ = hf.formGuess()
    D = Ps.cpu().numpy()
    return hf, np.asfortranarray(0.5 * (D + D.T))


def _check(mol, basis, thresh):
    bs = BasisSet(basis, mol.atoms, mol.coords)
    hf, D = _sad_density(mol, bs, thresh)
    ints = hf.ints
    ints.thresholdSchwartz = thresh
    PT, _ = ints.formPT(D)
    nq = ints.stats()["quartets"]
    hf.close()
    ob = O.OracleBasis.from_basis(bs)
    PTr, _, nr = O.form_pt(ob, D, thresh=thresh, nthreads=os.cpu_count())
    err = float(np.abs(PT - PTr).max())
    return nq, nr, err


@pytest.mark.slow
def test_h2o32_ccpvdz_sad_density_matches_oracle():
    nq, nr, err = _check(water_cluster(32, 1), "cc-pvdz", 1e-14)
    assert nq == nr
    assert err <= TOL_G, err


def test_water_631gd_sad_density_matches_oracle():
    nq, nr, err = _check(single_water(0), "6-31g*", 1e-12)
    assert nq == nr
    assert err <= TOL_G, err
