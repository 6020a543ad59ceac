"""Learned-guess host logic on the CPU: rotation matrices, invariance of the pair features
and local-frame blocks, exact reassembly, and the FP64 network oracle's gradients."""
import numpy as np
import pytest

from chronusq_public_b200 import guess_model as G
from chronusq_public_b200.basis import BasisSet
from chronusq_public_b200.molecule import Molecule, single_water, water_cluster
from oracle import mlp_ref
from oracle import oracle as O


def _rotation(seed):
    q, r = np.linalg.qr(np.random.default_rng(seed).normal(size=(3, 3)))
    q = q * np.sign(np.diag(r))
    return q if np.linalg.det(q) > 0 else -q


class _Geom:
    def __init__(self, atoms, coords):
        self.atoms = list(atoms)
        self.coords = np.asarray(coords)


@pytest.mark.parametrize("l", [2, 3])
def test_pure_rotations_form_an_orthogonal_representation(l):
    A, B = _rotation(1), _rotation(2)
    W = lambda F: G.pure_rotation(l, F[None])[0]
    assert np.abs(W(np.eye(3)) - np.eye(2 * l + 1)).max() < 1e-14
    assert np.abs(W(A).T @ W(A) - np.eye(2 * l + 1)).max() < 1e-13
    assert np.abs(W(A @ B) - W(A) @ W(B)).max() < 1e-13


@pytest.mark.parametrize("basis", ["6-31g*", "cc-pvdz"])
def test_local_blocks_and_features_are_invariant(basis):
    """The overlap matrix transforms like a density: its local-frame pair blocks, and
    the pair features, are the same for a rotated and translated copy of the cluster."""
    mol = water_cluster(3, 5)
    R = np.asarray(mol.coords)
    R2 = R @ _rotation(3).T + np.array([1.0, -2.0, 0.5])
    out = []
    for coords in (R, R2):
        bs = BasisSet(basis, mol.atoms, coords)
        S = O.one_e(O.OracleBasis.from_basis(bs), mol.atoms, coords)[0]
        out.append(G.molecule_samples(_Geom(mol.atoms, coords), bs, 100.0, S) + (S, bs))
    (l1, p1, F1, X1, T1, M1, S1, bs1), (l2, p2, F2, X2, T2, M2, S2, bs2) = out
    assert (p1 == p2).all() and (M1 == M2).all()
    assert np.abs(X1 - X2).max() < 1e-12
    assert np.abs(T1 - T2).max() < 1e-12
    # all pairs kept (cut-off above the cluster size): reassembly is exact
    assert np.abs(G.assemble_density(l1, p1, F1, T1, bs1.nbasis) - S1).max() < 1e-13
    assert np.abs(G.assemble_density(l2, p2, F2, T2, bs2.nbasis) - S2).max() < 1e-13


def test_cutoff_drops_far_pairs_and_small_molecules_work():
    mol = single_water(4)
    bs = BasisSet("6-31g*", mol.atoms, mol.coords)
    layout, pairs, F, X = G.molecule_samples(mol, bs, 8.0)
    assert len(pairs) == 6 and X.shape == (6, G.NFEAT) and np.isfinite(X).all()
    assert all(layout.Z[a] >= layout.Z[b] for a, b in pairs)
    for f in F:
        assert np.abs(f.T @ f - np.eye(3)).max() < 1e-12 and np.linalg.det(f) > 0
    big = water_cluster(6, 2)
    bsb = BasisSet("6-31g*", big.atoms, big.coords)
    _, pb, _, _ = G.molecule_samples(big, bsb, 4.0)
    d = np.linalg.norm(np.asarray(big.coords)[pb[:, 0]] - np.asarray(big.coords)[pb[:, 1]], axis=1)
    assert (d <= 4.0).all() and len(pb) < 18 * 19 // 2


def test_layout_rejects_atoms_beyond_the_output_head():
    mol = single_water(1)
    with pytest.raises(ValueError):
        G.AtomLayout(mol.atoms, BasisSet("cc-pvtz", mol.atoms, mol.coords))


def test_oracle_gradients_match_finite_differences():
    rng = np.random.default_rng(0)
    dims = [7, 9, 9, 5]
    W = [rng.normal(0, 0.5, (dims[i + 1], dims[i])) for i in range(3)]
    b = [rng.normal(0, 0.1, dims[i + 1]) for i in range(3)]
    X = rng.normal(size=(6, 7))
    T = rng.normal(size=(6, 5))
    M = (rng.uniform(size=(6, 5)) > 0.3).astype(float)
    out, cache = mlp_ref.forward(X, W, b)
    gW, gb = mlp_ref.backward(out, T, M, 1 / 6, W, cache)
    h = 1e-6
    for i in range(3):
        for idx in [(0, 0), (dims[i + 1] - 1, dims[i] - 1), (1, 2)]:
            Wp = [w.copy() for w in W]
            Wm = [w.copy() for w in W]
            Wp[i][idx] += h
            Wm[i][idx] -= h
            fd = (mlp_ref.loss(mlp_ref.forward(X, Wp, b)[0], T, M, 1 / 6)
                  - mlp_ref.loss(mlp_ref.forward(X, Wm, b)[0], T, M, 1 / 6)) / (2 * h)
            assert abs(fd - gW[i][idx]) < 1e-7 * max(1.0, abs(fd))
        bp = [x.copy() for x in b]
        bm = [x.copy() for x in b]
        bp[i][0] += h
        bm[i][0] -= h
        fd = (mlp_ref.loss(mlp_ref.forward(X, W, bp)[0], T, M, 1 / 6)
              - mlp_ref.loss(mlp_ref.forward(X, W, bm)[0], T, M, 1 / 6)) / (2 * h)
        assert abs(fd - gb[i][0]) < 1e-7 * max(1.0, abs(fd))
