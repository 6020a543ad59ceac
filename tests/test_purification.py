"""The batched SCF's density step by trace-correcting purification (batch_scf.occupied_projector)
against the eigenvector projector, on stacks of symmetric matrices with an open gap
(torch on the CPU; the same code runs on the GPU)."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from chronusq_public_b200.batch_scf import occupied_projector


def _stack(G, n, nocc, gap, seed):
    rng = np.random.default_rng(seed)
    F = np.zeros((G, n, n))
    for g in range(G):
        occ = np.sort(rng.uniform(-25.0, -gap / 2, nocc))           # core to valence
        virt = np.sort(rng.uniform(gap / 2, 8.0, n - nocc))
        Q, _ = np.linalg.qr(rng.normal(size=(n, n)))
        F[g] = (Q * np.concatenate([occ, virt])) @ Q.T
    return torch.tensor(F, dtype=torch.float64)


@pytest.mark.parametrize("G,n,nocc,gap", [(3, 18, 5, 0.6), (4, 90, 25, 0.4), (2, 216, 60, 0.3)])
def test_purification_gives_the_eigenvector_projector(G, n, nocc, gap):
    F = _stack(G, n, nocc, gap, n)
    P = occupied_projector(F, nocc)
    assert P is not None
    _, C = torch.linalg.eigh(F)
    Co = C[..., :nocc]
    Pref = Co @ Co.transpose(-1, -2)
    assert (P - Pref).abs().max().item() < 1e-12
    assert (P @ P - P).abs().max().item() < 1e-12
    tr = P.diagonal(dim1=-2, dim2=-1).sum(-1)
    assert (tr - nocc).abs().max().item() < 1e-10


def test_purification_reports_a_closed_gap():
    """Degenerate levels across the Fermi level: no projector (the caller diagonalises)."""
    n, nocc = 12, 5
    w = np.concatenate([np.linspace(-5, -1, nocc - 1), [0.0, 0.0], np.linspace(1, 5, n - nocc - 1)])
    Q, _ = np.linalg.qr(np.random.default_rng(3).normal(size=(n, n)))
    F = torch.tensor(((Q * w) @ Q.T)[None])
    assert occupied_projector(F, nocc, max_iter=60) is None
