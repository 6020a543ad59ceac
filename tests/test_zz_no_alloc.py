"""cqg_one_e_noalloc (one-electron integrals with a fixed module-scope charge table, no
allocation) against the allocating entry point cqg_one_e, both called through the C-ABI.

The entry point serves callers that cannot allocate device memory once they run: a host
program whose own memory pool already holds the GPU, or a loop that must not take the
device-wide synchronisation a cudaMalloc/cudaFree brings.

Named to be collected last, so it runs both after every other test and alone."""
import ctypes

import numpy as np
import pytest

from chronusq_public_b200 import _lib
from chronusq_public_b200.basis import BasisSet
from chronusq_public_b200.molecule import water_cluster

pytestmark = pytest.mark.gpu

MAX_CHARGES = 4096          # CQG_ONE_E_NOALLOC_MAX_CHARGES
TOL = {"S": 1e-12, "T": 1e-11, "V": 1e-10}


def _charges(mol, extra, seed):
    """The nuclei plus `extra` seeded point charges in the molecule's box (bohr)."""
    Z = np.asarray(mol.atoms, dtype=np.float64)
    R = np.asarray(mol.coords, dtype=np.float64).reshape(-1, 3)
    if extra:
        rng = np.random.default_rng(seed)
        Z = np.concatenate([Z, rng.uniform(-1.0, 1.0, extra)])
        R = np.concatenate([R, rng.uniform(R.min(0) - 2.0, R.max(0) + 2.0, (extra, 3))])
    return np.ascontiguousarray(Z), np.ascontiguousarray(R)


def _allocating(ai, Z, R, out, stream):
    L = ai._L
    d = ctypes.POINTER(ctypes.c_double)
    st = L.cqg_one_e(ai._ctx, len(Z), Z.ctypes.data_as(d), R.ctypes.data_as(d),
                     *[ctypes.c_void_p(x.data_ptr()) for x in out], ai.nBasis, 1, stream)
    _lib.check(st, ai._ctx)


def _no_alloc(ai, nq, zp, rp, out, stream, ld=None):
    return ai._L.cqg_one_e_noalloc(ai._ctx, nq, ctypes.c_void_p(zp), ctypes.c_void_p(rp),
                                   *[ctypes.c_void_p(x.data_ptr()) for x in out],
                                   ai.nBasis if ld is None else ld, stream)


@pytest.mark.parametrize("basis", ["6-31g*", "cc-pvdz"])
def test_no_alloc_matches_allocating_entry_point(basis):
    """Two calls in a row on a fresh context (host charges, then device charges with a
    padded leading dimension) match cqg_one_e, and neither call changes the device's free
    memory: the first call, which resolves the table's address, included."""
    import torch
    from chronusq_public_b200.aointegrals import AOIntegrals
    mol = water_cluster(2, 9)
    bs = BasisSet(basis, mol.atoms, mol.coords)
    ai = AOIntegrals(bs)
    n = ai.nBasis
    ldp = n + 3
    dev = torch.device("cuda", 0)
    stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    cases = [_charges(mol, 0, 1), _charges(mol, 300, 2)]
    # every buffer both calls need, allocated before the calls; the second call writes into
    # column-major n x n blocks of ldp x n arrays (stored as n rows of ldp in torch)
    ref = [[torch.zeros((n, n), dtype=torch.float64, device=dev) for _ in range(3)] for _ in cases]
    got0 = [torch.full((n, n), float("nan"), dtype=torch.float64, device=dev) for _ in range(3)]
    got1 = [torch.full((n, ldp), float("nan"), dtype=torch.float64, device=dev) for _ in range(3)]
    Zd = torch.tensor(cases[1][0], device=dev)
    Rd = torch.tensor(cases[1][1], device=dev)
    for (Z, R), out in zip(cases, ref):
        _allocating(ai, Z, R, out, stream)
    torch.cuda.synchronize(dev)

    Z0, R0 = cases[0]
    free0 = torch.cuda.mem_get_info(dev)[0]
    assert _no_alloc(ai, len(Z0), Z0.ctypes.data, R0.ctypes.data, got0, stream) == 0, ai._L.cqg_last_error(ai._ctx)
    torch.cuda.synchronize(dev)
    assert torch.cuda.mem_get_info(dev)[0] == free0
    assert _no_alloc(ai, len(cases[1][0]), Zd.data_ptr(), Rd.data_ptr(), got1, stream, ld=ldp) == 0
    torch.cuda.synchronize(dev)
    assert torch.cuda.mem_get_info(dev)[0] == free0

    for name, a, b in zip("STV", ref[0], got0):
        err = (a - b).abs().max().item()
        assert err < TOL[name], (basis, name, err)
    for name, a, b in zip("STV", ref[1], got1):
        # column j of the column-major result is row j of the torch array; the matrices
        # are symmetric, so the n x n block compares with either orientation
        err = (a - b[:, :n]).abs().max().item()
        assert err < TOL[name], (basis, name, err)
        assert torch.isnan(b[:, n:]).all(), (basis, name, "padding rows written")
    ai.close()


def test_no_alloc_rejects_bad_sizes_before_writing():
    """More charges than the table holds, or a leading dimension below nbf: status
    CQG_ERR_BAD_ARG with a message, and nothing written."""
    import torch
    from chronusq_public_b200.aointegrals import AOIntegrals
    mol = water_cluster(2, 4)
    bs = BasisSet("6-31g*", mol.atoms, mol.coords)
    ai = AOIntegrals(bs)
    n = ai.nBasis
    dev = torch.device("cuda", 0)
    stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    out = [torch.full((n, n), 7.0, dtype=torch.float64, device=dev) for _ in range(3)]
    Z = np.ones(MAX_CHARGES + 1)
    R = np.zeros((MAX_CHARGES + 1, 3))
    st = _no_alloc(ai, MAX_CHARGES + 1, Z.ctypes.data, R.ctypes.data, out, stream)
    assert st == 1                                   # CQG_ERR_BAD_ARG
    assert b"4096" in ai._L.cqg_last_error(ai._ctx)
    Zn, Rn = _charges(mol, 0, 0)
    st = _no_alloc(ai, len(Zn), Zn.ctypes.data, Rn.ctypes.data, out, stream, ld=n - 1)
    assert st == 1
    assert b"leading dimension" in ai._L.cqg_last_error(ai._ctx)
    torch.cuda.synchronize(dev)
    assert all(bool((x == 7.0).all()) for x in out)
    ai.close()
