"""cqg_one_e_noalloc (one-electron integrals with a fixed module-scope charge table, no
allocation) against the allocating entry point cqg_one_e, both called through the C-ABI.

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


def _no_alloc(ai, nq, zp, rp, out, stream):
    return ai._L.cqg_one_e_noalloc(ai._ctx, nq, ctypes.c_void_p(zp), ctypes.c_void_p(rp),
                                   *[ctypes.c_void_p(x.data_ptr()) for x in out], ai.nBasis, stream)


@pytest.mark.parametrize("basis", ["6-31g*", "cc-pvdz"])
def test_no_alloc_matches_allocating_entry_point(basis):
    import torch
    from chronusq_public_b200.aointegrals import AOIntegrals
    mol = water_cluster(2, 9)
    bs = BasisSet(basis, mol.atoms, mol.coords)
    ai = AOIntegrals(bs)
    n = ai.nBasis
    dev = torch.device("cuda", 0)
    stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    cases = [_charges(mol, 0, 1), _charges(mol, 300, 2)]
    # every buffer both calls need, allocated before the calls
    ref = [[torch.zeros((n, n), dtype=torch.float64, device=dev) for _ in range(3)] for _ in cases]
    got = [[torch.full((n, n), float("nan"), dtype=torch.float64, device=dev) for _ in range(3)] for _ in cases]
    Zd = torch.tensor(cases[1][0], device=dev)
    Rd = torch.tensor(cases[1][1], device=dev)
    for (Z, R), out in zip(cases, ref):
        _allocating(ai, Z, R, out, stream)
    torch.cuda.synchronize(dev)

    # two calls in a row: host charges first, device charges second
    Z0, R0 = cases[0]
    assert _no_alloc(ai, len(Z0), Z0.ctypes.data, R0.ctypes.data, got[0], stream) == 0, ai._L.cqg_last_error(ai._ctx)
    torch.cuda.synchronize(dev)
    free0 = torch.cuda.mem_get_info(dev)[0]
    assert _no_alloc(ai, len(cases[1][0]), Zd.data_ptr(), Rd.data_ptr(), got[1], stream) == 0
    torch.cuda.synchronize(dev)
    assert torch.cuda.mem_get_info(dev)[0] == free0

    for out_ref, out_got in zip(ref, got):
        for name, a, b in zip("STV", out_ref, out_got):
            err = (a - b).abs().max().item()
            assert err < TOL[name], (basis, name, err)
    ai.close()


def test_no_alloc_rejects_too_many_charges():
    import torch
    from chronusq_public_b200.aointegrals import AOIntegrals
    mol = water_cluster(2, 4)
    bs = BasisSet("6-31g*", mol.atoms, mol.coords)
    ai = AOIntegrals(bs)
    n = ai.nBasis
    dev = torch.device("cuda", 0)
    out = [torch.zeros((n, n), dtype=torch.float64, device=dev) for _ in range(3)]
    Z = np.ones(MAX_CHARGES + 1)
    R = np.zeros((MAX_CHARGES + 1, 3))
    st = _no_alloc(ai, MAX_CHARGES + 1, Z.ctypes.data, R.ctypes.data, out,
                   ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream))
    assert st == 1                                   # CQG_ERR_BAD_ARG
    assert b"4096" in ai._L.cqg_last_error(ai._ctx)
    ai.close()
