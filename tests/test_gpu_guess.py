"""Learned-guess kernels and SCF on the GPU: the BF16 GEMM against a torch FP32 product,
forward/backward gradients and Adam against the FP64 CPU oracle, a short training run,
and the learned guess converging to the SAD guess's energy."""
import ctypes
import os

import numpy as np
import pytest

from chronusq_public_b200 import _lib
from oracle import mlp_ref

pytestmark = pytest.mark.gpu


def _p(x):
    return ctypes.c_void_p(x.data_ptr()) if x is not None else None


@pytest.mark.parametrize("M,N,K,trans_a,epilogue", [(300, 196, 57, False, True), (256, 256, 256, True, False),
                                                     (17, 5, 33, False, True), (64, 64, 1000, True, True),
                                                     (20000, 256, 256, False, True), (20000, 196, 64, True, False),
                                                     (256, 196, 4096, True, False), (57, 256, 2000, True, False)])
def test_gemm_bf16_matches_torch_fp32(M, N, K, trans_a, epilogue):
    import torch
    L = _lib.lib()
    g = torch.Generator(device="cuda").manual_seed(M * 7 + K)
    A = torch.randn((K, M) if trans_a else (M, K), device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn((N, K), device="cuda", generator=g).to(torch.bfloat16)
    bias = torch.randn(N, device="cuda", generator=g) if epilogue else None
    C = torch.empty((M, N), device="cuda")
    Y = torch.empty((M, N), device="cuda", dtype=torch.bfloat16) if epilogue else None
    sam, sak = (1, M) if trans_a else (K, 1)
    st = L.cqg_mlp_gemm_bf16(_p(A), sam, sak, _p(B), K, 1, _p(C), N, M, N, K, _p(bias), _p(Y), N,
                             1 if epilogue else 0, 0, None)
    assert st == 0
    Af = (A.t() if trans_a else A).float()
    ref = Af @ B.float().t()
    if epilogue:
        ref = ref + bias
    scale = (Af.abs() @ B.float().abs().t()).max().item()
    torch.cuda.synchronize()
    assert (C - ref).abs().max().item() < 1e-5 * scale
    if epilogue:
        silu = ref * torch.sigmoid(ref)
        assert (Y.float() - silu).abs().max().item() < 1e-2 * silu.abs().max().item()


def test_forward_backward_match_fp64_oracle():
    import torch
    from chronusq_public_b200.guess_model import PairMLP, NFEAT, MAXF
    net = PairMLP(width=256, layers=4, seed=3)
    rng = np.random.default_rng(5)
    net.W[-1] = torch.tensor(rng.normal(0, 0.05, tuple(net.W[-1].shape)), dtype=torch.float32, device=net.dev)
    net.Wbf = [w.to(torch.bfloat16) for w in net.W]
    net.b = [torch.tensor(rng.normal(0, 0.1, b.numel()), dtype=torch.float32, device=net.dev) for b in net.b]
    M = 384
    X = rng.normal(size=(M, NFEAT))
    T = rng.normal(size=(M, MAXF * MAXF))
    Mk = (rng.uniform(size=(M, MAXF * MAXF)) > 0.4).astype(np.float32)
    Xbf = torch.tensor(X, dtype=torch.float32, device=net.dev).to(torch.bfloat16)
    out, cache = net.forward(Xbf, keep=True)
    loss, dout = net.loss_grad(out, torch.tensor(T, dtype=torch.float32, device=net.dev),
                               torch.tensor(Mk, device=net.dev), 1.0 / M)
    gW, gb = net.backward(dout, cache)
    torch.cuda.synchronize()
    Wq = [w.float().cpu().numpy().astype(np.float64) for w in net.Wbf]
    bq = [b.cpu().numpy().astype(np.float64) for b in net.b]
    ro, rc = mlp_ref.forward(Xbf.float().cpu().numpy(), Wq, bq)
    rl = mlp_ref.loss(ro, T, Mk, 1.0 / M)
    rW, rb = mlp_ref.backward(ro, T, Mk, 1.0 / M, Wq, rc)
    o = out.cpu().numpy()
    assert np.linalg.norm(o - ro) / np.linalg.norm(ro) < 2e-2
    assert abs(float(loss) - rl) / rl < 1e-2
    for i in range(len(Wq)):
        gw = gW[i].cpu().numpy()
        gbb = gb[i].cpu().numpy()
        assert np.linalg.norm(gw - rW[i]) / np.linalg.norm(rW[i]) < 3e-2, i
        assert np.linalg.norm(gbb - rb[i]) / np.linalg.norm(rb[i]) < 3e-2, i


def test_adam_matches_oracle():
    import torch
    L = _lib.lib()
    rng = np.random.default_rng(2)
    w0 = rng.normal(size=1000)
    g = rng.normal(size=1000)
    wd = torch.tensor(w0, dtype=torch.float32, device="cuda")
    m1 = torch.zeros_like(wd)
    m2 = torch.zeros_like(wd)
    wbf = torch.empty(1000, dtype=torch.bfloat16, device="cuda")
    gd = torch.tensor(g, dtype=torch.float32, device="cuda")
    rw, r1, r2 = w0.copy(), np.zeros(1000), np.zeros(1000)
    for step in (1, 2, 3):
        assert L.cqg_mlp_adam(_p(wd), _p(gd), _p(m1), _p(m2), 1000, 1e-2, 0.9, 0.999, 1e-8, step, 1e-3, _p(wbf),
                              None) == 0
        mlp_ref.adam_step(rw, g, r1, r2, step, 1e-2, wd=1e-3)
    torch.cuda.synchronize()
    assert np.abs(wd.cpu().numpy() - rw).max() < 1e-5
    assert np.abs(wbf.float().cpu().numpy() - wd.cpu().numpy()).max() < 1e-2


def test_training_lowers_loss_and_learned_guess_keeps_the_energy():
    from chronusq_public_b200.basis import BasisSet
    from chronusq_public_b200.guess_model import PairMLP
    from chronusq_public_b200.learned_guess import cluster_set, converged_densities, training_arrays
    from chronusq_public_b200.scf import SingleSlater
    mols = cluster_set(24, 2, 4, 11)
    P, E, its, _ = converged_densities(mols, "6-31g*")
    X, T, M = training_arrays(mols, "6-31g*", P, 8.0)
    net = PairMLP(width=256, layers=4, seed=1)
    hist = net.fit(X, T, M, epochs=30, batch=256)
    assert hist[-1] < 0.3 * hist[0]
    for mol in cluster_set(2, 2, 4, 12):
        bs = BasisSet("6-31g*", mol.atoms, mol.coords)
        Es = []
        for g in ("SAD", "LEARNED"):
            hf = SingleSlater(mol, bs, thresholdSchwartz=1e-12)
            hf.guess, hf.guess_model = g, net
            Es.append(hf.SCF3())
            assert hf.converged
            hf.close()
        assert abs(Es[0] - Es[1]) < 1e-8


WEIGHTS = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "chronusq_public_b200",
                       "guess_weights", "h2o_6-31gd.npz")


@pytest.mark.skipif(not os.path.exists(WEIGHTS), reason="no trained weights committed")
def test_trained_guess_needs_fewer_iterations_than_sad():
    """Held-out clusters (seed disjoint from training): the shipped network's guess
    converges in fewer SCF iterations than SAD, to the same energy within 1e-8 Eh."""
    from chronusq_public_b200.batch_scf import BatchSCF
    from chronusq_public_b200.guess_model import PairMLP
    from chronusq_public_b200.learned_guess import cluster_set
    net = PairMLP.load(WEIGHTS)
    mols = cluster_set(32, 2, 16, 99)
    res = {}
    for name, mdl in (("sad", None), ("learned", net)):
        b = BatchSCF(mols, "6-31g*", thresholdSchwartz=1e-12)
        res[name] = (b.run(model=mdl), b.iterations.copy())
        assert b.converged
        b.close()
    assert np.abs(res["sad"][0] - res["learned"][0]).max() < 1e-8
    assert res["learned"][1].mean() < res["sad"][1].mean()


WEIGHTS_DZ = os.path.join(os.path.dirname(WEIGHTS), "h2o_cc-pvdz.npz")
WEIGHTS_TZ = os.path.join(os.path.dirname(WEIGHTS), "h2o_cc-pvtz.npz")


def test_cc_pvtz_network_needs_fewer_iterations_than_sad():
    """The cc-pVTZ network (30-function head, trained on cc-pVTZ densities this engine
    converged, clusters of 2-8 waters) on held-out clusters from a disjoint seed: fewer
    batched SCF iterations than SAD, the same energies within 1e-8 Eh."""
    from chronusq_public_b200.batch_scf import BatchSCF
    from chronusq_public_b200.guess_model import PairMLP, default_weights
    from chronusq_public_b200.learned_guess import cluster_set
    assert default_weights("cc-pvtz") == WEIGHTS_TZ
    net = PairMLP.load(WEIGHTS_TZ)
    assert net.maxf == 30
    mols = cluster_set(6, 2, 5, 77)
    res = {}
    for name, mdl in (("sad", None), ("learned", net)):
        b = BatchSCF(mols, "cc-pvtz", thresholdSchwartz=1e-12)
        res[name] = (b.run(model=mdl), b.iterations.copy())
        assert b.converged
        if mdl is not None:
            assert b.guess_fallbacks == 0
        b.close()
    assert np.abs(res["sad"][0] - res["learned"][0]).max() < 1e-8
    assert res["learned"][1].mean() < res["sad"][1].mean()


@pytest.mark.skipif(not os.path.exists(WEIGHTS_DZ), reason="no trained weights committed")
def test_projected_learned_guess_in_a_larger_basis():
    """The cc-pVDZ network's density carried into cc-pVTZ by the overlap projection: the
    projection of a basis onto itself is the identity, and the SCF started from the
    projected prediction converges to the SAD-started energy within 1e-8 Eh."""
    import torch
    from chronusq_public_b200.basis import BasisSet
    from chronusq_public_b200.guess_model import PairMLP, project_density
    from chronusq_public_b200.molecule import water_cluster
    from chronusq_public_b200.scf import SingleSlater
    mol = water_cluster(2, 21)
    dz = BasisSet("cc-pvdz", mol.atoms, mol.coords)
    rng = np.random.default_rng(1)
    A = rng.normal(size=(dz.nbasis, dz.nbasis))
    P = A + A.T
    same = project_density(P, dz, dz)
    assert torch.abs(same - torch.as_tensor(P, device=same.device)).max().item() < 1e-9
    tz = BasisSet("cc-pvtz", mol.atoms, mol.coords)
    net = PairMLP.load(WEIGHTS_DZ)
    Es = []
    for g in ("SAD", "LEARNED"):
        hf = SingleSlater(mol, tz, thresholdSchwartz=1e-12)
        hf.guess, hf.guess_model, hf.guess_source_basis = g, net, "cc-pvdz"
        Es.append(hf.SCF3())
        assert hf.converged
        if g == "LEARNED":
            assert hf.guess_used == "LEARNED"
        hf.close()
    assert abs(Es[0] - Es[1]) < 1e-8


def test_graph_captured_training_matches_uncaptured():
    """fit() with the training step captured as a CUDA graph takes the same steps as the
    uncaptured loop: the same weights and loss history up to FP32 rounding (the weight and
    bias gradients are sums whose order is not fixed: split-K GEMM and column-sum atomics)."""
    import torch
    from chronusq_public_b200.guess_model import PairMLP, NFEAT, MAXF
    rng = np.random.default_rng(5)
    n = 5000
    X = rng.normal(size=(n, NFEAT)).astype(np.float32)
    X[:, -1] = 1.0
    T = rng.normal(size=(n, MAXF * MAXF)).astype(np.float32)
    M = (rng.uniform(size=T.shape) < 0.7).astype(np.float32)
    a = PairMLP(width=64, layers=2, seed=9)
    b = PairMLP(width=64, layers=2, seed=9)
    ha = a.fit(X, T, M, epochs=3, batch=512, graph=True)
    hb = b.fit(X, T, M, epochs=3, batch=512, graph=False)
    torch.cuda.synchronize()
    assert a.step == b.step
    for wa, wb in zip(a.W + a.b, b.W + b.b):
        assert (wa - wb).abs().max().item() <= 1e-5
    assert np.allclose(ha, hb, rtol=1e-3)
