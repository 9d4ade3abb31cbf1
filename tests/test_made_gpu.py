"""Proposal network on the GPU: the tensor-core GEMM against a PyTorch fp32 reference, the
hand-written backward pass against FP64 autograd (the CPU oracle), the sampler's log q (sample and
evaluate agree bit for bit; the distribution matches q), training raises the likelihood, and the
exact Metropolis-Hastings step leaves the Boltzmann distribution stationary (exact enumeration) with
a random and with a trained network."""

from __future__ import annotations

import numpy as np
import pytest

import oracle
from conftest import cuda_ready
from oracle import made_ref

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_ready(), reason="needs CUDA and libdrift_pt.so")]


def _gemm(A, B, **kw):
    import torch

    from drift_b200.made import Made

    m = Made.__new__(Made)
    m.torch, m.device = torch, A.device
    m.err = torch.zeros(1, dtype=torch.int32, device=A.device)
    m._bufs = {}
    M, N, K = A.shape[0], B.shape[0], A.shape[1]
    out = torch.zeros((M, N), dtype=torch.float32, device=A.device)
    m._gemm(A, B, M, N, K, out_f32=out, **kw)
    m.check()
    return out


@pytest.mark.parametrize("M,N,K", [(128, 64, 64), (200, 100, 72), (512, 1024, 512), (64, 512, 1024), (1024, 48, 256)])
def test_gemm_matches_fp32_reference(M, N, K):
    import torch

    g = torch.Generator().manual_seed(M + N + K)
    A = torch.randn(M, K, generator=g).to(torch.bfloat16)
    B = torch.randn(N, K, generator=g).to(torch.bfloat16)
    bias = torch.randn(N, generator=g)
    ref = A.float() @ B.float().T
    out = _gemm(A.cuda(), B.cuda()).cpu()
    tol = 1e-5 * K  # fp32 accumulation of bf16 products, in any order
    assert torch.allclose(out, ref, atol=tol, rtol=1e-5)
    out = _gemm(A.cuda(), B.cuda(), bias=bias.cuda(), act=1).cpu()
    assert torch.allclose(out, torch.relu(ref + bias), atol=tol, rtol=1e-5)
    R = torch.randn(M, N, generator=g).to(torch.bfloat16)
    out = _gemm(A.cuda(), B.cuda(), ref=R.cuda()).cpu()
    assert torch.allclose(out, ref * (R.float() > 0), atol=tol, rtol=1e-5)


@pytest.mark.parametrize("n,h,B", [(16, 32, 64), (64, 128, 256), (512, 1024, 128)])
def test_gradients_match_fp64_autograd(n, h, B):
    import torch

    from drift_b200.made import Made

    made = Made(n, (h, h), seed=3)
    rng = np.random.default_rng(5)
    x = np.where(rng.random((B, n)) < 0.5, -1, 1).astype(np.int8)
    W, b = made.weights_host()
    b = [rng.normal(scale=0.1, size=v.shape) for v in b]  # nonzero biases exercise the bias path
    for k in range(3):
        made.b[k].copy_(torch.from_numpy(b[k]).float())
    lq = made.loss_and_grad(torch.from_numpy(x).cuda()).cpu().numpy()
    made.check()
    got = [g.cpu().numpy() for g in made.gW] + [g.cpu().numpy() for g in made.gb]
    # (1) the same pass with the device's bf16 roundings, in FP64: only the FP32 accumulation order
    # (and the rare bf16 rounding it tips) differ
    lq_b, gW_b, gb_b = made_ref.logq_and_grads_bf16(W, b, x)
    assert np.max(np.abs(lq - lq_b)) <= 1e-4 * np.max(np.abs(lq_b))
    for g, ref in zip(got, gW_b + gb_b):
        rel = np.linalg.norm(g - ref) / max(np.linalg.norm(ref), 1e-30)
        assert rel < 5e-3, rel
    # (2) exact FP64 autograd of the same network: the bf16 activations and back-propagated signals
    # (8-bit mantissas, relative rounding 2^-9 per value) leave a few percent at most
    lq_ref, gW_ref, gb_ref, _ = made_ref.logq_and_grads(W, b, x)
    assert np.max(np.abs(lq - lq_ref)) <= 2e-2 * np.max(np.abs(lq_ref))
    for g, ref in zip(got, gW_ref + gb_ref):
        rel = np.linalg.norm(g - ref) / max(np.linalg.norm(ref), 1e-30)
        assert rel < 5e-2, rel


def test_sampler_logq_is_one_function_and_matches_fp64():
    import torch

    from drift_b200.made import Made

    n, h = 64, 128
    made = Made(n, (h, h), seed=7)
    for k in range(3):
        made.b[k].normal_(0.0, 0.3)
    x, lq = made.sample(40, seed=11, stream_id=2)
    lq_eval = made.logq(x)
    assert torch.equal(lq, lq_eval)  # bit for bit
    x2, lq2 = made.sample(40, seed=11, stream_id=2)
    assert torch.equal(x, x2) and torch.equal(lq, lq2)
    W, b = made.weights_host()
    ref = made_ref.logq(W, b, x.cpu().numpy())
    assert np.allclose(lq.cpu().numpy(), ref, rtol=1e-4, atol=1e-4)
    assert set(np.unique(x.cpu().numpy())) <= {-1, 1}


def test_sampler_draws_from_q():
    """Chi-square of 200,000 draws of an n = 8 network against its exact q."""
    from drift_b200.made import Made

    n = 8
    made = Made(n, (16, 16), seed=1)
    for k in range(3):
        made.b[k].normal_(0.0, 0.8)
    W, b = made.weights_host()
    xs, lq = made_ref.all_logq(W, b, n)
    p = np.exp(lq)
    x, _ = made.sample(200_000, seed=3)
    codes = ((x.cpu().numpy() > 0).astype(np.int64) * (1 << np.arange(n - 1, -1, -1))).sum(1)
    ref_codes = ((xs > 0).astype(np.int64) * (1 << np.arange(n - 1, -1, -1))).sum(1)
    counts = np.bincount(codes, minlength=1 << n)[ref_codes]
    expected = p * len(codes)
    keep = expected > 5
    chi2 = (((counts - expected) ** 2) / expected)[keep].sum()
    dof = keep.sum() - 1
    assert chi2 < dof + 6 * np.sqrt(2 * dof), (chi2, dof)


def test_suffix_sampler_keeps_the_prefix_and_its_logq_is_one_function():
    import torch

    from drift_b200.made import Made

    n, h = 64, 128
    made = Made(n, (h, h), seed=7)
    for k in range(3):
        made.b[k].normal_(0.0, 0.3)
    x0, _ = made.sample(40, seed=5, stream_id=1)
    x = x0.clone()
    lq = made.sample_suffix(x, 40, seed=11, stream_id=2)
    assert torch.equal(x[:, :40], x0[:, :40])
    assert not torch.equal(x[:, 40:], x0[:, 40:])
    assert torch.equal(lq, made.logq(x))  # bit for bit, as for whole draws
    y = x0.clone()
    assert torch.equal(made.sample_suffix(y, n, seed=11, stream_id=2), made.logq(x0)) and torch.equal(y, x0)


def test_suffix_sampler_draws_from_the_conditionals():
    """Chi-square of 100,000 redraws of the last 3 spins of an n = 8 network given fixed first 5,
    against the exact conditional q(x_5, x_6, x_7 | x_0..x_4)."""
    import torch

    from drift_b200.made import Made

    n, keep = 8, 5
    made = Made(n, (16, 16), seed=2)
    for k in range(3):
        made.b[k].normal_(0.0, 0.8)
    W, b = made.weights_host()
    xs, lq = made_ref.all_logq(W, b, n)
    prefix = np.array([1, -1, -1, 1, 1], np.int8)
    sel = np.all(xs[:, :keep] == prefix, axis=1)
    p = np.exp(lq[sel])
    p /= p.sum()
    N = 100_000
    x = torch.from_numpy(np.tile(np.concatenate([prefix, np.ones(n - keep, np.int8)]), (N, 1))).cuda()
    made.sample_suffix(x, keep, seed=4)
    xh = x.cpu().numpy()
    assert np.all(xh[:, :keep] == prefix)
    w = 1 << np.arange(n - keep - 1, -1, -1)
    codes = ((xh[:, keep:] > 0).astype(np.int64) * w).sum(1)
    ref_codes = ((xs[sel][:, keep:] > 0).astype(np.int64) * w).sum(1)
    counts = np.bincount(codes, minlength=1 << (n - keep))[ref_codes]
    expected = p * N
    chi2 = (((counts - expected) ** 2) / expected).sum()
    dof = len(p) - 1
    assert chi2 < dof + 6 * np.sqrt(2 * dof), (chi2, dof)


def test_training_raises_the_likelihood_of_the_data():
    import torch

    from drift_b200.made import Made

    n = 32
    rng = np.random.default_rng(2)
    # data: two ferromagnetic clusters with 5% flips
    base = np.where(rng.random(4096) < 0.5, -1, 1)[:, None] * np.ones((1, n))
    noise = np.where(rng.random((4096, n)) < 0.05, -1, 1)
    data = torch.from_numpy((base * noise).astype(np.int8)).cuda()
    made = Made(n, (64, 64), seed=0)
    hist = made.train(data, epochs=8, batch=256, lr=3e-3)
    assert hist[-1] > hist[0] + 5.0, hist
    # the data's entropy per configuration is log 2 + n H(0.05) = 0.69 + 32 * 0.199 = 7.05 nats
    assert hist[-1] > -9.0, hist


@pytest.mark.parametrize("trained,suffix", [(False, None), (True, None), (True, 6)])
def test_neural_pt_is_stationary_at_the_boltzmann_distribution(trained, suffix):
    """SK n = 16: per-rung mean energy of neural-proposal PT vs exact enumeration, with independent
    proposals and with conditional ones that redraw the last 6 spins."""
    from drift_b200.instances import sk_model
    from drift_b200.made import Made
    from drift_b200.neural import NeuralPT, collect_cold_samples
    from drift_b200.sk import SkEngine, SkModel

    n = 16
    sk = SkModel.from_model(sk_model(n, 11))
    betas = np.array([0.4, 0.8, 1.4, 2.2])
    made = Made(n, (32, 32), seed=0)
    if trained:
        pre = SkEngine(sk, betas, seed=9, sweeps_per_round=2)
        pre.init()
        data = collect_cold_samples(pre, 4096, n_cold=2)
        made.train(data, epochs=10, batch=256, lr=3e-3)
    ex = oracle.exact(sk.Jq * 2.0 ** -sk.shift, sk.hq * 2.0 ** -sk.shift, betas)
    npt = NeuralPT(sk, betas, made, seed=4, sweeps_per_round=1, n_cold=4, suffix=suffix)
    npt.init()
    npt.run(50)
    es = []
    for _ in range(1500):
        npt.run(1)
        slots = npt.eng.slot_of_rung.long()
        es.append(npt.eng.energy.index_select(0, slots).cpu().numpy())
    npt.eng.check()
    e = np.array(es, np.float64) * sk.energy_unit
    mean, sd = e.mean(0), e.std(0)
    # successive rounds are correlated; 8 naive standard errors
    assert np.all(np.abs(mean - ex.mean_e) <= 8 * sd / np.sqrt(len(e)) + 1e-9), (mean, ex.mean_e)
    acc = npt.acceptance()
    assert np.all(npt.prop_tried.cpu().numpy() > 0)
    if trained:
        assert np.nanmean(acc) > 0.05, acc


def test_trained_network_gains_over_the_untrained_one():
    """SK n = 64: trained on plain PT's cold configurations, the network's proposals are accepted
    far more often at the cold rungs than those of the same network untrained, and held-out cold
    configurations are far more likely under it."""
    import torch

    from drift_b200.instances import sk_model
    from drift_b200.made import Made
    from drift_b200.neural import NeuralPT, collect_cold_samples
    from drift_b200.sk import SkEngine, SkModel

    n = 64
    sk = SkModel.from_model(sk_model(n, 21))
    betas = 0.3 * 10.0 ** (np.arange(16) / 15)  # 0.3 .. 3.0
    pre = SkEngine(sk, betas, seed=2, sweeps_per_round=5)
    pre.init()
    pre.run(100)
    data = collect_cold_samples(pre, 8192 + 1024, n_cold=4)
    train, held = data[:8192], data[8192:]
    untrained = Made(n, (128, 128), seed=1)
    trained = Made(n, (128, 128), seed=1)
    trained.train(train, epochs=20, batch=256, lr=3e-3)
    ll_u = float(untrained.logq(held).mean().item())
    ll_t = float(trained.logq(held).mean().item())
    assert ll_t > ll_u + 10.0, (ll_t, ll_u)
    acc = {}
    for name, net in (("untrained", untrained), ("trained", trained)):
        npt = NeuralPT(sk, betas, net, seed=5, sweeps_per_round=5, n_cold=4)
        npt.init()
        npt.run(200)
        npt.eng.check()
        t = npt.prop_tried.cpu().numpy()[-4:].sum()
        a = npt.prop_accepted.cpu().numpy()[-4:].sum()
        acc[name] = a / t
    assert acc["trained"] > 0.02 and acc["trained"] > 5 * acc["untrained"], acc
