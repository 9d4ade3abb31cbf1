"""Batched neural proposals on the GPU: the gather equals the engine's own view, the MH step
replaces exactly what it accepts (energies recomputed exactly) and leaves everything else, the
grouped sampler equals the single-network sampler bit for bit, and neural-proposal PT on a batch
keeps every rung's Boltzmann distribution (exact enumeration)."""

from __future__ import annotations

import numpy as np
import pytest

import oracle
from conftest import cuda_ready

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_ready(), reason="needs CUDA and libdrift_pt.so")]


def small_batch(models, betas, seed=3, spr=1):
    from drift_b200.batch import BatchEngine, BatchProblem
    from drift_b200.engine import HostProblem

    bp = BatchProblem([HostProblem.from_model(m) for m in models], [betas] * len(models))
    return bp, BatchEngine(bp, seed=seed, sweeps_per_round=spr)


def batch_of_sizes(Ls):
    from drift_b200.instances import ea_2d_padded

    return [ea_2d_padded(L, 10 + k) for k, L in enumerate(Ls)]


def nets_for(bp, hidden=32):
    from drift_b200.made import Made

    return {k: Made(int(d["n"]), (hidden, hidden), seed=k) for k, d in enumerate(bp.desc)}


def test_gather_matches_the_engine_view():
    from drift_b200.batch_neural import BatchNeuralPT

    bp, eng = small_batch(batch_of_sizes((4, 5, 8, 11)), 0.3 * 10.0 ** (np.arange(8) / 7))
    eng.init()
    eng.run(3)
    eng.check()
    bn = BatchNeuralPT(eng, nets_for(bp), n_cold=3)
    bn.gather(bn.x_cur, bn.d_off)
    bn.check()
    x = bn.x_cur.cpu().numpy()
    for k, r, o in zip(bn.inst_h, bn.rung_h, bn.off_h):
        f = eng.fetch(int(k))
        n = int(bp.desc[k]["n"])
        assert np.array_equal(x[o:o + n], f["spins"][f["slot_of_rung"][r]])


@pytest.mark.parametrize("force", ["accept", "reject"])
def test_mh_replaces_exactly_what_it_accepts(force):
    import torch

    from drift_b200.batch_neural import BatchNeuralPT

    models = batch_of_sizes((4, 6, 9))
    bp, eng = small_batch(models, 0.3 * 10.0 ** (np.arange(6) / 5))
    eng.init()
    eng.run(2)
    eng.check()
    bn = BatchNeuralPT(eng, nets_for(bp), n_cold=4)
    before = [eng.fetch(k) for k in range(len(models))]
    rng = np.random.default_rng(5)
    xp = rng.choice(np.array([-1, 1], np.int8), size=bn.x_prop.numel())
    bn.x_prop.copy_(torch.from_numpy(xp))
    big = 1.0e6 if force == "accept" else -1.0e6
    bn.lq_cur.fill_(0.0)
    bn.lq_prop.fill_(-big)
    bn.mh(0)
    bn.check()
    pe = bn.prop_energy.cpu().numpy()
    for j, (k, r, o) in enumerate(zip(bn.inst_h, bn.rung_h, bn.off_h)):
        m = models[k]
        n = m.n
        assert pe[j] == m.energy(xp[o:o + n].astype(np.float64))  # exact recount on the device
        b, a = before[k], eng.fetch(int(k))
        slot = b["slot_of_rung"][r]
        if force == "accept":
            assert np.array_equal(a["spins"][slot], xp[o:o + n])
            assert a["energy_fixed"][slot] == pe[j]
            assert a["best_energy_fixed"][slot] == min(b["best_energy_fixed"][slot], pe[j])
        else:
            assert np.array_equal(a["spins"][slot], b["spins"][slot])
            assert a["energy_fixed"][slot] == b["energy_fixed"][slot]
    for k in range(len(models)):  # rungs without a request are untouched
        b, a = before[k], eng.fetch(k)
        for r in range(len(b["slot_of_rung"]) - 4):
            s = b["slot_of_rung"][r]
            assert np.array_equal(a["spins"][s], b["spins"][s])
    t, acc = bn.tried.cpu().numpy(), bn.accepted.cpu().numpy()
    assert np.all(t == 1) and np.all(acc == (1 if force == "accept" else 0))


def test_grouped_sampler_equals_single_networks():
    from drift_b200.batch_neural import BatchNeuralPT

    bp, eng = small_batch(batch_of_sizes((4, 8, 12)), 0.3 * 10.0 ** (np.arange(8) / 7))
    eng.init()
    eng.run(2)
    nets = nets_for(bp, hidden=48)
    bn = BatchNeuralPT(eng, nets, n_cold=5)
    G = len(bn.ks)
    for rnd in (0, 3):
        bn.propose(rnd)
        bn.check()
        xp, lqp = bn.x_prop.cpu().numpy(), bn.lq_prop.cpu().numpy()
        xc, lqc = bn.x_cur.cpu().numpy(), bn.lq_cur.cpu().numpy()
        for g, k in enumerate(bn.ks):
            made, n, j0 = nets[k], nets[k].n, bn.row0[k]
            o = int(bn.off_h[j0])
            x1, lq1 = made.sample(5, seed=bn.seed, stream_id=rnd * G + g)
            assert np.array_equal(x1.cpu().numpy().ravel(), xp[o:o + 5 * n])
            assert np.array_equal(lq1.cpu().numpy(), lqp[j0:j0 + 5])
            cur = bn.x_cur[o:o + 5 * n].view(5, n)
            assert np.array_equal(made.logq(cur).cpu().numpy(), lqc[j0:j0 + 5])
            assert np.array_equal(cur.cpu().numpy().ravel(), xc[o:o + 5 * n])


def test_batch_neural_pt_is_stationary_at_the_boltzmann_distribution():
    """Three 16-spin 2-D EA instances: per-rung mean energies of batched neural-proposal PT with
    trained networks vs exact enumeration, and the proposals are accepted."""
    import torch

    from drift_b200.batch_neural import BatchNeuralPT

    models = batch_of_sizes((4, 4, 4))
    betas = np.array([0.4, 0.8, 1.4, 2.2])
    bp, eng = small_batch(models, betas, seed=8)
    eng.init()
    nets = nets_for(bp, hidden=32)
    bn = BatchNeuralPT(eng, nets, n_cold=4)
    data = bn.collect(1024)
    for k, m in nets.items():
        m.train(data[k], epochs=8, batch=256, lr=3e-3)
    bn.run(50)
    R = len(betas)
    slot0 = torch.tensor([int(d["slot0"]) for d in bp.desc], device=bp.device)
    es = []
    for _ in range(1500):
        bn.run(1)
        idx = (slot0[:, None] + eng.slot_of_rung.view(len(models), R).long()).ravel()
        es.append(eng.energy.index_select(0, idx).view(len(models), R).cpu().numpy())
    bn.check()
    e = np.array(es, np.float64)  # [rounds][instance][rung]
    for k, m in enumerate(models):
        ex = oracle.exact(m.to_dense().J, np.zeros(m.n), betas)
        mean, sd = e[:, k].mean(0), e[:, k].std(0)
        # successive rounds are correlated; 8 naive standard errors
        assert np.all(np.abs(mean - ex.mean_e) <= 8 * sd / np.sqrt(len(e)) + 1e-9), (k, mean, ex.mean_e)
    acc = bn.acceptance()
    assert min(acc.values()) > 0.02, acc
