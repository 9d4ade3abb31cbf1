"""Dense-coupling engine (GPU): spins, energies, bests, rung permutation, exchange counts and
best history bit-exact against the dense-coupling oracle, over sizes that exercise padding
(n not a multiple of 128), a field, several replicas-per-CTA shapes and a partial last CTA;
resumed runs equal one long run; device energies equal exact recounts."""

from __future__ import annotations

import numpy as np
import pytest

import oracle
from conftest import cuda_ready

from drift_b200.sk import SkEngine, SkModel

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_ready(), reason="needs CUDA and libdrift_pt.so")]


def sk_couplings(n, seed, field=0.0):
    rng = np.random.default_rng(seed)
    J = np.triu(rng.normal(size=(n, n)) / np.sqrt(n), 1)
    J = J + J.T
    h = rng.normal(scale=field, size=n) if field else np.zeros(n)
    return J, h


def compare(eng, m, betas, rounds, spr, seed, instance):
    st = eng.fetch()
    o = oracle.sk_run(m.Jq, m.hq, m.shift, betas, m.scales(betas), n_rounds=rounds, sweeps_per_round=spr, seed=seed,
                      instance=instance)
    R = len(betas)
    assert np.array_equal(st["spins"], o.spins)
    assert np.array_equal(st["energy"], o.energy)
    assert np.array_equal(st["best_energy"], o.best_energy)
    assert np.array_equal(st["best_spins"], o.best_spins)
    assert np.array_equal(st["rung_of_slot"], o.rung_of_slot)
    assert np.array_equal(st["slot_of_rung"], o.slot_of_rung)
    assert np.array_equal(st["tried"], o.tried[: R - 1]) and np.array_equal(st["accepted"], o.accepted[: R - 1])
    if st["best_history"] is not None:
        assert np.array_equal(st["best_history"][:rounds], o.best_history)
    return st


@pytest.mark.parametrize("n,R,G,rounds,spr,field", [
    (512, 64, 4, 3, 2, 0.0),
    (512, 64, 1, 2, 1, 0.0),
    (512, 32, 12, 2, 2, 0.2),
    (200, 40, 12, 4, 2, 0.3),
    (100, 17, 3, 5, 1, 0.2),
    (33, 8, 0, 6, 3, 0.0),
])
def test_sk_matches_oracle(n, R, G, rounds, spr, field):
    J, h = sk_couplings(n, 4, field)
    m = SkModel(J, h)
    betas = np.geomspace(0.3, 3.0, R)
    eng = SkEngine(m, betas, seed=5, sweeps_per_round=spr, instance=2, replicas_per_cta=G)
    eng.init()
    eng.run(rounds, history=True)
    eng.check()
    st = compare(eng, m, betas, rounds, spr, 5, 2)
    # device recount of the final and best configurations
    import torch

    assert np.array_equal(eng.energies(torch.from_numpy(st["spins"]).cuda()), st["energy"])
    assert np.array_equal(eng.energies(torch.from_numpy(st["best_spins"]).cuda()), st["best_energy"])


def test_sk_resume_equals_one_run():
    J, h = sk_couplings(256, 7)
    m = SkModel(J, h)
    betas = np.geomspace(0.3, 3.0, 24)
    a = SkEngine(m, betas, seed=9, sweeps_per_round=2, replicas_per_cta=2)
    a.init()
    a.run(7)
    b = SkEngine(m, betas, seed=9, sweeps_per_round=2, replicas_per_cta=8)
    b.init()
    b.run(3)
    b.run(4)
    a.check()
    b.check()
    x, y = a.fetch(), b.fetch()
    for k in ("spins", "energy", "best_energy", "best_spins", "rung_of_slot", "tried", "accepted"):
        assert np.array_equal(x[k], y[k]), k


def test_sk_energies_track_the_unquantised_model():
    J, h = sk_couplings(512, 4)
    m = SkModel(J, h)
    betas = np.geomspace(0.3, 3.0, 64)
    eng = SkEngine(m, betas, seed=1, sweeps_per_round=5)
    eng.init()
    eng.run(4)
    eng.check()
    st = eng.fetch()
    e64 = m.energy_fp64(st["spins"])
    assert np.all(np.abs(st["energy"] * m.energy_unit - e64) <= (512 * 512 / 2 + 512) * m.energy_unit)
    # SK ground state per spin is about -0.763; after 20 sweeps the coldest rungs are well below -0.6 n
    assert st["best_energy"].min() * m.energy_unit < -0.6 * 512


def test_sk_chain_samples_the_unquantised_boltzmann_distribution():
    """The dense kernel runs the chain exactly on J quantised to 2^-25 (3 int8 limbs). This bounds the
    quantisation's effect on observables: on an SK instance of 16 spins with a field, the per-rung
    mean energy and |m| are within 3 standard errors (blocked; floored by the exact variance over
    the samples) of exact enumeration of the unquantised FP64 model (drift/solvers/exact.py:20-49,
    oracle/exact.c)."""
    import torch

    from drift_b200.observables import blocked

    J, h = sk_couplings(16, 12, field=0.3)
    m = SkModel(J, h)
    betas = np.geomspace(0.3, 3.0, 16)
    ex = oracle.exact(J, h, betas)
    eng = SkEngine(m, betas, seed=5, sweeps_per_round=2)
    eng.init()
    rounds = 4000
    E = torch.zeros((rounds, len(betas)), dtype=torch.int64, device="cuda")
    M = torch.zeros((rounds, len(betas)), dtype=torch.float64, device="cuda")
    for t in range(rounds):
        eng.run(1)
        at = eng.slot_of_rung.long()
        E[t] = eng.energy[at]
        M[t] = eng.spins[at].double().mean(dim=1).abs()
    eng.check()
    E = E.cpu().numpy().astype(np.float64) * m.energy_unit
    M = M.cpu().numpy()
    n_kept = rounds - int(rounds * 0.1)
    for x, mean, mean2 in ((E, ex.mean_e, ex.mean_e2), (M, ex.mean_absm, ex.mean_m2)):
        mx, sx = blocked(x)
        floor = np.sqrt(np.maximum(mean2 - mean ** 2, 0.0) / n_kept)
        assert np.all(np.abs(mx - mean) <= 3.0 * np.maximum(sx, floor) + 1e-9), (mx, mean, sx)
