"""Multispin lattice engine (GPU): words, energies, bests, rung permutation and exchange counts
bit-exact against the multispin oracle; energies equal to a direct recount of the unpacked spins."""

from __future__ import annotations

import numpy as np
import pytest

import oracle
from conftest import cuda_ready

from drift_b200.multispin import Lattice, MsEngine

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_ready(), reason="needs CUDA and libdrift_pt.so")]


def ladder(R, lo, hi):
    return lo * (hi / lo) ** (np.arange(R) / (R - 1))


@pytest.mark.parametrize("dims,L,R,rounds,spr", [(3, 4, 32, 6, 2), (3, 6, 64, 4, 3), (2, 8, 32, 10, 1), (2, 12, 96, 3, 2)])
def test_multispin_matches_oracle(dims, L, R, rounds, spr):
    lat = Lattice.edwards_anderson(dims, L, 7)
    betas = ladder(R, 0.2, 2.0)
    eng = MsEngine(lat, betas, seed=11, sweeps_per_round=spr, instance=3)
    eng.init()
    eng.run(rounds)
    eng.check()
    st = eng.fetch()
    ost = oracle.ms_run(dims, L, lat.jneg, betas, n_rounds=rounds, sweeps_per_round=spr, seed=11, instance=3)
    assert np.array_equal(st["words"], ost.words)
    assert np.array_equal(st["best_words"], ost.best_words)
    assert np.array_equal(st["energy"], ost.energy)
    assert np.array_equal(st["best_energy"], ost.best_energy)
    assert np.array_equal(st["rung_of_slot"], ost.rung_of_slot)
    assert np.array_equal(st["tried"], ost.tried[: R - 1]) and np.array_equal(st["accepted"], ost.accepted[: R - 1])
    assert np.array_equal(lat.energy(st["spins"]).astype(np.int64), st["energy"])
    assert np.array_equal(lat.energy(st["best_spins"]).astype(np.int64), st["best_energy"])


def test_multispin_resume_and_large_lattice_energies():
    lat = Lattice.edwards_anderson(3, 6, 2)
    betas = ladder(32, 0.2, 2.0)
    a = MsEngine(lat, betas, seed=4, sweeps_per_round=2)
    a.init()
    a.run(9)
    b = MsEngine(lat, betas, seed=4, sweeps_per_round=2)
    b.init()
    b.run(4)
    b.run(5)
    a.check()
    b.check()
    x, y = a.fetch(), b.fetch()
    for k in ("words", "best_words", "energy", "rung_of_slot", "tried", "accepted"):
        assert np.array_equal(x[k], y[k]), k
    # the 3-D L = 64 lattice: exact energies after a few rounds, 128 replicas
    big = Lattice.edwards_anderson(3, 64, 5)
    e = MsEngine(big, ladder(128, 0.2, 2.0), seed=1, sweeps_per_round=1)
    e.init()
    e.run(3)
    e.check()
    st = e.fetch()
    assert np.array_equal(big.energy(st["spins"][:8]).astype(np.int64), st["energy"][:8])
    assert np.all(st["best_energy"] <= st["energy"])


def _ms_series(lat, betas, rounds, spr, seed):
    """Per-round rung energies and |m| of the multispin engine (one launch per round)."""
    import torch

    eng = MsEngine(lat, betas, seed=seed, sweeps_per_round=spr)
    eng.init()
    R = len(betas)
    E = torch.zeros((rounds, R), dtype=torch.int64, device="cuda")
    words = torch.zeros((rounds, eng.W * lat.n), dtype=torch.int32, device="cuda")
    slots = torch.zeros((rounds, R), dtype=torch.int64, device="cuda")
    for t in range(rounds):
        eng.run(1)
        sor = eng.slot_of_rung.long()
        E[t] = eng.energy[sor]
        words[t] = eng.words
        slots[t] = sor
    eng.check()
    w = words.cpu().numpy().view(np.uint32).reshape(rounds, eng.W, lat.n)
    bits = (w[:, :, None, :] >> np.arange(32, dtype=np.uint32)[None, None, :, None]) & 1
    m = np.abs((1 - 2 * bits.astype(np.float64)).reshape(rounds, R, lat.n).mean(axis=2))
    absm = np.take_along_axis(m, slots.cpu().numpy(), axis=1)
    return E.cpu().numpy().astype(np.float64), absm


def test_multispin_engine_samples_the_boltzmann_distribution():
    """The kernel's chain on a 2-D +-J L = 4 lattice: per-rung mean energy and |m| within 3 standard
    errors (blocked; floored by the exact variance over the samples) of exact enumeration
    (drift/solvers/exact.py:20-49, oracle/exact.c)."""
    from drift_b200.observables import blocked
    from test_multispin import dense_couplings

    lat = Lattice.edwards_anderson(2, 4, 3)
    betas = ladder(32, 0.2, 3.0)
    ex = oracle.exact(dense_couplings(lat), np.zeros(lat.n), betas)
    E, M = _ms_series(lat, betas, 4000, 2, 9)
    n_kept = len(E) - int(len(E) * 0.1)
    for x, mean, mean2 in ((E, ex.mean_e, ex.mean_e2), (M, ex.mean_absm, ex.mean_m2)):
        mx, sx = blocked(x)
        floor = np.sqrt(np.maximum(mean2 - mean ** 2, 0.0) / n_kept)
        assert np.all(np.abs(mx - mean) <= 3.0 * np.maximum(sx, floor) + 1e-9), (mx, mean, sx)


@pytest.mark.parametrize("item_form", [1, 2])
def test_multispin_engine_agrees_with_the_int8_engine(item_form):
    """3-D +-J L = 4 (64 spins, beyond exact enumeration): the bit-packed chain and the int8 sparse
    engine (sliced-ELL gather or unit-regular form) have the same per-rung mean energies within 3
    combined standard errors (blocked)."""
    import torch

    from drift_b200.engine import DeviceProblem, HostProblem, PtEngine
    from drift_b200.instances import ea_3d
    from drift_b200.observables import blocked

    lat = Lattice.edwards_anderson(3, 4, 8)
    model = ea_3d(4, 8)
    s = np.random.default_rng(1).choice([-1.0, 1.0], size=(4, lat.n))
    assert np.allclose(lat.energy(s), model.energy_batch(s))  # the same couplings
    betas = ladder(32, 0.2, 2.0)
    rounds, spr = 4000, 2
    E_ms, _ = _ms_series(lat, betas, rounds, spr, 21)
    eng = PtEngine(DeviceProblem(HostProblem.from_model(model)), betas, seed=22, sweeps_per_round=spr,
                   item_form=item_form)
    eng.init()
    E = torch.zeros((rounds, len(betas)), dtype=torch.int64, device="cuda")
    for t in range(rounds):
        eng.run(1)
        E[t] = eng.energy[eng.slot_of_rung.long()]
    eng.check()
    m1, s1 = blocked(E_ms)
    m2, s2 = blocked(E.cpu().numpy().astype(np.float64))
    assert np.all(np.abs(m1 - m2) <= 3.0 * np.sqrt(s1 ** 2 + s2 ** 2) + 1e-9), (m1, m2, s1, s2)
