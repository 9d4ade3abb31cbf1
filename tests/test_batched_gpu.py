"""Batched engine (GPU): every instance of a batch is, bit for bit, the chain the single-instance
engine runs with instance = stream id and the same seed — whatever the launch shape, across resumed
calls and when the rounds are replayed from a captured CUDA graph."""

from __future__ import annotations

import numpy as np
import pytest

import oracle
from conftest import cuda_ready

from drift_b200.batch import BatchEngine, BatchProblem, autotune, tune_candidates
from drift_b200.engine import DeviceProblem, HostProblem, PtEngine, geometric_betas
from drift_b200.instances import ea_2d, er_gaussian, maxcut_3regular, maxcut_ising, pm_spin_glass, random_graph

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_ready(), reason="needs CUDA and libdrift_pt.so")]

KEYS = ("spins", "best_spins", "energy_fixed", "best_energy_fixed", "rung_of_slot", "slot_of_rung", "tried",
        "accepted")


def int_batch():
    models = [ea_2d(8, 1), maxcut_3regular(700, 2), ea_2d(20, 3), maxcut_ising(random_graph(40, 0.2, 7)),
              maxcut_3regular(3000, 5)]
    ladders = [geometric_betas(6, 0.3, 3.0), geometric_betas(12, 0.25, 5.0), geometric_betas(10, 0.4, 2.5),
               geometric_betas(5, 0.2, 4.0), geometric_betas(33, 0.25, 5.0)]
    return models, ladders


def f32_batch():
    models = [er_gaussian(300, 6, 1), er_gaussian(2000, 6, 2), er_gaussian(5000, 6, 3), pm_spin_glass(14, 7, 0.3)]
    ladders = [geometric_betas(8, 1 / 3.0, 10.0), geometric_betas(16, 1 / 3.0, 10.0),
               geometric_betas(32, 1 / 3.0, 10.0), geometric_betas(4, 0.2, 5.0)]
    return models, ladders


def single(model, betas, rounds, spr, seed, stream, integer_path):
    prob = DeviceProblem(HostProblem.from_model(model), integer_path=integer_path)
    eng = PtEngine(prob, betas, seed=seed, sweeps_per_round=spr, instance=stream)
    eng.init()
    eng.run(rounds)
    eng.check()
    return eng.fetch()


def run_batch(models, ladders, rounds, spr, seed, stream_ids=None, chunks=None, **shape):
    bp = BatchProblem([HostProblem.from_model(m) for m in models], ladders, stream_ids=stream_ids)
    eng = BatchEngine(bp, seed=seed, sweeps_per_round=spr, **shape)
    eng.init()
    for c in (chunks or [rounds]):
        eng.run(c)
    eng.check()
    return bp, eng


@pytest.mark.parametrize("which", ["int", "f32"])
def test_batch_matches_single_instance_runs(which):
    models, ladders = int_batch() if which == "int" else f32_batch()
    rounds, spr, seed = 12, 3, 17
    streams = [5, 9, 2, 40, 77, 3][: len(models)]
    bp, eng = run_batch(models, ladders, rounds, spr, seed, stream_ids=streams)
    assert bp.integer_path == (which == "int")
    for k, (m, b) in enumerate(zip(models, ladders)):
        ref = single(m, b, rounds, spr, seed, streams[k], bp.integer_path)
        got = eng.fetch(k)
        for key in KEYS:
            assert np.array_equal(got[key], ref[key]), f"instance {k}: {key}"


def test_degree_ordered_layout_matches_oracle():
    model = er_gaussian(3000, 6, 11)
    hp = HostProblem.from_model(model, order="degree")
    deg = np.diff(hp.row_ptr)
    for c in range(hp.n_colors):
        seg = hp.color_spins[hp.color_ptr[c]:hp.color_ptr[c + 1]]
        assert np.all(np.diff(deg[seg]) <= 0)
    betas = geometric_betas(8, 1 / 3.0, 10.0)
    bp = BatchProblem([hp], [betas], stream_ids=[3])
    eng = BatchEngine(bp, seed=5, sweeps_per_round=2)
    eng.init()
    eng.run(7)
    eng.check()
    prob = oracle.OracleProblem(hp.n, hp.row_ptr, hp.col_idx, hp.weight, hp.h, hp.color_ptr, hp.color_spins,
                                integer_path=False)
    ost = oracle.pt_run(prob, betas, n_rounds=7, sweeps_per_round=2, seed=5, instance=3)
    got = eng.fetch(0)
    assert np.array_equal(got["spins"], ost.spins)
    assert np.array_equal(got["energy_fixed"], ost.energy)
    assert np.array_equal(got["accepted"], ost.accepted[:7])


def test_batch_instance_matches_oracle():
    models, ladders = int_batch()
    rounds, spr, seed = 10, 2, 4
    bp, eng = run_batch(models, ladders, rounds, spr, seed, stream_ids=[0, 1, 2, 3, 4])
    k = 1
    hp = HostProblem.from_model(models[k])
    prob = oracle.OracleProblem(hp.n, hp.row_ptr, hp.col_idx, hp.weight, hp.h, hp.color_ptr, hp.color_spins,
                                integer_path=True)
    ost = oracle.pt_run(prob, ladders[k], n_rounds=rounds, sweeps_per_round=spr, seed=seed, instance=k)
    got = eng.fetch(k)
    assert np.array_equal(got["spins"], ost.spins)
    assert np.array_equal(got["energy_fixed"], ost.energy)
    assert np.array_equal(got["tried"], ost.tried[: len(ladders[k]) - 1])
    assert np.array_equal(got["accepted"], ost.accepted[: len(ladders[k]) - 1])


@pytest.mark.parametrize("shape", [dict(max_tile=32, threads_per_slot=16), dict(max_tile=8, threads_per_slot=32),
                                   dict(max_tile=4, threads_per_slot=64, ctas_per_sm=1),
                                   dict(max_tile=16, threads_per_slot=4, positions_per_item=8),
                                   dict(max_tile=2, threads_per_slot=128, positions_per_item=4)])
def test_batch_results_do_not_depend_on_launch_shape(shape):
    models, ladders = int_batch()
    rounds, spr, seed = 6, 2, 23
    _, base = run_batch(models, ladders, rounds, spr, seed)
    _, eng = run_batch(models, ladders, rounds, spr, seed, **shape)
    for k in range(len(models)):
        a, b = base.fetch(k), eng.fetch(k)
        for key in KEYS:
            assert np.array_equal(a[key], b[key]), f"{shape} instance {k}: {key}"


def test_batch_resume_equals_single_call():
    models, ladders = f32_batch()
    _, a = run_batch(models, ladders, 9, 2, 3)
    _, b = run_batch(models, ladders, 9, 2, 3, chunks=[2, 4, 3])
    for k in range(len(models)):
        x, y = a.fetch(k), b.fetch(k)
        for key in KEYS:
            assert np.array_equal(x[key], y[key]), f"instance {k}: {key}"


def test_batch_rounds_replayed_from_a_cuda_graph():
    import torch

    models, ladders = int_batch()
    rounds, spr, seed = 8, 2, 31
    _, eager = run_batch(models, ladders, rounds, spr, seed)
    bp = BatchProblem([HostProblem.from_model(m) for m in models], ladders)
    eng = BatchEngine(bp, seed=seed, sweeps_per_round=spr)
    eng.init()
    snapshot = [t.clone() for t in (eng.spins, eng.best_spins, eng.energy, eng.best_energy, eng.rung_of_slot,
                                    eng.slot_of_rung, eng.tried, eng.accepted)]
    eng.run(1)  # warm: sets the kernel attributes outside the capture
    torch.cuda.synchronize()
    for t, s in zip((eng.spins, eng.best_spins, eng.energy, eng.best_energy, eng.rung_of_slot, eng.slot_of_rung,
                     eng.tried, eng.accepted), snapshot):
        t.copy_(s)
    eng.rounds_done = 0
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        for _ in range(rounds // 2):  # four launches of 2 rounds each, one graph
            eng.run(2)
    g.replay()
    eng.check()
    for k in range(len(models)):
        a, b = eager.fetch(k), eng.fetch(k)
        for key in KEYS:
            assert np.array_equal(a[key], b[key]), f"instance {k}: {key}"


def test_whole_job_graph_replays_the_job():
    """BatchEngine.capture_job: initialisation and every round in one CUDA graph; each replay is the
    eager job bit for bit (one launch, or launches of 3 rounds)."""
    models, ladders = int_batch()
    rounds, spr, seed = 8, 2, 17
    _, eager = run_batch(models, ladders, rounds, spr, seed)
    for launch_rounds in (0, 3):
        bp = BatchProblem([HostProblem.from_model(m) for m in models], ladders)
        eng = BatchEngine(bp, seed=seed, sweeps_per_round=spr)
        job = eng.capture_job(rounds, launch_rounds)
        assert job.launches == (1 if launch_rounds == 0 else 3)
        for _ in range(2):
            job.replay()
            eng.check()
            for k in range(len(models)):
                a, b = eager.fetch(k), eng.fetch(k)
                for key in KEYS:
                    assert np.array_equal(a[key], b[key]), f"instance {k}: {key}"


def test_autotune_picks_a_shape_and_keeps_results():
    models, ladders = int_batch()
    rounds, spr, seed = 5, 2, 8
    _, base = run_batch(models, ladders, rounds, spr, seed)
    bp = BatchProblem([HostProblem.from_model(m) for m in models], ladders)
    eng = BatchEngine(bp, seed=seed, sweeps_per_round=spr)
    eng.init()
    cands = tune_candidates(bp)[:6]
    best = autotune(eng, rounds=1, candidates=cands)
    assert best in cands and eng.rounds_done == 0
    eng.run(rounds)
    eng.check()
    for k in range(len(models)):
        a, b = base.fetch(k), eng.fetch(k)
        for key in KEYS:
            assert np.array_equal(a[key], b[key]), f"instance {k}: {key}"
