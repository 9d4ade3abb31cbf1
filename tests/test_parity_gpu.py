"""Parity of the sm_100a engine with the oracle, through the C ABI (GPU required).

Bit-exact: final spins of every replica slot, fixed-point energies, per-slot best energies and
configurations, the rung permutation, per-pair exchange counts and the best-energy history, on
integer (+-J, MaxCut) and fp32 (Gaussian field / couplings) problems, for every launch shape,
and across resumed runs. Also: the reference's own GPU acceptance checks (tests/test_gpu.py,
tests/test_parallel_tempering.py of the reference) through the drop-in parallel_tempering_gpu.
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import oracle
from conftest import cuda_ready, dense_from_edges

from drift_b200 import _lib
from drift_b200.engine import DeviceProblem, HostProblem, PtEngine, geometric_betas
from drift_b200.gpu import parallel_tempering_gpu
from drift_b200.instances import (ea_2d, ea_3d, er_gaussian, gnp_pm, maxcut_3regular, maxcut_ising, pm_spin_glass,
                                  random_graph, sk_model)

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_ready(), reason="needs CUDA and libdrift_pt.so")]


def oracle_problem(hp: HostProblem, integer_path: bool):
    return oracle.OracleProblem(hp.n, hp.row_ptr, hp.col_idx, hp.weight, hp.h, hp.color_ptr, hp.color_spins,
                                integer_path=integer_path)


def run_engine(model, betas, rounds, spr, seed, *, rpc=0, threads=0, ppi=0, instance=0, chunks=None,
               integer_path=None, round_sync=0, item_form=0):
    import torch

    hp = HostProblem.from_model(model)
    prob = DeviceProblem(hp, integer_path=integer_path)
    eng = PtEngine(prob, betas, seed=seed, sweeps_per_round=spr, instance=instance, replicas_per_cta=rpc,
                   threads_per_cta=threads, positions_per_item=ppi, round_sync=round_sync, item_form=item_form)
    eng.init()
    hist = torch.zeros(max(rounds, 1), dtype=torch.float64, device="cuda")
    done = 0
    for c in (chunks or [rounds]):
        eng.run(c, history=hist[done:])
        done += c
    eng.check()
    return hp, prob, eng, eng.fetch(), hist.cpu().numpy()[:rounds]


def assert_bit_exact(st, ost, hist, rounds):
    assert np.array_equal(st["spins"], ost.spins)
    assert np.array_equal(st["energy_fixed"], ost.energy)
    assert np.array_equal(st["best_energy_fixed"], ost.best_energy)
    assert np.array_equal(st["best_spins"], ost.best_spins)
    assert np.array_equal(st["rung_of_slot"], ost.rung_of_slot)
    assert np.array_equal(st["slot_of_rung"], ost.slot_of_rung)
    R = len(ost.energy)
    assert np.array_equal(st["tried"], ost.tried[: R - 1])
    assert np.array_equal(st["accepted"], ost.accepted[: R - 1])
    assert np.array_equal(hist, ost.best_history[:rounds])


CASES = {
    # name: (model factory, R, (beta_hot, beta_cold) or T range, rounds, sweeps_per_round, seed)
    "ferro_chain_18": (lambda: dense_from_edges(18, {"i": list(range(17)), "j": list(range(1, 18)), "w": [1.0] * 17},
                                                [0.0] * 18), 12, (0.05, 3.0), 150, 4, 0),
    "maxcut_g16_s3": (lambda: maxcut_ising(random_graph(16, 0.5, 3)), 16, (0.05, 4.0), 200, 4, 1),
    "glass_n14_field_fp32": (lambda: pm_spin_glass(14, 7, field=0.3), 20, (0.05, 5.0), 300, 5, 2),
    "ea2d_L16_C1": (lambda: ea_2d(16, 1), 24, (1 / 3.0, 10.0), 2000, 1, 1),
    "maxcut_3reg_4096_C2": (lambda: maxcut_3regular(4096, 2), 64, (0.25, 5.0), 25, 4, 7),
    "er_gaussian_2000_fp32": (lambda: er_gaussian(2000, 6, 3), 8, (1 / 3.0, 10.0), 12, 2, 3),
    "sk_64_dense_fp32": (lambda: sk_model(64, 4), 8, (1 / 3.0, 1 / 0.3), 40, 2, 4),
}


def _isolated_spins():
    from drift_b200.ising import IsingModel

    J = gnp_pm(30, 0.15, 1).J.copy()
    J[:5] = 0.0
    J[:, :5] = 0.0
    return IsingModel(J, np.zeros(30))


def _pure_field(n, values, seed):
    from drift_b200.ising import IsingModel

    rng = np.random.default_rng(seed)
    h = rng.normal(size=n) if values is None else rng.choice(values, size=n)
    return IsingModel(np.zeros((n, n)), h)


EDGE_CASES = {
    # one replica (no exchange pair), two, an odd count; ragged sizes (25, 257 spins); isolated spins;
    # no couplings at all (an empty coupling table) on the fp32 and the integer path
    "one_replica": (lambda: maxcut_ising(random_graph(16, 0.5, 3)), 1, (0.2, 5.0), 60, 2, 5),
    "two_replicas": (lambda: maxcut_ising(random_graph(16, 0.5, 3)), 2, (0.2, 5.0), 60, 2, 6),
    "odd_ladder_ragged_25": (lambda: ea_2d(5, 2), 7, (0.2, 5.0), 80, 3, 7),
    "isolated_spins": (_isolated_spins, 9, (0.2, 5.0), 60, 2, 8),
    "ragged_257": (lambda: gnp_pm(257, 0.02, 4), 10, (0.2, 5.0), 40, 2, 9),
    "no_couplings_fp32": (lambda: _pure_field(12, None, 3), 6, (0.2, 5.0), 50, 2, 10),
    "no_couplings_int": (lambda: _pure_field(11, [-2.0, -1.0, 1.0, 2.0], 4), 5, (0.2, 5.0), 50, 2, 11),
}


@pytest.mark.parametrize("name", list(EDGE_CASES))
def test_edge_cases_match_oracle_bit_exact(name):
    make, R, (tmin, tmax), rounds, spr, seed = EDGE_CASES[name]
    model = make()
    betas = geometric_betas(R, tmin, tmax)
    hp, prob, eng, st, hist = run_engine(model, betas, rounds, spr, seed)
    ost = oracle.pt_run(oracle_problem(hp, prob.integer_path), betas, n_rounds=rounds, sweeps_per_round=spr,
                        seed=seed, thr=eng.thr)
    assert_bit_exact(st, ost, hist, rounds)


@pytest.mark.parametrize("item_form", [0, 1])
@pytest.mark.parametrize("name", list(CASES))
def test_engine_matches_oracle_bit_exact(name, item_form):
    """item_form 0 lets the engine choose (the unit-regular form for C1 and C2), 1 forces the
    sliced-ELL gather."""
    make, R, (tmin, tmax), rounds, spr, seed = CASES[name]
    model = make()
    betas = geometric_betas(R, tmin, tmax)
    hp, prob, eng, st, hist = run_engine(model, betas, rounds, spr, seed, item_form=item_form)
    ost = oracle.pt_run(oracle_problem(hp, prob.integer_path), betas, n_rounds=rounds, sweeps_per_round=spr,
                        seed=seed, thr=eng.thr)
    assert_bit_exact(st, ost, hist, rounds)


@pytest.mark.parametrize("rpc,threads,ppi,form", [(1, 64, 8, 1), (1, 512, 8, 1), (2, 256, 8, 1), (8, 512, 8, 1),
                                                   (64, 512, 8, 1), (1, 0, 4, 1), (1, 96, 4, 1), (4, 512, 4, 1),
                                                   (64, 512, 4, 1), (16, 0, 0, 0), (1, 0, 0, 2), (1, 0, 2, 2),
                                                   (1, 832, 2, 2), (1, 0, 4, 2), (1, 1024, 4, 2)])
def test_results_do_not_depend_on_launch_shape(rpc, threads, ppi, form):
    """Form 1 is the sliced-ELL gather, form 2 the unit-regular form (2 or 4 positions per item, the
    CTA as narrow as the largest class allows or as wide as the form allows)."""
    model = maxcut_3regular(2048, 5)
    R, rounds, spr, seed = 64, 10, 2, 11
    betas = geometric_betas(R, 0.25, 5.0)
    hp, prob, eng, st, hist = run_engine(model, betas, rounds, spr, seed, rpc=rpc, threads=threads, ppi=ppi,
                                         item_form=form)
    ost = oracle.pt_run(oracle_problem(hp, True), betas, n_rounds=rounds, sweeps_per_round=spr, seed=seed, thr=eng.thr)
    assert_bit_exact(st, ost, hist, rounds)


ROUND_SYNC_CASES = {
    # name: (model factory, R, T range, rounds, sweeps_per_round, seed, replicas per CTA)
    "ea2d_L16_R24": (lambda: ea_2d(16, 1), 24, (1 / 3.0, 10.0), 300, 1, 1, 0),
    "glass_field_fp32_R20": (lambda: pm_spin_glass(14, 7, field=0.3), 20, (0.05, 5.0), 120, 2, 2, 0),
    "ragged_257_R25_last_cta_short": (lambda: gnp_pm(257, 0.02, 4), 25, (0.2, 5.0), 60, 2, 3, 2),
    "three_replicas": (lambda: maxcut_ising(random_graph(16, 0.5, 3)), 3, (0.2, 5.0), 80, 3, 4, 0),
    "maxcut_2048_cluster_of_16": (lambda: maxcut_3regular(2048, 5), 16, (0.25, 5.0), 20, 2, 5, 1),
    "er_fp32_R32_four_per_cta": (lambda: er_gaussian(600, 6, 7), 32, (1 / 3.0, 10.0), 30, 2, 6, 4),
}


@pytest.mark.parametrize("round_sync", [1, 2])
@pytest.mark.parametrize("name", list(ROUND_SYNC_CASES))
def test_round_sync_forms_match_oracle_bit_exact(name, round_sync):
    """The grid form (bounded barrier in global memory) and the cluster form (energies through
    distributed shared memory) run the same chain."""
    make, R, (tmin, tmax), rounds, spr, seed, rpc = ROUND_SYNC_CASES[name]
    model = make()
    betas = geometric_betas(R, tmin, tmax)
    hp, prob, eng, st, hist = run_engine(model, betas, rounds, spr, seed, rpc=rpc, round_sync=round_sync)
    ost = oracle.pt_run(oracle_problem(hp, prob.integer_path), betas, n_rounds=rounds, sweeps_per_round=spr,
                        seed=seed, thr=eng.thr)
    assert_bit_exact(st, ost, hist, rounds)


ONE_POSITION_CASES = {
    # name: (model factory, R, T range, rounds, sweeps_per_round, seed)
    "ea2d_L16_R24": (lambda: ea_2d(16, 1), 24, (1 / 3.0, 10.0), 200, 1, 1),
    "ragged_25_R7": (lambda: ea_2d(5, 2), 7, (0.2, 5.0), 80, 3, 7),
    "int_field_R9": (lambda: _pure_field(40, [-2.0, -1.0, 1.0, 2.0], 5), 9, (0.2, 5.0), 40, 2, 12),
    "isolated_spins_R9": (_isolated_spins, 9, (0.2, 5.0), 60, 2, 8),
    "ragged_257_R10": (lambda: gnp_pm(257, 0.02, 4), 10, (0.2, 5.0), 40, 2, 9),
}


@pytest.mark.parametrize("round_sync", [1, 2])
@pytest.mark.parametrize("name", list(ONE_POSITION_CASES))
def test_one_position_per_item_matches_oracle_bit_exact(name, round_sync):
    make, R, (tmin, tmax), rounds, spr, seed = ONE_POSITION_CASES[name]
    model = make()
    betas = geometric_betas(R, tmin, tmax)
    hp, prob, eng, st, hist = run_engine(model, betas, rounds, spr, seed, ppi=1, round_sync=round_sync)
    assert prob.integer_path
    ost = oracle.pt_run(oracle_problem(hp, True), betas, n_rounds=rounds, sweeps_per_round=spr, seed=seed,
                        thr=eng.thr)
    assert_bit_exact(st, ost, hist, rounds)


def _ring_pm(n, seed):
    """A ring of n spins with +-1 couplings (every spin has 2)."""
    from drift_b200.ising import SparseIsingModel

    rng = np.random.default_rng(seed)
    i = np.arange(n)
    return SparseIsingModel(n, i, (i + 1) % n, rng.choice([-1.0, 1.0], size=n))


UNIT_CASES = {
    # name: (model factory, R, T range, rounds, sweeps_per_round, seed, round_sync)
    "ea2d_L16_R24_grid": (lambda: ea_2d(16, 1), 24, (1 / 3.0, 10.0), 400, 1, 1, 1),
    "ea2d_L16_R16_cluster": (lambda: ea_2d(16, 3), 16, (1 / 3.0, 10.0), 400, 1, 2, 2),
    "ea2d_L5_ragged_R7": (lambda: ea_2d(5, 2), 7, (0.2, 5.0), 80, 3, 7, 0),
    "ea3d_L6_W6_R20": (lambda: ea_3d(6, 4), 20, (0.2, 5.0), 60, 2, 3, 1),
    "ea3d_L4_W6_R12_cluster": (lambda: ea_3d(4, 5), 12, (0.2, 5.0), 60, 2, 4, 2),
    "ring_300_W2_R10": (lambda: _ring_pm(300, 6), 10, (0.2, 5.0), 80, 2, 5, 0),
    "ring_301_three_classes_R20": (lambda: _ring_pm(301, 7), 20, (0.2, 5.0), 60, 3, 11, 1),
    "maxcut_3reg_4096_R64_C2": (lambda: maxcut_3regular(4096, 2), 64, (0.25, 5.0), 25, 4, 7, 0),
    # padding positions (1800 spins in 2048) with the next round's first-sweep Philox blocks computed
    # in the round end (grid form, 352 threads: 256 beyond the first three warps for 225 groups)
    "maxcut_3reg_1800_R40_padded_deferred": (lambda: maxcut_3regular(1800, 9), 40, (0.25, 5.0), 30, 3, 13, 1),
    "maxcut_3reg_2048_R16_cluster": (lambda: maxcut_3regular(2048, 5), 16, (0.25, 5.0), 20, 2, 5, 2),
    "one_replica": (lambda: maxcut_3regular(512, 3), 1, (0.2, 5.0), 40, 2, 8, 0),
    "two_replicas": (lambda: maxcut_3regular(512, 3), 2, (0.2, 5.0), 40, 2, 9, 0),
    "maxcut_3reg_8192_R8_four_per_item": (lambda: maxcut_3regular(8192, 4), 8, (0.25, 5.0), 6, 2, 10, 1),
}


@pytest.mark.parametrize("name", list(UNIT_CASES))
def test_unit_regular_form_matches_oracle_bit_exact(name):
    """The unit-regular form (neighbour addresses, the rung's thresholds, a static schedule; compiled
    for 2 or 4 colour phases) runs the oracle's chain bit for bit: lattices in 2-D and 3-D, rings
    with 2 and 3 colour classes, MaxCut on 3-regular graphs, padding positions (25 spins in 256
    positions), one and two replicas, grid and cluster round ends."""
    make, R, (tmin, tmax), rounds, spr, seed, sync = UNIT_CASES[name]
    model = make()
    betas = geometric_betas(R, tmin, tmax)
    hp, prob, eng, st, hist = run_engine(model, betas, rounds, spr, seed, round_sync=sync, item_form=2)
    assert prob.unit_regular
    ost = oracle.pt_run(oracle_problem(hp, True), betas, n_rounds=rounds, sweeps_per_round=spr, seed=seed,
                        thr=eng.thr)
    assert_bit_exact(st, ost, hist, rounds)


def test_unit_regular_form_with_and_without_the_bank_placement():
    """The storage order of the spin words (drift_pt_unit_placement, on by default) changes no bit."""
    import torch

    model = maxcut_3regular(4096, 6)
    betas = geometric_betas(16, 0.25, 5.0)
    hp = HostProblem.from_model(model)
    ost = oracle.pt_run(oracle_problem(hp, True), betas, n_rounds=12, sweeps_per_round=2, seed=21,
                        thr=oracle.thresholds(betas, 3))
    for placed in (True, False):
        prob = DeviceProblem(hp)
        assert prob.d_unit_place is not None
        if not placed:
            prob.d_unit_place = None
        eng = PtEngine(prob, betas, seed=21, sweeps_per_round=2, item_form=2, round_sync=1)
        eng.init()
        hist = torch.zeros(12, dtype=torch.float64, device="cuda")
        eng.run(12, history=hist)
        eng.check()
        assert_bit_exact(eng.fetch(), ost, hist.cpu().numpy(), 12)


def test_unit_regular_form_resumes_and_checks_its_energy():
    model = maxcut_3regular(1024, 8)
    betas = geometric_betas(32, 0.25, 5.0)
    chunks = [5, 1, 7]
    hp, prob, eng, st, hist = run_engine(model, betas, sum(chunks), 3, 13, chunks=chunks, item_form=2)
    ost = oracle.pt_run(oracle_problem(hp, True), betas, n_rounds=sum(chunks), sweeps_per_round=3, seed=13,
                        thr=eng.thr)
    assert_bit_exact(st, ost, hist, sum(chunks))
    assert np.array_equal(eng.energy_fp64(), st["energy_fixed"].astype(np.float64))


def test_unit_regular_form_refuses_other_problems():
    betas = geometric_betas(8, 0.25, 5.0)
    with pytest.raises(_lib.EngineError, match="unit-regular"):
        run_engine(gnp_pm(64, 0.1, 2), betas, 2, 1, 0, item_form=2)  # irregular degrees
    with pytest.raises(_lib.EngineError, match="unit-regular"):
        run_engine(maxcut_3regular(512, 1), betas, 2, 1, 0, rpc=2, item_form=2)  # two replicas per CTA
    with pytest.raises(_lib.EngineError, match="item_form 2"):
        run_engine(maxcut_3regular(2048, 1), betas, 2, 1, 0, threads=64, item_form=2)  # one item per thread


def test_cluster_form_refuses_a_ladder_that_does_not_fit():
    betas = geometric_betas(64, 0.25, 5.0)
    with pytest.raises(_lib.EngineError, match="one cluster"):
        run_engine(maxcut_3regular(512, 1), betas, 2, 1, 0, rpc=1, round_sync=2)


def test_fp32_path_launch_shapes_and_resume():
    model = er_gaussian(1500, 6, 9)
    R, spr, seed = 16, 3, 5
    betas = geometric_betas(R, 1 / 3.0, 10.0)
    chunks = [3, 1, 6]
    hp, prob, eng, st, hist = run_engine(model, betas, sum(chunks), spr, seed, rpc=4, threads=128, chunks=chunks)
    ost = oracle.pt_run(oracle_problem(hp, False), betas, n_rounds=sum(chunks), sweeps_per_round=spr, seed=seed)
    assert_bit_exact(st, ost, hist, sum(chunks))


def test_resume_equals_single_run_integer():
    model = ea_2d(24, 3)
    R, spr, seed = 10, 2, 4
    betas = geometric_betas(R, 0.4, 3.0)
    chunks = [7, 13, 1, 9]
    hp, prob, eng, st, hist = run_engine(model, betas, sum(chunks), spr, seed, chunks=chunks)
    ost = oracle.pt_run(oracle_problem(hp, True), betas, n_rounds=sum(chunks), sweeps_per_round=spr, seed=seed,
                        thr=eng.thr)
    assert_bit_exact(st, ost, hist, sum(chunks))


@pytest.mark.parametrize("ppi", [8, 4])
def test_integer_field_and_wide_slices_small_items(ppi):
    # integer couplings with an integer field (kField) and degree-6 slices (W = 8) on short items
    from drift_b200.instances import ea_3d
    from drift_b200.ising import SparseIsingModel

    base = ea_3d(8, 2)
    rp, ci, w = base.csr()
    rows = np.repeat(np.arange(base.n), np.diff(rp))
    up = rows < ci
    rng = np.random.default_rng(1)
    model = SparseIsingModel(base.n, rows[up], ci[up], w[up], rng.integers(-2, 3, size=base.n).astype(float))
    betas = geometric_betas(12, 0.3, 3.0)
    hp, prob, eng, st, hist = run_engine(model, betas, 20, 3, 6, ppi=ppi)
    assert prob.integer_path and prob.info.has_field
    ost = oracle.pt_run(oracle_problem(hp, True), betas, n_rounds=20, sweeps_per_round=3, seed=6, thr=eng.thr)
    assert_bit_exact(st, ost, hist, 20)


def test_integer_couplings_forced_onto_fp32_path_match_oracle():
    model = ea_2d(16, 2)
    betas = geometric_betas(8, 0.3, 3.0)
    hp, prob, eng, st, hist = run_engine(model, betas, 30, 2, 3, integer_path=False)
    ost = oracle.pt_run(oracle_problem(hp, False), betas, n_rounds=30, sweeps_per_round=2, seed=3)
    assert_bit_exact(st, ost, hist, 30)


def test_instance_id_selects_an_independent_stream():
    model = maxcut_3regular(512, 1)
    betas = geometric_betas(8, 0.25, 5.0)
    _, _, eng0, st0, _ = run_engine(model, betas, 5, 2, 3, instance=0)
    hp, _, eng5, st5, hist = run_engine(model, betas, 5, 2, 3, instance=5)
    assert not np.array_equal(st0["spins"], st5["spins"])
    ost = oracle.pt_run(oracle_problem(hp, True), betas, n_rounds=5, sweeps_per_round=2, seed=3, instance=5, thr=eng5.thr)
    assert_bit_exact(st5, ost, hist, 5)


def test_energy_bookkeeping_against_fp64_recompute():
    # integer path: the incremental int64 energy equals the FP64 recompute exactly
    _, _, eng, st, _ = run_engine(maxcut_3regular(4096, 2), geometric_betas(16, 0.25, 5.0), 50, 4, 1)
    assert np.array_equal(eng.energy_fp64(), st["energy_fixed"].astype(np.float64))
    # fp32 path: fixed-point bookkeeping stays within 1e-5 relative of FP64 after 20k flips/spin
    model = er_gaussian(3000, 6, 4)
    _, _, eng, st, _ = run_engine(model, geometric_betas(8, 1 / 3.0, 10.0), 200, 100, 2)
    e64 = eng.energy_fp64()
    assert np.all(np.abs(st["energy"] - e64) <= 1e-5 * (1.0 + np.abs(e64)))
    for r in range(8):
        assert model.energy(st["spins"][r]) == pytest.approx(e64[r], rel=1e-9, abs=1e-9)


# ---- the reference's acceptance checks through the drop-in ----------------------------------

def test_gpu_reproduces_exact_on_small_maxcut(reference_instances):
    """tests/test_gpu.py:45-54 of the reference."""
    d = reference_instances["maxcut_g12_p05_s3"]
    model = dense_from_edges(d["n"], d["edges"], d["h"])
    res = parallel_tempering_gpu(model, n_replicas=16, T_min=0.05, T_max=4.0, n_rounds=200, sweeps_per_round=4,
                                 seed=1)
    assert res.best_E == pytest.approx(d["e_exact"])
    assert model.energy(res.best_s) == pytest.approx(res.best_E)
    assert 0.0 < res.swap_rate < 1.0 and res.throughput > 0 and res.seconds > 0
    assert len(res.best_history) == 200 and res.best_history[-1] == pytest.approx(res.best_E)


@pytest.mark.parametrize("name,kw", [
    ("maxcut_g16_p05_s3", dict(n_replicas=16, T_min=0.05, T_max=4.0, n_rounds=200, sweeps_per_round=4, seed=1)),
    ("maxcut_g18_p04_s8", dict(n_replicas=16, T_min=0.05, T_max=4.0, n_rounds=200, sweeps_per_round=4, seed=1)),
    ("glass_n14_s7_field", dict(n_replicas=20, T_min=0.05, T_max=5.0, n_rounds=300, sweeps_per_round=5, seed=2)),
    ("ferro_n18", dict(n_replicas=12, T_min=0.05, T_max=3.0, n_rounds=150, sweeps_per_round=4, seed=0)),
    ("maxcut_g20_p05_s2", dict(n_replicas=16, n_rounds=80, sweeps_per_round=4, seed=1)),
])
def test_drop_in_finds_exact_ground_states(reference_instances, name, kw):
    """tests/test_parallel_tempering.py:37-68 and experiments/phase14_gpu.py:38-65 of the reference."""
    d = reference_instances[name]
    model = dense_from_edges(d["n"], d["edges"], d["h"])
    res = parallel_tempering_gpu(model, **kw)
    assert np.isclose(res.best_E, d["e_exact"]), f"GPU PT {res.best_E} != exact {d['e_exact']}"
    assert res.rung_spins.shape == (kw["n_replicas"], d["n"])
    for r in range(kw["n_replicas"]):
        assert model.energy(res.rung_spins[r]) == pytest.approx(res.rung_energies[r], abs=1e-4)


def test_solve_abi_matches_device_layer():
    """drift_pt_solve (host buffers in and out) runs the same chain as the device layer."""
    model = maxcut_3regular(1024, 4)
    R, rounds, spr, seed = 32, 20, 3, 8
    hp = HostProblem.from_model(model)
    betas = geometric_betas(R, 0.25, 5.0)
    _, _, eng, st, hist = run_engine(model, betas, rounds, spr, seed)
    L = _lib.load()
    p = lambda a: a.ctypes.data_as(C.c_void_p)
    best_s = np.zeros(hp.n, np.float32)
    rung_spins = np.zeros((R, hp.n), np.int8)
    rung_e = np.zeros(R)
    tried = np.zeros(R - 1, np.int64)
    acc = np.zeros(R - 1, np.int64)
    bh = np.zeros(rounds)
    args = _lib.SolveArgs(R, rounds, spr, 0, seed, 0.0, 0.0, p(betas))
    res = _lib.SolveResult(0, 0, 0, 0, p(best_s), p(rung_spins), p(rung_e), p(tried), p(acc), p(bh))
    _lib.check(L.drift_pt_solve(C.byref(hp.c_csr()), C.byref(args), C.byref(res)), "drift_pt_solve")
    assert np.array_equal(tried, st["tried"]) and np.array_equal(acc, st["accepted"])
    assert np.array_equal(bh, hist)
    slot = st["slot_of_rung"]
    assert np.array_equal(rung_spins, st["spins"][slot])
    assert np.array_equal(rung_e, st["energy"][slot])
    b = int(np.argmin(st["best_energy_fixed"]))
    assert np.array_equal(best_s, st["best_spins"][b].astype(np.float32))
    assert res.best_E == pytest.approx(model.energy(best_s.astype(np.float64)))
    assert res.throughput > 0 and 0.0 < res.swap_rate < 1.0


def test_solve_calls_share_nothing_through_the_cached_arena():
    """drift_pt_solve keeps its device arena on the thread between calls: a call after a larger and a
    smaller one, and after drift_pt_solve_release, returns exactly what the same call returned first
    (every output, the swap counts and the best-energy history included)."""
    L = _lib.load()
    p = lambda a: a.ctypes.data_as(C.c_void_p)

    def solve(model, R, rounds, spr, seed):
        hp = HostProblem.from_model(model)
        betas = geometric_betas(R, 0.25, 5.0)
        out = {"best_s": np.zeros(hp.n, np.float32), "rung_spins": np.zeros((R, hp.n), np.int8),
               "rung_e": np.zeros(R), "tried": np.zeros(R - 1, np.int64), "acc": np.zeros(R - 1, np.int64),
               "hist": np.zeros(rounds)}
        args = _lib.SolveArgs(R, rounds, spr, 0, seed, 0.0, 0.0, p(betas))
        res = _lib.SolveResult(0, 0, 0, 0, p(out["best_s"]), p(out["rung_spins"]), p(out["rung_e"]),
                               p(out["tried"]), p(out["acc"]), p(out["hist"]))
        _lib.check(L.drift_pt_solve(C.byref(hp.c_csr()), C.byref(args), C.byref(res)), "drift_pt_solve")
        out["best_E"], out["swap_rate"] = res.best_E, res.swap_rate
        return out

    small = (maxcut_3regular(512, 3), 16, 12, 2, 5)
    first = solve(*small)
    solve(maxcut_3regular(2048, 6), 48, 30, 3, 9)  # a larger call grows the arena
    again = solve(*small)
    _lib.check(L.drift_pt_solve_release(), "drift_pt_solve_release")
    fresh = solve(*small)
    for k in first:
        assert np.array_equal(first[k], again[k]), k
        assert np.array_equal(first[k], fresh[k]), k
