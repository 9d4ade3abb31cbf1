"""Observables of the engine (GPU) on the C1 companion instance (G(20, 0.3), +-1 couplings, +-1
field): per-rung mean energy, |m| and site magnetisations against exact enumeration, and mean
energy, |m| and overlap q^2 (two independent ladders) within 3 sigma of the reference CPU PT
(oracle/ref_pt.py, the NumPy restatement of drift/solvers/parallel_tempering.py)."""

from __future__ import annotations

import numpy as np
import pytest

import oracle
from conftest import cuda_ready
from oracle import ref_pt
from test_observables import BETAS, R, check_against_exact, model

from drift_b200.observables import blocked, overlap, record

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_ready(), reason="needs CUDA and libdrift_pt.so")]


def _engine(m, seed):
    from drift_b200.engine import DeviceProblem, HostProblem, PtEngine

    eng = PtEngine(DeviceProblem(HostProblem.from_model(m)), BETAS, seed=seed, sweeps_per_round=5)
    eng.init()
    return eng


def test_engine_observables_match_exact_and_reference_cpu_pt():
    m = model()
    ex = oracle.exact(m.J, m.h, BETAS, site_mag=True)
    a = record(_engine(m, 1), 3000, spins=True)
    b = record(_engine(m, 2), 3000, spins=True)
    for run in (a, b):
        check_against_exact(run["energy"], run["absm"], run["spins"], ex)
    # the reference CPU PT: two independent ladders for the overlap
    ra = ref_pt.parallel_tempering(m, n_replicas=R, T_min=1.0 / 3.0, T_max=10.0, n_rounds=800, sweeps_per_round=5,
                                   seed=10, record=True, record_spins=True)
    rb = ref_pt.parallel_tempering(m, n_replicas=R, T_min=1.0 / 3.0, T_max=10.0, n_rounds=800, sweeps_per_round=5,
                                   seed=11, record=True, record_spins=True)
    ours = {"E": a["energy"], "absm": a["absm"], "q2": overlap(a["spins"], b["spins"]) ** 2}
    ref = {"E": ra["rung_energy"], "absm": ra["rung_absm"], "q2": overlap(ra["rung_spins"], rb["rung_spins"]) ** 2}
    for k in ("E", "absm", "q2"):
        mo, so = blocked(ours[k])
        mr, sr = blocked(ref[k])
        assert np.all(np.abs(mo - mr) <= 3.0 * np.sqrt(so ** 2 + sr ** 2) + 1e-9), (k, mo, mr, so, sr)
    assert a["energy"].min() >= ex.e_min - 1e-9


def test_engine_matches_the_reference_cpu_pt_on_c1():
    """C1 (2-D +-J L = 16, 24 rungs, T 1/3..10, one sweep per round): 16 independent ladders of the
    engine, each after the same burn-in, against 16 of the reference CPU PT (the fixture of
    tests/test_c1_observables.py): per-rung mean energy, |m| and overlap q^2 within 3 combined
    standard errors across runs."""
    from drift_b200.engine import DeviceProblem, PtEngine
    from test_c1_observables import assert_agrees_with_reference, c1_setup, summarise

    fx, hp, betas = c1_setup()
    prob = DeviceProblem(hp)
    E_runs, M_runs, S_runs = [], [], []
    for k in range(fx["runs"]):
        eng = PtEngine(prob, betas, seed=700 + k, sweeps_per_round=1)
        eng.init()
        eng.run(fx["burn_in"])
        run = record(eng, fx["rounds"], spins=True)
        E_runs.append(run["energy"])
        M_runs.append(run["absm"])
        S_runs.append(run["spins"])
    assert_agrees_with_reference(summarise(E_runs, M_runs, S_runs), fx)
