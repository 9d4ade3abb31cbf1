"""Observables on the C1 workload (2-D +-J L = 16, 24 rungs, T 1/3..10, an exchange after every
sweep) against the reference CPU PT (drift/solvers/parallel_tempering.py:52-124).

tests/golden/c1_observables.json holds, per rung, 16 independent reference runs' mean energy and
mean |m| and 8 run pairs' mean overlap q^2, each after a burn-in (tests/golden/make_c1_observables.py,
through the restatement oracle/ref_pt.py). Here the same protocol runs on the engine's chain: on the
CPU through the C oracle (the chain the kernels run bit for bit), and on the GPU through the engine
(tests/test_observables_gpu.py). Per rung, the mean over runs of each observable must agree with the
reference's within 3 combined standard errors taken across the independent runs.
"""

from __future__ import annotations

import json
import os

import numpy as np

import oracle

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "c1_observables.json")


def fixture() -> dict:
    with open(GOLDEN) as f:
        return json.load(f)


def c1_setup():
    from drift_b200.engine import HostProblem, geometric_betas
    from drift_b200.instances import ea_2d

    fx = fixture()
    hp = HostProblem.from_model(ea_2d(fx["L"], fx["seed"]))
    return fx, hp, geometric_betas(fx["R"], fx["T_min"], fx["T_max"])


def summarise(E_runs, M_runs, spins_runs):
    """Per-run rung means of E and |m| and per-pair mean q^2, from per-run series after burn-in."""
    E = np.array([e.mean(axis=0) for e in E_runs])
    M = np.array([m.mean(axis=0) for m in M_runs])
    q2 = []
    for k in range(0, len(spins_runs), 2):
        a, b = spins_runs[k].astype(np.float64), spins_runs[k + 1].astype(np.float64)
        q2.append(((a * b).mean(axis=2) ** 2).mean(axis=0))
    return {"energy": E, "absm": M, "q2": np.array(q2)}


def assert_agrees_with_reference(ours: dict, fx: dict) -> None:
    for key in ("energy", "absm", "q2"):
        a, b = np.asarray(ours[key]), np.asarray(fx[key])
        ma, mb = a.mean(axis=0), b.mean(axis=0)
        sa, sb = a.std(axis=0, ddof=1) / np.sqrt(len(a)), b.std(axis=0, ddof=1) / np.sqrt(len(b))
        assert np.all(np.abs(ma - mb) <= 3.0 * np.sqrt(sa ** 2 + sb ** 2) + 1e-12), (key, ma, mb, sa, sb)


def test_fixture_covers_the_c1_ladder():
    fx = fixture()
    assert fx["R"] == 24 and fx["L"] == 16 and len(fx["energy"]) == fx["runs"] == 16 and len(fx["q2"]) == 8
    E = np.array(fx["energy"]).mean(axis=0)
    assert np.all(np.diff(E) > 0)  # rung 0 is the coldest: hotter rungs, higher energies
    assert -2.0 * 256 <= E.min()  # at most every bond satisfied


def test_oracle_chain_matches_the_reference_cpu_pt_on_c1():
    fx, hp, betas = c1_setup()
    prob = oracle.OracleProblem(hp.n, hp.row_ptr, hp.col_idx, hp.weight, hp.h, hp.color_ptr, hp.color_spins)
    burn, rounds = fx["burn_in"], fx["rounds"]
    E_runs, M_runs, S_runs = [], [], []
    for k in range(fx["runs"]):
        st = oracle.pt_run(prob, betas, n_rounds=burn, sweeps_per_round=1, seed=500 + k)
        E = np.empty((rounds, fx["R"]))
        M = np.empty((rounds, fx["R"]))
        S = np.empty((rounds, fx["R"], hp.n), np.int8)
        for t in range(rounds):
            st = oracle.pt_run(prob, betas, n_rounds=1, sweeps_per_round=1, seed=500 + k, state=st,
                               round_offset=burn + t)
            sl = st.slot_of_rung
            E[t] = st.energy[sl]
            S[t] = st.spins[sl]
            M[t] = np.abs(S[t].astype(np.float64).mean(axis=1))
        E_runs.append(E)
        M_runs.append(M)
        S_runs.append(S)
    assert_agrees_with_reference(summarise(E_runs, M_runs, S_runs), fx)
