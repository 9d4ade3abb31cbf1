"""Generate tests/golden/c1_observables.json: equilibrium observables of the reference CPU PT on the
C1 workload (2-D Edwards-Anderson +-J, L = 16 periodic, 24 rungs on a geometric T ladder 1/3..10, one
sweep per round, an exchange step after every round).

    python tests/golden/make_c1_observables.py

The reference CPU algorithm is drift/solvers/parallel_tempering.py:52-124, run through its NumPy
restatement oracle/ref_pt.py (same draws in the same order; tests/golden/ref_pt.json pins it against
the reference itself), which also records what the reference computes but does not return: every
round's energy, |m| and configuration per rung. RUNS independent ladders are run in parallel
processes; each drops BURN_IN rounds and averages the next ROUNDS. The file holds, per rung, each
run's mean energy and mean |m|, and for each pair of runs (2k, 2k + 1) the mean overlap q^2 of their
configurations. Errors are then taken across independent runs, so no autocorrelation estimate is
needed. The colour-ordered sweep of the engine and the random-site sweep of the reference are
different Markov chains with the same stationary distribution; they are compared only after the
burn-in. The burn-in is set by the reference's chain: after 1000 rounds its coldest rungs are still
~0.6 above their equilibrium energy (-359.95 at T = 1/3, which the engine's chain reaches within
1000 rounds), so it runs 10000.
"""

from __future__ import annotations

import json
import multiprocessing as mp
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))

L, SEED, R, T_MIN, T_MAX = 16, 1, 24, 1.0 / 3.0, 10.0
RUNS, BURN_IN, ROUNDS = 16, 10000, 4000


def _run(seed: int):
    sys.path.insert(0, ROOT)
    from drift_b200.instances import ea_2d
    from oracle import ref_pt

    model = ea_2d(L, SEED).to_dense()
    out = ref_pt.parallel_tempering(model, n_replicas=R, T_min=T_MIN, T_max=T_MAX, n_rounds=BURN_IN + ROUNDS,
                                    sweeps_per_round=1, seed=seed, record=True, record_spins=True)
    return (out["rung_energy"][BURN_IN:].mean(axis=0), out["rung_absm"][BURN_IN:].mean(axis=0),
            out["rung_spins"][BURN_IN:])


def main() -> None:
    os.environ["OMP_NUM_THREADS"] = "1"
    with mp.get_context("spawn").Pool(min(RUNS, os.cpu_count() or 1)) as pool:
        res = pool.map(_run, [1000 + k for k in range(RUNS)])
    q2 = []
    for k in range(0, RUNS, 2):
        sa, sb = res[k][2].astype(np.float64), res[k + 1][2].astype(np.float64)
        q2.append(((sa * sb).mean(axis=2) ** 2).mean(axis=0).tolist())
    out = {"L": L, "seed": SEED, "R": R, "T_min": T_MIN, "T_max": T_MAX, "runs": RUNS, "burn_in": BURN_IN,
           "rounds": ROUNDS, "energy": [r[0].tolist() for r in res], "absm": [r[1].tolist() for r in res],
           "q2": q2}
    with open(os.path.join(HERE, "c1_observables.json"), "w") as f:
        json.dump(out, f)
    print(f"wrote {RUNS} runs to {HERE}/c1_observables.json")


if __name__ == "__main__":
    main()
