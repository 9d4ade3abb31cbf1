"""ORACLE - test infrastructure only.

NumPy restatement of the reference CPU parallel tempering, drift/solvers/parallel_tempering.py:52-124
(random-site Metropolis with PCG64 from ``numpy.random.default_rng(seed)``, adjacent-rung
configuration swaps with alternating parity, best-so-far per round). It makes the same random
draws in the same order as the reference, so on the same model and seed it returns the same
best_E, swap_rate and best_history; tests/golden/ref_pt.json pins that against outputs of the
reference itself. It also records per-round observables (energy and |m| per rung) that the
reference computes but does not return, for the statistical comparison with the engine.

It is the "reference" arm of bench.py: the reference's own CPU algorithm, timed on the host.
"""

from __future__ import annotations

import time

import numpy as np


def geometric_ladder(n_replicas: int, T_min: float, T_max: float) -> np.ndarray:
    """drift/solvers/parallel_tempering.py:29-36."""
    if n_replicas == 1:
        return np.array([T_min], dtype=np.float64)
    return T_min * (T_max / T_min) ** (np.arange(n_replicas) / (n_replicas - 1))


def parallel_tempering(model, *, n_replicas=16, T_min=0.1, T_max=5.0, n_rounds=300, sweeps_per_round=5, seed=0,
                       record=False, record_spins=False):
    """drift/solvers/parallel_tempering.py:52-124. Returns a dict; with ``record`` also the
    per-round rung energies (n_rounds, R) and |m| (n_rounds, R) after the sweeps; with
    ``record_spins`` the rung configurations (n_rounds, R, n) at the same points."""
    rng = np.random.default_rng(seed)
    n = model.n
    R = n_replicas
    temps = geometric_ladder(R, T_min, T_max)
    beta = 1.0 / np.maximum(temps, 1e-12)
    s = (rng.integers(0, 2, size=(R, n)) * 2 - 1).astype(np.float64)
    E = np.array([model.energy(s[r]) for r in range(R)])
    best_idx = int(np.argmin(E))
    best_s = s[best_idx].copy()
    best_E = float(E[best_idx])
    best_history = np.empty(n_rounds, dtype=np.float64)
    rec_E = np.empty((n_rounds, R)) if record else None
    rec_m = np.empty((n_rounds, R)) if record else None
    rec_s = np.empty((n_rounds, R, n), np.int8) if record_spins else None
    swaps_tried = 0
    swaps_done = 0
    J, h = model.J, model.h
    t_loop = time.perf_counter()
    for rnd in range(n_rounds):
        for r in range(R):
            inv_T = beta[r]
            sr = s[r]
            Er = E[r]
            for _ in range(sweeps_per_round * n):
                i = int(rng.integers(n))
                dE = float(2.0 * sr[i] * (J[i] @ sr + h[i]))  # drift/ising.py:63-68
                if dE <= 0.0 or rng.random() < np.exp(-dE * inv_T):
                    sr[i] = -sr[i]
                    Er += dE
            E[r] = Er
            if Er < best_E:
                best_E = float(Er)
                best_s = sr.copy()
        if record:
            rec_E[rnd] = E
            rec_m[rnd] = np.abs(s.mean(axis=1))
        if record_spins:
            rec_s[rnd] = s.astype(np.int8)
        start = rnd % 2
        for r in range(start, R - 1, 2):
            swaps_tried += 1
            delta = (beta[r] - beta[r + 1]) * (E[r] - E[r + 1])
            if delta >= 0.0 or rng.random() < np.exp(delta):
                s[[r, r + 1]] = s[[r + 1, r]]
                E[r], E[r + 1] = E[r + 1], E[r]
                swaps_done += 1
        best_history[rnd] = best_E
    loop_seconds = time.perf_counter() - t_loop
    out = {
        "best_s": best_s,
        "best_E": best_E,
        "temperatures": temps,
        "swap_rate": swaps_done / swaps_tried if swaps_tried else 0.0,
        "best_history": best_history,
        "attempts": float(R) * n_rounds * sweeps_per_round * n,
        "loop_seconds": loop_seconds,  # the round loop alone (initial energies excluded)
    }
    if record:
        out["rung_energy"] = rec_E
        out["rung_absm"] = rec_m
    if record_spins:
        out["rung_spins"] = rec_s
    return out
