"""Generate the golden fixtures in this folder by running the reference (DRiFT) itself.

    python tests/golden/make_golden.py /path/to/DRiFT

Needs the reference source tree on disk (it is imported, not copied). Writes:
  * reference.json - for each named instance: the reference's own J/h builders' output as an edge
    list, its exact ground energy (drift/solvers/exact.py:34-49), its greedy colouring
    (drift/gpu.py:122-145) and, for n <= 12, the full exact spectrum;
  * ref_pt.json    - outputs of the reference CPU parallel tempering
    (drift/solvers/parallel_tempering.py:52-124) for fixed seeds: best_E, swap_rate, best_history;
  * bank_fixtures.json - the reference instance bank's n=8 fixtures (J, h, known energy) as
    written by drift/benchmarks/instances/fixtures/*.json;
  * solve_dispatch.json - what the reference dispatcher drift.solve.solve (drift/solve.py:75-80)
    does on instances past its exact-enumeration size: the call it makes to
    drift.gpu.parallel_tempering_gpu (positional model, keyword arguments), recorded by replacing
    that function and drift.gpu.gpu_available, and how it turns the returned PtResult into its
    Solution (method, certified flag, energy and configuration taken from best_E and best_s).
The tests compare the oracle and the engine against these files; the reference is not needed to
run the tests.
"""

from __future__ import annotations

import glob
import json
import os
import sys

import numpy as np

OUT = os.path.dirname(os.path.abspath(__file__))


def edges(J: np.ndarray):
    iu, ju = np.nonzero(np.triu(J, 1))
    return {"i": iu.tolist(), "j": ju.tolist(), "w": J[iu, ju].tolist()}


def main(ref_root: str) -> None:
    sys.path.insert(0, ref_root)
    from drift.builders.qubo import maxcut_ising, random_graph
    from drift.gpu import _greedy_coloring
    from drift.ising import IsingModel
    from drift.solvers.exact import exact_ground_state
    from drift.solvers.parallel_tempering import parallel_tempering

    def glass(n, seed, field):
        rng = np.random.default_rng(seed)
        J = np.zeros((n, n))
        for i in range(n):
            for j in range(i + 1, n):
                J[i, j] = J[j, i] = rng.choice([-1.0, 1.0])
        h = rng.normal(scale=field, size=n) if field else np.zeros(n)
        return IsingModel(J=J, h=h)

    def ferro(n):
        J = np.zeros((n, n))
        for i in range(n - 1):
            J[i, i + 1] = J[i + 1, i] = 1.0
        return IsingModel(J=J, h=np.zeros(n))

    insts = {
        # tests/test_parallel_tempering.py:37-44, experiments/phase14_gpu.py:38-42
        "maxcut_g16_p05_s3": maxcut_ising(random_graph(16, p=0.5, seed=3)),
        "maxcut_g18_p04_s8": maxcut_ising(random_graph(18, p=0.4, seed=8)),
        # tests/test_gpu.py:47-54 and :57-67
        "maxcut_g12_p05_s3": maxcut_ising(random_graph(12, p=0.5, seed=3)),
        "maxcut_g20_p05_s2": maxcut_ising(random_graph(20, p=0.5, seed=2)),
        # tests/test_parallel_tempering.py:92-98
        "maxcut_g20_p04_s5": maxcut_ising(random_graph(20, p=0.4, seed=5)),
        # tests/test_parallel_tempering.py:47-59 (h ~ N(0, 0.3): the float path), :71-89, :62-68
        "glass_n14_s7_field": glass(14, 7, 0.3),
        "glass_n16_s11": glass(16, 11, 0.0),
        "ferro_n18": ferro(18),
        "maxcut_g10_weighted_s4": maxcut_ising(random_graph(10, p=0.6, seed=4, weighted=True)),
    }
    ref = {}
    for name, m in insts.items():
        s, e, spec = exact_ground_state(m)
        rows, cols = np.nonzero(m.J)
        row_ptr = np.zeros(m.n + 1, dtype=np.int64)
        row_ptr[1:] = np.cumsum(np.bincount(rows, minlength=m.n))
        k, cptr, cspins = _greedy_coloring(m.n, row_ptr, cols)
        ref[name] = {
            "n": m.n, "edges": edges(m.J), "h": m.h.tolist(), "e_exact": e,
            "coloring": {"k": int(k), "color_ptr": cptr.tolist(), "color_spins": cspins.tolist()},
            "spectrum": spec.tolist() if m.n <= 12 else None,
        }
    with open(os.path.join(OUT, "reference.json"), "w") as f:
        json.dump(ref, f)

    runs = [
        ("maxcut_g16_p05_s3", dict(n_replicas=16, T_min=0.05, T_max=4.0, n_rounds=40, sweeps_per_round=4, seed=1)),
        ("glass_n14_s7_field", dict(n_replicas=6, T_min=0.05, T_max=5.0, n_rounds=30, sweeps_per_round=5, seed=2)),
        ("maxcut_g20_p04_s5", dict(n_replicas=16, n_rounds=20, seed=6)),
        ("ferro_n18", dict(n_replicas=1, T_min=0.05, T_max=0.05, n_rounds=25, sweeps_per_round=5, seed=4)),
    ]
    pt = []
    for name, kw in runs:
        r = parallel_tempering(insts[name], **kw)
        pt.append({"instance": name, "kwargs": kw, "best_E": r.best_E, "swap_rate": r.swap_rate,
                   "best_history": r.best_history.tolist(), "best_s": r.best_s.tolist()})
    with open(os.path.join(OUT, "ref_pt.json"), "w") as f:
        json.dump(pt, f)

    bank = []
    for path in sorted(glob.glob(os.path.join(ref_root, "drift", "benchmarks", "instances", "fixtures", "*.json"))):
        with open(path) as f:
            d = json.load(f)
        J = np.asarray(d["J"], dtype=np.float64)
        bank.append({"id": d["id"], "n": d["n"], "edges": edges(J), "h": d["h"], "known_energy": d["known_energy"]})
    with open(os.path.join(OUT, "bank_fixtures.json"), "w") as f:
        json.dump(bank, f)
    dispatch = solve_dispatch()
    with open(os.path.join(OUT, "solve_dispatch.json"), "w") as f:
        json.dump(dispatch, f)
    print(f"wrote {len(ref)} instances, {len(pt)} PT runs, {len(bank)} bank fixtures, {len(dispatch)} solve() "
          f"dispatches to {OUT}")


def solve_dispatch():
    """Record drift.solve.solve's GPU branch on MaxCut G(n, 0.3) instances, n = 20..30."""
    import importlib

    ref_gpu = importlib.import_module("drift.gpu")
    ref_solve = importlib.import_module("drift.solve")  # the module (drift exports a function of that name)
    from drift.builders.qubo import maxcut_ising, random_graph
    from drift.solvers.parallel_tempering import PtResult

    out = []
    for n in (20, 24, 28, 30):
        model = maxcut_ising(random_graph(n, p=0.3, seed=n))
        calls = []
        marker = np.where(np.arange(n) % 3 == 0, -1.0, 1.0)

        def recorder(m, **kwargs):
            calls.append({"n": int(m.n), "kwargs": kwargs})
            return PtResult(best_s=marker.copy(), best_E=float(m.energy(marker)), temperatures=np.array([1.0]),
                            swap_rate=0.5)

        saved = ref_gpu.gpu_available, ref_gpu.parallel_tempering_gpu
        ref_gpu.gpu_available, ref_gpu.parallel_tempering_gpu = (lambda: True), recorder
        try:
            sol = ref_solve.solve(model)
        finally:
            ref_gpu.gpu_available, ref_gpu.parallel_tempering_gpu = saved
        assert len(calls) == 1
        out.append({"n": n, "edges": edges(model.J), "h": model.h.tolist(), "call": calls[0],
                    "method": sol.method, "certified": bool(sol.certified),
                    "energy_is_best_E": bool(sol.energy == float(model.energy(marker))),
                    "s_is_best_s": bool(np.array_equal(sol.s, marker))})
    return out


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("DRIFT_REFERENCE_TREE", "."))
