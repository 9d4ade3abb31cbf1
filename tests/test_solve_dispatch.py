"""The reference's solve() dispatcher reaches this engine (the f2 integration of the PT path).

drift.solve.solve (drift/solve.py:75-80) sends every instance past its exact-enumeration size to
drift.gpu.parallel_tempering_gpu(model, n_replicas=n_replicas or 256, n_rounds=..., sweeps_per_round=...,
seed=...) and returns Solution(s=best_s, energy=best_E, method="gpu-pt", certified=False). The
fixture tests/golden/solve_dispatch.json records exactly that call and mapping from the reference
itself (tests/golden/make_golden.py). The CPU tests check that the drop-in accepts the recorded call;
the GPU test makes the recorded calls through drift_b200.gpu and checks the Solution the dispatcher
builds from them against exact enumeration. Where the reference tree is importable
(DRIFT_REFERENCE_TREE), the GPU test also runs the reference's own solve() with drift.gpu pointed at
this engine, as INTEGRATION.md describes.
"""

from __future__ import annotations

import importlib
import inspect
import json
import os
import sys

import numpy as np
import pytest

import oracle
from conftest import cuda_ready, dense_from_edges

from drift_b200 import gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "solve_dispatch.json")


def _dispatches():
    with open(GOLDEN) as f:
        return json.load(f)


def test_recorded_dispatch_is_the_gpu_branch():
    d = _dispatches()
    assert [x["n"] for x in d] == [20, 24, 28, 30]
    for x in d:
        assert x["method"] == "gpu-pt" and x["certified"] is False
        assert x["energy_is_best_E"] and x["s_is_best_s"]
        assert x["call"]["n"] == x["n"]


def test_drop_in_accepts_the_recorded_call():
    sig = inspect.signature(gpu.parallel_tempering_gpu)
    for x in _dispatches():
        model = dense_from_edges(x["n"], x["edges"], x["h"])
        bound = sig.bind(model, **x["call"]["kwargs"])
        assert bound.arguments["n_replicas"] == 256


def _reference_solve_module():
    root = os.environ.get("DRIFT_REFERENCE_TREE")
    if not root or not os.path.isdir(os.path.join(root, "drift")):
        return None
    sys.dont_write_bytecode = True
    if root not in sys.path:
        sys.path.append(root)
    try:
        return importlib.import_module("drift.solve"), importlib.import_module("drift.gpu")
    except Exception:  # noqa: BLE001
        return None


@pytest.mark.gpu
@pytest.mark.skipif(not cuda_ready(), reason="needs CUDA and libdrift_pt.so")
def test_dispatcher_calls_reach_the_exact_ground_state(monkeypatch):
    for x in _dispatches():
        model = dense_from_edges(x["n"], x["edges"], x["h"])
        r = gpu.parallel_tempering_gpu(model, **x["call"]["kwargs"])
        # the Solution drift/solve.py:79-80 builds from the result
        s, energy = r.best_s, r.best_E
        e_exact = oracle.exact(model.J, model.h).e_min
        assert energy == pytest.approx(e_exact, abs=1e-9), x["n"]
        assert model.energy(s) == pytest.approx(energy, abs=1e-9)
        assert np.all(np.abs(s) == 1.0)
    ref = _reference_solve_module()
    if ref is None:
        return
    ref_solve, ref_gpu = ref
    monkeypatch.setattr(ref_gpu, "gpu_available", gpu.gpu_available)
    monkeypatch.setattr(ref_gpu, "parallel_tempering_gpu", gpu.parallel_tempering_gpu)
    for x in _dispatches():
        model = dense_from_edges(x["n"], x["edges"], x["h"])
        sol = ref_solve.solve(model)
        assert sol.method == "gpu-pt" and sol.certified is False
        assert sol.energy == pytest.approx(oracle.exact(model.J, model.h).e_min, abs=1e-9)
