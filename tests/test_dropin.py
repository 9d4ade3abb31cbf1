"""The drop-in module keeps the reference's PT interface (drift/gpu.py:33-52,
drift/solvers/parallel_tempering.py:39-61): the same names, the same keywords with the same
defaults and kinds, the same PtResult fields with extras only added after them. When the
reference tree is importable (read only), the signatures are also compared with its own."""

from __future__ import annotations

import dataclasses
import inspect
import os
import sys

import pytest

from drift_b200 import gpu

# the reference's keyword set and defaults (drift/gpu.py:43-52 = parallel_tempering.py:52-61)
REFERENCE_KEYWORDS = {"n_replicas": 16, "T_min": 0.1, "T_max": 5.0, "n_rounds": 300, "sweeps_per_round": 5, "seed": 0}
REFERENCE_RESULT_FIELDS = ["best_s", "best_E", "temperatures", "swap_rate", "best_history", "throughput", "seconds"]


def test_names_keywords_and_defaults_match_the_reference():
    assert callable(gpu.gpu_available) and callable(gpu.gpu_binary_path) and callable(gpu.parallel_tempering_gpu)
    assert isinstance(gpu.gpu_binary_path(), str)
    sig = inspect.signature(gpu.parallel_tempering_gpu)
    params = list(sig.parameters.values())
    assert params[0].name == "model" and params[0].kind == inspect.Parameter.POSITIONAL_OR_KEYWORD
    for name, default in REFERENCE_KEYWORDS.items():
        p = sig.parameters[name]
        assert p.kind == inspect.Parameter.KEYWORD_ONLY and p.default == default, name
    extra = [p for p in params[1:] if p.name not in REFERENCE_KEYWORDS]
    assert all(p.kind == inspect.Parameter.KEYWORD_ONLY and p.default is not inspect.Parameter.empty for p in extra)


def test_result_fields_extend_the_reference_record():
    names = [f.name for f in dataclasses.fields(gpu.PtResult)]
    assert names[: len(REFERENCE_RESULT_FIELDS)] == REFERENCE_RESULT_FIELDS
    required = [f.name for f in dataclasses.fields(gpu.PtResult)
                if f.default is dataclasses.MISSING and f.default_factory is dataclasses.MISSING]
    assert required == REFERENCE_RESULT_FIELDS[: len(required)]


def _reference():
    root = os.environ.get("DRIFT_REFERENCE_TREE")
    if not root or not os.path.isdir(os.path.join(root, "drift")):
        pytest.skip("DRIFT_REFERENCE_TREE does not name the reference tree")
    sys.dont_write_bytecode = True
    if root not in sys.path:
        sys.path.append(root)
    try:
        import drift.gpu as ref_gpu
        import drift.solvers.parallel_tempering as ref_pt
    except Exception as e:  # noqa: BLE001
        pytest.skip(f"reference not importable here: {e}")
    return ref_gpu, ref_pt


def test_signatures_equal_the_reference_modules():
    ref_gpu, ref_pt = _reference()
    mine = inspect.signature(gpu.parallel_tempering_gpu).parameters
    for fn in (ref_gpu.parallel_tempering_gpu, ref_pt.parallel_tempering):
        for name, p in inspect.signature(fn).parameters.items():
            assert name in mine, name
            assert mine[name].kind == p.kind and mine[name].default == p.default, name
    ref_fields = [f.name for f in dataclasses.fields(ref_pt.PtResult)]
    assert [f.name for f in dataclasses.fields(gpu.PtResult)][: len(ref_fields)] == ref_fields
