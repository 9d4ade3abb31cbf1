"""pytest configuration: the `gpu` marker and shared fixtures.

`-m "not gpu"` runs on a CPU-only machine (oracle vs golden vectors, host logic, the C ABI's
exports and host helpers); `-m gpu` runs the parity tests through the C ABI on a CUDA device.
"""

from __future__ import annotations

import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device and the built libdrift_pt.so")


def load_golden(name: str):
    with open(os.path.join(GOLDEN, name)) as f:
        return json.load(f)


def dense_from_edges(n, edges, h):
    from drift_b200.ising import IsingModel

    J = np.zeros((n, n))
    i, j, w = np.asarray(edges["i"], int), np.asarray(edges["j"], int), np.asarray(edges["w"], float)
    J[i, j] = w
    J[j, i] = w
    return IsingModel(J, np.asarray(h, dtype=np.float64))


@pytest.fixture(scope="session")
def reference_instances():
    return load_golden("reference.json")


def cuda_ready() -> bool:
    try:
        import torch

        from drift_b200 import _lib

        return torch.cuda.is_available() and _lib.available()
    except Exception:
        return False
