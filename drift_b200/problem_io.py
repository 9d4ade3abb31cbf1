"""The reference's problem.bin / result.bin files (drift/gpu.py:83-103, cuda/ising_pt.cu:40-45,
231-234): write a PT job for an `ising_pt`-style executable and read its result."""

from __future__ import annotations

import re
import struct

import numpy as np

from .engine import HostProblem

HEADER = struct.Struct("<Qiiiiiiff")  # seed, n, R, n_rounds, sweeps_per_round, nnz, k, T_min, T_max


def write_problem(path: str, model, *, n_replicas: int, T_min: float, T_max: float, n_rounds: int,
                  sweeps_per_round: int, seed: int) -> HostProblem:
    """CSR in np.nonzero order, fp32 weights and field, greedy colouring (drift/gpu.py:66-95)."""
    hp = HostProblem.from_model(model)
    k = hp.n_colors
    with open(path, "wb") as f:
        f.write(HEADER.pack(seed & 0xFFFFFFFFFFFFFFFF, hp.n, n_replicas, n_rounds, sweeps_per_round,
                            int(hp.col_idx.size), k, float(T_min), float(T_max)))
        for a, dt in ((hp.row_ptr, np.int32), (hp.col_idx, np.int32), (hp.weight, np.float32), (hp.h, np.float32),
                      (hp.color_ptr, np.int32), (hp.color_spins, np.int32)):
            f.write(np.ascontiguousarray(a, dtype=dt).tobytes())
    return hp


def read_result(path: str, n: int):
    """(best_E, best_s float64[n]) from a result file."""
    with open(path, "rb") as f:
        best_E = struct.unpack("<d", f.read(8))[0]
        best_s = np.frombuffer(f.read(4 * n), dtype=np.float32).astype(np.float64)
    return best_E, best_s


def parse_stderr(text: str) -> dict:
    """The time=...s and throughput=... fields drift/gpu.py:105-106 reads."""
    out = {}
    for key, pat in (("seconds", r"time=([\d.eE+-]+)s"), ("throughput", r"throughput=([\d.eE+-]+)")):
        m = re.search(pat, text)
        out[key] = float(m.group(1)) if m else None
    return out
