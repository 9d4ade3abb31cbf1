"""The problem.bin / result.bin boundary (CPU): the writer produces the reference's packed layout
(drift/gpu.py:86-95) byte for byte, and the `ising_pt` command rejects malformed files with exit
status 1 and a message before touching a GPU."""

from __future__ import annotations

import os
import struct
import subprocess

import numpy as np
import pytest

from drift_b200.build import CLI_PATH
from drift_b200.instances import gnp_pm
from drift_b200.problem_io import HEADER, write_problem


def test_problem_file_has_the_reference_layout(tmp_path):
    m = gnp_pm(20, 0.3, 2, field=1)
    path = str(tmp_path / "problem.bin")
    hp = write_problem(path, m, n_replicas=8, T_min=0.1, T_max=5.0, n_rounds=30, sweeps_per_round=5, seed=7)
    raw = open(path, "rb").read()
    seed, n, R, rounds, spr, nnz, k, tmin, tmax = struct.unpack("<Qiiiiiiff", raw[:40])
    assert (seed, n, R, rounds, spr) == (7, 20, 8, 30, 5) and HEADER.size == 40
    assert nnz == int(np.count_nonzero(m.J)) and k == hp.n_colors
    assert abs(tmin - 0.1) < 1e-7 and abs(tmax - 5.0) < 1e-7
    assert len(raw) == 40 + 4 * ((n + 1) + nnz + nnz + n + (k + 1) + n)
    # the CSR of drift/gpu.py:69-77: np.nonzero order, fp32 weights
    rows, cols = np.nonzero(m.J)
    off = 40 + 4 * (n + 1)
    assert np.array_equal(np.frombuffer(raw[off:off + 4 * nnz], np.int32), cols)
    assert np.array_equal(np.frombuffer(raw[off + 4 * nnz:off + 8 * nnz], np.float32), m.J[rows, cols].astype(np.float32))


def _run(*args):
    return subprocess.run([CLI_PATH, *args], capture_output=True, text=True, timeout=60)


@pytest.mark.skipif(not os.path.exists(CLI_PATH), reason="ising_pt command not built")
def test_cli_rejects_malformed_files(tmp_path):
    r = _run()
    assert r.returncode == 1 and "usage" in r.stderr
    r = _run(str(tmp_path / "missing.bin"), str(tmp_path / "out.bin"))
    assert r.returncode == 1 and "cannot read" in r.stderr
    short = tmp_path / "short.bin"
    short.write_bytes(b"\x00" * 20)
    r = _run(str(short), str(tmp_path / "out.bin"))
    assert r.returncode == 1 and "40-byte header" in r.stderr
    bad = tmp_path / "bad.bin"
    bad.write_bytes(struct.pack("<Qiiiiiiff", 1, 4, 2, 1, 1, 0, 0, 0.1, 1.0))  # k = 0
    r = _run(str(bad), str(tmp_path / "out.bin"))
    assert r.returncode == 1 and "out of range" in r.stderr
    good = str(tmp_path / "good.bin")
    write_problem(good, gnp_pm(12, 0.5, 1), n_replicas=4, T_min=0.1, T_max=5.0, n_rounds=2, sweeps_per_round=1, seed=1)
    raw = open(good, "rb").read()
    (tmp_path / "cut.bin").write_bytes(raw[:-4])
    r = _run(str(tmp_path / "cut.bin"), str(tmp_path / "out.bin"))
    assert r.returncode == 1 and "shorter" in r.stderr
    (tmp_path / "long.bin").write_bytes(raw + b"\x00\x00\x00\x00")
    r = _run(str(tmp_path / "long.bin"), str(tmp_path / "out.bin"))
    assert r.returncode == 1 and "longer" in r.stderr
    assert not (tmp_path / "out.bin").exists()
