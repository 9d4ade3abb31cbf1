"""The `ising_pt` command on the GPU: problem files written as drift/gpu.py writes them are solved
to the exact ground energies of the reference's own test instances, the result file and the stderr
fields are those drift/gpu.py reads, and - where the reference's engine was built from its source -
both executables agree on the ground energy."""

from __future__ import annotations

import os
import subprocess

import numpy as np
import pytest

import oracle
from conftest import cuda_ready, dense_from_edges, load_golden

from drift_b200.build import CLI_PATH
from drift_b200.problem_io import parse_stderr, read_result, write_problem

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_ready() or not os.path.exists(CLI_PATH),
                                                  reason="needs CUDA and the ising_pt command")]


@pytest.mark.parametrize("name", ["maxcut_g12_p05_s3", "maxcut_g16_p05_s3", "glass_n14_s7_field", "ferro_n18"])
def test_cli_solves_reference_problem_files(tmp_path, name):
    inst = load_golden("reference.json")[name]
    m = dense_from_edges(int(inst["n"]), inst["edges"], inst["h"])
    prob, res = str(tmp_path / "problem.bin"), str(tmp_path / "result.bin")
    write_problem(prob, m, n_replicas=16, T_min=0.1, T_max=5.0, n_rounds=300, sweeps_per_round=5, seed=0)
    binaries = [CLI_PATH] + ([oracle.REF_BIN] if os.path.exists(oracle.REF_BIN) else [])
    for binary in binaries:
        r = subprocess.run([binary, prob, res], capture_output=True, text=True, timeout=120)
        assert r.returncode == 0, r.stderr
        best_E, best_s = read_result(res, m.n)
        assert abs(best_E - inst["e_exact"]) < 1e-4, (binary, best_E, inst["e_exact"])
        assert set(np.unique(best_s)) <= {-1.0, 1.0}
        assert abs(m.energy(best_s) - best_E) < 1e-4
        f = parse_stderr(r.stderr)
        assert f["seconds"] is not None and f["throughput"] is not None and f["throughput"] > 0
