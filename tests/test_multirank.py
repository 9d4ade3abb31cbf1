"""The multi-GPU path is replicas only: with N ranks every rank runs its own copy of the job under
its own instance stream, and the only cross-rank operations are the timing barrier and the
max-over-ranks reduction. Checked here with two `gloo` ranks on the CPU: the collectives bench.py
uses, that each rank's chain equals the same chain run alone (no data crosses ranks) and differs
from the other rank's, the whole-job rate formula, and that the reference arm under torchrun does
its work on rank 0 only."""

from __future__ import annotations

import json
import os
import socket
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _small_problem():
    import oracle
    from drift_b200.engine import HostProblem
    from drift_b200.instances import ea_2d

    hp = HostProblem.from_model(ea_2d(6, 3))
    prob = oracle.OracleProblem(hp.n, hp.row_ptr, hp.col_idx, hp.weight, hp.h, hp.color_ptr, hp.color_spins)
    return prob, 0.2 * 10.0 ** (np.arange(8) / 7)


def _rank_main(rank: int, port: int, out_dir: str):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE="2",
                      LOCAL_RANK=str(rank), DRIFT_BENCH_BACKEND="gloo")
    sys.path.insert(0, ROOT)
    import torch
    import torch.distributed as dist

    import bench
    import oracle

    r, world, _ = bench.dist_setup(2)
    assert (r, world) == (rank, 2)
    mx = bench.reduce_max(float(10 * rank + 1), world, torch.device("cpu"))
    bench.barrier(world)
    prob, betas = _small_problem()
    st = oracle.pt_run(prob, betas, n_rounds=4, sweeps_per_round=2, seed=1, instance=rank)
    res = {"max": mx, "energy": st.energy.tolist(), "spins": st.spins.astype(int).ravel().tolist()}
    got = [None, None]
    dist.all_gather_object(got, res)
    with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
        json.dump({"mine": res, "all": got}, f)
    dist.destroy_process_group()


def test_two_gloo_ranks_run_independent_replicas(tmp_path):
    import torch.multiprocessing as mp

    port = _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_rank_main, args=(r, port, str(tmp_path))) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    import oracle

    prob, betas = _small_problem()
    outs = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(2)]
    for r, o in enumerate(outs):
        assert o["mine"]["max"] == 11.0  # max over ranks of 10 r + 1
        alone = oracle.pt_run(prob, betas, n_rounds=4, sweeps_per_round=2, seed=1, instance=r)
        assert o["mine"]["energy"] == alone.energy.tolist()  # nothing from the other rank entered
        assert o["all"][r] == o["mine"]
    assert outs[0]["mine"]["spins"] != outs[1]["mine"]["spins"]  # distinct instance streams


def test_whole_job_rate_is_all_ranks_attempts_over_the_slowest_rank():
    import bench

    assert bench.whole_job_rate(1e9, 4, 2, 0.5) == pytest.approx(1e9 * 4 * 2 / 0.5 / 1e9)


def test_reference_arm_under_torchrun_works_on_rank_zero_only():
    env = dict(os.environ, DRIFT_BENCH_BACKEND="gloo", OMP_NUM_THREADS="1")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2", "--master-addr",
           "127.0.0.1", "--master-port", str(_free_port()), "bench.py", "--impl", "reference", "--gpus", "2",
           "--steps", "1", "--warmup", "0", "--workload", "ea2d"]
    r = subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(ln) for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1 and lines[0]["impl"] == "reference" and lines[0]["n_gpus"] == 2
