"""Benchmark: spin-flip attempts per ns of the B200 parallel-tempering engine.

    python bench.py [--gpus N] [--steps K] [--warmup W]
                    [--workload maxcut3reg|ea2d|batched_er|ea3d64|maxcut3reg_r2048|ea2d_batch256|sk512]
                    [--impl b200|reference|reference-gpu]

Workload (default ``maxcut3reg``): plain PT on MaxCut as Ising over a random 3-regular graph,
N = 4096 (seeded), J = -1 on edges, h = 0, int8 spins, greedy colouring (4 colours), 64 replicas
on a geometric beta ladder 0.2..4.0, 1e5 sweeps = 25,000 rounds of 4 sweeps (the reference's
solve() default sweeps_per_round), one exchange step per round. One "step" is that whole job:
initialisation plus 1e5 sweeps of all 64 replicas = 2.62e10 attempts.

``value`` is device time (CUDA events around each step, inputs resident in HBM), summed over K
steps, max over ranks. L2 is flushed (a 256 MiB write) between steps, outside the timed events.
``e2e`` times the C ABI entry drift_pt_solve with host buffers (layout, upload, run, download).
With N > 1 (torchrun), every rank runs an independent copy (replicas only: the path has no
exchange across GPUs) and ``value`` is the sum of all ranks' attempts over the slowest rank's
time. ``--impl reference`` times the reference's own CPU algorithm (the NumPy restatement of
drift/solvers/parallel_tempering.py in oracle/ref_pt.py, one process per host core) on a bounded
sample of the same workload.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    "maxcut3reg": dict(desc="MaxCut random 3-regular N=4096 (J=-1), int8 spins, 64 replicas, beta 0.2-4.0, 1e5 sweeps",
                       n=4096, seed=2, R=64, beta=(0.2, 4.0), sweeps=100000, spr=4, bytes_per_attempt=2.0 + 3 * 5 / 64),
    "ea2d": dict(desc="2D EA +-J L=16 periodic (N=256), 24 replicas, beta 0.1-3.0, 2e4 sweeps, swap every sweep",
                 n=256, seed=1, R=24, beta=(0.1, 3.0), sweeps=20000, spr=1, bytes_per_attempt=2.0 + 4 * 5 / 24),
    # batched: 512 Erdos-Renyi instances, N ~ U{64..8192}, mean degree 6, J ~ N(0,1) fp32, h ~ N(0, 0.1),
    # 32 replicas each on a geometric beta ladder 0.1-3.0; 5e4 sweeps per job (one step times 100 rounds
    # of 5 sweeps, 1 % of the job: the full job takes about a minute per run)
    "batched_er": dict(desc="512 ER instances N~U[64,8192], deg 6, Gaussian J fp32, h~N(0,0.1), 32 replicas each, "
                            "beta 0.1-3.0; 500 of the job's 5e4 sweeps per step",
                       n_instances=512, seed=3, R=32, beta=(0.1, 3.0), sweeps=500, spr=5,
                       bytes_per_attempt=2.0 + 6 * 8 / 32 + 4 / 32),
    # 3-D Edwards-Anderson +-J, L = 64 periodic (N = 262,144), seed 5; 128 replicas packed 32 per
    # word; beta 0.2-2.0; 1e4 sweeps in rounds of 10. Algorithmic bytes per attempt: spin read and
    # write (2 bits) + 3 coupling bits per site shared by the 128 replicas = 0.253 B
    "ea3d64": dict(desc="3D EA +-J L=64 periodic (N=262144), 128 replicas (bit-packed), beta 0.2-2.0, 1e4 sweeps "
                        "in rounds of 10",
                   n=64 ** 3, L=64, seed=5, R=128, beta=(0.2, 2.0), sweeps=10000, spr=10,
                   bytes_per_attempt=2 / 8 + 3 / 8 / 128),
    # the MaxCut instance above with 2048 replicas, 32 per word, on the graph multispin engine
    # (clusters of CTAs per word chosen by the engine); 2e4 sweeps in rounds of 4 per step.
    # Algorithmic bytes per attempt: spin read and write (2 bits) + 3 neighbour bits = 5/8 B
    "maxcut3reg_r2048": dict(desc="MaxCut random 3-regular N=4096 (J=-1), 2048 replicas (bit-packed), beta 0.2-4.0, "
                                  "2e4 sweeps in rounds of 4",
                             n=4096, seed=2, R=2048, beta=(0.2, 4.0), sweeps=20000, spr=4, bytes_per_attempt=5 / 8),
    # uneven batch: 256 2-D EA +-J instances, L uniform in [8, 48] (seed 6), couplings of instance k
    # from seed k, each padded with uncoupled spins to a multiple of 8 (energies unchanged); 32
    # replicas each, beta 0.1-3.0, rounds of 10 sweeps; 1e3 sweeps per step. With --ttt: time to
    # the best energy of a 1e5-sweep plain run, plain vs neural proposals (one MADE per instance of
    # at most 512 spins). Algorithmic bytes per attempt as C3 with int8 couplings: 2 + 4 (4 + 1) / 32
    "ea2d_batch256": dict(desc="256 2D EA +-J instances L~U[8,48] (padded to 8k spins), 32 replicas each, "
                               "beta 0.1-3.0, rounds of 10 sweeps; 1e3 sweeps per step",
                          n_instances=256, seed=6, R=32, beta=(0.1, 3.0), sweeps=1000, spr=10,
                          bytes_per_attempt=2.0 + 4 * 5 / 32),
    # dense SK: J_ij ~ N(0, 1)/sqrt(N) (fp32 values) on the upper triangle, mirrored, h = 0, seed 4;
    # 64 replicas, beta 0.3-3.0, rounds of 10 sweeps; 1e4 sweeps per step. Tensor-core field
    # updates: the algorithmic work of an attempt is the 2N flops of J_i . s (drift/ising.py:68)
    # training of the proposal network of the dense workload: MADE 512-1024-1024-512 (bf16 weights,
    # fp32 accumulation), Adam on batches of 512 configurations; one step = 50 Adam steps. Algorithmic
    # work per Adam step: forward 2B(n h1 + h1 h2 + h2 n), the weight gradients the same again, the
    # activation gradients 2B(h2 n + h1 h2)
    "made_train": dict(desc="MADE 512-1024-1024-512 training (bf16 x bf16 -> fp32 tensor-core GEMMs), batch 512, "
                            "50 Adam steps per step", n=512, h=1024, batch=512, adam_steps=50,
                       flops_per_adam_step=2 * 512 * (2 * (512 * 1024 + 1024 * 1024 + 1024 * 512)
                                                       + (1024 * 512 + 1024 * 1024))),
    "sk512": dict(desc="SK N=512, J~N(0,1/N) fp32, 64 replicas, beta 0.3-3.0, 1e4 sweeps in rounds of 10",
                  n=512, seed=4, R=64, beta=(0.3, 3.0), sweeps=10000, spr=10, flops_per_attempt=2 * 512),
}


def make_batch_models(w):
    from drift_b200.instances import er_gaussian

    rng = np.random.default_rng(w["seed"])
    sizes = rng.integers(64, 8193, size=w["n_instances"])
    return [er_gaussian(int(n), 6, 1000 + i, field_sigma=0.1) for i, n in enumerate(sizes)]


def make_model(name):
    from drift_b200.instances import ea_2d, ea_2d_padded, er_gaussian, maxcut_3regular, sk_model

    w = WORKLOADS[name]
    if name == "sk512":
        return sk_model(w["n"], w["seed"])
    # the reference runs a batch one instance at a time: its CPU sample is the median-size instance
    if name == "batched_er":
        sizes = np.random.default_rng(w["seed"]).integers(64, 8193, size=w["n_instances"])
        i = int(np.argsort(sizes, kind="stable")[len(sizes) // 2])
        return er_gaussian(int(sizes[i]), 6, 1000 + i, field_sigma=0.1)
    if name == "ea2d_batch256":
        Ls = np.random.default_rng(w["seed"]).integers(8, 49, size=w["n_instances"])
        i = int(np.argsort(Ls, kind="stable")[len(Ls) // 2])
        return ea_2d_padded(int(Ls[i]), i)
    return maxcut_3regular(w["n"], w["seed"]) if name.startswith("maxcut3reg") else ea_2d(16, w["seed"])


def ladder(w):
    b_lo, b_hi = w["beta"]
    R = w["R"]
    return b_lo * (b_hi / b_lo) ** (np.arange(R) / (R - 1))


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def issue_basis(kernel_key, attempts_per_s, sm_mhz):
    """The issue ceiling of a kernel: warp instructions per attempt from its ncu capture
    (profiles/issue.json) times the measured attempt rate, against 4 warp instructions per SM cycle
    over the whole chip and over the SMs the launch occupies."""
    p = os.path.join(ROOT, "profiles", "issue.json")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        d = json.load(f).get(kernel_key)
    if not d:
        return None
    import torch

    sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    hz = float(sm_mhz or 1965.0) * 1e6
    achieved = attempts_per_s * d["warp_inst_per_attempt"] / 1e9
    chip = sms * 4 * hz / 1e9
    used = min(d["ctas"], sms) * 4 * hz / 1e9
    return {"unit": "G warp instructions/s", "warp_inst_per_attempt": d["warp_inst_per_attempt"], "achieved": achieved,
            "peak_chip": chip, "frac_chip": achieved / chip, "peak_used_sms": used, "frac_used_sms": achieved / used,
            "sms_used": min(d["ctas"], sms), "source": "profiles/issue.json (ncu smsp__inst_executed.sum)"}


def load_traffic(kernel_key):
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        d = json.load(f)
    return d.get(kernel_key)


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons while the timed region runs."""

    FIELDS = ("clocks.sm,clocks.max.sm,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.thread.join(timeout=2)
        # On B200 boxes, CUDA calls made shortly after an nvidia-smi process exits were seen to stall
        # for up to ~1 s on the host (kernel time unchanged): let that teardown pass before the next
        # timed region (the end-to-end calls follow right after).
        time.sleep(3.0)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                smax.append(float(parts[1]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[3:7]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(n_gpus):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist

        backend = "nccl" if os.environ.get("DRIFT_BENCH_BACKEND", "nccl") == "nccl" else "gloo"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return rank, world, local


def reduce_max(x: float, world: int, device) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(attempts_per_rank_step: float, steps: int, world: int, t_max_s: float) -> float:
    """Whole-job spin-flips/ns: every rank's attempts (replicas only: each rank runs its own copy of
    the job) over the slowest rank's device time."""
    return attempts_per_rank_step * steps * world / t_max_s / 1e9


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


# ---------------------------------------------------------------------------------------------

# seconds of host work per CPU baseline (the secondaries use less)
CPU_BUDGET_S = 12.0


def emit(args, line: dict) -> None:
    """Print a result line, or hand it to the caller that runs this workload as a secondary."""
    sink = getattr(args, "sink", None)
    if sink is not None:
        sink.append(line)
    else:
        print(json.dumps(line), flush=True)


REF_SAMPLE_RUNGS = 64
# attempts per process and step of the reference arm's sample (about 2-5 s of one core)
REF_SAMPLE_ATTEMPTS = 1.0e6
_REF_WORKER = {}


def _ref_worker_init(name):
    """Pool initializer: the reference's dense model of the workload, built once per process."""
    sys.path.insert(0, ROOT)
    model = make_model(name)
    _REF_WORKER["model"] = model.to_dense() if hasattr(model, "to_dense") else model


def ref_sample_shape(w, n):
    """(rungs, rounds) of one process's sample: the reference's cost is linear in rungs, so wide
    ladders are sampled with REF_SAMPLE_RUNGS rungs over the same temperature range, and rounds are
    added up to about REF_SAMPLE_ATTEMPTS attempts."""
    rungs = min(w["R"], REF_SAMPLE_RUNGS)
    return rungs, max(1, int(round(REF_SAMPLE_ATTEMPTS / (rungs * w["spr"] * n))))


def run_reference_sample(args_tuple):
    """One process: the reference CPU algorithm on a bounded sample; returns (attempts, seconds of
    the round loop alone)."""
    name, seed = args_tuple
    from oracle import ref_pt

    w = WORKLOADS[name]
    model = _REF_WORKER["model"]
    b = ladder(w)
    rungs, rounds = ref_sample_shape(w, model.n)
    out = ref_pt.parallel_tempering(model, n_replicas=rungs, T_min=1.0 / b[0], T_max=1.0 / b[-1], n_rounds=rounds,
                                    sweeps_per_round=w["spr"], seed=seed)
    return out["attempts"], out["loop_seconds"]


def bench_reference(args):
    rank, world, local = dist_setup(args.gpus)
    if rank != 0:
        return
    if args.workload == "ea3d64":
        print(json.dumps({"impl": "reference", "unavailable": "the reference CPU PT needs the dense J of the "
                          "L=64 lattice (262144^2 float64 = 550 GB); see the multispin oracle cpu_baseline instead"}),
              flush=True)
        return
    import multiprocessing as mp

    w = WORKLOADS[args.workload]
    n_sample = make_model(args.workload).n
    rungs, rounds = ref_sample_shape(w, n_sample)
    where = " of the batch's median-size instance" if "n_instances" in w else ""
    cores = os.cpu_count() or 1
    # one BLAS thread per process: the workers are spawned with this environment
    for var in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS"):
        os.environ[var] = "1"
    ctx = mp.get_context("spawn")
    with ctx.Pool(cores, initializer=_ref_worker_init, initargs=(args.workload,)) as pool:
        for s in range(args.warmup):
            pool.map(run_reference_sample, [(args.workload, 1000 * s + c) for c in range(cores)])
        total, t_sum = 0.0, 0.0
        for s in range(args.steps):
            res = pool.map(run_reference_sample, [(args.workload, 1000 * (s + args.warmup) + c) for c in range(cores)])
            total += sum(a for a, _ in res)
            t_sum += max(t for _, t in res)  # the processes run side by side: the step lasts as long as the slowest
    v = total / t_sum / 1e9
    sample = (f"{cores} processes x ({rounds} rounds x {w['spr']} sweeps x {rungs} rungs x {n_sample} spins{where}) "
              f"per step; each process's round loop timed (dense model built once per process, initial energies "
              f"excluded), the slowest process per step")
    print(json.dumps({
        "impl": "reference", "metric": "spin-flips/ns", "value": v, "unit": "flips/ns", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_sum / args.steps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": w["desc"], "sample": sample},
        "cpu_baseline": {"value": v, "unit": "flips/ns", "cores": cores, "kind": "port",
                         "sample": "oracle/ref_pt.py (the reference CPU PT restated, same NumPy stream): " + sample},
        "e2e": {"value": v, "unit": "flips/ns", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def bench_reference_gpu(args):
    """The reference's own GPU engine (cuda/ising_pt.cu compiled unchanged for sm_100a into
    oracle/_ref by oracle/Makefile) on the workload's problem file, as drift/gpu.py runs it."""
    rank, world, local = dist_setup(args.gpus)
    if rank != 0:
        return
    import tempfile

    import oracle
    from drift_b200.problem_io import parse_stderr, read_result, write_problem

    w = WORKLOADS[args.workload]
    if not os.path.exists(oracle.REF_BIN) or args.workload not in ("maxcut3reg", "ea2d", "sk512"):
        why = "oracle/_ref/ising_pt not built" if not os.path.exists(oracle.REF_BIN) else \
            "the reference engine runs one instance of a CSR model (no batched or bit-packed input)"
        emit(args, {"impl": "reference-gpu", "unavailable": why})
        return
    model = make_model(args.workload)
    b = ladder(w)
    # the reference's per-attempt loop is O(degree); the dense SK model runs a shortened job
    rounds = args.rounds or (200 if args.workload == "sk512" else w["sweeps"] // w["spr"])
    vals, walls, bests = [], [], []
    with tempfile.TemporaryDirectory() as d:
        prob, res = os.path.join(d, "problem.bin"), os.path.join(d, "result.bin")
        for s_ in range(args.warmup + args.steps):
            write_problem(prob, model, n_replicas=w["R"], T_min=1.0 / b[-1], T_max=1.0 / b[0], n_rounds=rounds,
                          sweeps_per_round=w["spr"], seed=1000 + s_)
            t0 = time.perf_counter()
            r = subprocess.run([oracle.REF_BIN, prob, res], capture_output=True, text=True, timeout=1800)
            wall = time.perf_counter() - t0
            if r.returncode != 0:
                emit(args, {"impl": "reference-gpu", "unavailable": f"reference engine failed: {r.stderr[-300:]}"})
                return
            if s_ >= args.warmup:
                f = parse_stderr(r.stderr)
                vals.append(f["throughput"] / 1e9)
                walls.append(float(w["R"]) * rounds * w["spr"] * w["n"] / wall / 1e9)
                bests.append(read_result(res, w["n"])[0])
    emit(args, {
        "impl": "reference-gpu", "metric": "spin-flips/ns", "value": float(np.median(vals)), "unit": "flips/ns",
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "dtype": "f64 field, f32 spins",
        "data": "synthetic",
        "config": {"workload": w["desc"], "rounds": rounds, "sweeps_per_round": w["spr"],
                   "timer": "the reference's own (round loop, device-synchronised)"},
        "wall_clock_flips_per_ns": float(np.median(walls)), "best_energy": float(np.min(bests)),
        "binary": "oracle/_ref/ising_pt: cuda/ising_pt.cu compiled unchanged with -gencode arch=compute_100a,code=sm_100a",
    })


def cpu_baseline_oracle(w, model_name, budget_s=None):
    """The C oracle (OpenMP over replicas) on the host cores: a bounded number of rounds."""
    budget_s = CPU_BUDGET_S if budget_s is None else budget_s
    import oracle

    from drift_b200.engine import HostProblem

    hp = HostProblem.from_model(make_model(model_name))
    prob = oracle.OracleProblem(hp.n, hp.row_ptr, hp.col_idx, hp.weight, hp.h, hp.color_ptr, hp.color_spins)
    b = ladder(w)
    threads = os.cpu_count() or 1
    st = oracle.pt_run(prob, b, n_rounds=1, sweeps_per_round=w["spr"], seed=3, threads=threads)
    t0 = time.perf_counter()
    rounds = 0
    chunk = 2
    while time.perf_counter() - t0 < budget_s:
        st = oracle.pt_run(prob, b, n_rounds=chunk, sweeps_per_round=w["spr"], seed=3, threads=threads, state=st,
                           round_offset=1 + rounds)
        rounds += chunk
        chunk = min(chunk * 2, 64)
    dt = time.perf_counter() - t0
    attempts = rounds * w["spr"] * w["R"] * w["n"]
    return {"value": attempts / dt / 1e9, "unit": "flips/ns", "cores": threads, "kind": "port",
            "sample": f"oracle/pt_oracle.c, {rounds} rounds x {w['spr']} sweeps x {w['R']} replicas x {w['n']} spins "
                      f"({attempts:.3g} attempts, {dt:.1f} s), OpenMP over replicas"}


def bench_b200(args):
    import ctypes as C

    import torch

    from drift_b200 import _lib
    from drift_b200.engine import DeviceProblem, HostProblem, PtEngine

    rank, world, local = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    w = WORKLOADS[args.workload]
    model = make_model(args.workload)
    hp = HostProblem.from_model(model)
    prob = DeviceProblem(hp, device=dev)
    betas = ladder(w)
    rounds = args.rounds or w["sweeps"] // w["spr"]
    eng = PtEngine(prob, betas, seed=1, sweeps_per_round=w["spr"], instance=rank, item_form=args.item_form,
                   positions_per_item=args.positions_per_item)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)
    attempts_per_step = float(w["R"]) * rounds * w["spr"] * w["n"]

    def step(seed):
        eng.seed = seed
        eng.init()
        ev_k0.record()
        eng.run(rounds)
        ev_k1.record()

    ev_k0, ev_k1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for s in range(args.warmup):
        step(100 + s)
    eng.check()
    sampler = ClockSampler(local)
    sampler.start()
    barrier(world)
    torch.cuda.synchronize()
    t_steps, t_kernel = 0.0, 0.0
    for s in range(args.steps):
        flush.fill_(s & 0xFF)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        step(1000 + s)
        e1.record()
        e1.synchronize()
        t_steps += e0.elapsed_time(e1) * 1e-3
        t_kernel += ev_k0.elapsed_time(ev_k1) * 1e-3
    torch.cuda.synchronize()
    barrier(world)
    clocks = sampler.stop()
    eng.check()
    t_max = reduce_max(t_steps, world, dev)
    tk_max = reduce_max(t_kernel, world, dev)
    value = whole_job_rate(attempts_per_step, args.steps, world, t_max)

    # ---- end to end through the C ABI with host buffers ----
    L = _lib.load()
    p = lambda a: a.ctypes.data_as(C.c_void_p)
    best_s = np.zeros(hp.n, np.float32)
    bh = np.zeros(rounds)
    sa = _lib.SolveArgs(w["R"], rounds, w["spr"], 0, 7 + rank, 0.0, 0.0, p(betas))
    sr = _lib.SolveResult(0, 0, 0, 0, p(best_s), None, None, None, None, p(bh))
    csr = hp.c_csr()
    _lib.check(L.drift_pt_solve(C.byref(csr), C.byref(sa), C.byref(sr)), "drift_pt_solve")  # warm
    e2e_steps = max(1, min(args.steps, 5))
    barrier(world)
    t0 = time.perf_counter()
    solve_ms = []  # per call: wall time, and the device time of its kernel as the call reports it
    for _ in range(e2e_steps):
        t1 = time.perf_counter()
        _lib.check(L.drift_pt_solve(C.byref(csr), C.byref(sa), C.byref(sr)), "drift_pt_solve")
        solve_ms.append([round((time.perf_counter() - t1) * 1e3, 2), round(sr.seconds * 1e3, 2)])
    t_e2e = reduce_max(time.perf_counter() - t0, world, dev)
    e2e = attempts_per_step * e2e_steps * world / t_e2e / 1e9
    info = prob.info
    h2d = (hp.n + 1 + prob.info.n_colors + 1 + info.n_slices + 1) * 4 + info.n_ell * 5 + info.n_pos * 4 + w["R"] * 8 \
        + w["R"] * prob.max_field * 4
    d2h = w["R"] * 8 * 3 + (w["R"] - 1) * 16 + info.n_pos + rounds * 8

    if rank == 0:
        peak, peak_kind = load_peaks()
        launch_s = tk_max / args.steps
        alg_bytes = attempts_per_step * w["bytes_per_attempt"]
        achieved = alg_bytes / launch_s / 1e9
        traffic = load_traffic(f"pt_run_kernel/{args.workload}")
        issue = issue_basis(f"pt_run_kernel/{args.workload}", attempts_per_step / launch_s, clocks.get("sm_mhz"))
        line = {
            "metric": "spin-flips/ns", "value": value, "unit": "flips/ns", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_max / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int8", "data": "synthetic",
            "config": {"workload": w["desc"] + (f" [shortened to {rounds} rounds]" if args.rounds else ""),
                       "rounds": rounds, "sweeps_per_round": w["spr"],
                       "attempts_per_step": attempts_per_step, "parallelism": f"replicas-only x{world}",
                       "l2": "flushed between steps (256 MiB write)",
                       "launch": {"rpc": eng.rpc or "auto", "threads": eng.threads or "auto",
                                  "item_form": {0: "auto", 1: "gather", 2: "unit-regular"}[args.item_form]}},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                         "kernel": "pt_run_kernel", "bytes_per_attempt": w["bytes_per_attempt"],
                         "kernel_ms": launch_s * 1e3, **({"issue": issue} if issue else {})},
            "e2e": {"value": e2e, "unit": "flips/ns", "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                    "api": "drift_pt_solve (C ABI, host buffers)", "solve_wall_and_kernel_ms": solve_ms},
            "gpu_launches": 4 * args.steps,
            "clocks": clocks,
        }
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline_oracle(w, args.workload)
        if (world == 1 and args.workload == "maxcut3reg" and not args.no_secondary and not args.rounds
                and not getattr(args, "sweeps_per_round", 0)):
            line["secondary"] = secondaries(args)
        emit(args, line)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


# The other benchmark workloads measured alongside the default line: (key, workload, overrides).
SECONDARIES = [
    ("ea2d_C1", "ea2d", {}),
    ("batched_er_C3", "batched_er", {}),
    ("sk512_C4", "sk512", {"ttt": True, "ttt_seeds": 3}),
    ("ea3d64_C5", "ea3d64", {}),
    ("ea2d_batch256_C5b", "ea2d_batch256", {}),
    ("maxcut3reg_r2048", "maxcut3reg_r2048", {}),
    ("made_train_C4_network", "made_train", {}),
]
# the reference's own GPU engine (cuda/ising_pt.cu built unchanged into oracle/_ref) on shortened jobs
REFERENCE_GPU = [("maxcut3reg_C2", "maxcut3reg", 2500), ("ea2d_C1", "ea2d", 20000)]


def secondaries(args) -> dict:
    """Run the other workloads with 3 warm-up and 3 timed steps each and collect their lines; then the
    reference GPU engine on C2 and C1. Each entry is that workload's own line (or an error)."""
    import copy

    global CPU_BUDGET_S
    saved_budget, CPU_BUDGET_S = CPU_BUDGET_S, 4.0
    out = {}
    for key, workload, over in SECONDARIES:
        a = copy.copy(args)
        a.workload, a.steps, a.warmup, a.rounds, a.sink = workload, 3, 3, 0, []
        a.item_form, a.positions_per_item, a.ttt = 0, 0, False
        for k, v in over.items():
            setattr(a, k, v)
        try:
            t0 = time.perf_counter()
            run_workload(a)
            out[key] = a.sink[-1] if a.sink else {"error": "no line"}
            out[key]["wall_s"] = time.perf_counter() - t0
        except Exception as e:  # noqa: BLE001 - a failing secondary must not lose the headline
            out[key] = {"error": f"{type(e).__name__}: {e}"[:300]}
    for key, workload, rounds in REFERENCE_GPU:
        a = copy.copy(args)
        a.workload, a.steps, a.warmup, a.rounds, a.sink = workload, 1, 1, rounds, []
        try:
            bench_reference_gpu(a)
            out["reference_gpu_" + key] = a.sink[-1] if a.sink else {"error": "no line"}
        except Exception as e:  # noqa: BLE001
            out["reference_gpu_" + key] = {"error": f"{type(e).__name__}: {e}"[:300]}
    CPU_BUDGET_S = saved_budget
    return out


def load_tensor_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d.get("bf16_tflops_sustained", d.get("bf16_tflops"))), "measured (bf16 sustained)"
    return 1400.0, "fallback (bf16 sustained)"


def cpu_baseline_sk(w, sk, budget_s=None):
    """The C oracle of the dense chain (OpenMP over replicas) on the host cores, bounded."""
    budget_s = CPU_BUDGET_S if budget_s is None else budget_s
    import oracle

    b = ladder(w)
    sc = sk.scales(b)
    threads = os.cpu_count() or 1
    st = oracle.sk_run(sk.Jq, sk.hq, sk.shift, b, sc, n_rounds=1, sweeps_per_round=1, seed=3, threads=threads)
    t0 = time.perf_counter()
    rounds = 0
    while time.perf_counter() - t0 < budget_s:
        st = oracle.sk_run(sk.Jq, sk.hq, sk.shift, b, sc, n_rounds=1, sweeps_per_round=w["spr"], seed=3,
                           threads=threads, state=st, round_offset=1 + rounds)
        rounds += 1
    dt = time.perf_counter() - t0
    attempts = rounds * w["spr"] * w["R"] * w["n"]
    return {"value": attempts / dt / 1e9, "unit": "flips/ns", "cores": threads, "kind": "port",
            "sample": f"oracle/sk_oracle.c, {rounds} rounds x {w['spr']} sweeps x {w['R']} replicas x {w['n']} spins "
                      f"({attempts:.3g} attempts, {dt:.1f} s), OpenMP over replicas"}


def bench_sk(args):
    import torch

    from drift_b200.sk import SkEngine, SkModel

    rank, world, local = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    w = WORKLOADS[args.workload]
    model = make_model(args.workload)
    sk = SkModel.from_model(model)
    betas = ladder(w)
    rounds = args.rounds or w["sweeps"] // w["spr"]
    eng = SkEngine(sk, betas, seed=1, sweeps_per_round=w["spr"], instance=rank, replicas_per_cta=args.sk_g,
                   device=dev)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)
    attempts_per_step = float(w["R"]) * rounds * w["spr"] * w["n"]
    ev_k0, ev_k1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def step(seed):
        eng.seed = seed
        eng.init()
        ev_k0.record()
        eng.run(rounds)
        ev_k1.record()

    for s_ in range(args.warmup):
        step(100 + s_)
    eng.check()
    sampler = ClockSampler(local)
    sampler.start()
    barrier(world)
    torch.cuda.synchronize()
    t_steps, t_kernel = 0.0, 0.0
    for s_ in range(args.steps):
        flush.fill_(s_ & 0xFF)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        step(1000 + s_)
        e1.record()
        e1.synchronize()
        t_steps += e0.elapsed_time(e1) * 1e-3
        t_kernel += ev_k0.elapsed_time(ev_k1) * 1e-3
    torch.cuda.synchronize()
    barrier(world)
    clocks = sampler.stop()
    eng.check()
    best = eng.fetch()["best_energy"].min() * sk.energy_unit
    t_max = reduce_max(t_steps, world, dev)
    tk_max = reduce_max(t_kernel, world, dev)
    value = whole_job_rate(attempts_per_step, args.steps, world, t_max)
    # end to end through the public Python API: quantisation and coupling table on the host, upload,
    # initialisation, the rounds, results downloaded
    e2e_steps = max(1, min(args.steps, 3))
    barrier(world)
    t0 = time.perf_counter()
    h2d = d2h = 0
    for k in range(e2e_steps):
        sk2 = SkModel.from_model(model)
        e2 = SkEngine(sk2, betas, seed=7 + k, sweeps_per_round=w["spr"], instance=rank, replicas_per_cta=args.sk_g,
                      device=dev)
        e2.init()
        e2.run(rounds)
        out = e2.fetch()
        h2d = sk2.Jq.nbytes + sk2.hq.nbytes + sk2.layout.nbytes + betas.nbytes + 4 * len(betas)
        d2h = sum(v.nbytes for v in out.values() if isinstance(v, np.ndarray))
    t_e2e = reduce_max(time.perf_counter() - t0, world, dev)
    if rank == 0:
        peak, peak_kind = load_tensor_peak()
        launch_s = tk_max / args.steps
        achieved = attempts_per_step * w["flops_per_attempt"] / launch_s / 1e12
        line = {
            "metric": "spin-flips/ns", "value": value, "unit": "flips/ns", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_max / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32 (int8 tensor-core limbs)", "data": "synthetic",
            "config": {"workload": w["desc"] + (f" [shortened to {rounds} rounds]" if args.rounds else ""),
                       "rounds": rounds, "sweeps_per_round": w["spr"], "attempts_per_step": attempts_per_step,
                       "parallelism": f"replicas-only x{world}", "l2": "flushed between steps (256 MiB write)",
                       "replicas_per_cta": eng.replicas_per_cta or "auto", "shift": sk.shift,
                       "best_energy_last_step": float(best)},
            "roofline": {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                         "frac": achieved / peak, "traffic": load_traffic("sk_run_kernel/sk512"), "peak_kind": peak_kind,
                         "kernel": "sk_run_kernel",
                         "flops_per_attempt": w["flops_per_attempt"], "kernel_ms": launch_s * 1e3,
                         "note": "sequential Metropolis chain: latency of the per-spin decision bounds the kernel"},
            "e2e": {"value": attempts_per_step * e2e_steps * world / t_e2e / 1e9, "unit": "flips/ns",
                    "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                    "api": "SkModel + SkEngine (Python over the C ABI), host J in, results out"},
            "gpu_launches": 2 * args.steps,
            "clocks": clocks,
        }
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline_sk(w, sk)
        if args.ttt:
            line["time_to_target"] = time_to_target(w, sk, args, dev)
        emit(args, line)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


def cpu_baseline_ms(w, lat, budget_s=None):
    """The multispin oracle (one replica bit at a time) on a bounded number of sweeps."""
    budget_s = CPU_BUDGET_S if budget_s is None else budget_s
    import oracle

    b = ladder(w)
    t0 = time.perf_counter()
    st = oracle.ms_run(3, w["L"], lat.jneg, b, n_rounds=1, sweeps_per_round=1, seed=3)
    sweeps = 1
    while time.perf_counter() - t0 < budget_s:
        st = oracle.ms_run(3, w["L"], lat.jneg, b, n_rounds=1, sweeps_per_round=1, seed=3, state=st,
                           round_offset=sweeps)
        sweeps += 1
    dt = time.perf_counter() - t0
    attempts = sweeps * w["R"] * w["n"]
    return {"value": attempts / dt / 1e9, "unit": "flips/ns", "cores": 1, "kind": "port",
            "sample": f"oracle/ms_oracle.c (scalar, one replica bit at a time), {sweeps} sweeps x {w['R']} replicas x "
                      f"{w['n']} sites incl. initialisation ({attempts:.3g} attempts, {dt:.1f} s)"}


def bench_ms(args):
    import torch

    from drift_b200.multispin import Lattice, MsEngine

    rank, world, local = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    w = WORKLOADS[args.workload]
    lat = Lattice.edwards_anderson(3, w["L"], w["seed"])
    betas = ladder(w)
    rounds = args.rounds or w["sweeps"] // w["spr"]
    eng = MsEngine(lat, betas, seed=1, sweeps_per_round=w["spr"], instance=rank, device=dev)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)
    attempts_per_step = float(w["R"]) * rounds * w["spr"] * w["n"]
    ev_k0, ev_k1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def step(seed):
        eng.seed = seed
        eng.init()
        ev_k0.record()
        eng.run(rounds)
        ev_k1.record()

    for s_ in range(args.warmup):
        step(100 + s_)
    eng.check()
    sampler = ClockSampler(local)
    sampler.start()
    barrier(world)
    torch.cuda.synchronize()
    t_steps, t_kernel = 0.0, 0.0
    for s_ in range(args.steps):
        flush.fill_(s_ & 0xFF)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        step(1000 + s_)
        e1.record()
        e1.synchronize()
        t_steps += e0.elapsed_time(e1) * 1e-3
        t_kernel += ev_k0.elapsed_time(ev_k1) * 1e-3
    torch.cuda.synchronize()
    barrier(world)
    clocks = sampler.stop()
    eng.check()
    t_max = reduce_max(t_steps, world, dev)
    tk_max = reduce_max(t_kernel, world, dev)
    value = whole_job_rate(attempts_per_step, args.steps, world, t_max)
    # end to end through the public Python API: couplings built on the host, uploaded, init, rounds,
    # energies downloaded
    e2e_steps = max(1, min(args.steps, 3))
    barrier(world)
    t0 = time.perf_counter()
    for k in range(e2e_steps):
        lat2 = Lattice.edwards_anderson(3, w["L"], w["seed"])
        e2 = MsEngine(lat2, betas, seed=7 + k, sweeps_per_round=w["spr"], instance=rank, device=dev)
        e2.init()
        e2.run(rounds)
        energies = e2.best_energy.cpu().numpy()
    t_e2e = reduce_max(time.perf_counter() - t0, world, dev)
    if rank == 0:
        peak, peak_kind = load_peaks()
        launch_s = tk_max / args.steps
        achieved = attempts_per_step * w["bytes_per_attempt"] / launch_s / 1e9
        line = {
            "metric": "spin-flips/ns", "value": value, "unit": "flips/ns", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_max / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u32 (1 bit per spin)", "data": "synthetic",
            "config": {"workload": w["desc"] + (f" [shortened to {rounds} rounds]" if args.rounds else ""),
                       "rounds": rounds, "sweeps_per_round": w["spr"], "attempts_per_step": attempts_per_step,
                       "parallelism": f"replicas-only x{world}", "l2": "flushed between steps (256 MiB write)",
                       "best_energy_per_spin": float(energies.min()) / w["n"]},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": load_traffic("ms_run_kernel/ea3d64"), "peak_kind": peak_kind,
                         "kernel": "ms_run_kernel", "bytes_per_attempt": w["bytes_per_attempt"],
                         "kernel_ms": launch_s * 1e3,
                         "note": "4 MiB of packed spins stay in L2: the HBM line is not the binding one"},
            "e2e": {"value": attempts_per_step * e2e_steps * world / t_e2e / 1e9, "unit": "flips/ns",
                    "h2d_bytes_per_step": int(lat.jneg.nbytes + betas.nbytes + 4 * w["R"] * 6),
                    "d2h_bytes_per_step": int(8 * w["R"]), "api": "Lattice + MsEngine (Python over the C ABI)"},
            "gpu_launches": 2 * args.steps,
            "clocks": clocks,
        }
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline_ms(w, lat)
        emit(args, line)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


def cpu_baseline_gms(w, lay, budget_s=None):
    """The graph multispin oracle (scalar, one replica bit at a time) on a bounded number of rounds."""
    budget_s = CPU_BUDGET_S if budget_s is None else budget_s
    import oracle

    b = ladder(w)
    t0 = time.perf_counter()
    st = oracle.gms_run(lay, b, n_rounds=1, sweeps_per_round=1, seed=3)
    sweeps = 1
    while time.perf_counter() - t0 < budget_s:
        st = oracle.gms_run(lay, b, n_rounds=1, sweeps_per_round=1, seed=3, state=st, round_offset=sweeps)
        sweeps += 1
    dt = time.perf_counter() - t0
    attempts = sweeps * w["R"] * w["n"]
    return {"value": attempts / dt / 1e9, "unit": "flips/ns", "cores": 1, "kind": "port",
            "sample": f"oracle/gms_oracle.c (scalar, one replica bit at a time), {sweeps} sweeps x {w['R']} replicas x "
                      f"{w['n']} spins incl. initialisation ({attempts:.3g} attempts, {dt:.1f} s)"}


def bench_gms(args):
    import torch

    from drift_b200.gms import GmsEngine, GmsLayout
    from drift_b200.instances import maxcut_3regular

    rank, world, local = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    w = WORKLOADS[args.workload]
    model = maxcut_3regular(w["n"], w["seed"])
    lay = GmsLayout.from_model(model)
    betas = ladder(w)
    rounds = args.rounds or w["sweeps"] // w["spr"]
    eng = GmsEngine(lay, betas, seed=1, sweeps_per_round=w["spr"], instance=rank, device=dev)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)
    attempts_per_step = float(w["R"]) * rounds * w["spr"] * w["n"]
    ev_k0, ev_k1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def step(seed):
        eng.seed = seed
        eng.init()
        ev_k0.record()
        eng.run(rounds)
        ev_k1.record()

    for s_ in range(args.warmup):
        step(100 + s_)
    eng.check()
    sampler = ClockSampler(local)
    sampler.start()
    barrier(world)
    torch.cuda.synchronize()
    t_steps, t_kernel = 0.0, 0.0
    for s_ in range(args.steps):
        flush.fill_(s_ & 0xFF)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        step(1000 + s_)
        e1.record()
        e1.synchronize()
        t_steps += e0.elapsed_time(e1) * 1e-3
        t_kernel += ev_k0.elapsed_time(ev_k1) * 1e-3
    torch.cuda.synchronize()
    barrier(world)
    clocks = sampler.stop()
    eng.check()
    t_max = reduce_max(t_steps, world, dev)
    tk_max = reduce_max(t_kernel, world, dev)
    value = whole_job_rate(attempts_per_step, args.steps, world, t_max)
    # end to end through the public Python API: layout built on the host from the model, uploaded,
    # init, rounds, best energies downloaded
    e2e_steps = max(1, min(args.steps, 3))
    barrier(world)
    t0 = time.perf_counter()
    for k in range(e2e_steps):
        lay2 = GmsLayout.from_model(model)
        e2 = GmsEngine(lay2, betas, seed=7 + k, sweeps_per_round=w["spr"], instance=rank, device=dev)
        e2.init()
        e2.run(rounds)
        energies = e2.best_energy.cpu().numpy()
    t_e2e = reduce_max(time.perf_counter() - t0, world, dev)
    if rank == 0:
        peak, peak_kind = load_peaks()
        launch_s = tk_max / args.steps
        achieved = attempts_per_step * w["bytes_per_attempt"] / launch_s / 1e9
        h2d = lay.color_ptr.nbytes + lay.ell_nbr.nbytes + lay.degree.nbytes + lay.jneg.nbytes + betas.nbytes
        # the engine's automatic shape: one CTA per word from 16 words up, else a cluster of CTAs per word
        kname = "gms_run_kernel" if w["R"] // 32 >= 16 else "gmc_run_kernel"
        line = {
            "metric": "spin-flips/ns", "value": value, "unit": "flips/ns", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_max / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u32 (1 bit per spin)", "data": "synthetic",
            "config": {"workload": w["desc"] + (f" [shortened to {rounds} rounds]" if args.rounds else ""),
                       "rounds": rounds, "sweeps_per_round": w["spr"], "attempts_per_step": attempts_per_step,
                       "parallelism": f"replicas-only x{world}", "l2": "flushed between steps (256 MiB write)",
                       "engine": "graph multispin (drift_pt_gms_run)",
                       "best_energy_per_spin": float(energies.min()) / w["n"]},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": load_traffic(f"{kname}/{args.workload}"), "peak_kind": peak_kind,
                         "kernel": kname, "bytes_per_attempt": w["bytes_per_attempt"],
                         "kernel_ms": launch_s * 1e3,
                         "note": "the packed words live in shared memory for the whole launch: the HBM line is "
                                 "not the binding one (the phases are latency-bound)"},
            "e2e": {"value": attempts_per_step * e2e_steps * world / t_e2e / 1e9, "unit": "flips/ns",
                    "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(8 * w["R"]),
                    "api": "GmsLayout + GmsEngine (Python over the C ABI)"},
            "gpu_launches": 2 * args.steps,
            "clocks": clocks,
        }
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline_gms(w, lay)
        emit(args, line)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


def time_to_target(w, sk, args, dev):
    """Wall time for plain PT and for neural-proposal PT (sample collection and training included)
    to reach the best energy of a long plain-PT run, within 1e-6 relative; a few seeds, bounded."""
    import torch

    from drift_b200.made import Made
    from drift_b200.neural import NeuralPT, collect_cold_samples
    from drift_b200.sk import SkEngine

    betas = ladder(w)
    unit = sk.energy_unit
    spr, chunk = w["spr"], 50
    ref = SkEngine(sk, betas, seed=100, sweeps_per_round=spr, replicas_per_cta=args.sk_g, device=dev)
    ref.init()
    ref.run(args.ttt_ref_sweeps // spr)
    ref.check()
    target = float(ref.best_energy.min().item()) * unit
    goal = target + 1e-6 * abs(target)

    def reached(eng):
        return float(eng.best_energy.min().item()) * unit <= goal

    out = {"target_energy": target, "target_from": f"plain PT, seed 100, {args.ttt_ref_sweeps} sweeps",
           "cap_s": args.ttt_cap_s, "plain": [], "neural": []}
    for seed in range(1, args.ttt_seeds + 1):
        eng = SkEngine(sk, betas, seed=seed, sweeps_per_round=spr, replicas_per_cta=args.sk_g, device=dev)
        eng.init()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        sweeps = 0
        while not reached(eng) and time.perf_counter() - t0 < args.ttt_cap_s:
            eng.run(chunk)
            sweeps += chunk * spr
        dt = time.perf_counter() - t0
        out["plain"].append({"seed": seed, "seconds": dt, "sweeps": sweeps, "reached": reached(eng)})
        # neural: the same start. Plain rounds collect the training set from the 8 coldest rungs;
        # the network then trains on a second stream while plain PT goes on in the first (the dense
        # kernel holds 32 of the 148 SMs), and proposals start when training is done
        eng = SkEngine(sk, betas, seed=seed, sweeps_per_round=spr, replicas_per_cta=args.sk_g, device=dev)
        eng.init()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        data = collect_cold_samples(eng, args.ttt_samples, n_cold=8)
        t_collect = time.perf_counter() - t0
        made = Made(w["n"], (1024, 1024), seed=seed, device=dev)
        main, side = torch.cuda.current_stream(), torch.cuda.Stream(device=dev)
        side.wait_stream(main)
        steps_done, slice_steps = 0, 8
        while steps_done < args.ttt_train_steps and not reached(eng) and time.perf_counter() - t0 < args.ttt_cap_s:
            eng.run(chunk // 10)
            with torch.cuda.stream(side):
                k = min(slice_steps, args.ttt_train_steps - steps_done)
                made.train_async(data, steps=k, batch=args.ttt_batch_size, lr=args.ttt_lr, seed=1000 * seed + steps_done)
            steps_done += k
        trained = torch.cuda.Event()
        trained.record(side)
        while not trained.query() and not reached(eng) and time.perf_counter() - t0 < args.ttt_cap_s:
            eng.run(chunk // 10)
        main.wait_stream(side)
        t_train = time.perf_counter() - t0 - t_collect
        npt = NeuralPT(sk, betas, made, n_cold=8, engine=eng, suffix=args.ttt_suffix or None)
        rounds = 0
        while not reached(eng) and time.perf_counter() - t0 < args.ttt_cap_s:
            npt.run(chunk // 10)
            rounds += chunk // 10
        dt = time.perf_counter() - t0
        acc = npt.acceptance()[-8:]
        out["neural"].append({"seed": seed, "seconds": dt, "reached": reached(eng), "collect_s": t_collect,
                              "train_s_overlapped_with_plain_pt": t_train, "train_steps": steps_done,
                              "proposal_rounds": rounds,
                              "proposal_acceptance_cold8": float(np.nanmean(acc)) if np.isfinite(acc).any() else None})
        if seed == 1:
            # acceptance at the 8 coldest rungs against the number of spins a proposal redraws (the last m
            # in the network's order; m = n is an independent whole configuration), from the state reached
            sweep_acc = {}
            for m in (4, 8, 16, 32, 64, 128, w["n"]):
                probe = NeuralPT(sk, betas, made, n_cold=8, engine=eng, suffix=None if m == w["n"] else m)
                t1 = time.perf_counter()
                probe.run(40)
                torch.cuda.synchronize()
                a8 = probe.acceptance()[-8:]
                sweep_acc[str(m)] = {"acceptance_cold8": float(np.nanmean(a8)) if np.isfinite(a8).any() else None,
                                     "ms_per_round": (time.perf_counter() - t1) / 40 * 1e3}
            out["acceptance_vs_redrawn_spins"] = sweep_acc
    for k in ("plain", "neural"):
        ts = [r["seconds"] for r in out[k]]
        out[k + "_median_s"] = float(np.median(ts))
    out["speedup_neural_over_plain"] = out["plain_median_s"] / out["neural_median_s"]
    return out


def bench_batched(args):
    import torch

    from drift_b200.batch import BatchEngine, BatchProblem, autotune
    from drift_b200.engine import HostProblem

    rank, world, local = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    w = WORKLOADS[args.workload]
    t_build0 = time.perf_counter()
    models = make_batch_models(w)
    hps = [HostProblem.from_model(m, order="degree") for m in models]
    ladders = [ladder(w)] * len(hps)
    bp = BatchProblem(hps, ladders, stream_ids=np.arange(len(hps)) + 1024 * rank, device=dev)
    t_build = time.perf_counter() - t_build0
    rounds = args.rounds or w["sweeps"] // w["spr"]
    eng = BatchEngine(bp, seed=1, sweeps_per_round=w["spr"])
    eng.init()
    shape = autotune(eng, rounds=2)
    total_n = int(sum(int(d["n"]) for d in bp.desc))
    attempts_per_step = float(w["R"]) * total_n * rounds * w["spr"]
    # the timed step is one replay of a job captured whole as a CUDA graph (BatchEngine.capture_job:
    # initialisation and the step's rounds, in 10 launches)
    job = eng.capture_job(rounds, max(1, rounds // 10))
    g = job.graph
    for _ in range(args.warmup):
        job.replay()
    eng.check()
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)
    sampler = ClockSampler(local)
    sampler.start()
    barrier(world)
    torch.cuda.synchronize()
    t_steps = 0.0
    for s_ in range(args.steps):
        flush.fill_(s_ & 0xFF)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        g.replay()
        e1.record()
        e1.synchronize()
        t_steps += e0.elapsed_time(e1) * 1e-3
    torch.cuda.synchronize()
    barrier(world)
    clocks = sampler.stop()
    eng.check()
    t_max = reduce_max(t_steps, world, dev)
    value = whole_job_rate(attempts_per_step, args.steps, world, t_max)
    # end to end through the public Python API: layouts and state uploaded from host, run, best
    # energies downloaded
    t0 = time.perf_counter()
    bp2 = BatchProblem(hps, ladders, stream_ids=np.arange(len(hps)) + 1024 * rank, device=dev)
    e2 = BatchEngine(bp2, seed=2, sweeps_per_round=w["spr"], **shape)
    e2.init()
    e2.run(rounds)
    best = e2.best_energies()
    t_e2e = reduce_max(time.perf_counter() - t0, world, dev)
    if rank == 0:
        peak, peak_kind = load_peaks()
        achieved = attempts_per_step * w["bytes_per_attempt"] / (t_max / args.steps) / 1e9
        h2d = int(sum(t.numel() * t.element_size() for t in (bp2.d_desc, bp2.d_color_ptr, bp2.d_slice_off,
                                                             bp2.d_ell_nbr, bp2.d_ell_w, bp2.d_h_pos, bp2.d_betas)))
        line = {
            "metric": "spin-flips/ns", "value": value, "unit": "flips/ns", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_max / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": w["desc"], "instances": len(hps), "total_spins": total_n, "rounds": rounds,
                       "sweeps_per_round": w["spr"], "attempts_per_step": attempts_per_step,
                       "parallelism": f"replicas-only x{world}", "l2": "flushed between steps (256 MiB write)",
                       "launch": shape, "cuda_graph": True, "host_build_s": t_build},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": load_traffic("pt_batched_kernel/batched_er"), "peak_kind": peak_kind,
                         "kernel": "pt_batched_kernel", "bytes_per_attempt": w["bytes_per_attempt"]},
            "e2e": {"value": attempts_per_step * world / t_e2e / 1e9, "unit": "flips/ns", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": int(bp2.total_slots * 8), "api": "BatchProblem + BatchEngine (Python)",
                    "best_energy_mean": float(np.mean(best))},
            # per replay: the job's sweep launches and drift_pt_batch_init's three kernels per instance
            "gpu_launches": (job.launches + 3 * bp.n_instances) * args.steps,
            "clocks": clocks,
        }
        emit(args, line)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


def ttt_batch(w, bp, hps, args, dev):
    """Time for every instance of the batch to reach the best energy of a 10x longer plain run:
    plain batched PT vs the same with neural proposals (sample collection, network construction
    and training inside the clock). Per instance the first time its best reaches its target is
    kept; the batch's time is the last of them (None when the cap came first)."""
    import torch

    from drift_b200.batch import BatchEngine
    from drift_b200.batch_neural import BatchNeuralPT, make_nets

    spr, chunk = w["spr"], 10
    K = bp.n_instances
    ref = BatchEngine(bp, seed=100, sweeps_per_round=spr)
    ref.init()
    t_ref0 = time.perf_counter()
    ref_rounds = args.ttt_ref_sweeps // spr
    done = 0
    while done < ref_rounds:
        ref.run(min(500, ref_rounds - done))
        done += min(500, ref_rounds - done)
    ref.check()
    target = ref.best_energies()
    t_ref = time.perf_counter() - t_ref0
    sizes = np.array([int(d["n"]) for d in bp.desc])

    def track(step, eng, cap):
        t0 = time.perf_counter()
        first = np.full(K, np.nan)
        while time.perf_counter() - t0 < cap:
            step()
            hit = eng.best_energies() <= target
            now = time.perf_counter() - t0
            first[np.isnan(first) & hit] = now
            if not np.isnan(first).any():
                break
        return first

    def summary(first, extra=None):
        ok = ~np.isnan(first)
        small = sizes <= 512
        r = {"all_reached_s": float(first.max()) if ok.all() else None, "fraction_reached": float(ok.mean()),
             "median_instance_s": float(np.median(first[ok])) if ok.any() else None,
             "median_instance_s_n_le_512": float(np.median(first[ok & small])) if (ok & small).any() else None,
             "reached_n_le_512": float(ok[small].mean())}
        r.update(extra or {})
        return r

    out = {"target_from": f"plain batched PT, seed 100, {args.ttt_ref_sweeps} sweeps ({t_ref:.1f} s)",
           "cap_s": args.ttt_cap_s, "networks": int((sizes <= 512).sum()), "plain": [], "neural": []}
    for seed in range(1, args.ttt_seeds + 1):
        eng = BatchEngine(bp, seed=seed, sweeps_per_round=spr)
        eng.init()
        torch.cuda.synchronize()
        first = track(lambda: eng.run(chunk), eng, args.ttt_cap_s)
        out["plain"].append(summary(first, {"seed": seed}))
        eng = BatchEngine(bp, seed=seed, sweeps_per_round=spr)
        eng.init()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        nets = make_nets(bp, seed=seed)
        bn = BatchNeuralPT(eng, nets, n_cold=8)
        data = bn.collect(args.ttt_batch_rounds)
        t_collect = time.perf_counter() - t0
        for k, m in nets.items():
            m.train(data[k], epochs=args.ttt_epochs, batch=args.ttt_batch_size, lr=args.ttt_lr)
        torch.cuda.synchronize()
        t_train = time.perf_counter() - t0 - t_collect
        every = max(1, min(chunk, args.ttt_propose_every))

        def neural_step():
            # chunk rounds, a proposal after every `every`-th
            for r in range(chunk):
                if (r + 1) % every == 0:
                    bn.run(1)
                else:
                    eng.run(1)
        # instances that reached their target during collection count at its end (an upper bound)
        reached_early = eng.best_energies() <= target
        first = track(neural_step, eng, args.ttt_cap_s - t_collect - t_train) + (t_collect + t_train)
        first[reached_early] = t_collect
        acc = bn.acceptance()
        out["neural"].append(summary(first, {"seed": seed, "collect_s": t_collect, "train_s": t_train,
                                             "propose_every_rounds": every, "epochs": args.ttt_epochs,
                                             "lr": args.ttt_lr, "train_samples_per_net": 8 * args.ttt_batch_rounds,
                                             "proposal_acceptance_mean": float(np.nanmean(list(acc.values()))),
                                             "proposal_acceptance_max": float(np.nanmax(list(acc.values())))}))
    for k in ("plain", "neural"):
        v = [r["all_reached_s"] for r in out[k]]
        out[k + "_all_reached_median_s"] = float(np.median(v)) if all(x is not None for x in v) else None
    if out["plain_all_reached_median_s"] and out["neural_all_reached_median_s"]:
        out["speedup_neural_over_plain"] = out["plain_all_reached_median_s"] / out["neural_all_reached_median_s"]
    return out


def bench_ea2d_batch(args):
    import torch

    from drift_b200.batch import BatchEngine, BatchProblem, autotune
    from drift_b200.engine import HostProblem
    from drift_b200.instances import ea2d_batch

    rank, world, local = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    w = WORKLOADS[args.workload]
    models = ea2d_batch(w["n_instances"], w["seed"])
    hps = [HostProblem.from_model(m) for m in models]
    ladders = [ladder(w)] * len(hps)
    bp = BatchProblem(hps, ladders, stream_ids=np.arange(len(hps)) + 1024 * rank, device=dev)
    rounds = args.rounds or w["sweeps"] // w["spr"]
    eng = BatchEngine(bp, seed=1, sweeps_per_round=w["spr"])
    eng.init()
    shape = autotune(eng, rounds=2)
    total_n = int(sum(int(d["n"]) for d in bp.desc))
    attempts_per_step = float(w["R"]) * total_n * rounds * w["spr"]
    for _ in range(args.warmup):
        eng.run(rounds)
    eng.check()
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)
    sampler = ClockSampler(local)
    sampler.start()
    barrier(world)
    torch.cuda.synchronize()
    t_steps = 0.0
    for s_ in range(args.steps):
        flush.fill_(s_ & 0xFF)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        eng.run(rounds)
        e1.record()
        e1.synchronize()
        t_steps += e0.elapsed_time(e1) * 1e-3
    torch.cuda.synchronize()
    barrier(world)
    clocks = sampler.stop()
    eng.check()
    t_max = reduce_max(t_steps, world, dev)
    value = whole_job_rate(attempts_per_step, args.steps, world, t_max)
    t0 = time.perf_counter()
    bp2 = BatchProblem(hps, ladders, stream_ids=np.arange(len(hps)) + 1024 * rank, device=dev)
    e2 = BatchEngine(bp2, seed=2, sweeps_per_round=w["spr"], **shape)
    e2.init()
    e2.run(rounds)
    best = e2.best_energies()
    t_e2e = reduce_max(time.perf_counter() - t0, world, dev)
    if rank == 0:
        peak, peak_kind = load_peaks()
        achieved = attempts_per_step * w["bytes_per_attempt"] / (t_max / args.steps) / 1e9
        h2d = int(sum(t.numel() * t.element_size() for t in (bp2.d_desc, bp2.d_color_ptr, bp2.d_slice_off,
                                                             bp2.d_ell_nbr, bp2.d_ell_w, bp2.d_h_pos, bp2.d_betas)))
        line = {
            "metric": "spin-flips/ns", "value": value, "unit": "flips/ns", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_max / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int8", "data": "synthetic",
            "config": {"workload": w["desc"], "instances": len(hps), "total_spins": total_n, "rounds": rounds,
                       "sweeps_per_round": w["spr"], "attempts_per_step": attempts_per_step,
                       "parallelism": f"replicas-only x{world}", "l2": "flushed between steps (256 MiB write)",
                       "launch": shape},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": load_traffic("pt_batched_kernel/ea2d_batch256"), "peak_kind": peak_kind,
                         "kernel": "pt_batched_kernel",
                         "bytes_per_attempt": w["bytes_per_attempt"]},
            "e2e": {"value": attempts_per_step * world / t_e2e / 1e9, "unit": "flips/ns", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": int(bp2.total_slots * 8), "api": "BatchProblem + BatchEngine (Python)",
                    "best_energy_mean": float(np.mean(best))},
            "gpu_launches": args.steps,
            "clocks": clocks,
        }
        if args.ttt and world == 1:
            line["time_to_target"] = ttt_batch(w, bp, hps, args, dev)
        emit(args, line)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference", "reference-gpu"])
    ap.add_argument("--workload", default="maxcut3reg", choices=list(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--sk-g", type=int, default=2, help="dense workload: replicas per CTA (1..12)")
    ap.add_argument("--ttt", action="store_true", help="dense workload: add time-to-target, neural vs plain PT")
    ap.add_argument("--ttt-seeds", type=int, default=3)
    ap.add_argument("--ttt-cap-s", type=float, default=20.0)
    ap.add_argument("--ttt-ref-sweeps", type=int, default=100000)
    ap.add_argument("--ttt-samples", type=int, default=8192, help="neural PT (dense): training configurations")
    ap.add_argument("--ttt-epochs", type=int, default=5)
    ap.add_argument("--ttt-lr", type=float, default=1e-3, help="neural PT: Adam learning rate")
    ap.add_argument("--ttt-batch-size", type=int, default=512, help="neural PT: training batch")
    ap.add_argument("--ttt-train-steps", type=int, default=600, help="neural PT (dense): Adam steps")
    ap.add_argument("--ttt-suffix", type=int, default=0,
                    help="neural PT (dense): redraw the last m spins per proposal (0 = whole configurations)")
    ap.add_argument("--ttt-propose-every", type=int, default=1,
                    help="batched neural PT: rounds between proposals (1 = after every round)")
    ap.add_argument("--ttt-batch-rounds", type=int, default=256,
                    help="batched neural PT: plain rounds that collect each network's training set (8 per round)")
    ap.add_argument("--item-form", type=int, default=0, choices=[0, 1, 2],
                    help="sparse workloads: 0 = the engine's choice, 1 = sliced-ELL gather, 2 = unit-regular form")
    ap.add_argument("--positions-per-item", type=int, default=0, choices=[0, 1, 2, 4, 8],
                    help="sparse workloads: positions per item (0 = the engine's choice)")
    ap.add_argument("--rounds", type=int, default=0,
                    help="override the rounds per step (profiling of a short case; the line then says so)")
    ap.add_argument("--no-secondary", action="store_true",
                    help="default workload: skip the other workloads' lines (the 'secondary' object)")
    ap.add_argument("--sweeps-per-round", type=int, default=0,
                    help="sparse workloads: override the sweeps per round (same sweeps per job; the line then says so)")
    args = ap.parse_args()
    if args.sweeps_per_round:
        w = WORKLOADS[args.workload]
        if args.workload not in ("maxcut3reg", "ea2d"):
            ap.error("--sweeps-per-round applies to the maxcut3reg and ea2d workloads")
        WORKLOADS[args.workload] = dict(w, spr=args.sweeps_per_round,
                                        desc=w["desc"] + f" [{args.sweeps_per_round} sweeps per round]")
    if args.impl == "reference":
        bench_reference(args)
    elif args.impl == "reference-gpu":
        bench_reference_gpu(args)
    else:
        run_workload(args)


def bench_made_train(args):
    """Adam steps of the proposal network at the dense workload's shape (tensor-core GEMMs plus the
    element-wise training kernels), CUDA events around each step of 50 Adam steps."""
    import torch

    from drift_b200.made import Made

    rank, world, local = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    w = WORKLOADS[args.workload]
    n, h, B, K = w["n"], w["h"], w["batch"], w["adam_steps"]
    made = Made(n, (h, h), seed=1, device=dev)
    g = torch.Generator(device=dev).manual_seed(5)
    data = (torch.randint(0, 2, (8 * B, n), device=dev, generator=g) * 2 - 1).to(torch.int8)
    ev = []

    def step(s_):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        made.train_async(data, steps=K, batch=B, lr=1e-4, seed=s_)
        e1.record()
        ev.append((e0, e1))

    for s_ in range(args.warmup):
        step(s_)
    made.check()
    ev.clear()
    sampler = ClockSampler(local)
    sampler.start()
    torch.cuda.synchronize()
    for s_ in range(args.steps):
        step(100 + s_)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    made.check()
    t = sum(a.elapsed_time(b) for a, b in ev) * 1e-3
    t_max = reduce_max(t, world, dev)
    flops = float(w["flops_per_adam_step"]) * K * args.steps * world
    if rank == 0:
        peak, peak_kind = load_tensor_peak()
        achieved = flops / t_max / 1e12
        emit(args, {
            "metric": "MADE training TFLOP/s", "value": achieved, "unit": "TFLOP/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_max / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "bf16 x bf16 -> fp32",
            "data": "synthetic (random +-1 configurations)",
            "config": {"workload": w["desc"], "adam_steps_per_step": K, "flops_per_adam_step": w["flops_per_adam_step"]},
            "roofline": {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                         "frac": achieved / peak, "traffic": None, "peak_kind": peak_kind,
                         "kernel": "the whole Adam step (gemm_bf16_kernel and the element-wise training kernels)"},
            # per Adam step: spins to bf16, 3 forward and 5 backward GEMMs, the loss, 6 transposes, 3 bias
            # sums, 6 Adam updates
            "gpu_launches": 25 * K * args.steps, "clocks": clocks,
        })
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


def run_workload(args):
    if args.workload == "made_train":
        bench_made_train(args)
        return
    if args.workload == "batched_er":
        bench_batched(args)
    elif args.workload == "sk512":
        bench_sk(args)
    elif args.workload == "ea3d64":
        bench_ms(args)
    elif args.workload == "maxcut3reg_r2048":
        bench_gms(args)
    elif args.workload == "ea2d_batch256":
        bench_ea2d_batch(args)
    else:
        bench_b200(args)


if __name__ == "__main__":
    main()
