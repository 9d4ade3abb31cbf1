"""drift_b200.gpu - drop-in for the reference's GPU parallel-tempering entry point.

Same names, keywords, return type and error behaviour as drift/gpu.py:29-114:

    gpu_binary_path() -> str            path of the engine (here: libdrift_pt.so)
    gpu_available()   -> bool           True iff the engine is built and a CUDA device is visible
    parallel_tempering_gpu(model, *, n_replicas=16, T_min=0.1, T_max=5.0, n_rounds=300,
                           sweeps_per_round=5, seed=0) -> PtResult

Instead of serialising problem.bin and running a subprocess (drift/gpu.py:83-103), the call
compiles the CSR and colouring through the C ABI and runs one persistent sm_100a launch. The
result keeps every PtResult field of drift/solvers/parallel_tempering.py:39-49 (and fills the
ones the reference GPU path leaves None: swap_rate, best_history) and adds per-rung final
spins/energies and per-pair swap counts. Extra keywords (all optional): ``betas`` (explicit ladder,
one beta per rung, overrides T_min/T_max), ``instance`` (stream id), ``replicas_per_cta`` and
``threads_per_cta`` (launch shape; results do not depend on it).
"""

from __future__ import annotations

import time
from dataclasses import dataclass, field

import numpy as np

from . import _lib


def geometric_ladder(n_replicas: int, T_min: float, T_max: float) -> np.ndarray:
    """Geometric temperature ladder T_min..T_max (drift/solvers/parallel_tempering.py:29-36)."""
    if n_replicas == 1:
        return np.array([T_min], dtype=np.float64)
    return T_min * (T_max / T_min) ** (np.arange(n_replicas) / (n_replicas - 1))


@dataclass
class PtResult:
    """Outcome of a PT run: the fields of drift/solvers/parallel_tempering.py:39-49, plus extras."""

    best_s: np.ndarray
    best_E: float
    temperatures: np.ndarray
    swap_rate: float
    best_history: np.ndarray = field(default=None)
    throughput: float = None     # attempted spin flips per second (device time of the round loop)
    seconds: float = None
    rung_spins: np.ndarray = field(default=None)     # (R, n) final configuration at each rung
    rung_energies: np.ndarray = field(default=None)  # (R,)
    swap_tried: np.ndarray = field(default=None)     # (R-1,) per adjacent rung pair
    swap_accepted: np.ndarray = field(default=None)


def gpu_binary_path() -> str:
    """Absolute path where the compiled engine is expected."""
    return _lib.lib_path()


def gpu_available() -> bool:
    """True iff the engine library is built and a CUDA device is visible."""
    if not _lib.available():
        return False
    try:
        import torch

        return bool(torch.cuda.is_available())
    except Exception:
        return False


def parallel_tempering_gpu(
    model,
    *,
    n_replicas: int = 16,
    T_min: float = 0.1,
    T_max: float = 5.0,
    n_rounds: int = 300,
    sweeps_per_round: int = 5,
    seed: int = 0,
    betas=None,
    instance: int = 0,
    replicas_per_cta: int = 0,
    threads_per_cta: int = 0,
) -> PtResult:
    """Solve `model` by parallel tempering on the GPU. Same signature/return as the CPU reference."""
    if not gpu_available():
        raise RuntimeError(
            f"GPU engine not built or no CUDA device: expected {gpu_binary_path()}.\n"
            "Build it with: python -m drift_b200.build"
        )
    import torch

    from .engine import DeviceProblem, HostProblem, PtEngine

    if betas is None:
        temps = geometric_ladder(n_replicas, T_min, T_max)
        beta_arr = 1.0 / np.maximum(temps, 1e-12)
    else:
        beta_arr = np.ascontiguousarray(betas, dtype=np.float64)
        if beta_arr.shape != (n_replicas,):
            raise ValueError(f"betas must have shape ({n_replicas},)")
        temps = 1.0 / np.maximum(beta_arr, 1e-300)
    hp = HostProblem.from_model(model)
    prob = DeviceProblem(hp)
    eng = PtEngine(prob, beta_arr, seed=seed, sweeps_per_round=sweeps_per_round, instance=instance,
                   replicas_per_cta=replicas_per_cta, threads_per_cta=threads_per_cta)
    hist = torch.empty(max(n_rounds, 1), dtype=torch.float64, device=prob.device)
    eng.init()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record()
    eng.run(n_rounds, history=hist)
    end.record()
    eng.check()
    secs = start.elapsed_time(end) * 1e-3
    st = eng.fetch()
    best_slot = int(np.argmin(st["best_energy_fixed"]))
    best_s = st["best_spins"][best_slot].astype(np.float64)
    best_E = float(model.energy(best_s))
    R = n_replicas
    tried, acc = st["tried"], st["accepted"]
    swap_rate = float(acc.sum() / tried.sum()) if tried.sum() else 0.0
    attempts = float(R) * n_rounds * sweeps_per_round * hp.n
    rung_slot = st["slot_of_rung"]
    return PtResult(
        best_s=best_s,
        best_E=best_E,
        temperatures=temps,
        swap_rate=swap_rate,
        best_history=hist.cpu().numpy()[:n_rounds] if n_rounds > 0 else np.zeros(0),
        throughput=attempts / secs if secs > 0 else None,
        seconds=secs,
        rung_spins=st["spins"][rung_slot],
        rung_energies=st["energy"][rung_slot],
        swap_tried=tried,
        swap_accepted=acc,
    )
