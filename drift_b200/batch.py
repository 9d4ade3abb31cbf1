"""Batched parallel tempering: many independent instances (uneven sizes, own ladders, own replica
counts) advanced by one persistent sm_100a launch per call (include/drift_pt.h, batched layer).

Instance k is bit for bit the chain that the single-instance engine runs with
``instance = stream_ids[k]`` and the same seed; batching changes speed, never results.

The launch shape (replicas per work item, threads per replica, CTAs per SM, positions per item)
is picked by ``autotune``, which times a few rounds of each candidate shape and caches the winner
by problem signature; since results do not depend on the shape, the tuner is free to choose.
"""

from __future__ import annotations

import ctypes as C
import json
import os
import time

import numpy as np

from . import _lib
from .engine import HostProblem, _ptr

DESC_DTYPE = np.dtype([("n", "<i4"), ("n_pos", "<i4"), ("n_slices", "<i4"), ("n_colors", "<i4"),
                       ("n_replicas", "<i4"), ("max_field", "<i4"), ("stream_id", "<i4"), ("reserved", "<i4"),
                       ("color_ptr", "<i8"), ("slice_off", "<i8"), ("ell", "<i8"), ("pos", "<i8"),
                       ("slot0", "<i8"), ("spin0", "<i8"), ("thr", "<i8")])
assert DESC_DTYPE.itemsize == 88

SPIN_BUDGET = 160 * 1024  # shared-memory bytes for one item's spins


class BatchSizesC(C.Structure):
    _fields_ = [("color_ptr", C.c_int64), ("slice_off", C.c_int64), ("ell", C.c_int64), ("pos", C.c_int64),
                ("sites", C.c_int64), ("all_integer", C.c_int32), ("reserved", C.c_int32)]


class BatchLayoutC(C.Structure):
    _fields_ = [("color_ptr", C.c_void_p), ("slice_off", C.c_void_p), ("ell_nbr", C.c_void_p), ("ell_w", C.c_void_p),
                ("h_pos", C.c_void_p), ("site_of_pos", C.c_void_p), ("pos_of_site", C.c_void_p)]


def _bind():
    L = _lib.load()
    if not getattr(L, "_blay_bound", False):
        vp = C.c_void_p
        L.drift_pt_batch_layout_query.argtypes = [C.c_int32, vp, vp, C.POINTER(BatchSizesC)]
        L.drift_pt_batch_layout_fill.argtypes = [C.c_int32, vp, vp, C.c_int32, vp, vp, vp, vp, vp,
                                                 C.POINTER(BatchLayoutC)]
        L._blay_bound = True
    return L


class BatchProblem:
    """Concatenated device layouts of several HostProblems with a ladder (betas) each."""

    def __init__(self, problems: list[HostProblem], ladders: list, *, stream_ids=None, device="cuda",
                 integer_path: bool | None = None):
        import torch

        if len(problems) != len(ladders) or not problems:
            raise ValueError("need one ladder per problem")
        L = _bind()
        K = len(problems)
        csrs = (_lib.Csr * K)(*[hp.c_csr() for hp in problems])
        infos = (_lib.LayoutInfo * K)()
        sizes = BatchSizesC()
        _lib.check(L.drift_pt_batch_layout_query(K, csrs, infos, C.byref(sizes)), "drift_pt_batch_layout_query")
        all_int = bool(sizes.all_integer)
        if integer_path is None:
            integer_path = all_int
        if integer_path and not all_int:
            raise ValueError("integer path requested but some instance has non-integer couplings")
        self.integer_path = bool(integer_path)
        self.n_instances = K
        self.stream_ids = np.arange(K, dtype=np.int64) if stream_ids is None else np.asarray(stream_ids, np.int64)
        if self.stream_ids.shape != (K,) or np.any(self.stream_ids < 0) or np.any(self.stream_ids >= 2 ** 24):
            raise ValueError("stream_ids must be K values in [0, 2^24)")
        self.ladders = [np.ascontiguousarray(b, dtype=np.float64) for b in ladders]
        R = np.array([len(b) for b in self.ladders], np.int32)
        if np.any(R < 1):
            raise ValueError(f"instance {int(np.argmin(R))}: empty ladder")
        betas = np.concatenate(self.ladders)
        F = np.array([i.max_field for i in infos], np.int64) if self.integer_path else np.zeros(K, np.int64)
        wd = np.int8 if self.integer_path else np.float32
        hd = np.int32 if self.integer_path else np.float32
        cp = np.zeros(sizes.color_ptr, np.int32)
        so = np.zeros(sizes.slice_off, np.int32)
        nb = np.zeros(sizes.ell + 4, np.int32)  # tails: the kernels may read a vector past the last entry
        w = np.zeros(sizes.ell + 16, wd)
        h = np.zeros(sizes.pos, hd)
        sop = np.zeros(sizes.pos, np.int32)
        pos = np.zeros(sizes.sites, np.int32)
        thr = np.zeros(max(int((R * F).sum()), 1), np.uint32)
        desc = np.zeros(K, dtype=DESC_DTYPE)
        out = BatchLayoutC(_ptr(cp), _ptr(so), _ptr(nb), _ptr(w), _ptr(h), _ptr(sop), _ptr(pos))
        sid = self.stream_ids.astype(np.int32)
        _lib.check(L.drift_pt_batch_layout_fill(K, csrs, infos, 1 if self.integer_path else 0, _ptr(R), _ptr(sid),
                                                _ptr(betas), desc.ctypes.data, _ptr(thr), C.byref(out)),
                   "drift_pt_batch_layout_fill")
        self.desc = desc
        self.infos = list(infos)
        self.site_of_pos = [sop[int(d["pos"]): int(d["pos"]) + int(d["n_pos"])] for d in desc]
        site0 = np.concatenate([[0], np.cumsum([int(d["n"]) for d in desc])])
        self.pos_of_site = [pos[site0[k]: site0[k + 1]] for k in range(K)]
        self.total_slots = int(R.sum())
        self.total_spin_bytes = int(sum(int(d["n_replicas"]) * int(d["n_pos"]) for d in desc))
        self.max_n_pos = int(max(i.n_pos for i in infos))
        self.max_colors = int(max(i.n_colors for i in infos))
        self.max_width = int(max(i.max_degree for i in infos))
        self.min_width = int(min(i.min_width for i in infos))
        self.max_field = int(F.max()) if self.integer_path else 0
        self.has_field = int(any(i.has_field for i in infos))
        self.device = dev = torch.device(device)
        t = lambda a: torch.from_numpy(a).to(dev)
        self.d_desc = t(desc.view(np.uint8))
        self.d_color_ptr = t(cp)
        self.d_slice_off = t(so)
        self.d_ell_nbr = t(nb)
        self.d_ell_w = t(w)
        self.d_h_pos = t(h)
        self.d_betas = t(betas)
        self.d_thr = t(thr.view(np.int32)) if self.integer_path else None

    def c_problem(self) -> "_lib.BatchProblem":
        return _lib.BatchProblem(self.n_instances, 1 if self.integer_path else 0, self.has_field, self.max_width,
                                 self.min_width, self.max_field, self.max_n_pos, self.max_colors, self.total_slots,
                                 self.d_desc.data_ptr(), self.d_color_ptr.data_ptr(), self.d_slice_off.data_ptr(),
                                 self.d_ell_nbr.data_ptr(), self.d_ell_w.data_ptr(), self.d_h_pos.data_ptr(),
                                 self.d_betas.data_ptr(), self.d_thr.data_ptr() if self.d_thr is not None else None)

    def energy_scale(self) -> float:
        return 1.0 if self.integer_path else 2.0 ** -32

    def signature(self) -> str:
        n = sorted(int(i.n) for i in self.infos)
        R = sorted(len(b) for b in self.ladders)
        return json.dumps([self.n_instances, n[0], n[len(n) // 2], n[-1], R[0], R[-1], self.max_width,
                           self.integer_path])


class BatchEngine:
    """State of a batch on the device; ``run`` advances every instance by n_rounds rounds."""

    def __init__(self, bp: BatchProblem, *, seed: int = 0, sweeps_per_round: int = 1, max_tile: int = 0,
                 threads_per_slot: int = 0, ctas_per_sm: int = 0, positions_per_item: int = 0,
                 timeout_s: float = 10.0):
        import torch

        self.torch = torch
        self.bp = bp
        self.seed, self.spr = int(seed), int(sweeps_per_round)
        dev = bp.device
        S = bp.total_slots
        self.spins = torch.empty(bp.total_spin_bytes, dtype=torch.int8, device=dev)
        self.best_spins = torch.empty(bp.total_spin_bytes, dtype=torch.int8, device=dev)
        self.energy = torch.empty(S, dtype=torch.int64, device=dev)
        self.best_energy = torch.empty(S, dtype=torch.int64, device=dev)
        self.rung_of_slot = torch.empty(S, dtype=torch.int32, device=dev)
        self.slot_of_rung = torch.empty(S, dtype=torch.int32, device=dev)
        self.tried = torch.zeros(S, dtype=torch.int64, device=dev)
        self.accepted = torch.zeros(S, dtype=torch.int64, device=dev)
        self.workspace = torch.zeros(256, dtype=torch.uint8, device=dev)
        self.timeout_s = float(timeout_s)
        self.rounds_done = 0
        self.set_shape(max_tile, threads_per_slot, ctas_per_sm, positions_per_item)

    def set_shape(self, max_tile=0, threads_per_slot=0, ctas_per_sm=0, positions_per_item=0):
        bp = self.bp
        R_max = max(len(b) for b in bp.ladders)
        if max_tile <= 0:
            max_tile = min(32, R_max)
        if threads_per_slot <= 0:
            threads_per_slot = 32 if max_tile <= 16 else 16
            while max_tile * threads_per_slot > 512:
                threads_per_slot //= 2
            while (max_tile * threads_per_slot) % 32:
                threads_per_slot *= 2
        self.shape = dict(max_tile=int(max_tile), threads_per_slot=int(threads_per_slot),
                          ctas_per_sm=int(ctas_per_sm), positions_per_item=int(positions_per_item))
        L = _lib.load()
        n_pos = np.array([d["n_pos"] for d in bp.desc], np.int32)
        n_rep = np.array([d["n_replicas"] for d in bp.desc], np.int32)
        n_items = C.c_int32(0)
        _lib.check(L.drift_pt_batch_items(bp.n_instances, _ptr(n_pos), _ptr(n_rep), max_tile, SPIN_BUDGET, None,
                                          C.byref(n_items)), "batch_items")
        items = np.zeros(3 * n_items.value, np.int32)
        _lib.check(L.drift_pt_batch_items(bp.n_instances, _ptr(n_pos), _ptr(n_rep), max_tile, SPIN_BUDGET,
                                          _ptr(items), C.byref(n_items)), "batch_items")
        items = items.reshape(-1, 3)
        self.items = items
        self.max_item_bytes = int(max(n_pos[i] * c for i, _, c in items))
        self.d_items = self.torch.from_numpy(items.ravel().copy()).to(bp.device)

    def _args(self, n_rounds: int) -> "_lib.BatchRunArgs":
        s = self.shape
        return _lib.BatchRunArgs(n_rounds, self.spr, self.rounds_done, self.seed & 0xFFFFFFFFFFFFFFFF,
                                 self.d_items.data_ptr(), len(self.items), int(self.items[:, 2].max()),
                                 s["threads_per_slot"], s["ctas_per_sm"], s["positions_per_item"],
                                 self.max_item_bytes, self.timeout_s)

    def _state(self) -> "_lib.DeviceState":
        return _lib.DeviceState(self.spins.data_ptr(), self.energy.data_ptr(), self.best_energy.data_ptr(),
                                self.best_spins.data_ptr(), self.rung_of_slot.data_ptr(),
                                self.slot_of_rung.data_ptr(), self.tried.data_ptr(), self.accepted.data_ptr(), None)

    def stream(self):
        return C.c_void_p(self.torch.cuda.current_stream(self.bp.device).cuda_stream)

    def init(self) -> None:
        L = _lib.load()
        P, A, S = self.bp.c_problem(), self._args(0), self._state()
        _lib.check(L.drift_pt_batch_init(C.byref(P), C.byref(A), C.byref(S), self.stream()), "drift_pt_batch_init")
        self.rounds_done = 0

    def run(self, n_rounds: int) -> None:
        L = _lib.load()
        P, A, S = self.bp.c_problem(), self._args(n_rounds), self._state()
        _lib.check(L.drift_pt_batch_run(C.byref(P), C.byref(A), C.byref(S), C.c_void_p(self.workspace.data_ptr()),
                                        self.workspace.numel(), self.stream()), "drift_pt_batch_run")
        self.rounds_done += n_rounds

    def check(self) -> None:
        self.torch.cuda.synchronize(self.bp.device)
        flag = int(self.workspace[16:20].view(self.torch.int32).item())
        if flag:
            raise _lib.EngineError(_lib.ETIMEOUT, "drift_pt_batch_run", "a bounded in-kernel wait timed out")

    def fetch(self, k: int) -> dict:
        """Host copy of instance k's state, spins in its original site order (as PtEngine.fetch)."""
        d = self.bp.desc[k]
        R, n_pos, s0, p0 = int(d["n_replicas"]), int(d["n_pos"]), int(d["slot0"]), int(d["spin0"])
        pos = self.bp.pos_of_site[k]
        sc = self.bp.energy_scale()
        sp = self.spins[p0:p0 + R * n_pos].view(R, n_pos).cpu().numpy()
        bsp = self.best_spins[p0:p0 + R * n_pos].view(R, n_pos).cpu().numpy()
        out = {
            "spins": sp[:, pos], "best_spins": bsp[:, pos],
            "energy_fixed": self.energy[s0:s0 + R].cpu().numpy(),
            "best_energy_fixed": self.best_energy[s0:s0 + R].cpu().numpy(),
            "rung_of_slot": self.rung_of_slot[s0:s0 + R].cpu().numpy(),
            "slot_of_rung": self.slot_of_rung[s0:s0 + R].cpu().numpy(),
            "tried": self.tried[s0:s0 + R - 1].cpu().numpy(),
            "accepted": self.accepted[s0:s0 + R - 1].cpu().numpy(),
        }
        out["energy"] = out["energy_fixed"] * sc
        out["best_energy"] = out["best_energy_fixed"] * sc
        return out

    def capture_job(self, n_rounds: int, launch_rounds: int = 0) -> "JobGraph":
        """A whole job captured as one CUDA graph: the initialisation and n_rounds rounds, as
        launches of launch_rounds rounds each (0: one launch). Replaying it runs the job from the
        start with this engine's seed, so every replay gives the same bits as `init(); run(n_rounds)`."""
        return JobGraph(self, n_rounds, launch_rounds)

    def best_energies(self) -> np.ndarray:
        """Lowest energy of every instance so far (model units)."""
        be = self.best_energy.cpu().numpy()
        return np.array([be[int(d["slot0"]):int(d["slot0"]) + int(d["n_replicas"])].min() for d in self.bp.desc]) \
            * self.bp.energy_scale()


class JobGraph:
    """A batched PT job (drift_pt_batch_init plus every round) captured once as a CUDA graph, so a
    whole run is one graph launch. The engine's kernel attributes are set by one eager round before
    the capture (no attribute or occupancy call is made inside it); the state buffers are the
    engine's own, and the graph writes them on every replay."""

    def __init__(self, eng: BatchEngine, n_rounds: int, launch_rounds: int = 0):
        torch = eng.torch
        if n_rounds < 1:
            raise ValueError("a job has at least one round")
        self.eng, self.n_rounds = eng, int(n_rounds)
        step = int(launch_rounds) if launch_rounds > 0 else self.n_rounds
        eng.init()
        eng.run(1)  # outside the capture: kernel attributes, the launch plan's caches
        torch.cuda.synchronize(eng.bp.device)
        self.launches = 0
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph):
            eng.init()
            done = 0
            while done < self.n_rounds:
                c = min(step, self.n_rounds - done)
                eng.run(c)
                done += c
                self.launches += 1
        eng.rounds_done = self.n_rounds

    def replay(self) -> None:
        """Run the whole job again (asynchronously on the current stream)."""
        self.graph.replay()
        self.eng.rounds_done = self.n_rounds


_TUNE_CACHE: dict = {}


def tune_candidates(bp: BatchProblem):
    R_max = max(len(b) for b in bp.ladders)
    tiles = sorted({min(R_max, t) for t in (32, 16, 8, 4)}, reverse=True)
    out = []
    for tile in tiles:
        for tps in (4, 8, 16, 32, 64):
            th = tile * tps
            if th < 64 or th > 512 or th % 32:
                continue
            for P in ((4, 8) if bp.integer_path else (8,)):
                for cps in (0, 1):
                    out.append(dict(max_tile=tile, threads_per_slot=tps, ctas_per_sm=cps, positions_per_item=P))
    return out


def autotune(eng: BatchEngine, *, rounds: int = 2, candidates=None, cache_path: str | None = None) -> dict:
    """Time every candidate launch shape on ``rounds`` rounds from the current state and keep the
    fastest (the state is restored afterwards). Results are cached by problem signature, sweeps per
    round and SM count, in memory and, if given, in a JSON file."""
    torch = eng.torch
    props = torch.cuda.get_device_properties(eng.bp.device)
    key = json.dumps([eng.bp.signature(), eng.spr, props.multi_processor_count])
    if cache_path and os.path.exists(cache_path) and key not in _TUNE_CACHE:
        with open(cache_path) as f:
            _TUNE_CACHE.update(json.load(f))
    if key in _TUNE_CACHE:
        eng.set_shape(**_TUNE_CACHE[key])
        return _TUNE_CACHE[key]
    saved = [t.clone() for t in (eng.spins, eng.best_spins, eng.energy, eng.best_energy, eng.rung_of_slot,
                                 eng.slot_of_rung, eng.tried, eng.accepted)]
    done0 = eng.rounds_done
    best, best_t = None, float("inf")
    for cand in (candidates or tune_candidates(eng.bp)):
        try:
            eng.set_shape(**cand)
            eng.run(1)  # warm
            torch.cuda.synchronize(eng.bp.device)
            t0 = time.perf_counter()
            eng.run(rounds)
            torch.cuda.synchronize(eng.bp.device)
            dt = time.perf_counter() - t0
        except _lib.EngineError:
            continue
        if dt < best_t:
            best, best_t = cand, dt
    for t, s in zip((eng.spins, eng.best_spins, eng.energy, eng.best_energy, eng.rung_of_slot, eng.slot_of_rung,
                     eng.tried, eng.accepted), saved):
        t.copy_(s)
    eng.rounds_done = done0
    if best is None:
        raise RuntimeError("autotune: no candidate launch shape ran")
    eng.set_shape(**best)
    _TUNE_CACHE[key] = best
    if cache_path:
        with open(cache_path, "w") as f:
            json.dump(_TUNE_CACHE, f)
    return best
