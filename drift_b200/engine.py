"""Device-resident PT engine: compiled problem and replica state in torch-owned device memory,
driven through the C ABI (include/drift_pt.h). torch supplies allocation and the stream only.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib
from .ising import model_csr


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


def greedy_coloring(n: int, row_ptr: np.ndarray, col_idx: np.ndarray):
    """(k, color_ptr, color_spins): greedy colouring + stable colour order (drift/gpu.py:122-145)."""
    L = _lib.load()
    color = np.zeros(max(n, 1), dtype=np.int32)
    k = C.c_int32(0)
    _lib.check(L.drift_pt_greedy_coloring(n, _ptr(row_ptr), _ptr(col_idx), _ptr(color), C.byref(k)), "greedy_coloring")
    color_ptr = np.zeros(k.value + 1, dtype=np.int32)
    color_spins = np.zeros(max(n, 1), dtype=np.int32)
    _lib.check(L.drift_pt_color_order(n, _ptr(color), k.value, _ptr(color_ptr), _ptr(color_spins)), "color_order")
    return k.value, color_ptr, color_spins[:n]


def geometric_betas(n_replicas: int, T_min: float, T_max: float) -> np.ndarray:
    """beta per rung of the geometric temperature ladder (drift/solvers/parallel_tempering.py:29-36,73)."""
    if n_replicas == 1:
        T = np.array([T_min], dtype=np.float64)
    else:
        T = T_min * (T_max / T_min) ** (np.arange(n_replicas) / (n_replicas - 1))
    return 1.0 / np.maximum(T, 1e-12)


@dataclass
class HostProblem:
    """A problem in the reference's own CSR terms plus its colouring (the content of problem.bin)."""

    n: int
    row_ptr: np.ndarray
    col_idx: np.ndarray
    weight: np.ndarray
    h: np.ndarray
    color_ptr: np.ndarray
    color_spins: np.ndarray

    @classmethod
    def from_model(cls, model, order: str = "index") -> "HostProblem":
        """Greedy colouring of the model's couplings (drift/gpu.py:122-145). ``order`` sets the
        order of the spins inside each colour class: "index" (the reference's stable order) or
        "degree" (descending degree, then index), which gives slices of nearly uniform width on
        irregular graphs. Any order inside a class is an equally valid sweep; the uniforms follow
        the positions, so runs are reproducible for a given order."""
        n, row_ptr, col_idx, weight, h = model_csr(model)
        _, color_ptr, color_spins = greedy_coloring(n, row_ptr, col_idx)
        if order == "degree":
            deg = np.diff(row_ptr)
            for c in range(len(color_ptr) - 1):
                seg = color_spins[color_ptr[c]:color_ptr[c + 1]]
                color_spins[color_ptr[c]:color_ptr[c + 1]] = seg[np.lexsort((seg, -deg[seg]))]
        elif order != "index":
            raise ValueError("order must be 'index' or 'degree'")
        return cls(n, row_ptr, col_idx, weight, h, color_ptr, color_spins)

    @property
    def n_colors(self) -> int:
        return len(self.color_ptr) - 1

    def c_csr(self) -> _lib.Csr:
        return _lib.Csr(self.n, int(self.col_idx.size), _ptr(self.row_ptr), _ptr(self.col_idx), _ptr(self.weight),
                        _ptr(self.h), self.n_colors, _ptr(self.color_ptr), _ptr(self.color_spins))


class DeviceProblem:
    """The compiled sliced-ELL layout of a HostProblem, uploaded to the current CUDA device."""

    def __init__(self, hp: HostProblem, device="cuda", integer_path: bool | None = None):
        import torch

        L = _lib.load()
        self.host = hp
        csr = hp.c_csr()
        info = _lib.LayoutInfo()
        _lib.check(L.drift_pt_layout_query(C.byref(csr), C.byref(info)), "layout_query")
        if integer_path is None:
            integer_path = bool(info.integer_couplings)
        if integer_path and not info.integer_couplings:
            raise ValueError("integer path requested for non-integer couplings")
        self.info = info
        self.integer_path = bool(integer_path)
        self.n, self.n_pos, self.n_slices, self.n_ell = info.n, info.n_pos, info.n_slices, info.n_ell
        self.max_field = info.max_field if integer_path else 0
        color_ptr = np.zeros(info.n_colors + 1, np.int32)
        slice_off = np.zeros(info.n_slices + 1, np.int32)
        ell_nbr = np.zeros(max(info.n_ell, 1), np.int32)
        ell_w = np.zeros(max(info.n_ell, 1), np.int8 if integer_path else np.float32)
        h_pos = np.zeros(info.n_pos, np.int32 if integer_path else np.float32)
        self.site_of_pos = np.zeros(info.n_pos, np.int32)
        self.pos_of_site = np.zeros(info.n, np.int32)
        lay = _lib.Layout(_ptr(color_ptr), _ptr(slice_off), _ptr(ell_nbr), _ptr(ell_w), _ptr(h_pos),
                          _ptr(self.site_of_pos), _ptr(self.pos_of_site))
        _lib.check(L.drift_pt_layout_fill(C.byref(csr), 1 if integer_path else 0, C.byref(lay)), "layout_fill")
        self.color_ptr_host = color_ptr
        self.max_class = int(np.max(np.diff(color_ptr)))
        self.max_width = int(np.max(np.diff(slice_off))) if slice_off.size > 1 else 0
        self.min_width = int(np.min(np.diff(slice_off))) if slice_off.size > 1 else 0
        self.unit_regular = int(info.unit_regular) if integer_path else 0
        # the unit-regular form's bank-aware storage order of the spin bytes (drift_pt_unit_placement)
        self.unit_place = None
        if self.unit_regular:
            place = np.zeros(info.n_pos // 4, np.uint16)
            _lib.check(L.drift_pt_unit_placement(C.byref(csr), 0, _ptr(place)), "unit_placement")
            self.unit_place = place
        self.device = torch.device(device)
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(self.device)
        self.d_color_ptr, self.d_slice_off, self.d_ell_nbr = t(color_ptr), t(slice_off), t(ell_nbr)
        self.d_ell_w, self.d_h_pos = t(ell_w), t(h_pos)
        self.d_unit_place = t(self.unit_place.view(np.int16)) if self.unit_place is not None else None

    def c_problem(self) -> _lib.DeviceProblem:
        return _lib.DeviceProblem(self.n, self.n_pos, self.n_slices, self.info.n_colors, 1 if self.integer_path else 0,
                                  self.max_field, self.max_width, self.max_class, self.info.has_field,
                                  self.min_width, self.unit_regular, self.n_ell,
                                  self.d_color_ptr.data_ptr(), self.d_slice_off.data_ptr(), self.d_ell_nbr.data_ptr(),
                                  self.d_ell_w.data_ptr(), self.d_h_pos.data_ptr(),
                                  self.d_unit_place.data_ptr() if self.d_unit_place is not None else None)

    def energy_scale(self) -> float:
        return 1.0 if self.integer_path else 2.0 ** -32


class PtEngine:
    """R replicas of one problem on a beta ladder; state stays on the device between runs."""

    def __init__(self, prob: DeviceProblem, betas, *, seed: int = 0, sweeps_per_round: int = 1, instance: int = 0,
                 replicas_per_cta: int = 0, threads_per_cta: int = 0, positions_per_item: int = 0,
                 timeout_s: float = 10.0, round_sync: int = 0, item_form: int = 0):
        import torch

        self.torch = torch
        self.prob = prob
        self.betas = np.ascontiguousarray(betas, dtype=np.float64)
        R = self.R = len(self.betas)
        if R < 1:
            raise ValueError("need at least one replica")
        if not np.all(np.isfinite(self.betas)) or np.any(self.betas < 0):
            raise ValueError("betas must be finite and >= 0")
        self.seed, self.instance, self.spr = int(seed), int(instance), int(sweeps_per_round)
        if self.spr < 1:
            raise ValueError("sweeps_per_round must be >= 1")
        self.rpc, self.threads, self.timeout_s = int(replicas_per_cta), int(threads_per_cta), float(timeout_s)
        self.ppi = int(positions_per_item)
        self.round_sync = int(round_sync)  # 0 auto, 1 grid barrier, 2 one cluster
        self.item_form = int(item_form)  # 0 auto, 1 sliced-ELL gather, 2 unit-regular sweep
        dev = prob.device
        L = _lib.load()
        self.d_betas = torch.from_numpy(self.betas).to(dev)
        self.thr = None
        if prob.integer_path:
            thr = np.zeros(R * prob.max_field, dtype=np.uint32)
            _lib.check(L.drift_pt_thresholds(R, _ptr(self.betas), prob.max_field, _ptr(thr)), "thresholds")
            self.thr = thr.reshape(R, prob.max_field)
            self.d_thr = torch.from_numpy(thr.view(np.int32)).to(dev)
        n_pos = prob.n_pos
        self.spins = torch.empty((R, n_pos), dtype=torch.int8, device=dev)
        self.best_spins = torch.empty((R, n_pos), dtype=torch.int8, device=dev)
        self.energy = torch.empty(R, dtype=torch.int64, device=dev)
        self.best_energy = torch.empty(R, dtype=torch.int64, device=dev)
        self.rung_of_slot = torch.empty(R, dtype=torch.int32, device=dev)
        self.slot_of_rung = torch.empty(R, dtype=torch.int32, device=dev)
        self.tried = torch.zeros(max(R - 1, 1), dtype=torch.int64, device=dev)
        self.accepted = torch.zeros(max(R - 1, 1), dtype=torch.int64, device=dev)
        ws = C.c_size_t(0)
        _lib.check(L.drift_pt_workspace_bytes(R, C.byref(ws)), "workspace_bytes")
        self.workspace = torch.zeros(ws.value, dtype=torch.uint8, device=dev)
        self.rounds_done = 0
        self.history = None

    def _args(self, n_rounds: int) -> _lib.RunArgs:
        return _lib.RunArgs(self.R, n_rounds, self.spr, self.round_sync, self.rounds_done, self.seed & 0xFFFFFFFFFFFFFFFF,
                            self.instance, self.rpc, self.threads, self.ppi, self.item_form, self.d_betas.data_ptr(),
                            self.d_thr.data_ptr() if self.thr is not None else None, self.timeout_s)

    def _state(self, history=None) -> _lib.DeviceState:
        return _lib.DeviceState(self.spins.data_ptr(), self.energy.data_ptr(), self.best_energy.data_ptr(),
                                self.best_spins.data_ptr(), self.rung_of_slot.data_ptr(),
                                self.slot_of_rung.data_ptr(), self.tried.data_ptr(), self.accepted.data_ptr(),
                                history.data_ptr() if history is not None else None)

    def stream(self):
        return C.c_void_p(self.torch.cuda.current_stream(self.prob.device).cuda_stream)

    def init(self) -> None:
        L = _lib.load()
        P, A, S = self.prob.c_problem(), self._args(0), self._state()
        _lib.check(L.drift_pt_init(C.byref(P), C.byref(A), C.byref(S), self.stream()), "drift_pt_init")
        self.rounds_done = 0

    def run(self, n_rounds: int, history=None) -> None:
        """Enqueue n_rounds rounds (asynchronous). ``history``: optional device float64[n_rounds]."""
        L = _lib.load()
        P, A, S = self.prob.c_problem(), self._args(n_rounds), self._state(history)
        _lib.check(L.drift_pt_run(C.byref(P), C.byref(A), C.byref(S), C.c_void_p(self.workspace.data_ptr()),
                                  self.workspace.numel(), self.stream()), "drift_pt_run")
        self.rounds_done += n_rounds

    def check(self) -> None:
        L = _lib.load()
        _lib.check(L.drift_pt_check(C.c_void_p(self.workspace.data_ptr()), self.stream()), "drift_pt_check")

    def energy_fp64(self, which: str = "spins") -> np.ndarray:
        """FP64 recompute of each slot's energy (of its current or best spins)."""
        L = _lib.load()
        out = self.torch.empty(self.R, dtype=self.torch.float64, device=self.prob.device)
        sp = self.spins if which == "spins" else self.best_spins
        P = self.prob.c_problem()
        _lib.check(L.drift_pt_energy_fp64(C.byref(P), C.c_void_p(sp.data_ptr()), self.R, C.c_void_p(out.data_ptr()),
                                          self.stream()), "drift_pt_energy_fp64")
        return out.cpu().numpy()

    def fetch(self) -> dict:
        """Host copy of the state, spins in the original site order, energies in model units."""
        pos = self.prob.pos_of_site
        sc = self.prob.energy_scale()
        out = {
            "spins": self.spins.cpu().numpy()[:, pos],
            "best_spins": self.best_spins.cpu().numpy()[:, pos],
            "energy_fixed": self.energy.cpu().numpy(),
            "best_energy_fixed": self.best_energy.cpu().numpy(),
            "rung_of_slot": self.rung_of_slot.cpu().numpy(),
            "slot_of_rung": self.slot_of_rung.cpu().numpy(),
            "tried": self.tried.cpu().numpy()[: max(self.R - 1, 0)],
            "accepted": self.accepted.cpu().numpy()[: max(self.R - 1, 0)],
        }
        out["energy"] = out["energy_fixed"] * sc
        out["best_energy"] = out["best_energy_fixed"] * sc
        return out
