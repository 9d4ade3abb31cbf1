"""Dense-coupling (Sherrington-Kirkpatrick type) parallel tempering (include/drift_pt.h, dense
layer): sequential-order Metropolis sweeps with exact integer local fields, updated on the tensor
cores.

The reference runs a dense model through its sparse CSR kernel (cuda/ising_pt.cu:109-122), where
every spin is its own colour class and each attempt walks n - 1 neighbours. This layer keeps each
replica's local fields F = J s + h and adds J delta after every block of 32 spins with int8
tensor-core products (three limbs of 24-bit fixed-point couplings), so every field and energy is
an exact integer.

Couplings are quantised once: Jq = rint(J 2^shift), hq = rint(h 2^shift), shift the largest that
keeps every coupling within 24 bits and every field below 2^30 (for J_ij ~ N(0, 1/n), n = 512:
shift = 25, i.e. an absolute resolution of 3e-8). Energies reported in float are E2 2^-(shift+1);
``SkEngine.energy_fp64`` recomputes them from the unquantised model.
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .engine import _ptr

MAX_N = 512
MAX_R = 512


class SkProblemC(C.Structure):
    _fields_ = [("n", C.c_int32), ("shift", C.c_int32), ("Jq", C.c_void_p), ("hq", C.c_void_p), ("layout", C.c_void_p)]


class SkStateC(C.Structure):
    _fields_ = [("spins", C.c_void_p), ("best_spins", C.c_void_p), ("energy", C.c_void_p),
                ("best_energy", C.c_void_p), ("rung_of_slot", C.c_void_p), ("slot_of_rung", C.c_void_p),
                ("swap_tried", C.c_void_p), ("swap_accepted", C.c_void_p), ("best_history", C.c_void_p)]


class SkRunArgsC(C.Structure):
    _fields_ = [("n_replicas", C.c_int32), ("n_rounds", C.c_int32), ("sweeps_per_round", C.c_int32),
                ("replicas_per_cta", C.c_int32), ("round_offset", C.c_int64), ("seed", C.c_uint64),
                ("instance", C.c_uint32), ("reserved", C.c_int32), ("betas", C.c_void_p), ("scales", C.c_void_p),
                ("timeout_s", C.c_double)]


def _bind():
    L = _lib.load()
    if not getattr(L, "_sk_bound", False):
        vp, i32 = C.c_void_p, C.c_int32
        L.drift_pt_sk_quantize.argtypes = [i32, vp, vp, vp, vp, C.POINTER(i32)]
        L.drift_pt_sk_layout_bytes.argtypes = [i32, C.POINTER(C.c_size_t)]
        L.drift_pt_sk_layout_fill.argtypes = [i32, vp, vp]
        L.drift_pt_sk_scales.argtypes = [i32, vp, i32, vp]
        L.drift_pt_sk_workspace_bytes.argtypes = [i32, C.POINTER(C.c_size_t)]
        L.drift_pt_sk_init.argtypes = [C.POINTER(SkProblemC), C.POINTER(SkRunArgsC), C.POINTER(SkStateC), vp]
        L.drift_pt_sk_run.argtypes = [C.POINTER(SkProblemC), C.POINTER(SkRunArgsC), C.POINTER(SkStateC), vp,
                                      C.c_size_t, vp]
        L.drift_pt_sk_energy.argtypes = [C.POINTER(SkProblemC), i32, vp, vp, vp]
        L._sk_bound = True
    return L


class SkModel:
    """Host side of a dense model: fixed-point couplings, the device coupling table (bytes)."""

    def __init__(self, J: np.ndarray, h: np.ndarray | None = None):
        J = np.ascontiguousarray(J, np.float64)
        n = J.shape[0]
        if J.shape != (n, n):
            raise ValueError("J must be square")
        self.n = n
        self.J = J
        self.h = np.zeros(n) if h is None else np.ascontiguousarray(h, np.float64)
        L = _bind()
        self.Jq = np.zeros((n, n), np.int32)
        self.hq = np.zeros(n, np.int32)
        sh = C.c_int32(0)
        _lib.check(L.drift_pt_sk_quantize(n, _ptr(J), _ptr(self.h), _ptr(self.Jq), _ptr(self.hq), C.byref(sh)),
                   "drift_pt_sk_quantize")
        self.shift = sh.value
        nbytes = C.c_size_t(0)
        _lib.check(L.drift_pt_sk_layout_bytes(n, C.byref(nbytes)), "drift_pt_sk_layout_bytes")
        self.layout = np.zeros(nbytes.value, np.uint8)
        _lib.check(L.drift_pt_sk_layout_fill(n, _ptr(self.Jq), _ptr(self.layout)), "drift_pt_sk_layout_fill")

    @classmethod
    def from_model(cls, model) -> "SkModel":
        return cls(np.asarray(model.J, np.float64), np.asarray(model.h, np.float64))

    def scales(self, betas) -> np.ndarray:
        betas = np.ascontiguousarray(betas, np.float64)
        out = np.zeros(len(betas), np.float32)
        _lib.check(_bind().drift_pt_sk_scales(len(betas), _ptr(betas), self.shift, _ptr(out)), "drift_pt_sk_scales")
        return out

    @property
    def energy_unit(self) -> float:
        """Energy of one unit of E2."""
        return 2.0 ** -(self.shift + 1)

    def energy_fp64(self, spins: np.ndarray) -> np.ndarray:
        """E = -1/2 s^T J s - h^T s of the unquantised model (drift/ising.py:50-60)."""
        s = np.asarray(spins, np.float64)
        return -0.5 * np.einsum("...i,ij,...j->...", s, self.J, s) - s @ self.h


class SkEngine:
    """R replicas of an SkModel on a beta ladder; state on the device."""

    def __init__(self, model: SkModel, betas, *, seed: int = 0, sweeps_per_round: int = 1, instance: int = 0,
                 replicas_per_cta: int = 0, device="cuda", timeout_s: float = 10.0):
        import torch

        self.torch = torch
        self.model = model
        self.betas = np.ascontiguousarray(betas, np.float64)
        R = self.R = len(self.betas)
        if R < 2 or R > MAX_R:
            raise ValueError(f"the dense engine needs 2..{MAX_R} replicas")
        self.seed, self.spr, self.instance = int(seed), int(sweeps_per_round), int(instance)
        self.replicas_per_cta, self.timeout_s = int(replicas_per_cta), float(timeout_s)
        L = _bind()
        dev = self.device = torch.device(device)
        n = model.n
        self.d_Jq = torch.from_numpy(model.Jq).to(dev)
        self.d_hq = torch.from_numpy(model.hq).to(dev)
        self.d_layout = torch.from_numpy(model.layout).to(dev)
        self.d_betas = torch.from_numpy(self.betas).to(dev)
        self.d_scales = torch.from_numpy(model.scales(self.betas)).to(dev)
        self.spins = torch.empty((R, n), dtype=torch.int8, device=dev)
        self.best_spins = torch.empty((R, n), dtype=torch.int8, device=dev)
        self.energy = torch.empty(R, dtype=torch.int64, device=dev)
        self.best_energy = torch.empty(R, dtype=torch.int64, device=dev)
        self.rung_of_slot = torch.empty(R, dtype=torch.int32, device=dev)
        self.slot_of_rung = torch.empty(R, dtype=torch.int32, device=dev)
        self.tried = torch.zeros(R, dtype=torch.int64, device=dev)
        self.accepted = torch.zeros(R, dtype=torch.int64, device=dev)
        self.best_history = None
        ws = C.c_size_t(0)
        _lib.check(L.drift_pt_sk_workspace_bytes(R, C.byref(ws)), "drift_pt_sk_workspace_bytes")
        self.workspace = torch.zeros(ws.value, dtype=torch.uint8, device=dev)
        self.rounds_done = 0

    def _problem(self):
        return SkProblemC(self.model.n, self.model.shift, self.d_Jq.data_ptr(), self.d_hq.data_ptr(),
                          self.d_layout.data_ptr())

    def _args(self, n_rounds):
        return SkRunArgsC(self.R, n_rounds, self.spr, self.replicas_per_cta, self.rounds_done,
                          self.seed & 0xFFFFFFFFFFFFFFFF, self.instance, 0, self.d_betas.data_ptr(),
                          self.d_scales.data_ptr(), self.timeout_s)

    def _state(self):
        return SkStateC(self.spins.data_ptr(), self.best_spins.data_ptr(), self.energy.data_ptr(),
                        self.best_energy.data_ptr(), self.rung_of_slot.data_ptr(), self.slot_of_rung.data_ptr(),
                        self.tried.data_ptr(), self.accepted.data_ptr(),
                        self.best_history.data_ptr() if self.best_history is not None else None)

    def stream(self):
        return C.c_void_p(self.torch.cuda.current_stream(self.device).cuda_stream)

    def init(self):
        P, A, S = self._problem(), self._args(0), self._state()
        _lib.check(_bind().drift_pt_sk_init(C.byref(P), C.byref(A), C.byref(S), self.stream()), "drift_pt_sk_init")
        self.tried.zero_()
        self.accepted.zero_()
        self.rounds_done = 0

    def run(self, n_rounds: int, history: bool = False):
        self.best_history = (self.torch.zeros(max(n_rounds, 1), dtype=self.torch.int64, device=self.device)
                             if history else None)
        P, A, S = self._problem(), self._args(n_rounds), self._state()
        _lib.check(_bind().drift_pt_sk_run(C.byref(P), C.byref(A), C.byref(S), C.c_void_p(self.workspace.data_ptr()),
                                           self.workspace.numel(), self.stream()), "drift_pt_sk_run")
        self.rounds_done += n_rounds

    def check(self):
        self.torch.cuda.synchronize(self.device)
        if int(self.workspace[8:12].view(self.torch.int32).item()):
            raise _lib.EngineError(_lib.ETIMEOUT, "drift_pt_sk_run", "a bounded in-kernel wait timed out")

    def energies(self, spins) -> np.ndarray:
        """Exact E2 of device configurations [k][n] (int8), computed on the device."""
        spins = spins.contiguous()
        out = self.torch.empty(spins.shape[0], dtype=self.torch.int64, device=self.device)
        P = self._problem()
        _lib.check(_bind().drift_pt_sk_energy(C.byref(P), spins.shape[0], C.c_void_p(spins.data_ptr()),
                                              C.c_void_p(out.data_ptr()), self.stream()), "drift_pt_sk_energy")
        return out.cpu().numpy()

    def fetch(self) -> dict:
        R = self.R
        return {
            "spins": self.spins.cpu().numpy(),
            "best_spins": self.best_spins.cpu().numpy(),
            "energy": self.energy.cpu().numpy(),
            "best_energy": self.best_energy.cpu().numpy(),
            "rung_of_slot": self.rung_of_slot.cpu().numpy(),
            "slot_of_rung": self.slot_of_rung.cpu().numpy(),
            "tried": self.tried.cpu().numpy()[: R - 1],
            "accepted": self.accepted.cpu().numpy()[: R - 1],
            "best_history": self.best_history.cpu().numpy() if self.best_history is not None else None,
        }
