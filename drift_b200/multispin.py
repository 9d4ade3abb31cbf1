"""Multispin (bit-packed) parallel tempering on +-J cubic lattices (include/drift_pt.h, multispin
layer): 32 replicas per 32-bit word, checkerboard sweeps, exact energies, adjacent-rung exchange.

For lattices far beyond what a dense IsingModel can hold (a 3-D L = 64 lattice has 262,144 spins;
its dense J would take 550 GB), ``Lattice.edwards_anderson`` builds the couplings directly, with the
same random draws as ``drift_b200.instances.ea_2d`` / ``ea_3d``.
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .engine import _ptr


class LatticeC(C.Structure):
    _fields_ = [("dims", C.c_int32), ("L", C.c_int32), ("jneg", C.c_void_p)]


class MsStateC(C.Structure):
    _fields_ = [("words", C.c_void_p), ("best_words", C.c_void_p), ("energy", C.c_void_p),
                ("best_energy", C.c_void_p), ("rung_of_slot", C.c_void_p), ("slot_of_rung", C.c_void_p),
                ("swap_tried", C.c_void_p), ("swap_accepted", C.c_void_p)]


class MsRunArgsC(C.Structure):
    _fields_ = [("n_words", C.c_int32), ("n_rounds", C.c_int32), ("sweeps_per_round", C.c_int32),
                ("ctas_per_sm", C.c_int32), ("round_offset", C.c_int64), ("seed", C.c_uint64),
                ("instance", C.c_uint32), ("reserved", C.c_int32), ("betas", C.c_void_p),
                ("thresholds", C.c_void_p), ("timeout_s", C.c_double)]


def _bind():
    L = _lib.load()
    if not getattr(L, "_ms_bound", False):
        L.drift_pt_ms_workspace_bytes.argtypes = [C.c_int32, C.POINTER(C.c_size_t)]
        L.drift_pt_ms_workspace_bytes.restype = C.c_int
        L.drift_pt_ms_init.argtypes = [C.POINTER(LatticeC), C.POINTER(MsRunArgsC), C.POINTER(MsStateC), C.c_void_p]
        L.drift_pt_ms_init.restype = C.c_int
        L.drift_pt_ms_run.argtypes = [C.POINTER(LatticeC), C.POINTER(MsRunArgsC), C.POINTER(MsStateC), C.c_void_p,
                                      C.c_size_t, C.c_void_p]
        L.drift_pt_ms_run.restype = C.c_int
        L._ms_bound = True
    return L


class Lattice:
    """+-J couplings of a d-dimensional periodic cubic lattice (d = 2, 3; even L; no field), stored
    as one byte per site in colour-split order: bit d set when J(site, site + e_d) = -1."""

    def __init__(self, dims: int, L: int, jneg_by_site: np.ndarray):
        if dims not in (2, 3) or L < 4 or L % 2:
            raise ValueError("dims must be 2 or 3 and L even >= 4")
        self.dims, self.L = dims, L
        self.n = L ** dims
        idx = np.arange(self.n)
        x, y = idx % L, (idx // L) % L
        z = idx // (L * L) if dims == 3 else np.zeros_like(idx)
        colour = (x + y + z) & 1
        self.q_of_site = (colour * (self.n // 2) + (x >> 1) + (L // 2) * (y + L * z)).astype(np.int64)
        self.site_of_q = np.empty(self.n, np.int64)
        self.site_of_q[self.q_of_site] = idx
        jb = np.asarray(jneg_by_site, np.uint8)
        if jb.shape != (self.n,):
            raise ValueError("one coupling byte per site")
        self.jneg = np.ascontiguousarray(jb[self.site_of_q])

    @classmethod
    def edwards_anderson(cls, dims: int, L: int, seed: int) -> "Lattice":
        """+-J with p = 1/2: the draws of drift_b200.instances.ea_2d / ea_3d (bond +x of every site,
        then +y, then +z)."""
        rng = np.random.default_rng(seed)
        n = L ** dims
        w = rng.integers(0, 2, size=dims * n) * 2.0 - 1.0
        jb = np.zeros(n, np.uint8)
        for d in range(dims):
            jb |= ((w[d * n:(d + 1) * n] < 0).astype(np.uint8) << d)
        return cls(dims, L, jb)

    def couplings(self):
        """(i, j, J) bond list in natural site order (x + L (y + L z))."""
        L, n = self.L, self.n
        idx = np.arange(n)
        x, y = idx % L, (idx // L) % L
        z = idx // (L * L) if self.dims == 3 else np.zeros_like(idx)
        jb = self.jneg[self.q_of_site]
        nbs = [((x + 1) % L) + L * (y + L * z), x + L * (((y + 1) % L) + L * z), x + L * (y + L * ((z + 1) % L))]
        i = np.concatenate([idx] * self.dims)
        j = np.concatenate(nbs[: self.dims])
        J = np.concatenate([np.where((jb >> d) & 1, -1.0, 1.0) for d in range(self.dims)])
        return i, j, J

    def energy(self, spins: np.ndarray) -> np.ndarray:
        """E = -sum_bonds J s_i s_j for spins (..., n) in natural site order."""
        i, j, J = self.couplings()
        s = np.asarray(spins, np.float64)
        return -(s[..., i] * s[..., j] * J).sum(axis=-1)


class MsEngine:
    """R = 32 W replicas of a Lattice on a beta ladder, state on the device."""

    def __init__(self, lat: Lattice, betas, *, seed: int = 0, sweeps_per_round: int = 1, instance: int = 0,
                 device="cuda", ctas_per_sm: int = 0, timeout_s: float = 10.0):
        import torch

        self.torch = torch
        self.lat = lat
        self.betas = np.ascontiguousarray(betas, np.float64)
        R = len(self.betas)
        if R % 32 or R < 32:
            raise ValueError("the multispin engine needs a multiple of 32 replicas")
        self.R, self.W = R, R // 32
        self.seed, self.spr, self.instance = int(seed), int(sweeps_per_round), int(instance)
        self.ctas_per_sm, self.timeout_s = int(ctas_per_sm), float(timeout_s)
        L = _bind()
        dev = self.device = torch.device(device)
        thr = np.zeros(R * 2 * lat.dims, np.uint32)
        _lib.check(L.drift_pt_thresholds(R, _ptr(self.betas), 2 * lat.dims, _ptr(thr)), "thresholds")
        self.d_thr = torch.from_numpy(thr.view(np.int32)).to(dev)
        self.d_betas = torch.from_numpy(self.betas).to(dev)
        self.d_jneg = torch.from_numpy(lat.jneg).to(dev)
        N = lat.n
        self.words = torch.empty(self.W * N, dtype=torch.int32, device=dev)
        self.best_words = torch.empty(self.W * N, dtype=torch.int32, device=dev)
        self.energy = torch.empty(R, dtype=torch.int64, device=dev)
        self.best_energy = torch.empty(R, dtype=torch.int64, device=dev)
        self.rung_of_slot = torch.empty(R, dtype=torch.int32, device=dev)
        self.slot_of_rung = torch.empty(R, dtype=torch.int32, device=dev)
        self.tried = torch.zeros(R, dtype=torch.int64, device=dev)
        self.accepted = torch.zeros(R, dtype=torch.int64, device=dev)
        ws = C.c_size_t(0)
        _lib.check(L.drift_pt_ms_workspace_bytes(self.W, C.byref(ws)), "ms_workspace_bytes")
        self.workspace = torch.zeros(ws.value, dtype=torch.uint8, device=dev)
        self.rounds_done = 0

    def _c(self, n_rounds):
        lat = LatticeC(self.lat.dims, self.lat.L, self.d_jneg.data_ptr())
        args = MsRunArgsC(self.W, n_rounds, self.spr, self.ctas_per_sm, self.rounds_done,
                          self.seed & 0xFFFFFFFFFFFFFFFF, self.instance, 0, self.d_betas.data_ptr(),
                          self.d_thr.data_ptr(), self.timeout_s)
        st = MsStateC(self.words.data_ptr(), self.best_words.data_ptr(), self.energy.data_ptr(),
                      self.best_energy.data_ptr(), self.rung_of_slot.data_ptr(), self.slot_of_rung.data_ptr(),
                      self.tried.data_ptr(), self.accepted.data_ptr())
        return lat, args, st

    def stream(self):
        return C.c_void_p(self.torch.cuda.current_stream(self.device).cuda_stream)

    def init(self):
        L = _bind()
        lat, args, st = self._c(0)
        _lib.check(L.drift_pt_ms_init(C.byref(lat), C.byref(args), C.byref(st), self.stream()), "drift_pt_ms_init")
        self.rounds_done = 0

    def run(self, n_rounds: int):
        L = _bind()
        lat, args, st = self._c(n_rounds)
        _lib.check(L.drift_pt_ms_run(C.byref(lat), C.byref(args), C.byref(st), C.c_void_p(self.workspace.data_ptr()),
                                     self.workspace.numel(), self.stream()), "drift_pt_ms_run")
        self.rounds_done += n_rounds

    def check(self):
        self.torch.cuda.synchronize(self.device)
        if int(self.workspace[8:12].view(self.torch.int32).item()):
            raise _lib.EngineError(_lib.ETIMEOUT, "drift_pt_ms_run", "a bounded in-kernel wait timed out")

    def _unpack(self, words: np.ndarray) -> np.ndarray:
        """(R, n) spins +-1 in natural site order from [W][N] words."""
        w = words.reshape(self.W, self.lat.n).view(np.uint32)
        bits = (w[:, None, :] >> np.arange(32, dtype=np.uint32)[None, :, None]) & 1  # (W, 32, N)
        s = (1 - 2 * bits.astype(np.int8)).reshape(self.R, self.lat.n)
        return s[:, self.lat.q_of_site]

    def fetch(self) -> dict:
        return {
            "words": self.words.cpu().numpy().view(np.uint32).reshape(self.W, self.lat.n),
            "best_words": self.best_words.cpu().numpy().view(np.uint32).reshape(self.W, self.lat.n),
            "spins": self._unpack(self.words.cpu().numpy()),
            "best_spins": self._unpack(self.best_words.cpu().numpy()),
            "energy": self.energy.cpu().numpy(),
            "best_energy": self.best_energy.cpu().numpy(),
            "rung_of_slot": self.rung_of_slot.cpu().numpy(),
            "slot_of_rung": self.slot_of_rung.cpu().numpy(),
            "tried": self.tried.cpu().numpy()[: self.R - 1],
            "accepted": self.accepted.cpu().numpy()[: self.R - 1],
        }
