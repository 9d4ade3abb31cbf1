"""Bit-packed (multispin) parallel tempering on any graph with +-1 couplings and no field
(include/drift_pt.h, graph multispin layer): 32 replicas per 32-bit word, one CTA per word with its
state in shared memory, colour-ordered sweeps, exact energies, adjacent-rung exchange.

For models like MaxCut on sparse graphs (J = -1 on edges) with a multiple of 32 replicas this
layer does the work of a colour phase for 32 replicas with one word operation per bond instead of
one per bond and replica.
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .engine import HostProblem, _ptr


class GmsLayoutInfoC(C.Structure):
    _fields_ = [("n", C.c_int32), ("n_pos", C.c_int32), ("n_colors", C.c_int32), ("max_degree", C.c_int32),
                ("n_bonds", C.c_int64), ("max_class", C.c_int32), ("reserved", C.c_int32)]


class GmsLayoutC(C.Structure):
    _fields_ = [("color_ptr", C.c_void_p), ("ell_nbr", C.c_void_p), ("degree", C.c_void_p), ("jneg", C.c_void_p),
                ("pos_of_site", C.c_void_p), ("site_of_pos", C.c_void_p)]


class GmsProblemC(C.Structure):
    _fields_ = [("n", C.c_int32), ("n_pos", C.c_int32), ("n_colors", C.c_int32), ("max_degree", C.c_int32),
                ("n_bonds", C.c_int64), ("max_class", C.c_int32), ("reserved", C.c_int32), ("color_ptr", C.c_void_p),
                ("ell_nbr", C.c_void_p), ("degree", C.c_void_p),
                ("jneg", C.c_void_p)]


class GmsStateC(C.Structure):
    _fields_ = [("words", C.c_void_p), ("best_words", C.c_void_p), ("energy", C.c_void_p),
                ("best_energy", C.c_void_p), ("rung_of_slot", C.c_void_p), ("slot_of_rung", C.c_void_p),
                ("swap_tried", C.c_void_p), ("swap_accepted", C.c_void_p)]


class GmsRunArgsC(C.Structure):
    _fields_ = [("n_words", C.c_int32), ("n_rounds", C.c_int32), ("sweeps_per_round", C.c_int32),
                ("threads_per_cta", C.c_int32), ("round_offset", C.c_int64), ("seed", C.c_uint64),
                ("instance", C.c_uint32), ("cluster_size", C.c_int32), ("betas", C.c_void_p), ("thresholds", C.c_void_p),
                ("timeout_s", C.c_double)]


def _bind():
    L = _lib.load()
    if not getattr(L, "_gms_bound", False):
        vp = C.c_void_p
        L.drift_pt_gms_layout_query.argtypes = [C.POINTER(_lib.Csr), C.POINTER(GmsLayoutInfoC)]
        L.drift_pt_gms_layout_fill.argtypes = [C.POINTER(_lib.Csr), C.POINTER(GmsLayoutC)]
        L.drift_pt_gms_workspace_bytes.argtypes = [C.c_int32, C.POINTER(C.c_size_t)]
        L.drift_pt_gms_init.argtypes = [C.POINTER(GmsProblemC), C.POINTER(GmsRunArgsC), C.POINTER(GmsStateC), vp]
        L.drift_pt_gms_run.argtypes = [C.POINTER(GmsProblemC), C.POINTER(GmsRunArgsC), C.POINTER(GmsStateC), vp,
                                       C.c_size_t, vp]
        L._gms_bound = True
    return L


class GmsLayout:
    """Host layout of a +-1 graph: positions in colour order, neighbour table, coupling signs."""

    def __init__(self, hp: HostProblem):
        L = _bind()
        csr = hp.c_csr()
        info = GmsLayoutInfoC()
        _lib.check(L.drift_pt_gms_layout_query(C.byref(csr), C.byref(info)), "drift_pt_gms_layout_query")
        self.n, self.n_pos, self.n_colors, self.max_degree, self.n_bonds = (info.n, info.n_pos, info.n_colors,
                                                                             info.max_degree, info.n_bonds)
        self.max_class = info.max_class
        self.color_ptr = np.zeros(self.n_colors + 1, np.int32)
        self.ell_nbr = np.zeros((self.max_degree, self.n_pos), np.int32)
        self.degree = np.zeros(self.n_pos, np.uint8)
        self.jneg = np.zeros(self.n_pos, np.uint8)
        self.pos_of_site = np.zeros(self.n, np.int32)
        self.site_of_pos = np.zeros(self.n_pos, np.int32)
        out = GmsLayoutC(_ptr(self.color_ptr), _ptr(self.ell_nbr), _ptr(self.degree), _ptr(self.jneg),
                         _ptr(self.pos_of_site), _ptr(self.site_of_pos))
        _lib.check(L.drift_pt_gms_layout_fill(C.byref(csr), C.byref(out)), "drift_pt_gms_layout_fill")

    @classmethod
    def from_model(cls, model) -> "GmsLayout":
        return cls(HostProblem.from_model(model))


class GmsEngine:
    """R = 32 W replicas of a GmsLayout on a beta ladder; state on the device."""

    def __init__(self, lay: GmsLayout, betas, *, seed: int = 0, sweeps_per_round: int = 1, instance: int = 0,
                 threads_per_cta: int = 0, cluster_size: int = 0, device="cuda", timeout_s: float = 10.0):
        import torch

        self.torch = torch
        self.lay = lay
        self.betas = np.ascontiguousarray(betas, np.float64)
        R = len(self.betas)
        if R % 32 or R < 32:
            raise ValueError("the multispin engine needs a multiple of 32 replicas")
        self.R, self.W = R, R // 32
        self.seed, self.spr, self.instance = int(seed), int(sweeps_per_round), int(instance)
        self.threads, self.cluster, self.timeout_s = int(threads_per_cta), int(cluster_size), float(timeout_s)
        L = _bind()
        dev = self.device = torch.device(device)
        thr = np.zeros(R * lay.max_degree, np.uint32)
        _lib.check(L.drift_pt_thresholds(R, _ptr(self.betas), lay.max_degree, _ptr(thr)), "thresholds")
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
        self.d_thr = t(thr.view(np.int32))
        self.d_betas = t(self.betas)
        self.d_color_ptr, self.d_ell = t(lay.color_ptr), t(lay.ell_nbr)
        self.d_degree, self.d_jneg = t(lay.degree), t(lay.jneg)
        self.words = torch.empty(self.W * lay.n_pos, dtype=torch.int32, device=dev)
        self.best_words = torch.empty(self.W * lay.n_pos, dtype=torch.int32, device=dev)
        self.energy = torch.empty(R, dtype=torch.int64, device=dev)
        self.best_energy = torch.empty(R, dtype=torch.int64, device=dev)
        self.rung_of_slot = torch.empty(R, dtype=torch.int32, device=dev)
        self.slot_of_rung = torch.empty(R, dtype=torch.int32, device=dev)
        self.tried = torch.zeros(R, dtype=torch.int64, device=dev)
        self.accepted = torch.zeros(R, dtype=torch.int64, device=dev)
        ws = C.c_size_t(0)
        _lib.check(L.drift_pt_gms_workspace_bytes(self.W, C.byref(ws)), "drift_pt_gms_workspace_bytes")
        self.workspace = torch.zeros(ws.value, dtype=torch.uint8, device=dev)
        self.rounds_done = 0

    def _c(self, n_rounds):
        lay = self.lay
        P = GmsProblemC(lay.n, lay.n_pos, lay.n_colors, lay.max_degree, lay.n_bonds, lay.max_class, 0,
                        self.d_color_ptr.data_ptr(),
                        self.d_ell.data_ptr(), self.d_degree.data_ptr(), self.d_jneg.data_ptr())
        A = GmsRunArgsC(self.W, n_rounds, self.spr, self.threads, self.rounds_done, self.seed & 0xFFFFFFFFFFFFFFFF,
                        self.instance, self.cluster, self.d_betas.data_ptr(), self.d_thr.data_ptr(), self.timeout_s)
        S = GmsStateC(self.words.data_ptr(), self.best_words.data_ptr(), self.energy.data_ptr(),
                      self.best_energy.data_ptr(), self.rung_of_slot.data_ptr(), self.slot_of_rung.data_ptr(),
                      self.tried.data_ptr(), self.accepted.data_ptr())
        return P, A, S

    def stream(self):
        return C.c_void_p(self.torch.cuda.current_stream(self.device).cuda_stream)

    def init(self):
        P, A, S = self._c(0)
        _lib.check(_bind().drift_pt_gms_init(C.byref(P), C.byref(A), C.byref(S), self.stream()), "drift_pt_gms_init")
        self.tried.zero_()
        self.accepted.zero_()
        self.rounds_done = 0

    def run(self, n_rounds: int):
        P, A, S = self._c(n_rounds)
        _lib.check(_bind().drift_pt_gms_run(C.byref(P), C.byref(A), C.byref(S), C.c_void_p(self.workspace.data_ptr()),
                                            self.workspace.numel(), self.stream()), "drift_pt_gms_run")
        self.rounds_done += n_rounds

    def check(self):
        self.torch.cuda.synchronize(self.device)
        code = int(self.workspace[8:12].view(self.torch.int32).item())
        if code == _lib.ETIMEOUT:
            raise _lib.EngineError(code, "drift_pt_gms_run", "a bounded in-kernel wait timed out")
        if code:
            raise _lib.EngineError(code, "drift_pt_gms_run", "the device layout is inconsistent (colour table or "
                                   "neighbour index out of range)")

    def unpack(self, words: np.ndarray) -> np.ndarray:
        """(R, n) spins +-1 in the original site order from [W][n_pos] words."""
        w = np.asarray(words).view(np.uint32).reshape(self.W, self.lay.n_pos)
        bits = (w[:, None, :] >> np.arange(32, dtype=np.uint32)[None, :, None]) & 1
        s = (1 - 2 * bits.astype(np.int8)).reshape(self.R, self.lay.n_pos)
        return s[:, self.lay.pos_of_site]

    def fetch(self) -> dict:
        words = self.words.cpu().numpy()
        best = self.best_words.cpu().numpy()
        return {
            "words": words.view(np.uint32).reshape(self.W, self.lay.n_pos),
            "best_words": best.view(np.uint32).reshape(self.W, self.lay.n_pos),
            "spins": self.unpack(words), "best_spins": self.unpack(best),
            "energy": self.energy.cpu().numpy(), "best_energy": self.best_energy.cpu().numpy(),
            "rung_of_slot": self.rung_of_slot.cpu().numpy(), "slot_of_rung": self.slot_of_rung.cpu().numpy(),
            "tried": self.tried.cpu().numpy()[: self.R - 1], "accepted": self.accepted.cpu().numpy()[: self.R - 1],
        }
