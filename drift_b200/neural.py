"""Neural-proposal parallel tempering on dense models: plain PT rounds of the dense-coupling engine
(drift_b200.sk) alternated with proposals from a trained MADE (drift_b200.made) at the coldest rungs,
each accepted by the exact Metropolis-Hastings test of drift_pt_made_mh.

Two kinds of proposal: independent whole configurations x' ~ q, or (``suffix=m``) conditional ones
that keep a replica's first n - m spins and redraw the last m from q's conditionals given them. For
both, the test's ratio is q(x) / q(x') (for the conditional proposal the kept spins' factors of q
cancel between the forward and the reverse move). Energies are exact integers, so the stationary
distribution of every rung is the same Boltzmann distribution as plain PT's, and plain PT remains
the fallback between proposals.
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .made import Made
from .sk import SkEngine, SkModel


def _bind():
    L = _lib.load()
    if not getattr(L, "_mh_bound", False):
        from .sk import SkProblemC, SkRunArgsC, SkStateC

        vp = C.c_void_p
        L.drift_pt_made_mh.argtypes = [C.POINTER(SkProblemC), C.POINTER(SkRunArgsC), C.POINTER(SkStateC), vp, vp, vp,
                                       vp, vp, vp, vp, C.c_int64, vp]
        L.drift_pt_made_mh.restype = C.c_int
        L._mh_bound = True
    return L


def collect_cold_samples(eng: SkEngine, n_samples: int, n_cold: int = 8):
    """Run plain PT rounds and keep the configurations of the n_cold coldest rungs after each round:
    an int8 [n_samples][n] device tensor (the training set of the proposal network)."""
    torch = eng.torch
    R = eng.R
    out = torch.empty((n_samples, eng.model.n), dtype=torch.int8, device=eng.device)
    got = 0
    while got < n_samples:
        eng.run(1)
        slots = eng.slot_of_rung[R - n_cold:].long()
        take = min(n_cold, n_samples - got)
        out[got:got + take] = eng.spins.index_select(0, slots[:take])
        got += take
    eng.check()
    return out


class NeuralPT:
    """An SkEngine plus a Made: `run(n)` does n rounds of (sweeps_per_round plain sweeps, then one
    proposal per replica at the n_cold coldest rungs)."""

    def __init__(self, model: SkModel, betas, made: Made, *, seed: int = 0, sweeps_per_round: int = 10,
                 n_cold: int = 8, replicas_per_cta: int = 0, instance: int = 0, device="cuda",
                 engine: SkEngine | None = None, suffix: int | None = None):
        # `engine`: continue an existing plain-PT run (e.g. the one whose samples trained `made`)
        self.eng = engine or SkEngine(model, betas, seed=seed, sweeps_per_round=sweeps_per_round, instance=instance,
                                      replicas_per_cta=replicas_per_cta, device=device)
        self.made = made
        self.n_cold = n_cold
        if suffix is not None and not 1 <= suffix <= model.n:
            raise ValueError("suffix must be in [1, n]")
        self.suffix = suffix  # None: independent proposals; m: redraw the last m spins
        torch = self.torch = self.eng.torch
        R = self.eng.R
        self.prop_tried = torch.zeros(R, dtype=torch.int64, device=self.eng.device)
        self.prop_accepted = torch.zeros(R, dtype=torch.int64, device=self.eng.device)
        self.active = torch.zeros(R, dtype=torch.uint8, device=self.eng.device)

    def init(self):
        self.eng.init()
        self.prop_tried.zero_()
        self.prop_accepted.zero_()

    def propose(self, round_index: int):
        eng, made = self.eng, self.made
        R = eng.R
        if self.suffix is None:
            xp, lq_p = made.sample(R, seed=eng.seed ^ 0x5EED, stream_id=round_index)
        else:
            xp = eng.spins.clone()
            lq_p = made.sample_suffix(xp, made.n - self.suffix, seed=eng.seed ^ 0x5EED, stream_id=round_index)
        lq_c = made.logq(eng.spins)
        e_p = self.torch.empty(R, dtype=self.torch.int64, device=eng.device)
        P = eng._problem()
        _lib.check(_lib.load().drift_pt_sk_energy(C.byref(P), R, C.c_void_p(xp.data_ptr()), C.c_void_p(e_p.data_ptr()),
                                                  eng.stream()), "drift_pt_sk_energy")
        self.active.copy_((eng.rung_of_slot >= R - self.n_cold).to(self.torch.uint8))
        A, S = eng._args(0), eng._state()
        _lib.check(_bind().drift_pt_made_mh(C.byref(P), C.byref(A), C.byref(S), C.c_void_p(xp.data_ptr()),
                                            C.c_void_p(e_p.data_ptr()), C.c_void_p(lq_p.data_ptr()),
                                            C.c_void_p(lq_c.data_ptr()), C.c_void_p(self.active.data_ptr()),
                                            C.c_void_p(self.prop_tried.data_ptr()),
                                            C.c_void_p(self.prop_accepted.data_ptr()), round_index, eng.stream()),
                   "drift_pt_made_mh")

    def run(self, n_rounds: int):
        for _ in range(n_rounds):
            r = self.eng.rounds_done
            self.eng.run(1)
            self.propose(r)

    def acceptance(self) -> np.ndarray:
        """Accepted / tried proposals per rung (NaN where none were tried)."""
        t = self.prop_tried.cpu().numpy().astype(np.float64)
        a = self.prop_accepted.cpu().numpy().astype(np.float64)
        with np.errstate(invalid="ignore", divide="ignore"):
            return a / t
