"""Neural-proposal parallel tempering on a batch of instances (integer couplings): the batched plain-PT
engine (drift_b200.batch) plus, for every instance that has a proposal network, whole-configuration
proposals at its n_cold coldest rungs after every round. Each proposal is accepted by the exact
Metropolis-Hastings test of drift_pt_batch_mh (energies recomputed exactly on the device, log-ratio
in double), so every rung keeps plain PT's Boltzmann distribution. Instances without a network run
plain PT only, the method's fallback.

Networks are independent MADEs (drift_b200.made), one per instance of at most 512 spins (the
sampler's limit), trained on configurations the batch itself samples at the coldest rungs. All the
networks of a batch evaluate and draw in one launch each (drift_pt_made_group_run); the gather of
the current configurations and the MH step are one launch each, whatever the number of instances.
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .batch import BatchEngine
from .made import Made, MadeNetC

MAX_NET_SPINS = 512


def _bind():
    L = _lib.load()
    if not getattr(L, "_bmh_bound", False):
        vp = C.c_void_p
        L.drift_pt_made_group_bytes.argtypes = [C.c_int32, C.POINTER(C.c_size_t)]
        L.drift_pt_made_group_fill.argtypes = [C.c_int32, C.POINTER(MadeNetC), vp, C.c_int32, vp, vp, C.c_uint64,
                                               vp, vp]
        L.drift_pt_made_group_run.argtypes = [vp, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_uint32,
                                              vp]
        L.drift_pt_batch_gather.argtypes = [C.POINTER(_lib.BatchProblem), C.POINTER(_lib.DeviceState), C.c_int32,
                                            vp, vp, vp, vp, vp, vp, C.c_int64, vp, vp, vp]
        L.drift_pt_batch_mh.argtypes = [C.POINTER(_lib.BatchProblem), C.POINTER(_lib.DeviceState), C.c_uint64,
                                        C.c_int32, vp, vp, vp, vp, vp, vp, vp, vp, C.c_int64, vp, vp, vp, vp, vp, vp]
        L._bmh_bound = True
    return L


def default_hidden(n: int) -> int:
    """Hidden width of an instance's network: 2n, a multiple of 8, at most 1024 and at most
    4 (n - 1) (the sampler's units-per-degree bound)."""
    h = min(1024, 2 * n, 4 * (n - 1))
    return max(8, h - h % 8)


class BatchNeuralPT:
    """A BatchEngine plus one Made per instance in `nets` ({instance index: Made}); `propose(r)`
    offers every networked instance a fresh draw at each of its n_cold coldest rungs."""

    def __init__(self, eng: BatchEngine, nets: dict, *, n_cold: int = 8):
        torch = self.torch = eng.torch
        self.eng, self.bp = eng, eng.bp
        bp = self.bp
        dev = self.device = bp.device
        self.nets = dict(nets)
        self.ks = sorted(self.nets)
        self.n_cold = int(n_cold)
        K = bp.n_instances
        n_of = [int(d["n"]) for d in bp.desc]
        R_of = [int(d["n_replicas"]) for d in bp.desc]
        if not self.ks:
            raise ValueError("no instance has a network")
        for k in self.ks:
            m = self.nets[k]
            if not 0 <= k < K:
                raise ValueError(f"network for instance {k} outside the batch")
            if m.n != n_of[k]:
                raise ValueError(f"instance {k}: network has {m.n} spins, the instance {n_of[k]}")
            if self.n_cold > R_of[k]:
                raise ValueError(f"instance {k}: n_cold {n_cold} exceeds its {R_of[k]} rungs")
        site_off = np.zeros(K, np.int64)
        site_off[1:] = np.cumsum(n_of)[:-1]
        inst, rung, off = [], [], []
        o = 0
        self.row0 = {}  # first request of instance k
        for k in self.ks:
            self.row0[k] = len(inst)
            for c in range(self.n_cold):
                inst.append(k)
                rung.append(R_of[k] - self.n_cold + c)
                off.append(o)
                o += n_of[k]
        self.count = len(inst)
        self.inst_h, self.rung_h, self.off_h = (np.array(inst, np.int32), np.array(rung, np.int32),
                                                np.array(off, np.int64))
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
        self.d_inst, self.d_rung, self.d_off = t(self.inst_h), t(self.rung_h), t(self.off_h)
        self.d_site_off = t(site_off)
        self.d_pos_of_site = t(np.concatenate([np.asarray(p, np.int32) for p in bp.pos_of_site]))
        self.x_prop = torch.zeros(o, dtype=torch.int8, device=dev)
        self.x_cur = torch.zeros(o, dtype=torch.int8, device=dev)
        self.lq_prop = torch.zeros(self.count, dtype=torch.float32, device=dev)
        self.lq_cur = torch.zeros(self.count, dtype=torch.float32, device=dev)
        self.prop_energy = torch.zeros(self.count, dtype=torch.int64, device=dev)
        self.tried = torch.zeros(self.count, dtype=torch.int64, device=dev)
        self.accepted = torch.zeros(self.count, dtype=torch.int64, device=dev)
        self.scratch = torch.zeros(self.count * bp.max_n_pos, dtype=torch.int8, device=dev)
        self.err = torch.zeros(1, dtype=torch.int32, device=dev)
        self.seed = eng.seed ^ 0x5EED
        self.tables = None

    # ------------------------------------------------------------------ plumbing
    def _ps(self):
        return self.bp.c_problem(), self.eng._state()

    def _tables(self):
        """Group tables of the networks (draw and evaluate). The weights are updated in place by
        training, so the tables stay valid once built."""
        if self.tables is not None:
            return self.tables
        L = _bind()
        torch = self.torch
        G = len(self.ks)
        nets = (MadeNetC * G)(*[self.nets[k].net_c() for k in self.ks])
        counts = np.full(G, self.n_cold, np.int32)
        xs_p = (C.c_void_p * G)(*[self.x_prop.data_ptr() + int(self.off_h[self.row0[k]]) for k in self.ks])
        xs_c = (C.c_void_p * G)(*[self.x_cur.data_ptr() + int(self.off_h[self.row0[k]]) for k in self.ks])
        lq_p = (C.c_void_p * G)(*[self.lq_prop.data_ptr() + 4 * self.row0[k] for k in self.ks])
        lq_c = (C.c_void_p * G)(*[self.lq_cur.data_ptr() + 4 * self.row0[k] for k in self.ks])
        streams = np.arange(G, dtype=np.uint32)
        nb = C.c_size_t(0)
        _lib.check(L.drift_pt_made_group_bytes(G, C.byref(nb)), "drift_pt_made_group_bytes")
        tab_s = torch.zeros(nb.value, dtype=torch.uint8, device=self.device)
        tab_e = torch.zeros(nb.value, dtype=torch.uint8, device=self.device)
        _lib.check(L.drift_pt_made_group_fill(G, nets, counts.ctypes.data, 0, xs_p, lq_p, self.seed & 0xFFFFFFFFFFFFFFFF,
                                              streams.ctypes.data, C.c_void_p(tab_s.data_ptr())),
                   "drift_pt_made_group_fill")
        _lib.check(L.drift_pt_made_group_fill(G, nets, counts.ctypes.data, 1, xs_c, lq_c, 0, None,
                                              C.c_void_p(tab_e.data_ptr())), "drift_pt_made_group_fill")
        m = [self.nets[k] for k in self.ks]
        self.sizes = (max(x.n for x in m), max(x.h1 for x in m), max(x.h2 for x in m))
        self.tables = (tab_s, tab_e)
        return self.tables

    # ------------------------------------------------------------------ data
    def gather(self, out, out_off, out_step=None, rep: int = 0):
        """Configurations at every request's (instance, rung), site order, into out + out_off[j] +
        rep * out_step[j] (device int64 arrays)."""
        P, S = self._ps()
        _lib.check(_bind().drift_pt_batch_gather(
            C.byref(P), C.byref(S), self.count, C.c_void_p(self.d_inst.data_ptr()), C.c_void_p(self.d_rung.data_ptr()),
            C.c_void_p(self.d_site_off.data_ptr()), C.c_void_p(self.d_pos_of_site.data_ptr()),
            C.c_void_p(out_off.data_ptr()), C.c_void_p(out_step.data_ptr()) if out_step is not None else None,
            int(rep), C.c_void_p(out.data_ptr()), C.c_void_p(self.err.data_ptr()), self.eng.stream()),
            "drift_pt_batch_gather")

    def collect(self, n_rounds: int) -> dict:
        """Run n_rounds plain rounds and keep the n_cold coldest configurations of every networked
        instance after each: {instance: int8 [n_rounds * n_cold][n] device tensor} (training sets)."""
        torch = self.torch
        n_of = {k: int(self.bp.desc[k]["n"]) for k in self.ks}
        base, o = {}, 0
        for k in self.ks:
            base[k] = o
            o += n_rounds * self.n_cold * n_of[k]
        data = torch.empty(o, dtype=torch.int8, device=self.device)
        off = np.array([base[k] + c * n_of[k] for k in self.ks for c in range(self.n_cold)], np.int64)
        step = np.array([self.n_cold * n_of[k] for k in self.ks for _ in range(self.n_cold)], np.int64)
        d_off, d_step = torch.from_numpy(off).to(self.device), torch.from_numpy(step).to(self.device)
        for r in range(n_rounds):
            self.eng.run(1)
            self.gather(data, d_off, d_step, rep=r)
        self.check()
        return {k: data[base[k]: base[k] + n_rounds * self.n_cold * n_of[k]].view(n_rounds * self.n_cold, n_of[k])
                for k in self.ks}

    # ------------------------------------------------------------------ proposals
    def propose(self, round_index: int):
        """One proposal per request: log q of the current configurations, fresh draws, exact MH."""
        L = _bind()
        tab_s, tab_e = self._tables()
        G = len(self.ks)
        mn, mh1, mh2 = self.sizes
        st = self.eng.stream()
        self.gather(self.x_cur, self.d_off)
        _lib.check(L.drift_pt_made_group_run(C.c_void_p(tab_e.data_ptr()), G, self.n_cold, mn, mh1, mh2, 0, st),
                   "drift_pt_made_group_run")
        _lib.check(L.drift_pt_made_group_run(C.c_void_p(tab_s.data_ptr()), G, self.n_cold, mn, mh1, mh2,
                                             (round_index * G) & 0xFFFFFFFF, st), "drift_pt_made_group_run")
        self.mh(round_index)

    def mh(self, round_index: int):
        """The exact MH step for the proposals in x_prop (log q values lq_prop) against the current
        configurations' lq_cur."""
        P, S = self._ps()
        _lib.check(_bind().drift_pt_batch_mh(
            C.byref(P), C.byref(S), self.seed & 0xFFFFFFFFFFFFFFFF, self.count, C.c_void_p(self.d_inst.data_ptr()),
            C.c_void_p(self.d_rung.data_ptr()), C.c_void_p(self.d_site_off.data_ptr()),
            C.c_void_p(self.d_pos_of_site.data_ptr()), C.c_void_p(self.d_off.data_ptr()),
            C.c_void_p(self.x_prop.data_ptr()), C.c_void_p(self.lq_prop.data_ptr()), C.c_void_p(self.lq_cur.data_ptr()),
            int(round_index), C.c_void_p(self.scratch.data_ptr()), C.c_void_p(self.prop_energy.data_ptr()),
            C.c_void_p(self.tried.data_ptr()), C.c_void_p(self.accepted.data_ptr()), C.c_void_p(self.err.data_ptr()),
            self.eng.stream()), "drift_pt_batch_mh")

    def run(self, n_rounds: int):
        """n_rounds of (one plain round of every instance, then one proposal per request)."""
        for _ in range(n_rounds):
            r = self.eng.rounds_done
            self.eng.run(1)
            self.propose(r)

    def check(self):
        self.eng.check()
        if int(self.err.item()):
            raise _lib.EngineError(_lib.EINVAL, "drift_pt_batch_mh", "a proposal request is out of range")

    def acceptance(self) -> dict:
        """{instance: accepted / tried over its requests} (NaN where none were tried)."""
        t = self.tried.cpu().numpy().astype(np.float64)
        a = self.accepted.cpu().numpy().astype(np.float64)
        out = {}
        for k in self.ks:
            j0 = self.row0[k]
            tt, aa = t[j0:j0 + self.n_cold].sum(), a[j0:j0 + self.n_cold].sum()
            out[k] = aa / tt if tt else float("nan")
        return out


def make_nets(bp, *, seed: int = 0, max_spins: int = MAX_NET_SPINS, hidden=None) -> dict:
    """One untrained Made per instance of at most max_spins spins (n a multiple of 8)."""
    nets = {}
    for k, d in enumerate(bp.desc):
        n = int(d["n"])
        if 8 <= n <= max_spins and n % 8 == 0:
            h = hidden(n) if hidden else default_hidden(n)
            nets[k] = Made(n, hidden=(h, h), seed=seed + k, device=bp.device)
    return nets
