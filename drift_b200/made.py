"""Proposal network for neural-proposal parallel tempering: a masked autoregressive MLP (MADE,
Germain et al., ICML 2015) over n spins, trained on configurations that plain PT samples at its
coldest rungs, and the exact Metropolis-Hastings step that lets its whole-configuration proposals
enter a replica (include/drift_pt.h, proposal-network section).

Everything runs on the device through the C ABI: the products of the forward and backward passes on
the tensor cores (drift_pt_gemm_bf16: BF16 operands, FP32 accumulation), the log-likelihood and its
gradient, bias sums, transposes and Adam in element-wise kernels, sampling and log q evaluation in
one kernel whose arithmetic is the same for both (so q(x') used to draw a proposal is the q the
acceptance ratio divides by).
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib


class GemmC(C.Structure):
    _fields_ = [("M", C.c_int32), ("N", C.c_int32), ("K", C.c_int32), ("lda", C.c_int32), ("ldb", C.c_int32),
                ("ldc", C.c_int32), ("act", C.c_int32), ("reserved", C.c_int32), ("A", C.c_void_p),
                ("B", C.c_void_p), ("bias", C.c_void_p), ("relu_ref", C.c_void_p), ("out_f32", C.c_void_p),
                ("out_bf16", C.c_void_p)]


class MadeNetC(C.Structure):
    _fields_ = [("n", C.c_int32), ("h1", C.c_int32), ("h2", C.c_int32), ("max_units_per_degree", C.c_int32),
                ("w1t", C.c_void_p), ("w2t", C.c_void_p), ("w3t", C.c_void_p), ("b1", C.c_void_p),
                ("b2", C.c_void_p), ("b3", C.c_void_p), ("ord1", C.c_void_p), ("off1", C.c_void_p),
                ("ord2", C.c_void_p), ("off2", C.c_void_p)]


def _bind():
    L = _lib.load()
    if not getattr(L, "_made_bound", False):
        vp, i32, i64, f32 = C.c_void_p, C.c_int32, C.c_int64, C.c_float
        L.drift_pt_gemm_bf16.argtypes = [C.POINTER(GemmC), vp, vp]
        L.drift_pt_made_loss.argtypes = [i32, i32, vp, vp, vp, vp, f32, vp]
        L.drift_pt_made_spins_to_bf16.argtypes = [i64, vp, vp, vp]
        L.drift_pt_transpose_bf16.argtypes = [i32, i32, vp, vp, vp]
        L.drift_pt_colsum_bf16.argtypes = [i32, i32, vp, vp, vp]
        L.drift_pt_adam.argtypes = [i32, i32, vp, vp, vp, vp, vp, f32, f32, f32, f32, i32, vp, vp, vp]
        L.drift_pt_made_sample.argtypes = [C.POINTER(MadeNetC), i32, i32, vp, vp, C.c_uint64, C.c_uint32, vp]
        L.drift_pt_made_sample_suffix.argtypes = [C.POINTER(MadeNetC), i32, i32, vp, vp, C.c_uint64, C.c_uint32, vp]
        for name in ("drift_pt_gemm_bf16", "drift_pt_made_loss", "drift_pt_made_spins_to_bf16",
                     "drift_pt_transpose_bf16", "drift_pt_colsum_bf16", "drift_pt_adam", "drift_pt_made_sample",
                     "drift_pt_made_sample_suffix"):
            getattr(L, name).restype = C.c_int
        L._made_bound = True
    return L


def degrees(n: int, h: int) -> np.ndarray:
    """Hidden-unit degrees 1 .. n-1, assigned cyclically (unit k: 1 + k mod (n-1))."""
    return 1 + (np.arange(h) % (n - 1))


def masks(n: int, h1: int, h2: int):
    """MADE masks: M1 [h1][n], M2 [h2][h1], M3 [n][h2] (1 = connection kept)."""
    m0 = np.arange(n) + 1
    m1, m2 = degrees(n, h1), degrees(n, h2)
    M1 = (m1[:, None] >= m0[None, :]).astype(np.uint8)
    M2 = (m2[:, None] >= m1[None, :]).astype(np.uint8)
    M3 = (m0[:, None] > m2[None, :]).astype(np.uint8)
    return M1, M2, M3


def _order(n: int, deg: np.ndarray):
    ord_ = np.argsort(deg, kind="stable").astype(np.int32)
    counts = np.bincount(deg, minlength=n + 1)[1:n + 1]  # degrees 1..n
    off = np.zeros(n + 1, np.int32)
    off[1:] = np.cumsum(counts)
    return ord_, off, int(counts.max())


class Made:
    """MADE with two hidden layers on the device; fp32 master weights, bf16 working copies."""

    def __init__(self, n: int, hidden=(1024, 1024), seed: int = 0, device="cuda"):
        import torch

        self.torch = torch
        self.n, (self.h1, self.h2) = n, hidden
        if n < 2 or n % 8 or self.h1 % 8 or self.h2 % 8:
            raise ValueError("n and the hidden widths must be multiples of 8 (n >= 8)")
        self.device = torch.device(device)
        dev = self.device
        rng = np.random.default_rng(seed)
        M1, M2, M3 = masks(n, self.h1, self.h2)
        shapes = [(self.h1, n), (self.h2, self.h1), (n, self.h2)]
        self.masks = [torch.from_numpy(M).to(dev) for M in (M1, M2, M3)]
        self.W, self.Wb, self.Wt, self.b = [], [], [], []
        for (o, i), M in zip(shapes, (M1, M2, M3)):
            lim = 1.0 / np.sqrt(i)
            w = (rng.uniform(-lim, lim, size=(o, i)) * M).astype(np.float32)
            self.W.append(torch.from_numpy(w).to(dev))
            self.Wb.append(torch.from_numpy(w).to(dev).to(torch.bfloat16).contiguous())
            self.Wt.append(torch.from_numpy(np.ascontiguousarray(w.T)).to(dev).to(torch.bfloat16).contiguous())
            self.b.append(torch.zeros(o, dtype=torch.float32, device=dev))
        self.mW = [torch.zeros_like(w) for w in self.W]
        self.vW = [torch.zeros_like(w) for w in self.W]
        self.mb = [torch.zeros_like(b) for b in self.b]
        self.vb = [torch.zeros_like(b) for b in self.b]
        self.gW = [torch.zeros_like(w) for w in self.W]
        self.gb = [torch.zeros_like(b) for b in self.b]
        o1, f1, u1 = _order(n, degrees(n, self.h1))
        o2, f2, u2 = _order(n, degrees(n, self.h2))
        if max(u1, u2) > 4:
            raise ValueError("at most 4 hidden units per degree (hidden width <= 4 (n - 1))")
        self.ord1, self.off1 = torch.from_numpy(o1).to(dev), torch.from_numpy(f1).to(dev)
        self.ord2, self.off2 = torch.from_numpy(o2).to(dev), torch.from_numpy(f2).to(dev)
        self.max_units = max(u1, u2)
        self.steps = 0
        self.err = torch.zeros(1, dtype=torch.int32, device=dev)
        self._bufs = {}

    # ------------------------------------------------------------------ plumbing
    def _stream(self):
        return C.c_void_p(self.torch.cuda.current_stream(self.device).cuda_stream)

    @staticmethod
    def _p(t):
        return C.c_void_p(t.data_ptr()) if t is not None else None

    def _buf(self, name, shape, dtype):
        t = self._bufs.get(name)
        if t is None or tuple(t.shape) != tuple(shape) or t.dtype != dtype:
            t = self.torch.empty(shape, dtype=dtype, device=self.device)
            self._bufs[name] = t
        return t

    def _gemm(self, A, Bm, M, N, K, *, bias=None, act=0, ref=None, out_f32=None, out_bf16=None, ldc=None):
        g = GemmC(M, N, K, A.shape[-1], Bm.shape[-1], ldc or N, act, 0, A.data_ptr(), Bm.data_ptr(),
                  bias.data_ptr() if bias is not None else None, ref.data_ptr() if ref is not None else None,
                  out_f32.data_ptr() if out_f32 is not None else None,
                  out_bf16.data_ptr() if out_bf16 is not None else None)
        _lib.check(_bind().drift_pt_gemm_bf16(C.byref(g), self._p(self.err), self._stream()), "drift_pt_gemm_bf16")

    def _t(self, x, name):
        rows, cols = x.shape
        out = self._buf(name, (cols, rows), x.dtype)
        _lib.check(_bind().drift_pt_transpose_bf16(rows, cols, self._p(x), self._p(out), self._stream()),
                   "drift_pt_transpose_bf16")
        return out

    def net_c(self) -> MadeNetC:
        return MadeNetC(self.n, self.h1, self.h2, self.max_units, self.Wt[0].data_ptr(), self.Wt[1].data_ptr(),
                        self.Wt[2].data_ptr(), self.b[0].data_ptr(), self.b[1].data_ptr(), self.b[2].data_ptr(),
                        self.ord1.data_ptr(), self.off1.data_ptr(), self.ord2.data_ptr(), self.off2.data_ptr())

    # ------------------------------------------------------------------ training
    def forward(self, x):
        """Logits [B][n] fp32 of int8 spins x [B][n] (tensor-core path)."""
        torch = self.torch
        B, n = x.shape
        X = self._buf("X", (B, n), torch.bfloat16)
        _lib.check(_bind().drift_pt_made_spins_to_bf16(B * n, self._p(x), self._p(X), self._stream()), "spins_to_bf16")
        h1 = self._buf("h1", (B, self.h1), torch.bfloat16)
        h2 = self._buf("h2", (B, self.h2), torch.bfloat16)
        logits = self._buf("logits", (B, n), torch.float32)
        self._gemm(X, self.Wb[0], B, self.h1, n, bias=self.b[0], act=1, out_bf16=h1)
        self._gemm(h1, self.Wb[1], B, self.h2, self.h1, bias=self.b[1], act=1, out_bf16=h2)
        self._gemm(h2, self.Wb[2], B, n, self.h2, bias=self.b[2], out_f32=logits)
        return logits

    def loss_and_grad(self, x):
        """Mean log q over the batch; gradients of -mean log q into gW / gb."""
        torch = self.torch
        B, n = x.shape
        logits = self.forward(x)
        X, h1, h2 = self._bufs["X"], self._bufs["h1"], self._bufs["h2"]
        logq = self._buf("logq", (B,), torch.float32)
        dl = self._buf("dl", (B, n), torch.bfloat16)
        _lib.check(_bind().drift_pt_made_loss(B, n, self._p(logits), self._p(x), self._p(logq), self._p(dl),
                                              1.0 / B, self._stream()), "drift_pt_made_loss")
        L = _bind()
        s = self._stream()
        # layer 3
        self._gemm(self._t(dl, "dlT"), self._t(h2, "h2T"), n, self.h2, B, out_f32=self.gW[2])
        _lib.check(L.drift_pt_colsum_bf16(B, n, self._p(dl), self._p(self.gb[2]), s), "colsum")
        dh2 = self._buf("dh2", (B, self.h2), torch.bfloat16)
        self._gemm(dl, self.Wt[2], B, self.h2, n, ref=h2, out_bf16=dh2)
        # layer 2
        self._gemm(self._t(dh2, "dh2T"), self._t(h1, "h1T"), self.h2, self.h1, B, out_f32=self.gW[1])
        _lib.check(L.drift_pt_colsum_bf16(B, self.h2, self._p(dh2), self._p(self.gb[1]), s), "colsum")
        dh1 = self._buf("dh1", (B, self.h1), torch.bfloat16)
        self._gemm(dh2, self.Wt[1], B, self.h1, self.h2, ref=h1, out_bf16=dh1)
        # layer 1
        self._gemm(self._t(dh1, "dh1T"), self._t(X, "XT"), self.h1, n, B, out_f32=self.gW[0])
        _lib.check(L.drift_pt_colsum_bf16(B, self.h1, self._p(dh1), self._p(self.gb[0]), s), "colsum")
        return logq

    def step(self, lr: float = 1e-3, beta1: float = 0.9, beta2: float = 0.999, eps: float = 1e-8):
        self.steps += 1
        L = _bind()
        s = self._stream()
        for k in range(3):
            o, i = self.W[k].shape
            _lib.check(L.drift_pt_adam(o, i, self._p(self.W[k]), self._p(self.gW[k]), self._p(self.mW[k]),
                                       self._p(self.vW[k]), self._p(self.masks[k]), lr, beta1, beta2, eps, self.steps,
                                       self._p(self.Wb[k]), self._p(self.Wt[k]), s), "drift_pt_adam")
            _lib.check(L.drift_pt_adam(1, o, self._p(self.b[k]), self._p(self.gb[k]), self._p(self.mb[k]),
                                       self._p(self.vb[k]), None, lr, beta1, beta2, eps, self.steps, None, None, s),
                       "drift_pt_adam")

    def train(self, data, *, epochs: int = 1, batch: int = 512, lr: float = 1e-3, seed: int = 0):
        """Minibatch Adam on int8 configurations data [M][n] (device); returns mean log q per epoch."""
        torch = self.torch
        M = data.shape[0]
        batch = min(batch, M - M % 8) if M >= 8 else M
        g = torch.Generator(device="cpu").manual_seed(seed)
        hist = []
        for _ in range(epochs):
            perm = torch.randperm(M, generator=g).to(self.device)
            tot, cnt = torch.zeros((), device=self.device), 0
            for s0 in range(0, M - batch + 1, batch):
                xb = data.index_select(0, perm[s0:s0 + batch]).contiguous()
                lq = self.loss_and_grad(xb)
                self.step(lr)
                tot += lq.sum()
                cnt += batch
            hist.append(float(tot.item()) / max(cnt, 1))
        self.check()
        return hist

    def train_async(self, data, *, steps: int, batch: int = 512, lr: float = 1e-3, seed: int = 0):
        """Enqueue `steps` minibatch Adam steps on the current stream without synchronising the host:
        minibatches are drawn on the device (uniform with replacement from data [M][n]), and the
        mean log q of each step's batch is left in a device tensor [steps] (returned). Lets the
        network train on a side stream while other work (plain PT) runs on another."""
        torch = self.torch
        M = data.shape[0]
        batch = min(batch, M - M % 8) if M >= 8 else M
        g = torch.Generator(device=self.device).manual_seed(seed)
        idx = torch.randint(0, M, (steps, batch), device=self.device, generator=g)
        out = torch.empty(steps, dtype=torch.float32, device=self.device)
        for k in range(steps):
            xb = data.index_select(0, idx[k]).contiguous()
            lq = self.loss_and_grad(xb)
            self.step(lr)
            out[k] = lq.mean()
        return out

    def check(self):
        self.torch.cuda.synchronize(self.device)
        if int(self.err.item()):
            raise _lib.EngineError(_lib.ETIMEOUT, "drift_pt_gemm_bf16", "a bounded in-kernel wait timed out")

    # ------------------------------------------------------------------ sampling
    def sample(self, count: int, seed: int, stream_id: int = 0):
        """(x int8 [count][n], log q fp32 [count]) drawn from q."""
        x = self.torch.empty((count, self.n), dtype=self.torch.int8, device=self.device)
        lq = self.torch.empty(count, dtype=self.torch.float32, device=self.device)
        net = self.net_c()
        _lib.check(_bind().drift_pt_made_sample(C.byref(net), count, 0, self._p(x), self._p(lq),
                                                seed & 0xFFFFFFFFFFFFFFFF, stream_id & 0xFFFFFFFF, self._stream()),
                   "drift_pt_made_sample")
        return x, lq

    def sample_suffix(self, x, keep: int, seed: int, stream_id: int = 0):
        """In place on int8 configurations x [count][n]: keep spins 0..keep-1, draw the others from
        q's conditionals; returns the log q (fp32 [count]) of the results."""
        lq = self.torch.empty(x.shape[0], dtype=self.torch.float32, device=self.device)
        net = self.net_c()
        _lib.check(_bind().drift_pt_made_sample_suffix(C.byref(net), x.shape[0], int(keep), self._p(x), self._p(lq),
                                                       seed & 0xFFFFFFFFFFFFFFFF, stream_id & 0xFFFFFFFF,
                                                       self._stream()), "drift_pt_made_sample_suffix")
        return lq

    def logq(self, x):
        """log q of int8 configurations x [count][n] (same arithmetic as sample())."""
        x = x.contiguous()
        lq = self.torch.empty(x.shape[0], dtype=self.torch.float32, device=self.device)
        net = self.net_c()
        _lib.check(_bind().drift_pt_made_sample(C.byref(net), x.shape[0], 1, self._p(x), self._p(lq), 0, 0,
                                                self._stream()), "drift_pt_made_sample")
        return lq

    # ------------------------------------------------------------------ host copies (tests)
    def weights_host(self):
        """bf16-rounded weights (as float64) and biases, as the device computes with them."""
        return ([w.to(self.torch.float32).cpu().numpy().astype(np.float64) for w in self.Wb],
                [b.cpu().numpy().astype(np.float64) for b in self.b])
