"""ORACLE (test infrastructure only): the proposal network restated on the CPU in FP64.

The masked autoregressive MLP of drift_b200/made.py (MADE, Germain et al., ICML 2015), written
independently from its definition: input i has degree i+1, hidden unit k of a layer of width h has
degree 1 + k mod (n-1), W1[k][i] is kept iff m1(k) >= i+1, W2[k'][k] iff m2(k') >= m1(k), W3[i][k']
iff i+1 > m2(k'); q(x) = prod_i sigma(x_i l_i). Gradients come from PyTorch CPU autograd in
float64 (the checker for the device's hand-written backward pass); `all_logq` enumerates q over
every configuration of a small n.
"""

from __future__ import annotations

import itertools

import numpy as np


def degrees(n: int, h: int) -> np.ndarray:
    return 1 + (np.arange(h) % (n - 1))


def masks(n: int, h1: int, h2: int):
    d_in = np.arange(1, n + 1)
    d1, d2 = degrees(n, h1), degrees(n, h2)
    return ((d1[:, None] >= d_in[None, :]).astype(np.float64), (d2[:, None] >= d1[None, :]).astype(np.float64),
            (d_in[:, None] > d2[None, :]).astype(np.float64))


def logq_and_grads(W, b, x):
    """log q(x) per row of x (+-1, [B][n]) and the gradients of -mean log q w.r.t. W and b."""
    import torch

    Wt = [torch.tensor(w, dtype=torch.float64, requires_grad=True) for w in W]
    bt = [torch.tensor(v, dtype=torch.float64, requires_grad=True) for v in b]
    X = torch.tensor(np.asarray(x, np.float64))
    h1 = torch.relu(X @ Wt[0].T + bt[0])
    h2 = torch.relu(h1 @ Wt[1].T + bt[1])
    logits = h2 @ Wt[2].T + bt[2]
    logq = torch.nn.functional.logsigmoid(X * logits).sum(dim=1)
    loss = -logq.mean()
    loss.backward()
    return (logq.detach().numpy(), [w.grad.numpy() for w in Wt], [v.grad.numpy() for v in bt],
            logits.detach().numpy())


def logq(W, b, x) -> np.ndarray:
    X = np.asarray(x, np.float64)
    h1 = np.maximum(X @ W[0].T + b[0], 0.0)
    h2 = np.maximum(h1 @ W[1].T + b[1], 0.0)
    z = X * (h2 @ W[2].T + b[2])
    return (np.minimum(z, 0.0) - np.log1p(np.exp(-np.abs(z)))).sum(axis=1)


def all_configs(n: int) -> np.ndarray:
    return np.array(list(itertools.product((-1, 1), repeat=n)), dtype=np.int8)


def all_logq(W, b, n: int):
    xs = all_configs(n)
    return xs, logq(W, b, xs)


def to_bf16(a) -> np.ndarray:
    """Round to the nearest bfloat16 (ties to even), returned as float64."""
    f = np.asarray(a, np.float64).astype(np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def logq_and_grads_bf16(W, b, x):
    """The device's training pass restated in FP64 with bf16 roundings at the same points: the
    hidden activations, the logit gradient and the back-propagated hidden gradients are stored as
    bf16; products accumulate exactly (FP64 here, FP32 on the device)."""
    X = np.asarray(x, np.float64)
    B = X.shape[0]
    h1 = to_bf16(np.maximum(X @ W[0].T + b[0], 0.0))
    h2 = to_bf16(np.maximum(h1 @ W[1].T + b[1], 0.0))
    logits = (h2 @ W[2].T + b[2]).astype(np.float32).astype(np.float64)
    z = X * logits
    logq = (np.minimum(z, 0.0) - np.log1p(np.exp(-np.abs(z)))).sum(axis=1)
    dl = to_bf16(-(1.0 / B) * X / (1.0 + np.exp(z)))
    gW3, gb3 = dl.T @ h2, dl.sum(0)
    dh2 = to_bf16((dl @ W[2]) * (h2 > 0))
    gW2, gb2 = dh2.T @ h1, dh2.sum(0)
    dh1 = to_bf16((dh2 @ W[1]) * (h1 > 0))
    gW1, gb1 = dh1.T @ X, dh1.sum(0)
    return logq, [gW1, gW2, gW3], [gb1, gb2, gb3]
