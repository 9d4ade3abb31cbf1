"""Per-rung observables of a PT run: energy, |magnetisation| and, from two independent
ladders, the overlap q = (1/n) sum_i s_i^a s_i^b, recorded after every round, plus blocked means
and standard errors for comparing runs."""

from __future__ import annotations

import numpy as np


def record(engine, n_rounds: int, spins: bool = False) -> dict:
    """Run `n_rounds` single rounds of a PtEngine; after each, the rung-ordered energies (model
    units), |m| and, with `spins`, the rung configurations in the original site order."""
    torch = engine.torch
    prob = engine.prob
    dev = engine.spins.device
    R, n = engine.R, prob.n
    valid = torch.from_numpy((prob.site_of_pos >= 0).astype(np.float64)).to(dev)
    pos = torch.from_numpy(prob.pos_of_site.astype(np.int64)).to(dev)
    scale = prob.energy_scale()
    E = torch.empty((n_rounds, R), dtype=torch.float64, device=dev)
    M = torch.empty((n_rounds, R), dtype=torch.float64, device=dev)
    S = torch.empty((n_rounds, R, n), dtype=torch.int8, device=dev) if spins else None
    for t in range(n_rounds):
        engine.run(1)
        slots = engine.slot_of_rung.long()
        E[t] = engine.energy.index_select(0, slots).double() * scale
        sp = engine.spins.index_select(0, slots)
        M[t] = (sp.double() * valid).sum(1).abs() / n
        if spins:
            S[t] = sp.index_select(1, pos)
    engine.check()
    return {"energy": E.cpu().numpy(), "absm": M.cpu().numpy(), "spins": S.cpu().numpy() if spins else None}


def overlap(spins_a: np.ndarray, spins_b: np.ndarray) -> np.ndarray:
    """q per round and rung of two independent ladders' recorded configurations [T][R][n]."""
    return (spins_a.astype(np.float64) * spins_b.astype(np.float64)).mean(axis=2)


def blocked(x: np.ndarray, blocks: int = 20, discard: float = 0.1):
    """Mean and standard error per column of a time series [T][...], after dropping the first
    `discard` fraction, from `blocks` block means (successive rounds are correlated)."""
    x = np.asarray(x, np.float64)
    x = x[int(len(x) * discard):]
    T = len(x) - len(x) % blocks
    bm = x[:T].reshape(blocks, T // blocks, *x.shape[1:]).mean(axis=1)
    return bm.mean(axis=0), bm.std(axis=0, ddof=1) / np.sqrt(blocks)
