"""Where a block of the dense (SK) kernel spends its time: the clock64 stamps of the profiling build.

    python -m drift_b200.build --sk-stamps      # libdrift_pt_skstamp.so, the stamps compiled in
    python -m drift_b200.sk_stamps              # SK N = 512, 64 replicas, 2 per CTA: the breakdown

The dense kernel resolves a replica's spins 32 at a time (one block) and keeps the fields current
through a pipeline of hand-offs between warp roles: the resolver publishes its block's spin changes
(delta), the producer issues the tensor-core MMAs once every resolver of the CTA has, a loader reads
the updated fields of block j + 2 from tensor memory and stages them, and the resolver picks block
j + 2 up. The profiling build stamps CTA 0 at each hand-off; this prints the median cycles of each
leg over the steady part of a 200-sweep run, and the median period of a block.
"""

from __future__ import annotations

import ctypes as C
import json
import sys

import numpy as np

LEGS = [
    ("resolve: block picked up -> delta published (resolver 0)", lambda S, j: S[1, j] - S[0, j]),
    ("delta published -> producer has every resolver's delta", lambda S, j: S[2, j] - S[1, j]),
    ("producer: deltas -> the loaders' reads of the accumulator set done", lambda S, j: S[3, j] - S[2, j]),
    ("producer: reads done -> MMAs issued and committed", lambda S, j: S[4, j] - S[3, j]),
    ("MMAs of block j-2 committed -> loader of block j sees them complete", lambda S, j: S[5, j] - S[4, j - 2]),
    ("loader: second field read + thresholds -> stage released", lambda S, j: S[6, j] - S[5, j]),
    ("stage released -> resolver picks the block up", lambda S, j: S[0, j] - S[6, j]),
]


def main(argv=None) -> dict:
    from . import _lib
    from . import build as b

    _lib.LIB_PATH = b.SK_STAMP_LIB_PATH
    L = _lib.load()
    L.drift_pt_sk_stamps.argtypes = [C.c_void_p]
    L.drift_pt_sk_stamps.restype = C.c_int
    import torch

    from .instances import sk_model
    from .sk import SkEngine, SkModel

    sk = SkModel.from_model(sk_model(512, 4))
    betas = 0.3 * 10.0 ** (np.arange(64) / 63)
    eng = SkEngine(sk, betas, seed=1, sweeps_per_round=10, replicas_per_cta=2)
    eng.init()
    eng.run(2)
    torch.cuda.synchronize()
    eng.run(20)  # 200 sweeps x 16 blocks = 3200 steps, all stamped
    eng.check()
    buf = np.zeros((8, 4096), np.uint64)
    _lib.check(L.drift_pt_sk_stamps(buf.ctypes.data_as(C.c_void_p)), "drift_pt_sk_stamps")
    S = buf.astype(np.int64)
    j = np.arange(200, 20 * 10 * 16 - 4)
    out = {"block period (resolver 0 picks up block j+1 after block j)": float(np.median(S[0, j + 1] - S[0, j]))}
    for name, f in LEGS:
        out[name] = float(np.median(f(S, j)))
    out["two-block cycle: resolve(j-2) start -> resolve(j) start"] = float(np.median(S[0, j] - S[0, j - 2]))
    for k, v in out.items():
        print(f"{k:72s} {v:8.0f} cycles")
    if argv and "--json" in argv:
        print(json.dumps(out))
    return out


if __name__ == "__main__":
    main(sys.argv[1:])
