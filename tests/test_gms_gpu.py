"""Graph multispin layer on the GPU: words, energies, bests, rung permutation and exchange counts
bit-exact against the oracle (regular, irregular and lattice graphs, 1-3 words, the full MaxCut
N = 4096 instance), resumed runs equal one run, energies equal a recount of the spins."""

from __future__ import annotations

import numpy as np
import pytest

import oracle
from conftest import cuda_ready

from drift_b200.gms import GmsEngine, GmsLayout
from drift_b200.instances import ea_2d, gnp_pm, maxcut_3regular

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_ready(), reason="needs CUDA and libdrift_pt.so")]


def ladder(R, lo, hi):
    return lo * (hi / lo) ** (np.arange(R) / (R - 1))


CASES = {
    "3reg256": (maxcut_3regular(256, 1), 32, 6, 2),
    "gnp40": (gnp_pm(40, 0.1, 7), 64, 5, 3),
    "ea2d8": (ea_2d(8, 2), 96, 4, 2),
    "3reg4096": (maxcut_3regular(4096, 2), 64, 3, 4),
}


@pytest.mark.parametrize("case,cluster,thr", [
    ("3reg256", 1, 0), ("3reg256", 4, 64), ("3reg256", 16, 32),
    ("gnp40", 1, 64), ("gnp40", 2, 0), ("gnp40", 0, 0),
    ("ea2d8", 1, 0), ("ea2d8", 8, 96),
    ("3reg4096", 1, 0), ("3reg4096", 16, 128), ("3reg4096", 0, 0),
])
def test_gms_matches_oracle(case, cluster, thr):
    """One CTA per word and clusters of 2-16 CTAs per word run the same chain."""
    model, R, rounds, spr = CASES[case]
    lay = GmsLayout.from_model(model)
    betas = ladder(R, 0.2, 4.0)
    eng = GmsEngine(lay, betas, seed=9, sweeps_per_round=spr, instance=5, threads_per_cta=thr, cluster_size=cluster)
    eng.init()
    eng.run(rounds)
    eng.check()
    st = eng.fetch()
    o = oracle.gms_run(lay, betas, n_rounds=rounds, sweeps_per_round=spr, seed=9, instance=5)
    assert np.array_equal(st["words"], o.words)
    assert np.array_equal(st["best_words"], o.best_words)
    assert np.array_equal(st["energy"], o.energy) and np.array_equal(st["best_energy"], o.best_energy)
    assert np.array_equal(st["rung_of_slot"], o.rung_of_slot)
    assert np.array_equal(st["tried"], o.tried[: R - 1]) and np.array_equal(st["accepted"], o.accepted[: R - 1])
    s = st["spins"].astype(np.float64)
    J = model.to_dense().J if hasattr(model, "to_dense") else model.J
    ref = -0.5 * np.einsum("ri,ij,rj->r", s, J, s)
    assert np.array_equal(ref.astype(np.int64), st["energy"])


@pytest.mark.parametrize("cluster", [1, 8])
def test_gms_resume_equals_one_run(cluster):
    lay = GmsLayout.from_model(maxcut_3regular(512, 3))
    betas = ladder(64, 0.2, 4.0)
    a = GmsEngine(lay, betas, seed=2, sweeps_per_round=3, cluster_size=cluster)
    a.init()
    a.run(9)
    b = GmsEngine(lay, betas, seed=2, sweeps_per_round=3, cluster_size=1)
    b.init()
    b.run(4)
    b.run(5)
    a.check()
    b.check()
    x, y = a.fetch(), b.fetch()
    for k in ("words", "best_words", "energy", "best_energy", "rung_of_slot", "tried", "accepted"):
        assert np.array_equal(x[k], y[k]), k
