"""The oracle, pinned: Philox against the Random123 known-answer vectors, the exact enumerator,
the colouring and the NumPy reference-PT restatement against outputs of the reference itself
(tests/golden/, made by tests/golden/make_golden.py), and the C oracle chain against the
reference's own acceptance checks (tests/test_parallel_tempering.py of the reference)."""

from __future__ import annotations

import math

import numpy as np
import pytest

import oracle
from oracle import ref_pt
from conftest import dense_from_edges, load_golden

from drift_b200.engine import geometric_betas
from drift_b200.instances import ea_2d, maxcut_3regular, maxcut_ising, random_graph


# Random123 known-answer vectors for philox4x32-10 (kat_vectors of the Random123 distribution).
PHILOX_KAT = [
    ((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
    ((0xFFFFFFFF,) * 4, (0xFFFFFFFF,) * 2, (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
    ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
     (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)),
]


@pytest.mark.parametrize("ctr,key,expect", PHILOX_KAT)
def test_philox_known_answers(ctr, key, expect):
    assert tuple(int(x) for x in oracle.philox(ctr, key)) == expect


def test_philox_uniformity():
    # 2^16 outputs: every byte value appears close to 1/256 of the time (chi-square, 255 dof)
    words = np.array([oracle.philox((i, 7, 3, 1), (11, 13)) for i in range(16384)], dtype=np.uint32).ravel()
    counts = np.bincount((words & 0xFF).astype(np.int64), minlength=256)
    exp = words.size / 256
    chi2 = float(((counts - exp) ** 2 / exp).sum())
    assert chi2 < 340.0  # p ~ 3e-4 upper tail for 255 dof


@pytest.mark.parametrize("x", [0.0, -1e-12, -0.25, -0.6931471805599453, -1.0, -2.5, -7.75, -30.0, -300.0, -707.5])
def test_exp_matches_libm(x):
    assert oracle.exp_neg_d(x) == pytest.approx(math.exp(x), rel=4e-16, abs=0.0)
    if x > -87:
        assert oracle.exp_neg_f(x) == pytest.approx(math.exp(np.float32(x)), rel=3e-7)


def test_exp_edges():
    assert oracle.exp_neg_d(-800.0) == 0.0
    assert oracle.exp_neg_d(0.5) == 1.0  # positive arguments saturate (acceptance probability 1)
    assert oracle.exp_neg_f(-100.0) == 0.0


def test_integer_thresholds_are_floor_of_exp():
    for beta in (0.0, 0.1, 0.5, 1.0, 3.0, 4.0):
        for x in range(1, 13):
            t = oracle.threshold_int(beta, x)
            exact = math.exp(-2.0 * x * beta) * 2.0 ** 32
            assert abs(t - min(math.floor(exact), 2 ** 32 - 1)) <= 1


def test_exact_enumeration_matches_reference(reference_instances):
    for name, d in reference_instances.items():
        m = dense_from_edges(d["n"], d["edges"], d["h"])
        ex = oracle.exact(m.J, m.h, spectrum=d["spectrum"] is not None)
        assert ex.e_min == pytest.approx(d["e_exact"], abs=1e-9), name
        if d["spectrum"] is not None:
            assert np.allclose(ex.spectrum, d["spectrum"], atol=1e-9), name


def test_exact_enumeration_bank_fixtures():
    for d in load_golden("bank_fixtures.json"):
        m = dense_from_edges(d["n"], d["edges"], d["h"])
        assert oracle.exact(m.J, m.h).e_min == pytest.approx(d["known_energy"], abs=1e-9), d["id"]


def test_exact_boltzmann_averages_small_chain():
    # open ferromagnetic chain of 3 spins: closed form <E> = -2 tanh(beta)
    J = np.zeros((3, 3))
    J[0, 1] = J[1, 0] = J[1, 2] = J[2, 1] = 1.0
    betas = np.array([0.2, 1.0, 2.5])
    ex = oracle.exact(J, np.zeros(3), betas)
    assert np.allclose(ex.mean_e, -2.0 * np.tanh(betas), atol=1e-12)


def test_greedy_coloring_matches_reference(reference_instances):
    for name, d in reference_instances.items():
        m = dense_from_edges(d["n"], d["edges"], d["h"])
        row_ptr, col_idx, _ = m.csr()
        k, _, cptr, cs = oracle.greedy_coloring(m.n, row_ptr, col_idx)
        assert k == d["coloring"]["k"], name
        assert cptr.tolist() == d["coloring"]["color_ptr"], name
        assert cs.tolist() == d["coloring"]["color_spins"], name


def test_instance_builders_match_reference(reference_instances):
    for name, (n, p, seed) in {"maxcut_g16_p05_s3": (16, 0.5, 3), "maxcut_g12_p05_s3": (12, 0.5, 3),
                               "maxcut_g20_p04_s5": (20, 0.4, 5)}.items():
        m = maxcut_ising(random_graph(n, p, seed))
        ref = dense_from_edges(n, reference_instances[name]["edges"], reference_instances[name]["h"])
        assert np.array_equal(m.J, ref.J), name
    w = maxcut_ising(random_graph(10, 0.6, 4, weighted=True))
    ref = reference_instances["maxcut_g10_weighted_s4"]
    assert np.allclose(w.J, dense_from_edges(10, ref["edges"], ref["h"]).J)


def test_ref_pt_restatement_reproduces_reference(reference_instances):
    for run in load_golden("ref_pt.json"):
        d = reference_instances[run["instance"]]
        m = dense_from_edges(d["n"], d["edges"], d["h"])
        out = ref_pt.parallel_tempering(m, **run["kwargs"])
        assert out["best_E"] == run["best_E"], run["instance"]
        assert out["swap_rate"] == run["swap_rate"], run["instance"]
        assert np.array_equal(out["best_history"], np.asarray(run["best_history"])), run["instance"]
        assert np.array_equal(out["best_s"], np.asarray(run["best_s"])), run["instance"]


def _oracle_problem(model):
    row_ptr, col_idx, w = model.csr()
    return oracle.OracleProblem(model.n, row_ptr, col_idx, w, model.h)


@pytest.mark.parametrize("name,kw", [
    ("maxcut_g16_p05_s3", dict(R=16, T=(0.05, 4.0), rounds=200, spr=4, seed=1)),   # test_parallel_tempering.py:37-44
    ("glass_n14_s7_field", dict(R=20, T=(0.05, 5.0), rounds=300, spr=5, seed=2)),  # :47-59 (float path)
    ("ferro_n18", dict(R=12, T=(0.05, 3.0), rounds=150, spr=4, seed=0)),           # :62-68
    ("maxcut_g18_p04_s8", dict(R=16, T=(0.05, 4.0), rounds=200, spr=4, seed=1)),   # phase14_gpu.py:38-42
])
def test_oracle_chain_finds_exact_ground_state(reference_instances, name, kw):
    d = reference_instances[name]
    m = dense_from_edges(d["n"], d["edges"], d["h"])
    prob = _oracle_problem(m)
    betas = geometric_betas(kw["R"], *kw["T"])
    st = oracle.pt_run(prob, betas, n_rounds=kw["rounds"], sweeps_per_round=kw["spr"], seed=kw["seed"])
    scale = 1.0 if prob.integer_path else 2.0 ** -32
    best = int(np.argmin(st.best_energy))
    assert m.energy(st.best_spins[best].astype(float)) == pytest.approx(d["e_exact"], abs=1e-6)
    assert st.best_energy[best] * scale == pytest.approx(d["e_exact"], abs=1e-4)
    # incremental energies equal a full recompute (exactly on the integer path)
    for r in range(kw["R"]):
        e = m.energy(st.spins[r].astype(float))
        if prob.integer_path:
            assert st.energy[r] == int(round(e))
        else:
            assert st.energy[r] * scale == pytest.approx(e, abs=1e-4)
    assert st.best_history[kw["rounds"] - 1] == pytest.approx(st.best_energy[best] * scale)


def test_oracle_exchange_beats_single_cold_walker(reference_instances):
    """tests/test_parallel_tempering.py:71-89 of the reference, on the oracle chain."""
    d = reference_instances["glass_n16_s11"]
    m = dense_from_edges(d["n"], d["edges"], d["h"])
    prob = _oracle_problem(m)
    seeds = range(12)
    full = [oracle.pt_run(prob, geometric_betas(20, 0.05, 5.0), n_rounds=300, sweeps_per_round=5,
                          seed=s).best_energy.min() for s in seeds]
    cold = [oracle.pt_run(prob, geometric_betas(1, 0.05, 0.05), n_rounds=300, sweeps_per_round=5,
                          seed=s).best_energy.min() for s in seeds]
    assert all(e == d["e_exact"] for e in full)
    # the lone cold walker freezes above the ground state on most seeds
    assert sum(e > d["e_exact"] for e in cold) >= len(seeds) // 2


def test_oracle_resume_equals_single_run():
    m = ea_2d(8, 3)
    prob = _oracle_problem(m)
    betas = geometric_betas(6, 0.4, 3.0)
    a = oracle.pt_run(prob, betas, n_rounds=30, sweeps_per_round=2, seed=9)
    b = oracle.pt_run(prob, betas, n_rounds=12, sweeps_per_round=2, seed=9)
    b = oracle.pt_run(prob, betas, n_rounds=18, sweeps_per_round=2, seed=9, state=b, round_offset=12)
    for f in ("spins", "energy", "best_energy", "best_spins", "rung_of_slot", "tried", "accepted"):
        assert np.array_equal(getattr(a, f), getattr(b, f)), f


def test_oracle_thread_count_does_not_change_results():
    m = maxcut_3regular(512, 1)
    prob = _oracle_problem(m)
    betas = geometric_betas(8, 0.25, 5.0)
    a = oracle.pt_run(prob, betas, n_rounds=10, sweeps_per_round=2, seed=5, threads=1)
    b = oracle.pt_run(prob, betas, n_rounds=10, sweeps_per_round=2, seed=5, threads=4)
    for f in ("spins", "energy", "best_energy", "rung_of_slot", "tried", "accepted"):
        assert np.array_equal(getattr(a, f), getattr(b, f)), f


_FRESH_PROCESS_CHAIN = """
import hashlib, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
import oracle
rng = np.random.default_rng(11)
n, m = 3000, 9000
e = rng.integers(0, n, size=(m, 2))
e = e[e[:, 0] != e[:, 1]]
J = np.zeros((n, n), np.float32)
J[e[:, 0], e[:, 1]] = rng.standard_normal(len(e)).astype(np.float32)
J = np.triu(J, 1); J = J + J.T
row_ptr = np.concatenate([[0], np.cumsum((J != 0).sum(1))]).astype(np.int32)
col_idx = np.nonzero(J)[1].astype(np.int32)
w = J[J != 0].astype(np.float32)
h = (0.1 * rng.standard_normal(n)).astype(np.float32)
_, _, cp, cs = oracle.greedy_coloring(n, row_ptr, col_idx)
prob = oracle.OracleProblem(n, row_ptr, col_idx, w, h, cp, cs, integer_path=False)
st = oracle.pt_run(prob, 1.0 / np.geomspace(3.0, 0.1, 8), n_rounds=2, sweeps_per_round=2, seed=5, threads=8)
print(hashlib.sha256(st.spins.tobytes() + st.energy.tobytes()).hexdigest())
"""


def test_oracle_fp32_chain_is_the_same_in_fresh_processes():
    """The first exponentials of a process are evaluated by several replica threads at once; the
    chain must not depend on which thread gets there first (run in new processes, 8 threads)."""
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    outs = {subprocess.run([sys.executable, "-c", _FRESH_PROCESS_CHAIN, root], capture_output=True, text=True,
                           check=True, timeout=120).stdout.strip() for _ in range(10)}
    assert len(outs) == 1, outs


def test_oracle_swap_rate_matches_reference_cpu_statistically(reference_instances):
    """Equilibrium swap acceptance depends only on the Boltzmann energy distributions, so the
    colour-ordered chain and the reference's random-site chain agree within sampling noise."""
    d = reference_instances["maxcut_g20_p04_s5"]
    m = dense_from_edges(d["n"], d["edges"], d["h"])
    prob = _oracle_problem(m)
    R, rounds = 8, 600
    betas = geometric_betas(R, 0.3, 3.0)
    st = oracle.pt_run(prob, betas, n_rounds=rounds, sweeps_per_round=2, seed=21)
    ours = st.accepted.sum() / st.tried.sum()
    ref = ref_pt.parallel_tempering(m, n_replicas=R, T_min=1 / 3.0, T_max=1 / 0.3, n_rounds=rounds,
                                    sweeps_per_round=2, seed=21)["swap_rate"]
    # R-1 pairs x rounds/2 attempts each; generous 4-sigma band on a proportion
    n_att = st.tried.sum()
    sig = math.sqrt(max(ours * (1 - ours), 1e-3) / n_att) * math.sqrt(2) * 2.0  # autocorrelation allowance
    assert abs(ours - ref) < 4 * sig + 0.02
