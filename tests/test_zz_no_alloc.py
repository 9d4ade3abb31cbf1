"""drift_pt_run_noalloc: the round loop for callers that cannot allocate device memory.

Such callers (a process whose framework already holds the device memory, a loop that may not call
cudaMalloc after start-up, a binding that only gets pointers to other people's buffers) cannot
provide drift_pt_run's workspace. The allocation-free entry point uses the library's built-in
scratch array instead; apart from that it must run the very same chain. This test calls it through
the C ABI twice in a row (a fresh chain, then a resumed one) and compares every output with the
workspace entry point's, bit for bit as the other parity tests do, checking after each call with
drift_pt_noalloc_check that no bounded wait gave up. It also checks the size limit at its exact
boundary (the largest replica count, whose scratch fills the array) and one past it, and that a run
whose wait limit runs out is reported by drift_pt_noalloc_check and leaves the next run clean.

The file is named to be collected last, so a run that stops at the first failure has run every
other test before this one; it does not depend on them and passes alone in a fresh process.
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import cuda_ready

from drift_b200 import _lib
from drift_b200.engine import DeviceProblem, HostProblem, PtEngine, geometric_betas
from drift_b200.instances import maxcut_3regular
from drift_b200.ising import IsingModel

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_ready(), reason="needs CUDA and libdrift_pt.so")]


def _run_noalloc(eng: PtEngine, n_rounds: int, hist=None, timeout_s: float | None = None) -> None:
    L = _lib.load()
    P, A, S = eng.prob.c_problem(), eng._args(n_rounds), eng._state(hist)
    if timeout_s is not None:
        A.timeout_s = timeout_s
    _lib.check(L.drift_pt_run_noalloc(C.byref(P), C.byref(A), C.byref(S), eng.stream()), "drift_pt_run_noalloc")
    eng.rounds_done += n_rounds


def _noalloc_check(eng: PtEngine) -> int:
    return _lib.load().drift_pt_noalloc_check(eng.stream())


def test_noalloc_entry_matches_workspace_entry_on_two_calls():
    import torch

    model = maxcut_3regular(1024, 3)
    R, spr, seed = 32, 2, 5
    betas = geometric_betas(R, 0.25, 5.0)
    prob = DeviceProblem(HostProblem.from_model(model))
    # 32 replicas, one per CTA: every round meets at the grid barrier that lives in the scratch
    ref = PtEngine(prob, betas, seed=seed, sweeps_per_round=spr, replicas_per_cta=1)
    nal = PtEngine(prob, betas, seed=seed, sweeps_per_round=spr, replicas_per_cta=1)
    ref.init()
    nal.init()
    for call, n_rounds in enumerate((6, 9)):
        h_ref = torch.zeros(n_rounds, dtype=torch.float64, device=prob.device)
        h_nal = torch.zeros(n_rounds, dtype=torch.float64, device=prob.device)
        ref.run(n_rounds, history=h_ref)
        _run_noalloc(nal, n_rounds, h_nal)
        ref.check()
        assert _noalloc_check(nal) == _lib.OK, f"call {call}: a bounded wait gave up"
        torch.cuda.synchronize()
        a, b = ref.fetch(), nal.fetch()
        for key in ("spins", "best_spins", "energy_fixed", "best_energy_fixed", "rung_of_slot", "slot_of_rung",
                    "tried", "accepted"):
            assert np.array_equal(a[key], b[key]), f"call {call}: {key} differs"
        assert torch.equal(h_ref, h_nal), f"call {call}: best history differs"
        assert np.array_equal(nal.energy_fp64(), b["energy_fixed"].astype(np.float64))


def test_noalloc_entry_rejects_too_many_replicas():
    model = maxcut_3regular(64, 1)
    prob = DeviceProblem(HostProblem.from_model(model))
    eng = PtEngine(prob, geometric_betas(2, 0.5, 2.0), seed=1)
    eng.init()
    args = eng._args(1)
    args.n_replicas = 4097
    L = _lib.load()
    rc = L.drift_pt_run_noalloc(C.byref(prob.c_problem()), C.byref(args), C.byref(eng._state()), eng.stream())
    assert rc == _lib.EUNSUPPORTED
    assert "4096" in L.drift_pt_last_error().decode()


def test_noalloc_entry_at_its_replica_limit():
    """R = DRIFT_PT_NOALLOC_MAX_REPLICAS: the scratch the run needs is exactly the built-in array."""
    import torch

    R = 4096
    need = C.c_size_t(0)
    L = _lib.load()
    _lib.check(L.drift_pt_workspace_bytes(R, C.byref(need)), "drift_pt_workspace_bytes")
    assert need.value == 256 + 32 * R  # the array's size
    # 4096 replicas fit the sweep kernel's shared memory when the largest local field is 1: 16 spins
    # with fields of +-1 and no couplings
    h = np.random.default_rng(3).choice([-1.0, 1.0], size=16)
    model = IsingModel(np.zeros((16, 16)), h)
    prob = DeviceProblem(HostProblem.from_model(model))
    assert prob.integer_path and prob.max_field == 1
    betas = geometric_betas(R, 0.2, 4.0)
    ref = PtEngine(prob, betas, seed=3, sweeps_per_round=1)
    nal = PtEngine(prob, betas, seed=3, sweeps_per_round=1)
    ref.init()
    nal.init()
    h_ref = torch.zeros(1, dtype=torch.float64, device=prob.device)
    h_nal = torch.zeros(1, dtype=torch.float64, device=prob.device)
    ref.run(1, history=h_ref)
    _run_noalloc(nal, 1, h_nal)
    ref.check()
    assert _noalloc_check(nal) == _lib.OK
    a, b = ref.fetch(), nal.fetch()
    for key in ("spins", "best_spins", "energy_fixed", "best_energy_fixed", "rung_of_slot", "slot_of_rung",
                "tried", "accepted"):
        assert np.array_equal(a[key], b[key]), key
    assert torch.equal(h_ref, h_nal)


def test_noalloc_check_reports_a_wait_that_ran_out():
    """A wait limit of 1 ns runs out at the first grid-wide wait that is not satisfied at once; the
    kernel gives up (it sets the error flag, every CTA leaves its round loop) and the check reports it.
    A run only waits when some CTA reaches a round end noticeably before another (about a microsecond
    of skew), which happened in every one of 30 fresh-process trials of this shape on B200 but is not
    certain, so up to five runs are made; each that does not time out must report success. The next
    call with the default limit starts from a cleared scratch and is clean."""
    model = maxcut_3regular(1024, 4)
    prob = DeviceProblem(HostProblem.from_model(model))
    betas = geometric_betas(32, 0.25, 5.0)
    eng = PtEngine(prob, betas, seed=9, sweeps_per_round=1, replicas_per_cta=1, round_sync=1)
    rc = _lib.OK
    for _ in range(5):
        eng.init()
        _run_noalloc(eng, 2000, timeout_s=1e-9)
        rc = _noalloc_check(eng)
        if rc == _lib.ETIMEOUT:
            break
        assert rc == _lib.OK, rc
    assert rc == _lib.ETIMEOUT, rc
    assert "timed out" in _lib.load().drift_pt_last_error().decode()
    eng.init()
    _run_noalloc(eng, 3)
    assert _noalloc_check(eng) == _lib.OK
    st = eng.fetch()
    assert np.array_equal(eng.energy_fp64(), st["energy_fixed"].astype(np.float64))
