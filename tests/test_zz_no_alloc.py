"""drift_pt_run_noalloc: the round loop for callers that cannot allocate device memory.

Such callers (a process whose framework already holds the device memory, a loop that may not call
cudaMalloc after start-up, a binding that only gets pointers to other people's buffers) cannot
provide drift_pt_run's workspace. The allocation-free entry point uses the library's built-in
scratch array instead; apart from that it must run the very same chain. This test calls it through
the C ABI twice in a row (a fresh chain, then a resumed one) and compares every output with the
workspace entry point's, bit for bit as the other parity tests do. It also checks the size limit.

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

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_ready(), reason="needs CUDA and libdrift_pt.so")]


def _run_noalloc(eng: PtEngine, n_rounds: int, hist) -> None:
    L = _lib.load()
    P, A, S = eng.prob.c_problem(), eng._args(n_rounds), eng._state(hist)
    _lib.check(L.drift_pt_run_noalloc(C.byref(P), C.byref(A), C.byref(S), eng.stream()), "drift_pt_run_noalloc")
    eng.rounds_done += n_rounds


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
