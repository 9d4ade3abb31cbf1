"""Dense-coupling layer, CPU side: fixed-point quantisation, the device coupling table (decoded
back from the tensor-core operand layout), acceptance scales, the oracle's -ln and threshold
against NumPy, and the oracle chain itself (exact energies, Boltzmann statistics against exact
enumeration)."""

from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import oracle
from drift_b200 import _lib
from drift_b200.sk import SkModel


def sk_couplings(n, seed, field=0.0):
    rng = np.random.default_rng(seed)
    J = np.triu(rng.normal(size=(n, n)) / np.sqrt(n), 1)
    J = J + J.T
    h = rng.normal(scale=field, size=n) if field else np.zeros(n)
    return J, h


def core_offset(row, k):
    return (row >> 3) * 256 + (k >> 4) * 128 + (row & 7) * 16 + (k & 15)


@pytest.mark.parametrize("n,field", [(512, 0.0), (100, 0.3), (7, 0.0)])
def test_quantize_rule(n, field):
    J, h = sk_couplings(n, 4, field)
    m = SkModel(J, h)
    s = m.shift
    rows = np.abs(J).sum(1) + np.abs(h)

    def fits(sh):
        return np.abs(J).max() * 2.0 ** sh <= 2 ** 23 - 2 ** 16 and rows.max() * 2.0 ** sh + n <= 2 ** 30

    assert fits(s) and not fits(s + 1)
    assert np.array_equal(m.Jq, np.rint(J * 2.0 ** s).astype(np.int32))
    assert np.array_equal(m.hq, np.rint(h * 2.0 ** s).astype(np.int32))
    assert (np.abs(m.Jq).sum(1) + np.abs(m.hq)).max() < 2 ** 30
    if n == 512 and field == 0.0:
        assert s == 25  # SK at n = 512: resolution 2^-25 ~ 3e-8


def test_quantize_rejects_bad_models():
    L = _lib.load()
    from drift_b200.sk import _bind

    _bind()
    n = 4
    J = np.zeros((n, n))
    J[0, 1] = 1.0
    Jq = np.zeros((n, n), np.int32)
    hq = np.zeros(n, np.int32)
    sh = C.c_int32(0)
    p = lambda a: a.ctypes.data_as(C.c_void_p)
    assert L.drift_pt_sk_quantize(n, p(J), None, p(Jq), p(hq), C.byref(sh)) == _lib.EINVAL  # not symmetric
    assert "symmetric" in L.drift_pt_last_error().decode()
    J[1, 0] = 1.0
    J[2, 2] = 0.5
    assert L.drift_pt_sk_quantize(n, p(J), None, p(Jq), p(hq), C.byref(sh)) == _lib.EINVAL  # diagonal
    J[2, 2] = 0.0
    assert L.drift_pt_sk_quantize(n, p(J), None, p(Jq), p(hq), C.byref(sh)) == _lib.OK
    assert L.drift_pt_sk_quantize(513, p(J), None, p(Jq), p(hq), C.byref(sh)) == _lib.EINVAL


@pytest.mark.parametrize("n", [512, 200, 33])
def test_layout_decodes_to_the_couplings(n):
    J, h = sk_couplings(n, 9, 0.2)
    m = SkModel(J, h)
    nt = (n + 127) // 128
    nb = 4 * nt
    eb = nt * 3 * 4096 + 8192
    assert m.layout.size == nb * eb
    lay = m.layout.view(np.int8)
    rows = np.arange(128)
    ks = np.arange(32)
    off = core_offset(rows[:, None], ks[None, :])
    Jp = np.zeros((128 * nt, 32 * nb), np.int64)
    Jp[:n, :n] = m.Jq
    for B in range(nb):
        e = lay[B * eb:(B + 1) * eb]
        for t in range(nt):
            limbs = [e[(t * 3 + k) * 4096:(t * 3 + k + 1) * 4096][off].astype(np.int64) for k in range(3)]
            val = limbs[0] + 256 * limbs[1] + 65536 * limbs[2]
            assert np.array_equal(val, Jp[128 * t:128 * (t + 1), 32 * B:32 * (B + 1)]), (B, t)
        dg = e[nt * 3 * 4096:nt * 3 * 4096 + 4096].view(np.int32).reshape(32, 32)
        assert np.array_equal(dg, Jp[32 * B:32 * (B + 1), 32 * B:32 * (B + 1)])
        pv = e[nt * 3 * 4096 + 4096:].view(np.int32).reshape(32, 32)
        Bp = (B - 1) % nb
        assert np.array_equal(pv, Jp[32 * Bp:32 * (Bp + 1), 32 * B:32 * (B + 1)])


def test_scales():
    m = SkModel(*sk_couplings(64, 1))
    betas = np.geomspace(0.3, 3.0, 16)
    assert np.array_equal(m.scales(betas), (2.0 ** m.shift / (2 * betas)).astype(np.float32))


def test_neg_log_and_threshold_against_numpy():
    us = ((2 * np.arange(0, 1 << 23, 997) + 1) * 2.0 ** -24).astype(np.float32)
    got = np.array([oracle.neg_log_unit(float(u)) for u in us])
    ref = -np.log(us.astype(np.float64))
    assert np.all(np.abs(got - ref) <= 4e-7 * np.maximum(ref, 1e-3))
    rng = np.random.default_rng(0)
    for c in (1.0, 5.6e7, 3.3e8, 1e12):
        for w in rng.integers(0, 2 ** 32, size=200, dtype=np.uint64):
            D = oracle.sk_threshold(int(w), float(np.float32(c)))
            u = (2 * (int(w) >> 9) + 1) * 2.0 ** -24
            ref = -np.log(u) * float(np.float32(c))
            if ref >= 2 ** 31:
                assert D == 2 ** 31 - 1
            else:
                assert abs(D - np.floor(ref)) <= 1 + 1e-6 * ref


def test_oracle_energies_are_exact_and_match_fp64():
    J, h = sk_couplings(96, 5, 0.2)
    m = SkModel(J, h)
    betas = np.geomspace(0.3, 3.0, 12)
    st = oracle.sk_run(m.Jq, m.hq, m.shift, betas, m.scales(betas), n_rounds=6, sweeps_per_round=3, seed=7)
    for r in range(12):
        assert oracle.sk_energy(m.Jq, m.hq, st.spins[r]) == st.energy[r]
        assert oracle.sk_energy(m.Jq, m.hq, st.best_spins[r]) == st.best_energy[r]
    # quantised energies vs the unquantised model: |dE| <= (n^2/2 + n) 2^-(shift+1) at most
    e64 = m.energy_fp64(st.spins)
    assert np.all(np.abs(st.energy * m.energy_unit - e64) <= (96 * 96 / 2 + 96) * m.energy_unit)
    assert np.all(st.best_history == np.minimum.accumulate(st.best_history))
    assert (st.accepted[:11] > 0).any() and np.all(st.accepted <= st.tried)


def test_oracle_chain_samples_the_boltzmann_distribution():
    """<E> per rung of a long run vs exact enumeration (n = 10): the log-domain acceptance rule is
    the Metropolis rule."""
    n = 10
    J, h = sk_couplings(n, 3, 0.4)
    m = SkModel(J, h)
    betas = np.array([0.3, 0.7, 1.2, 2.0])
    ex = oracle.exact(m.Jq * 2.0 ** -m.shift, m.hq * 2.0 ** -m.shift, betas)
    st = None
    means = np.zeros(len(betas))
    sq = np.zeros(len(betas))
    k = 0
    for rnd in range(400):
        st = oracle.sk_run(m.Jq, m.hq, m.shift, betas, m.scales(betas), n_rounds=1, sweeps_per_round=5, seed=11,
                           state=st, round_offset=rnd)
        if rnd >= 40:
            e = st.energy[st.slot_of_rung] * m.energy_unit
            means += e
            sq += e * e
            k += 1
    means /= k
    sd = np.sqrt(np.maximum(sq / k - means ** 2, 1e-12))
    # consecutive rounds are correlated: allow 6 naive standard errors
    assert np.all(np.abs(means - ex.mean_e) <= 6 * sd / np.sqrt(k) + 1e-9), (means, ex.mean_e)


def test_device_entry_points_validate_before_touching_the_gpu():
    """Shape and argument errors come back as EINVAL from the host side of the call."""
    from drift_b200.sk import SkProblemC, SkRunArgsC, SkStateC, _bind

    L = _bind()
    fake = 64  # never dereferenced: validation fails first
    P = SkProblemC(512, 25, fake, fake, fake)
    S = SkStateC(*([fake] * 8), None)

    def run(**kw):
        args = dict(n_replicas=64, n_rounds=1, sweeps_per_round=1, replicas_per_cta=4, round_offset=0, seed=0,
                    instance=0, reserved=0, betas=fake, scales=fake, timeout_s=1.0)
        args.update(kw)
        A = SkRunArgsC(*args.values())
        return L.drift_pt_sk_run(C.byref(P), C.byref(A), C.byref(S), C.c_void_p(fake), 1 << 20, None)

    assert run(replicas_per_cta=13) == _lib.EINVAL
    assert "replicas_per_cta" in L.drift_pt_last_error().decode()
    assert run(n_replicas=1) == _lib.EINVAL
    assert run(n_replicas=513) == _lib.EINVAL
    assert run(sweeps_per_round=0) == _lib.EINVAL
    assert run(instance=1 << 24) == _lib.EINVAL
    assert L.drift_pt_sk_run(C.byref(P), C.byref(SkRunArgsC(64, 1, 1, 4, 0, 0, 0, 0, fake, fake, 1.0)), C.byref(S),
                             C.c_void_p(fake), 16, None) == _lib.EINVAL  # workspace too small
    assert "workspace" in L.drift_pt_last_error().decode()
    bad = SkProblemC(600, 25, fake, fake, fake)
    assert L.drift_pt_sk_init(C.byref(bad), C.byref(SkRunArgsC(64, 1, 1, 4, 0, 0, 0, 0, fake, fake, 1.0)),
                              C.byref(S), None) == _lib.EINVAL
