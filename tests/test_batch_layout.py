"""The batch layout built in two calls (drift_pt_batch_layout_query/fill, instances split over host
threads) equals the concatenation of the per-instance layouts and thresholds, on the integer and the
fp32 path, with the descriptor offsets pointing at each instance's part."""

from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from drift_b200 import _lib
from drift_b200.batch import BatchProblem
from drift_b200.engine import HostProblem, _ptr
from drift_b200.instances import ea_2d, er_gaussian, maxcut_3regular


def per_instance(hp, integer_path, betas):
    L = _lib.load()
    info = _lib.LayoutInfo()
    _lib.check(L.drift_pt_layout_query(C.byref(hp.c_csr()), C.byref(info)), "layout_query")
    cp = np.zeros(info.n_colors + 1, np.int32)
    so = np.zeros(info.n_slices + 1, np.int32)
    nb = np.zeros(max(info.n_ell, 1), np.int32)
    w = np.zeros(max(info.n_ell, 1), np.int8 if integer_path else np.float32)
    h = np.zeros(info.n_pos, np.int32 if integer_path else np.float32)
    sop = np.zeros(info.n_pos, np.int32)
    pos = np.zeros(info.n, np.int32)
    lay = _lib.Layout(_ptr(cp), _ptr(so), _ptr(nb), _ptr(w), _ptr(h), _ptr(sop), _ptr(pos))
    _lib.check(L.drift_pt_layout_fill(C.byref(hp.c_csr()), 1 if integer_path else 0, C.byref(lay)), "layout_fill")
    thr = np.zeros(len(betas) * info.max_field, np.uint32)
    if integer_path:
        _lib.check(L.drift_pt_thresholds(len(betas), _ptr(np.ascontiguousarray(betas)), info.max_field, _ptr(thr)),
                   "thresholds")
    return info, cp, so, nb[: info.n_ell], w[: info.n_ell], h, sop, pos, thr


@pytest.mark.parametrize("integer_path", [True, False])
def test_batch_layout_equals_the_per_instance_layouts(integer_path):
    if integer_path:
        models = [ea_2d(L, k) for k, L in enumerate((4, 9, 16, 23, 5))] + [maxcut_3regular(300, 1)]
    else:
        models = [er_gaussian(n, 6, 40 + n, field_sigma=0.1) for n in (64, 301, 1000, 77)]
    hps = [HostProblem.from_model(m) for m in models]
    rng = np.random.default_rng(1)
    ladders = [0.1 * 30.0 ** (np.arange(R) / (R - 1)) for R in rng.integers(2, 40, size=len(hps))]
    sid = np.arange(len(hps)) * 7 + 3
    bp = BatchProblem(hps, ladders, stream_ids=sid, device="cpu", integer_path=integer_path)
    parts = [per_instance(hp, integer_path, b) for hp, b in zip(hps, ladders)]
    cat = lambda i: np.concatenate([p[i] for p in parts])
    assert np.array_equal(bp.d_color_ptr.numpy(), cat(1))
    assert np.array_equal(bp.d_slice_off.numpy(), cat(2))
    assert np.array_equal(bp.d_ell_nbr.numpy()[:-4], cat(3)) and np.all(bp.d_ell_nbr.numpy()[-4:] == 0)
    assert np.array_equal(bp.d_ell_w.numpy()[:-16], cat(4))
    assert np.array_equal(bp.d_h_pos.numpy(), cat(5))
    for k, p in enumerate(parts):
        d = bp.desc[k]
        assert (d["n"], d["n_pos"], d["n_slices"], d["n_colors"]) == (p[0].n, p[0].n_pos, p[0].n_slices, p[0].n_colors)
        assert d["n_replicas"] == len(ladders[k]) and d["stream_id"] == sid[k]
        assert d["max_field"] == (p[0].max_field if integer_path else 0)
        assert np.array_equal(bp.site_of_pos[k], p[6]) and np.array_equal(bp.pos_of_site[k], p[7])
        off = int(d["pos"])
        assert np.array_equal(bp.d_h_pos.numpy()[off: off + p[0].n_pos], p[5])
        if integer_path:
            t = bp.d_thr.numpy().view(np.uint32)[int(d["thr"]): int(d["thr"]) + len(p[8])]
            assert np.array_equal(t, p[8])
    assert bp.total_slots == sum(len(b) for b in ladders)


def test_batch_layout_rejects_bad_input_with_the_instance_named():
    hps = [HostProblem.from_model(ea_2d(4, 1)), HostProblem.from_model(er_gaussian(50, 6, 2))]
    with pytest.raises(ValueError, match="non-integer"):
        BatchProblem(hps, [np.ones(4), np.ones(4)], device="cpu", integer_path=True)
    with pytest.raises(ValueError, match="stream_ids"):
        BatchProblem(hps, [np.ones(4), np.ones(4)], device="cpu", stream_ids=[0, 1 << 24])
