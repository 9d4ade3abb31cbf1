"""C ABI without a GPU: the library loads, exports every symbol include/drift_pt.h declares, and its
host helpers (colouring, layout, thresholds, argument checks) agree with the oracle."""

from __future__ import annotations

import ctypes as C
import os
import re

import numpy as np
import pytest

import oracle
from conftest import ROOT, dense_from_edges

from drift_b200 import _lib, gpu
from drift_b200.engine import HostProblem, greedy_coloring
from drift_b200.instances import ea_2d, er_gaussian, maxcut_3regular, sk_model


def header_symbols():
    with open(os.path.join(ROOT, "include", "drift_pt.h")) as f:
        return sorted(set(re.findall(r"DRIFT_PT_API\s+[\w\s\*]+?\b(drift_pt_\w+)\(", f.read())))


def test_library_exports_every_declared_symbol():
    L = _lib.load()
    declared = header_symbols()
    assert len(declared) >= 13
    assert sorted(_lib.EXPORTED) == declared
    for name in declared:
        assert hasattr(L, name), name
    assert L.drift_pt_version().decode().startswith("drift-b200-pt")


def test_gpu_available_is_a_bool():
    assert isinstance(gpu.gpu_available(), bool)


def test_missing_engine_raises_not_built(monkeypatch, tmp_path):
    monkeypatch.setattr(_lib, "LIB_PATH", str(tmp_path / "missing.so"))
    monkeypatch.setattr(_lib, "_lib", None)
    assert gpu.gpu_available() is False
    with pytest.raises(RuntimeError, match="not built"):
        gpu.parallel_tempering_gpu(dense_from_edges(4, {"i": [0, 1, 2], "j": [1, 2, 3], "w": [1.0] * 3}, [0.0] * 4),
                                   n_replicas=2, n_rounds=2)
    with pytest.raises(RuntimeError, match="not built"):
        _lib.load()


def test_greedy_coloring_matches_oracle_and_reference(reference_instances):
    for name, d in reference_instances.items():
        m = dense_from_edges(d["n"], d["edges"], d["h"])
        rp, ci, _ = m.csr()
        k, cptr, cs = greedy_coloring(m.n, rp, ci)
        assert k == d["coloring"]["k"] and cptr.tolist() == d["coloring"]["color_ptr"], name
        assert cs.tolist() == d["coloring"]["color_spins"], name
    for m in (ea_2d(16, 1), maxcut_3regular(4096, 2), er_gaussian(3000, 6, 5)):
        rp, ci, _ = m.csr()
        k, cptr, cs = greedy_coloring(m.n, rp, ci)
        ko, _, cpo, cso = oracle.greedy_coloring(m.n, rp, ci)
        assert k == ko and np.array_equal(cptr, cpo) and np.array_equal(cs, cso)
    assert greedy_coloring(256, *ea_2d(16, 1).csr()[:2])[0] == 2  # checkerboard


def _layout(hp, integer_path):
    L = _lib.load()
    csr = hp.c_csr()
    info = _lib.LayoutInfo()
    _lib.check(L.drift_pt_layout_query(C.byref(csr), C.byref(info)), "query")
    arrs = dict(color_ptr=np.zeros(info.n_colors + 1, np.int32), slice_off=np.zeros(info.n_slices + 1, np.int32),
                ell_nbr=np.zeros(max(info.n_ell, 1), np.int32),
                ell_w=np.zeros(max(info.n_ell, 1), np.int8 if integer_path else np.float32),
                h_pos=np.zeros(info.n_pos, np.int32 if integer_path else np.float32),
                site_of_pos=np.zeros(info.n_pos, np.int32), pos_of_site=np.zeros(info.n, np.int32))
    p = lambda a: a.ctypes.data_as(C.c_void_p)
    lay = _lib.Layout(*(p(arrs[k]) for k in ("color_ptr", "slice_off", "ell_nbr", "ell_w", "h_pos", "site_of_pos",
                                             "pos_of_site")))
    _lib.check(L.drift_pt_layout_fill(C.byref(csr), 1 if integer_path else 0, C.byref(lay)), "fill")
    return info, arrs


@pytest.mark.parametrize("make,integer", [(lambda: ea_2d(16, 1), True), (lambda: maxcut_3regular(1024, 3), True),
                                          (lambda: er_gaussian(700, 6, 2), False), (lambda: sk_model(64, 4), False)])
def test_layout_decodes_back_to_the_csr(make, integer):
    m = make()
    hp = HostProblem.from_model(m)
    info, a = _layout(hp, integer)
    assert info.integer_couplings == (1 if integer else 0)
    n = hp.n
    assert np.array_equal(a["site_of_pos"][:n], hp.color_spins)
    assert np.all(a["site_of_pos"][n:] == -1)
    assert np.array_equal(a["pos_of_site"][hp.color_spins], np.arange(n))
    so = a["slice_off"]
    for p in range(info.n_pos):
        S, lane, q = p // 256, (p % 256) // 8, p % 8
        width = so[S + 1] - so[S]
        i = a["site_of_pos"][p]
        hv = a["h_pos"][S * 256 + q * 32 + lane]
        if i < 0:
            assert hv == 0
            continue
        assert hv == hp.h[i]
        lo, hi = hp.row_ptr[i], hp.row_ptr[i + 1]
        deg = hi - lo
        assert deg <= width
        for d in range(width):
            e = so[S] * 256 + (d * 8 + q) * 32 + lane
            if d < deg:
                assert a["ell_nbr"][e] == a["pos_of_site"][hp.col_idx[lo + d]]
                assert a["ell_w"][e] == hp.weight[lo + d]
            else:
                assert a["ell_w"][e] == 0 and a["ell_nbr"][e] == p


def test_integer_detection_and_max_field():
    hp = HostProblem.from_model(maxcut_3regular(1024, 3))
    info, _ = _layout(hp, True)
    assert info.integer_couplings == 1 and info.max_field == 3
    hp = HostProblem.from_model(er_gaussian(500, 6, 1))
    info, _ = _layout(hp, False)
    assert info.integer_couplings == 0


def test_thresholds_match_oracle():
    L = _lib.load()
    betas = np.array([0.0, 0.1, 0.25, 0.333, 1.0, 2.0, 3.0, 4.0])
    F = 12
    thr = np.zeros(len(betas) * F, np.uint32)
    _lib.check(L.drift_pt_thresholds(len(betas), betas.ctypes.data_as(C.c_void_p), F,
                                     thr.ctypes.data_as(C.c_void_p)), "thresholds")
    assert np.array_equal(thr.reshape(len(betas), F), oracle.thresholds(betas, F))
    assert np.all(thr.reshape(len(betas), F)[0] == 0xFFFFFFFF)  # beta = 0 accepts everything


def test_invalid_inputs_are_rejected_with_a_message():
    L = _lib.load()
    m = ea_2d(4, 0)
    hp = HostProblem.from_model(m)
    bad = HostProblem(hp.n, hp.row_ptr, hp.col_idx, hp.weight, hp.h, np.array([0, hp.n], np.int32),
                      np.arange(hp.n, dtype=np.int32))  # one colour: coupled spins share it
    info = _lib.LayoutInfo()
    rc = L.drift_pt_layout_query(C.byref(bad.c_csr()), C.byref(info))
    assert rc == _lib.EINVAL
    assert "invalid colouring" in L.drift_pt_last_error().decode()
    perm = hp.color_spins.copy()
    perm[0] = perm[1]
    bad2 = HostProblem(hp.n, hp.row_ptr, hp.col_idx, hp.weight, hp.h, hp.color_ptr, perm)
    assert L.drift_pt_layout_query(C.byref(bad2.c_csr()), C.byref(info)) == _lib.EINVAL
    assert "permutation" in L.drift_pt_last_error().decode()
    ws = C.c_size_t(0)
    assert L.drift_pt_workspace_bytes(0, C.byref(ws)) == _lib.EINVAL
    assert L.drift_pt_workspace_bytes(64, C.byref(ws)) == _lib.OK and ws.value >= 64 * 16
    # device entry points reject NULL problems before touching the GPU
    assert L.drift_pt_init(None, None, None, None) == _lib.EINVAL
    assert L.drift_pt_run(None, None, None, None, 0, None) == _lib.EINVAL


def test_ctypes_structs_match_the_header(tmp_path):
    """Every struct of include/drift_pt.h has the same size and field offsets as its ctypes mirror."""
    import shutil
    import subprocess

    from drift_b200.batch import DESC_DTYPE
    from drift_b200.gms import GmsLayoutC, GmsLayoutInfoC, GmsProblemC, GmsRunArgsC, GmsStateC
    from drift_b200.multispin import LatticeC, MsRunArgsC, MsStateC
    from drift_b200.sk import SkProblemC, SkRunArgsC, SkStateC

    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    mirrors = {"DriftPtCsr": _lib.Csr, "DriftPtLayoutInfo": _lib.LayoutInfo, "DriftPtLayout": _lib.Layout,
               "DriftPtDeviceProblem": _lib.DeviceProblem, "DriftPtDeviceState": _lib.DeviceState,
               "DriftPtRunArgs": _lib.RunArgs, "DriftPtSolveArgs": _lib.SolveArgs,
               "DriftPtSolveResult": _lib.SolveResult, "DriftPtBatchProblem": _lib.BatchProblem,
               "DriftPtBatchRunArgs": _lib.BatchRunArgs, "DriftPtLattice": LatticeC, "DriftPtMsState": MsStateC,
               "DriftPtMsRunArgs": MsRunArgsC, "DriftPtSkProblem": SkProblemC, "DriftPtSkState": SkStateC,
               "DriftPtSkRunArgs": SkRunArgsC, "DriftPtGmsProblem": GmsProblemC,
               "DriftPtGmsLayoutInfo": GmsLayoutInfoC, "DriftPtGmsLayout": GmsLayoutC, "DriftPtGmsState": GmsStateC,
               "DriftPtGmsRunArgs": GmsRunArgsC}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "drift_pt.h"', "int main(void) {"]
    for cname, py in mirrors.items():
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            lines.append(f'printf("{cname}.{fname} %zu\\n", offsetof({cname}, {fname}));')
    lines.append('printf("DriftPtInstanceDesc size %zu\\n", sizeof(DriftPtInstanceDesc));')
    for fname in DESC_DTYPE.names:
        lines.append(f'printf("DriftPtInstanceDesc.{fname} %zu\\n", offsetof(DriftPtInstanceDesc, {fname}));')
    lines.append("return 0; }")
    src = tmp_path / "probe.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "probe"
    subprocess.run([cc, "-I", os.path.join(ROOT, "include"), "-o", str(exe), str(src)], check=True)
    got = dict(l.rsplit(" ", 1) for l in subprocess.run([str(exe)], capture_output=True, text=True,
                                                         check=True).stdout.splitlines())
    for cname, py in mirrors.items():
        assert int(got[f"{cname} size"]) == C.sizeof(py), cname
        for fname, _ in py._fields_:
            assert int(got[f"{cname}.{fname}"]) == getattr(py, fname).offset, f"{cname}.{fname}"
    assert int(got["DriftPtInstanceDesc size"]) == DESC_DTYPE.itemsize
    for fname in DESC_DTYPE.names:
        assert int(got[f"DriftPtInstanceDesc.{fname}"]) == DESC_DTYPE.fields[fname][1], fname
