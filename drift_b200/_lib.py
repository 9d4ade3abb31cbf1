"""ctypes binding of libdrift_pt.so (declarations in include/drift_pt.h).

The library is the only compute path: if it is missing, every entry point raises RuntimeError
with "not built" in the message (the reference's convention, drift/gpu.py:59-64).
"""

from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libdrift_pt.so")

OK, EINVAL, ECUDA, ETIMEOUT, ENOMEM, EUNSUPPORTED = 0, 1, 2, 3, 4, 5

# Every symbol include/drift_pt.h declares.
EXPORTED = (
    "drift_pt_version", "drift_pt_last_error", "drift_pt_greedy_coloring", "drift_pt_color_order",
    "drift_pt_layout_query", "drift_pt_layout_fill", "drift_pt_unit_placement", "drift_pt_thresholds",
    "drift_pt_workspace_bytes",
    "drift_pt_init", "drift_pt_run", "drift_pt_check", "drift_pt_energy_fp64", "drift_pt_solve", "drift_pt_solve_release",
    "drift_pt_run_noalloc", "drift_pt_noalloc_check", "drift_pt_batch_items", "drift_pt_batch_init", "drift_pt_batch_workspace_bytes",
    "drift_pt_batch_run", "drift_pt_ms_workspace_bytes", "drift_pt_ms_init", "drift_pt_ms_run",
    "drift_pt_sk_quantize", "drift_pt_sk_layout_bytes", "drift_pt_sk_layout_fill", "drift_pt_sk_scales",
    "drift_pt_sk_workspace_bytes", "drift_pt_sk_init", "drift_pt_sk_run", "drift_pt_sk_energy",
    "drift_pt_gemm_bf16", "drift_pt_made_loss", "drift_pt_made_spins_to_bf16", "drift_pt_transpose_bf16",
    "drift_pt_colsum_bf16", "drift_pt_adam", "drift_pt_made_sample", "drift_pt_made_sample_suffix", "drift_pt_made_mh",
    "drift_pt_gms_layout_query", "drift_pt_gms_layout_fill", "drift_pt_gms_workspace_bytes", "drift_pt_gms_init",
    "drift_pt_gms_run", "drift_pt_made_group_bytes", "drift_pt_made_group_fill", "drift_pt_made_group_run",
    "drift_pt_batch_gather", "drift_pt_batch_mh", "drift_pt_batch_layout_query", "drift_pt_batch_layout_fill",
)

vp = C.c_void_p


class Csr(C.Structure):
    _fields_ = [("n", C.c_int32), ("nnz", C.c_int64), ("row_ptr", vp), ("col_idx", vp), ("weight", vp), ("h", vp),
                ("n_colors", C.c_int32), ("color_ptr", vp), ("color_spins", vp)]


class LayoutInfo(C.Structure):
    _fields_ = [("n", C.c_int32), ("n_pos", C.c_int32), ("n_slices", C.c_int32), ("n_colors", C.c_int32),
                ("n_ell", C.c_int64), ("max_degree", C.c_int32), ("integer_couplings", C.c_int32),
                ("max_field", C.c_int32), ("has_field", C.c_int32), ("min_width", C.c_int32),
                ("unit_regular", C.c_int32)]


class Layout(C.Structure):
    _fields_ = [("color_ptr", vp), ("slice_off", vp), ("ell_nbr", vp), ("ell_w", vp), ("h_pos", vp),
                ("site_of_pos", vp), ("pos_of_site", vp)]


class DeviceProblem(C.Structure):
    _fields_ = [("n", C.c_int32), ("n_pos", C.c_int32), ("n_slices", C.c_int32), ("n_colors", C.c_int32),
                ("integer_path", C.c_int32), ("max_field", C.c_int32), ("max_width", C.c_int32),
                ("max_class", C.c_int32), ("has_field", C.c_int32), ("min_width", C.c_int32),
                ("unit_regular", C.c_int32), ("n_ell", C.c_int64),
                ("color_ptr", vp), ("slice_off", vp), ("ell_nbr", vp), ("ell_w", vp), ("h_pos", vp),
                ("unit_place", vp)]


class DeviceState(C.Structure):
    _fields_ = [("spins", vp), ("energy", vp), ("best_energy", vp), ("best_spins", vp), ("rung_of_slot", vp),
                ("slot_of_rung", vp), ("swap_tried", vp), ("swap_accepted", vp), ("best_history", vp)]


class RunArgs(C.Structure):
    _fields_ = [("n_replicas", C.c_int32), ("n_rounds", C.c_int32), ("sweeps_per_round", C.c_int32),
                ("round_sync", C.c_int32), ("round_offset", C.c_int64), ("seed", C.c_uint64),
                ("instance", C.c_uint32), ("replicas_per_cta", C.c_int32), ("threads_per_cta", C.c_int32),
                ("positions_per_item", C.c_int32), ("item_form", C.c_int32), ("betas", vp), ("thresholds", vp),
                ("timeout_s", C.c_double)]


class SolveArgs(C.Structure):
    _fields_ = [("n_replicas", C.c_int32), ("n_rounds", C.c_int32), ("sweeps_per_round", C.c_int32),
                ("reserved0", C.c_int32), ("seed", C.c_uint64), ("T_min", C.c_double), ("T_max", C.c_double),
                ("betas", vp)]


class SolveResult(C.Structure):
    _fields_ = [("best_E", C.c_double), ("seconds", C.c_double), ("throughput", C.c_double),
                ("swap_rate", C.c_double), ("best_s", vp), ("rung_spins", vp), ("rung_energy", vp),
                ("swap_tried", vp), ("swap_accepted", vp), ("best_history", vp)]


class BatchProblem(C.Structure):
    _fields_ = [("n_instances", C.c_int32), ("integer_path", C.c_int32), ("has_field", C.c_int32),
                ("max_width", C.c_int32), ("min_width", C.c_int32), ("max_field", C.c_int32),
                ("max_n_pos", C.c_int32), ("max_colors", C.c_int32), ("total_slots", C.c_int64),
                ("desc", vp), ("color_ptr", vp), ("slice_off", vp), ("ell_nbr", vp), ("ell_w", vp), ("h_pos", vp),
                ("betas", vp), ("thresholds", vp)]


class BatchRunArgs(C.Structure):
    _fields_ = [("n_rounds", C.c_int32), ("sweeps_per_round", C.c_int32), ("round_offset", C.c_int64),
                ("seed", C.c_uint64), ("items", vp), ("n_items", C.c_int32), ("max_tile", C.c_int32),
                ("threads_per_slot", C.c_int32), ("ctas_per_sm", C.c_int32), ("positions_per_item", C.c_int32),
                ("max_item_bytes", C.c_int32), ("timeout_s", C.c_double)]


_lib = None


def lib_path() -> str:
    return LIB_PATH


def available() -> bool:
    return os.path.exists(LIB_PATH)


def load():
    """Load libdrift_pt.so (raises RuntimeError "... not built ..." if it is absent)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"B200 PT engine not built at {LIB_PATH}.\nBuild it with: python -m drift_b200.build")
    L = C.CDLL(LIB_PATH)
    L.drift_pt_version.restype = C.c_char_p
    L.drift_pt_last_error.restype = C.c_char_p
    L.drift_pt_greedy_coloring.argtypes = [C.c_int32, vp, vp, vp, C.POINTER(C.c_int32)]
    L.drift_pt_color_order.argtypes = [C.c_int32, vp, C.c_int32, vp, vp]
    L.drift_pt_layout_query.argtypes = [C.POINTER(Csr), C.POINTER(LayoutInfo)]
    L.drift_pt_layout_fill.argtypes = [C.POINTER(Csr), C.c_int32, C.POINTER(Layout)]
    L.drift_pt_thresholds.argtypes = [C.c_int32, vp, C.c_int32, vp]
    L.drift_pt_unit_placement.argtypes = [C.POINTER(Csr), C.c_int32, vp]
    L.drift_pt_workspace_bytes.argtypes = [C.c_int32, C.POINTER(C.c_size_t)]
    L.drift_pt_init.argtypes = [C.POINTER(DeviceProblem), C.POINTER(RunArgs), C.POINTER(DeviceState), vp]
    L.drift_pt_run.argtypes = [C.POINTER(DeviceProblem), C.POINTER(RunArgs), C.POINTER(DeviceState), vp,
                               C.c_size_t, vp]
    L.drift_pt_run_noalloc.argtypes = [C.POINTER(DeviceProblem), C.POINTER(RunArgs), C.POINTER(DeviceState), vp]
    L.drift_pt_check.argtypes = [vp, vp]
    L.drift_pt_noalloc_check.argtypes = [vp]
    L.drift_pt_batch_items.argtypes = [C.c_int32, vp, vp, C.c_int32, C.c_int64, vp, C.POINTER(C.c_int32)]
    L.drift_pt_batch_init.argtypes = [C.POINTER(BatchProblem), C.POINTER(BatchRunArgs), C.POINTER(DeviceState), vp]
    L.drift_pt_batch_workspace_bytes.argtypes = [C.POINTER(BatchProblem), C.POINTER(C.c_size_t)]
    L.drift_pt_batch_run.argtypes = [C.POINTER(BatchProblem), C.POINTER(BatchRunArgs), C.POINTER(DeviceState), vp,
                                     C.c_size_t, vp]
    L.drift_pt_energy_fp64.argtypes = [C.POINTER(DeviceProblem), vp, C.c_int32, vp, vp]
    L.drift_pt_solve.argtypes = [C.POINTER(Csr), C.POINTER(SolveArgs), C.POINTER(SolveResult)]
    for name in EXPORTED:
        if name not in ("drift_pt_version", "drift_pt_last_error"):
            getattr(L, name).restype = C.c_int
    _lib = L
    return L


class EngineError(RuntimeError):
    def __init__(self, code: int, where: str, msg: str):
        super().__init__(f"{where} failed (status {code}): {msg}")
        self.code = code


def check(rc: int, where: str) -> None:
    if rc != OK:
        msg = load().drift_pt_last_error().decode(errors="replace")
        raise EngineError(rc, where, msg)
