"""ORACLE - test infrastructure only.

CPU restatements of the reference's parallel-tempering path, used as the checker by the tests,
by ``__graft_entry__.smoke()`` and as the timed CPU baseline of ``bench.py``. Nothing in the
product (``drift_b200``) imports this package.

  * ``liboracle.so`` (built from ``pt_oracle.c`` and ``exact.c`` by ``Makefile``):
      - ``philox``          Philox4x32-10 (Salmon et al., SC'11), written independently of the
                            engine's copy;
      - ``greedy_coloring`` drift/gpu.py:122-145;
      - ``pt_run``          the colour-ordered sweep of cuda/ising_pt.cu:109-135 and the
                            adjacent-rung exchange of drift/solvers/parallel_tempering.py:104-113,
                            driven by the same counter-based uniforms as the engine, so spins,
                            energies and swap counts can be compared bit for bit;
      - ``exact``           drift/solvers/exact.py:20-49 as a Gray-code walk (n <= 30), plus
                            Boltzmann averages;
      - ``ms_run``          the bit-packed lattice chain (ms_oracle.c);
      - ``sk_run``          the dense-coupling chain on fixed-point couplings (sk_oracle.c);
      - ``gms_run``         the bit-packed chain on a +-1 graph (gms_oracle.c).
  * ``ref_pt`` - NumPy restatement of the reference CPU parallel tempering
    (drift/solvers/parallel_tempering.py:29-124) with the same NumPy random stream, pinned to the
    reference by golden outputs in tests/golden/.

Parity pins: Philox against the Random123 known-answer vectors, the exact enumerator and
``ref_pt`` against outputs of the reference itself (tests/golden/, generated by
tests/golden/make_golden.py). The engine-specific definitions (uniform layout, thresholds,
fixed-point energies) have no reference counterpart; they are pinned by restating them here
independently.
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

_lib = None


def build(force: bool = False) -> str:
    srcs = [os.path.join(HERE, f) for f in ("pt_oracle.c", "exact.c", "ms_oracle.c", "sk_oracle.c", "gms_oracle.c",
                                             "Makefile")]
    if force or not os.path.exists(LIB_PATH) or any(os.path.getmtime(s) > os.path.getmtime(LIB_PATH) for s in srcs):
        r = subprocess.run(["make", "-s", "-C", HERE, "-B" if force else "all"], capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"oracle build failed:\n{r.stdout}\n{r.stderr}")
    return LIB_PATH


REF_BIN = os.path.join(HERE, "_ref", "ising_pt")


def reference_tree() -> str | None:
    """The reference (DRiFT) source tree named by the DRIFT_REFERENCE_TREE environment variable, if
    it is set and holds the tree; None otherwise."""
    root = os.environ.get("DRIFT_REFERENCE_TREE")
    return root if root and os.path.isdir(os.path.join(root, "cuda")) else None


def build_ref() -> str | None:
    """Compile the reference's own GPU engine (cuda/ising_pt.cu, unchanged) into _ref/ when its
    source tree is named by DRIFT_REFERENCE_TREE; returns the binary's path if it exists afterwards."""
    root = reference_tree()
    if root is not None and os.path.exists(os.path.join(root, "cuda", "ising_pt.cu")):
        r = subprocess.run(["make", "-s", "-C", HERE, "ref", f"REFERENCE={root}"], capture_output=True,
                           text=True)
        if r.returncode != 0:
            raise RuntimeError(f"reference GPU engine build failed:\n{r.stdout}\n{r.stderr}")
    return REF_BIN if os.path.exists(REF_BIN) else None


class _Problem(C.Structure):
    _fields_ = [("n", C.c_int32), ("row_ptr", C.c_void_p), ("col_idx", C.c_void_p), ("weight", C.c_void_p),
                ("h", C.c_void_p), ("n_colors", C.c_int32), ("color_ptr", C.c_void_p), ("color_spins", C.c_void_p),
                ("integer_path", C.c_int32), ("max_field", C.c_int32)]


class _Run(C.Structure):
    _fields_ = [("R", C.c_int32), ("n_rounds", C.c_int32), ("sweeps_per_round", C.c_int32), ("threads", C.c_int32),
                ("round_offset", C.c_int64), ("seed", C.c_uint64), ("instance", C.c_uint32),
                ("betas", C.c_void_p), ("thr", C.c_void_p), ("init", C.c_int32)]


class _State(C.Structure):
    _fields_ = [("spins", C.c_void_p), ("energy", C.c_void_p), ("best_energy", C.c_void_p),
                ("best_spins", C.c_void_p), ("rung_of_slot", C.c_void_p), ("slot_of_rung", C.c_void_p),
                ("tried", C.c_void_p), ("accepted", C.c_void_p), ("best_history", C.c_void_p)]


class _ExactOut(C.Structure):
    _fields_ = [("e_min", C.c_double), ("argmin", C.c_uint64), ("mean_e", C.c_void_p), ("mean_e2", C.c_void_p),
                ("mean_absm", C.c_void_p), ("mean_m2", C.c_void_p), ("site_mag", C.c_void_p),
                ("spectrum", C.c_void_p)]


class _MsOracle(C.Structure):
    _fields_ = [("dims", C.c_int32), ("L", C.c_int32), ("W", C.c_int32), ("jneg", C.c_void_p), ("betas", C.c_void_p),
                ("thr", C.c_void_p), ("seed", C.c_uint64), ("instance", C.c_uint32), ("n_rounds", C.c_int32),
                ("spr", C.c_int32), ("init", C.c_int32), ("round_offset", C.c_int64), ("words", C.c_void_p),
                ("best_words", C.c_void_p), ("energy", C.c_void_p), ("best_energy", C.c_void_p),
                ("rung_of_slot", C.c_void_p), ("slot_of_rung", C.c_void_p), ("tried", C.c_void_p),
                ("accepted", C.c_void_p)]


class _SkOracle(C.Structure):
    _fields_ = [("n", C.c_int32), ("R", C.c_int32), ("n_rounds", C.c_int32), ("spr", C.c_int32), ("init", C.c_int32),
                ("threads", C.c_int32), ("Jq", C.c_void_p), ("hq", C.c_void_p), ("betas", C.c_void_p),
                ("scales", C.c_void_p), ("escale", C.c_double), ("seed", C.c_uint64), ("instance", C.c_uint32),
                ("reserved", C.c_int32), ("round_offset", C.c_int64), ("spins", C.c_void_p),
                ("best_spins", C.c_void_p), ("energy", C.c_void_p), ("best_energy", C.c_void_p),
                ("rung_of_slot", C.c_void_p), ("slot_of_rung", C.c_void_p), ("tried", C.c_void_p),
                ("accepted", C.c_void_p), ("best_history", C.c_void_p)]


class _GmsOracle(C.Structure):
    _fields_ = [("n", C.c_int32), ("n_pos", C.c_int32), ("k", C.c_int32), ("D", C.c_int32), ("W", C.c_int32),
                ("n_rounds", C.c_int32), ("spr", C.c_int32), ("init", C.c_int32), ("color_ptr", C.c_void_p),
                ("ell", C.c_void_p), ("degree", C.c_void_p), ("jneg", C.c_void_p), ("n_bonds", C.c_int64),
                ("betas", C.c_void_p), ("thr", C.c_void_p), ("seed", C.c_uint64), ("instance", C.c_uint32),
                ("reserved", C.c_int32), ("round_offset", C.c_int64), ("words", C.c_void_p),
                ("best_words", C.c_void_p), ("energy", C.c_void_p), ("best_energy", C.c_void_p),
                ("rung_of_slot", C.c_void_p), ("slot_of_rung", C.c_void_p), ("tried", C.c_void_p),
                ("accepted", C.c_void_p)]


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB_PATH)
        L.oracle_philox4x32_10.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.oracle_greedy_coloring.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.oracle_greedy_coloring.restype = C.c_int
        L.oracle_pt_run.argtypes = [C.POINTER(_Problem), C.POINTER(_Run), C.POINTER(_State)]
        L.oracle_pt_run.restype = C.c_int
        L.oracle_exact.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.POINTER(_ExactOut)]
        L.oracle_exact.restype = C.c_int
        L.oracle_exp_neg_d.argtypes = [C.c_double]
        L.oracle_exp_neg_d.restype = C.c_double
        L.oracle_exp_neg_f.argtypes = [C.c_float]
        L.oracle_exp_neg_f.restype = C.c_float
        L.oracle_threshold_int.argtypes = [C.c_double, C.c_int]
        L.oracle_threshold_int.restype = C.c_uint32
        L.oracle_energy_fp64.argtypes = [C.POINTER(_Problem), C.c_void_p]
        L.oracle_energy_fp64.restype = C.c_double
        L.oracle_ms_run.argtypes = [C.POINTER(_MsOracle)]
        L.oracle_ms_run.restype = C.c_int
        L.oracle_gms_run.argtypes = [C.POINTER(_GmsOracle)]
        L.oracle_gms_run.restype = C.c_int
        L.oracle_sk_run.argtypes = [C.POINTER(_SkOracle)]
        L.oracle_sk_run.restype = C.c_int
        L.oracle_sk_energy.argtypes = [C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p]
        L.oracle_sk_energy.restype = C.c_int64
        L.oracle_neg_log_unit.argtypes = [C.c_float]
        L.oracle_neg_log_unit.restype = C.c_float
        L.oracle_sk_threshold.argtypes = [C.c_uint32, C.c_float]
        L.oracle_sk_threshold.restype = C.c_int32
        _lib = L
    return _lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


def philox(ctr, key) -> np.ndarray:
    c = np.ascontiguousarray(ctr, dtype=np.uint32)
    k = np.ascontiguousarray(key, dtype=np.uint32)
    o = np.zeros(4, dtype=np.uint32)
    lib().oracle_philox4x32_10(_p(c), _p(k), _p(o))
    return o


def exp_neg_d(x: float) -> float:
    return lib().oracle_exp_neg_d(float(x))


def exp_neg_f(x: float) -> float:
    return lib().oracle_exp_neg_f(float(x))


def threshold_int(beta: float, x: int) -> int:
    return int(lib().oracle_threshold_int(float(beta), int(x)))


def greedy_coloring(n: int, row_ptr: np.ndarray, col_idx: np.ndarray):
    """(k, color, color_ptr, color_spins) - drift/gpu.py:122-145."""
    rp = np.ascontiguousarray(row_ptr, dtype=np.int32)
    ci = np.ascontiguousarray(col_idx, dtype=np.int32)
    color = np.zeros(max(n, 1), dtype=np.int32)
    cptr = np.zeros(n + 2, dtype=np.int32)
    cs = np.zeros(max(n, 1), dtype=np.int32)
    k = lib().oracle_greedy_coloring(n, _p(rp), _p(ci), _p(color), _p(cptr), _p(cs))
    return k, color[:n], cptr[:k + 1], cs[:n]


class OracleProblem:
    """CSR problem in the reference's own terms (drift/gpu.py:66-81) plus its colouring."""

    def __init__(self, n, row_ptr, col_idx, weight, h, color_ptr=None, color_spins=None, integer_path=None):
        self.n = int(n)
        self.row_ptr = np.ascontiguousarray(row_ptr, dtype=np.int32)
        self.col_idx = np.ascontiguousarray(col_idx, dtype=np.int32)
        self.weight = np.ascontiguousarray(weight, dtype=np.float32)
        self.h = np.ascontiguousarray(h, dtype=np.float32)
        if color_ptr is None:
            _, _, color_ptr, color_spins = greedy_coloring(self.n, self.row_ptr, self.col_idx)
        self.color_ptr = np.ascontiguousarray(color_ptr, dtype=np.int32)
        self.color_spins = np.ascontiguousarray(color_spins, dtype=np.int32)
        is_int = bool(np.all(np.round(self.weight) == self.weight) and np.all(np.abs(self.weight) <= 127)
                      and np.all(np.round(self.h) == self.h) and np.all(np.abs(self.h) <= 2 ** 20))
        if integer_path is None:
            integer_path = is_int
        self.integer_path = bool(integer_path)
        F = 0
        if self.integer_path:
            absw = np.abs(self.weight).astype(np.int64)
            rowsum = np.add.reduceat(absw, self.row_ptr[:-1]) if absw.size else np.zeros(self.n, np.int64)
            rowsum = np.where(np.diff(self.row_ptr) > 0, rowsum, 0)
            F = int(max(1, int(np.max(rowsum + np.abs(self.h).astype(np.int64)))))
        self.max_field = F

    def _c(self):
        return _Problem(self.n, _p(self.row_ptr), _p(self.col_idx), _p(self.weight), _p(self.h),
                        len(self.color_ptr) - 1, _p(self.color_ptr), _p(self.color_spins),
                        1 if self.integer_path else 0, self.max_field)


class OracleState:
    def __init__(self, n: int, R: int, n_rounds: int = 0):
        self.spins = np.zeros((R, n), dtype=np.int8)
        self.energy = np.zeros(R, dtype=np.int64)
        self.best_energy = np.zeros(R, dtype=np.int64)
        self.best_spins = np.zeros((R, n), dtype=np.int8)
        self.rung_of_slot = np.arange(R, dtype=np.int32)
        self.slot_of_rung = np.arange(R, dtype=np.int32)
        self.tried = np.zeros(max(R - 1, 1), dtype=np.int64)
        self.accepted = np.zeros(max(R - 1, 1), dtype=np.int64)
        self.best_history = np.zeros(max(n_rounds, 1), dtype=np.float64)


def thresholds(betas: np.ndarray, F: int) -> np.ndarray:
    return np.array([[threshold_int(b, x) for x in range(1, F + 1)] for b in betas], dtype=np.uint32)


def pt_run(prob: OracleProblem, betas, *, n_rounds: int, sweeps_per_round: int, seed: int, instance: int = 0,
           state: OracleState | None = None, round_offset: int = 0, thr: np.ndarray | None = None,
           threads: int = 0) -> OracleState:
    """Run (or continue, with ``state`` and ``round_offset``) the oracle chain."""
    betas = np.ascontiguousarray(betas, dtype=np.float64)
    R = len(betas)
    init = state is None
    if state is None:
        state = OracleState(prob.n, R, n_rounds)
    if len(state.best_history) < max(n_rounds, 1):
        state.best_history = np.zeros(max(n_rounds, 1), dtype=np.float64)
    if prob.integer_path and thr is None:
        thr = thresholds(betas, prob.max_field)
    thr = np.ascontiguousarray(thr, dtype=np.uint32) if thr is not None else None
    P = prob._c()
    A = _Run(R, n_rounds, sweeps_per_round, threads, round_offset, seed & 0xFFFFFFFFFFFFFFFF, instance,
             _p(betas), _p(thr) if thr is not None else None, 1 if init else 0)
    S = _State(_p(state.spins), _p(state.energy), _p(state.best_energy), _p(state.best_spins),
               _p(state.rung_of_slot), _p(state.slot_of_rung), _p(state.tried), _p(state.accepted),
               _p(state.best_history))
    rc = lib().oracle_pt_run(C.byref(P), C.byref(A), C.byref(S))
    if rc != 0:
        raise ValueError("oracle_pt_run: invalid arguments")
    return state


def energy_fp64(prob: OracleProblem, spins: np.ndarray) -> float:
    s = np.ascontiguousarray(spins, dtype=np.int8)
    P = prob._c()
    return float(lib().oracle_energy_fp64(C.byref(P), _p(s)))


class ExactResult:
    def __init__(self, e_min, argmin, mean_e, mean_e2, mean_absm, mean_m2, site_mag, spectrum):
        self.e_min, self.argmin = e_min, argmin
        self.mean_e, self.mean_e2, self.mean_absm, self.mean_m2 = mean_e, mean_e2, mean_absm, mean_m2
        self.site_mag, self.spectrum = site_mag, spectrum


def exact(J: np.ndarray, h: np.ndarray, betas=(), spectrum: bool = False, site_mag: bool = False) -> ExactResult:
    """Exact enumeration (drift/solvers/exact.py:34-49) plus Boltzmann averages at ``betas``."""
    J = np.ascontiguousarray(J, dtype=np.float64)
    h = np.ascontiguousarray(h, dtype=np.float64)
    n = h.shape[0]
    betas = np.ascontiguousarray(betas, dtype=np.float64)
    nb = len(betas)
    me, me2, ma, mm2 = (np.zeros(max(nb, 1)) for _ in range(4))
    sm = np.zeros((max(nb, 1), n)) if site_mag else None
    spec = np.zeros(1 << n) if spectrum else None
    out = _ExactOut(0.0, 0, _p(me), _p(me2), _p(ma), _p(mm2), _p(sm) if sm is not None else None,
                    _p(spec) if spec is not None else None)
    rc = lib().oracle_exact(n, _p(J), _p(h), nb, _p(betas) if nb else None, C.byref(out))
    if rc != 0:
        raise ValueError("oracle_exact: n must be in 1..30")
    return ExactResult(out.e_min, out.argmin, me[:nb], me2[:nb], ma[:nb], mm2[:nb],
                       sm[:nb] if sm is not None else None, spec)


class MsState:
    def __init__(self, W: int, N: int):
        R = 32 * W
        self.words = np.zeros((W, N), np.uint32)
        self.best_words = np.zeros((W, N), np.uint32)
        self.energy = np.zeros(R, np.int64)
        self.best_energy = np.zeros(R, np.int64)
        self.rung_of_slot = np.arange(R, dtype=np.int32)
        self.slot_of_rung = np.arange(R, dtype=np.int32)
        self.tried = np.zeros(max(R - 1, 1), np.int64)
        self.accepted = np.zeros(max(R - 1, 1), np.int64)


def ms_run(dims: int, L: int, jneg: np.ndarray, betas, *, n_rounds: int, sweeps_per_round: int, seed: int,
           instance: int = 0, state: MsState | None = None, round_offset: int = 0) -> MsState:
    """The multispin lattice chain (ms_oracle.c): jneg in colour-split site order, R = len(betas)."""
    betas = np.ascontiguousarray(betas, np.float64)
    R = len(betas)
    if R % 32:
        raise ValueError("multispin needs a multiple of 32 replicas")
    W, N = R // 32, L ** dims
    jneg = np.ascontiguousarray(jneg, np.uint8)
    thr = np.ascontiguousarray(thresholds(betas, 2 * dims), np.uint32)
    init = state is None
    if state is None:
        state = MsState(W, N)
    o = _MsOracle(dims, L, W, _p(jneg), _p(betas), _p(thr), seed & 0xFFFFFFFFFFFFFFFF, instance, n_rounds,
                  sweeps_per_round, 1 if init else 0, round_offset, _p(state.words), _p(state.best_words),
                  _p(state.energy), _p(state.best_energy), _p(state.rung_of_slot), _p(state.slot_of_rung),
                  _p(state.tried), _p(state.accepted))
    if lib().oracle_ms_run(C.byref(o)) != 0:
        raise ValueError("oracle_ms_run failed")
    return state


def neg_log_unit(u: float) -> float:
    return float(lib().oracle_neg_log_unit(u))


def sk_threshold(word: int, c: float) -> int:
    return int(lib().oracle_sk_threshold(word & 0xFFFFFFFF, c))


def sk_energy(Jq: np.ndarray, hq: np.ndarray, spins: np.ndarray) -> int:
    """E2 = -sum_i s_i (sum_j Jq_ij s_j + 2 hq_i), exact."""
    Jq = np.ascontiguousarray(Jq, np.int32)
    hq = np.ascontiguousarray(hq, np.int32)
    s = np.ascontiguousarray(spins, np.int8)
    return int(lib().oracle_sk_energy(len(hq), _p(Jq), _p(hq), _p(s)))


class SkState:
    def __init__(self, R: int, n: int):
        self.spins = np.zeros((R, n), np.int8)
        self.best_spins = np.zeros((R, n), np.int8)
        self.energy = np.zeros(R, np.int64)
        self.best_energy = np.zeros(R, np.int64)
        self.rung_of_slot = np.arange(R, dtype=np.int32)
        self.slot_of_rung = np.arange(R, dtype=np.int32)
        self.tried = np.zeros(R, np.int64)
        self.accepted = np.zeros(R, np.int64)
        self.best_history = None


def sk_run(Jq: np.ndarray, hq: np.ndarray, shift: int, betas, scales, *, n_rounds: int, sweeps_per_round: int,
           seed: int, instance: int = 0, state: SkState | None = None, round_offset: int = 0,
           threads: int = 0) -> SkState:
    """The dense-coupling chain (sk_oracle.c) on fixed-point couplings Jq, hq; R = len(betas)."""
    Jq = np.ascontiguousarray(Jq, np.int32)
    hq = np.ascontiguousarray(hq, np.int32)
    betas = np.ascontiguousarray(betas, np.float64)
    scales = np.ascontiguousarray(scales, np.float32)
    n, R = len(hq), len(betas)
    init = state is None
    if state is None:
        state = SkState(R, n)
    hist = np.zeros(max(n_rounds, 1), np.int64)
    o = _SkOracle(n, R, n_rounds, sweeps_per_round, 1 if init else 0, threads, _p(Jq), _p(hq), _p(betas), _p(scales),
                  2.0 ** -(shift + 1), seed & 0xFFFFFFFFFFFFFFFF, instance, 0, round_offset, _p(state.spins),
                  _p(state.best_spins), _p(state.energy), _p(state.best_energy), _p(state.rung_of_slot),
                  _p(state.slot_of_rung), _p(state.tried), _p(state.accepted), _p(hist))
    if lib().oracle_sk_run(C.byref(o)) != 0:
        raise ValueError("oracle_sk_run failed")
    state.best_history = hist[:n_rounds]
    return state


class GmsState:
    def __init__(self, W: int, n_pos: int):
        R = 32 * W
        self.words = np.zeros((W, n_pos), np.uint32)
        self.best_words = np.zeros((W, n_pos), np.uint32)
        self.energy = np.zeros(R, np.int64)
        self.best_energy = np.zeros(R, np.int64)
        self.rung_of_slot = np.arange(R, dtype=np.int32)
        self.slot_of_rung = np.arange(R, dtype=np.int32)
        self.tried = np.zeros(R, np.int64)
        self.accepted = np.zeros(R, np.int64)


def gms_run(layout, betas, *, n_rounds: int, sweeps_per_round: int, seed: int, instance: int = 0,
            state: GmsState | None = None, round_offset: int = 0) -> GmsState:
    """The bit-packed graph chain (gms_oracle.c); `layout` has n, n_pos, n_colors, max_degree,
    n_bonds, color_ptr, ell_nbr [D][n_pos], degree, jneg (host arrays)."""
    betas = np.ascontiguousarray(betas, np.float64)
    R = len(betas)
    if R % 32:
        raise ValueError("the multispin chain needs a multiple of 32 replicas")
    W = R // 32
    thr = np.ascontiguousarray(thresholds(betas, layout.max_degree), np.uint32)
    init = state is None
    if state is None:
        state = GmsState(W, layout.n_pos)
    cp = np.ascontiguousarray(layout.color_ptr, np.int32)
    ell = np.ascontiguousarray(layout.ell_nbr, np.int32)
    deg = np.ascontiguousarray(layout.degree, np.uint8)
    jn = np.ascontiguousarray(layout.jneg, np.uint8)
    o = _GmsOracle(layout.n, layout.n_pos, layout.n_colors, layout.max_degree, W, n_rounds, sweeps_per_round,
                   1 if init else 0, _p(cp), _p(ell), _p(deg), _p(jn), layout.n_bonds, _p(betas), _p(thr),
                   seed & 0xFFFFFFFFFFFFFFFF, instance, 0, round_offset, _p(state.words), _p(state.best_words),
                   _p(state.energy), _p(state.best_energy), _p(state.rung_of_slot), _p(state.slot_of_rung),
                   _p(state.tried), _p(state.accepted))
    if lib().oracle_gms_run(C.byref(o)) != 0:
        raise ValueError("oracle_gms_run failed")
    return state
