"""drift_pt_unit_placement (CPU): the unit-regular form's storage order of spin words is a permutation
that fills every shared-memory bank equally, and it lowers the number of shared-memory passes of the
form's neighbour gathers, counted here from the kernel's item schedule (item = glo * (8 / P) + lt,
warp = lt / 32, load index i W + d): on MaxCut N = 4096 by at least a fifth, and never above the
positions' own order. The chain does not depend on it (the GPU parity tests run with it)."""

from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from drift_b200 import _lib
from drift_b200.engine import HostProblem, _ptr
from drift_b200.instances import ea_2d, gnp_pm, maxcut_3regular


def placement(hp: HostProblem, P: int = 0) -> np.ndarray:
    n_pos = ((hp.n + 255) // 256) * 256
    out = np.zeros(n_pos // 4, np.uint16)
    _lib.check(_lib.load().drift_pt_unit_placement(C.byref(hp.c_csr()), P, _ptr(out)), "unit_placement")
    return out


def gather_passes(hp: HostProblem, word_slot: np.ndarray, P: int) -> int:
    """Shared-memory passes of one sweep's gathers and own-word accesses (max distinct words per bank)."""
    n = hp.n
    pos_of_site = np.empty(n, np.int64)
    pos_of_site[hp.color_spins] = np.arange(n)
    NB = 8 // P
    sets: dict = {}
    cp = hp.color_ptr
    for c in range(len(cp) - 1):
        lo, hi = int(cp[c]), int(cp[c + 1])
        glo, ghi = lo >> 3, (hi + 7) >> 3
        for lt in range((ghi - glo) * NB):
            item, w = glo * NB + lt, lt >> 5
            sets.setdefault((c, w, "own"), set()).add(item * P // 4)
            for i in range(P):
                p = item * P + i
                if p >= n:
                    continue
                s = hp.color_spins[p]
                for d, q in enumerate(pos_of_site[hp.col_idx[hp.row_ptr[s]:hp.row_ptr[s + 1]]]):
                    sets.setdefault((c, w, i, d), set()).add(int(q) // 4)
    return sum(int(np.bincount([int(word_slot[u]) % 32 for u in us], minlength=32).max()) for us in sets.values())


@pytest.mark.parametrize("make", [lambda: maxcut_3regular(4096, 2), lambda: maxcut_3regular(1024, 7),
                                  lambda: ea_2d(16, 1), lambda: ea_2d(5, 2)])
def test_placement_is_a_balanced_permutation(make):
    hp = HostProblem.from_model(make())
    ws = placement(hp)
    words = len(ws)
    assert np.array_equal(np.sort(ws.astype(np.int64)), np.arange(words))
    assert np.all(np.bincount(ws.astype(np.int64) % 32, minlength=32) == words // 32)


def test_placement_lowers_the_gather_passes():
    hp = HostProblem.from_model(maxcut_3regular(4096, 2))
    words = ((hp.n + 255) // 256) * 64
    for P in (2, 4):
        ours = gather_passes(hp, placement(hp, P), P)
        plain = gather_passes(hp, np.arange(words), P)
        assert ours <= 0.8 * plain, (P, ours, plain)
    lat = HostProblem.from_model(ea_2d(16, 1))  # a lattice: its own order is conflict-free already
    assert gather_passes(lat, placement(lat, 2), 2) <= gather_passes(lat, np.arange(64), 2)


def test_placement_refuses_problems_outside_the_form():
    hp = HostProblem.from_model(gnp_pm(40, 0.2, 3))
    out = np.zeros(64, np.uint16)
    assert _lib.load().drift_pt_unit_placement(C.byref(hp.c_csr()), 0, _ptr(out)) == _lib.EUNSUPPORTED
