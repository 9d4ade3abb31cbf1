"""Graph multispin layer, CPU side: the layout (colour-ordered positions, neighbour table, coupling
signs), what it rejects, and the oracle's bit-packed chain: exact energies, and Boltzmann averages
of exact enumeration per rung."""

from __future__ import annotations

import numpy as np
import pytest

import oracle
from drift_b200 import _lib
from drift_b200.engine import HostProblem
from drift_b200.gms import GmsLayout
from drift_b200.instances import ea_2d, gnp_pm, maxcut_3regular


def dense_J(model):
    return model.to_dense().J if hasattr(model, "to_dense") else model.J


def with_isolated(model, extra):
    """The model with `extra` uncoupled spins appended (degree-0 positions)."""
    from drift_b200.ising import IsingModel

    J = dense_J(model)
    n = J.shape[0] + extra
    Jx = np.zeros((n, n))
    Jx[: J.shape[0], : J.shape[0]] = J
    return IsingModel(Jx, np.zeros(n))


@pytest.mark.parametrize("model", [maxcut_3regular(64, 1), gnp_pm(40, 0.1, 7), ea_2d(8, 2),
                                   with_isolated(gnp_pm(16, 0.3, 5), 3)])
def test_layout_decodes_to_the_graph(model):
    hp = HostProblem.from_model(model)
    lay = GmsLayout(hp)
    n = model.n
    assert lay.n == n and lay.n_pos % 32 == 0 and np.array_equal(lay.color_ptr, hp.color_ptr)
    assert np.array_equal(lay.site_of_pos[:n], hp.color_spins) and np.all(lay.site_of_pos[n:] == -1)
    J = dense_J(model)
    for p in range(n):
        i = lay.site_of_pos[p]
        nbrs = np.nonzero(J[i])[0]
        assert lay.degree[p] == len(nbrs)
        for d, j in enumerate(nbrs):
            assert lay.ell_nbr[d, p] == lay.pos_of_site[j]
            assert ((lay.jneg[p] >> d) & 1) == (J[i, j] < 0)
    assert lay.n_bonds == np.count_nonzero(np.triu(J, 1))


def test_layout_rejects_what_it_cannot_run():
    m = gnp_pm(20, 0.3, 2)
    m.h[:] = 1.0
    with pytest.raises(_lib.EngineError, match="no field"):
        GmsLayout.from_model(m)
    m = gnp_pm(20, 0.3, 2)
    m.J[m.J != 0] *= 2.0
    with pytest.raises(_lib.EngineError, match=r"\+-1"):
        GmsLayout.from_model(m)
    from drift_b200.ising import IsingModel

    J = np.ones((10, 10)) - np.eye(10)  # degree 9
    with pytest.raises(_lib.EngineError, match="degree"):
        GmsLayout.from_model(IsingModel(J, np.zeros(10)))


def _unpack(words, lay, W):
    w = np.asarray(words, np.uint32).reshape(W, lay.n_pos)
    bits = (w[:, None, :] >> np.arange(32, dtype=np.uint32)[None, :, None]) & 1
    return (1 - 2 * bits.astype(np.int8)).reshape(32 * W, lay.n_pos)[:, lay.pos_of_site]


def test_oracle_energies_are_exact():
    m = gnp_pm(40, 0.1, 7)
    lay = GmsLayout.from_model(m)
    betas = 0.1 * 30.0 ** (np.arange(64) / 63)
    st = oracle.gms_run(lay, betas, n_rounds=5, sweeps_per_round=2, seed=4)
    for words, e in ((st.words, st.energy), (st.best_words, st.best_energy)):
        s = _unpack(words, lay, 2)
        ref = -0.5 * np.einsum("ri,ij,rj->r", s.astype(np.float64), m.J, s.astype(np.float64))
        assert np.array_equal(ref.astype(np.int64), e)


def test_oracle_chain_samples_the_boltzmann_distribution():
    m = gnp_pm(16, 0.3, 5)
    lay = GmsLayout.from_model(m)
    betas = 0.2 * 15.0 ** (np.arange(32) / 31)
    ex = oracle.exact(m.J, m.h, betas)
    st = None
    E = []
    for t in range(600):
        st = oracle.gms_run(lay, betas, n_rounds=1, sweeps_per_round=2, seed=6, state=st, round_offset=t)
        E.append(st.energy[st.slot_of_rung].copy())
    from drift_b200.observables import blocked

    mE, sE = blocked(np.array(E, np.float64))
    assert np.all(np.abs(mE - ex.mean_e) <= 3.0 * sE + 1e-9), (mE, ex.mean_e, sE)
