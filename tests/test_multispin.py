"""Multispin lattice chain without a GPU: the oracle's chain (ms_oracle.c, the chain the multispin
kernel runs bit for bit) samples the Boltzmann distribution of the lattice.

The multispin layer draws its uniforms as bit planes and decides a flip from the number of
unsatisfied bonds, so it shares no code path with the sparse engine's acceptance test. Agreement
with the exact Boltzmann averages of exact enumeration (drift/solvers/exact.py:20-49, restated in
oracle/exact.c) pins its Metropolis rule and its energy convention: per rung, the mean energy and
the mean |m| of a 2-D +-J lattice with L = 4 (16 spins) lie within 3 standard errors (blocked) of the
exact values at all 32 temperatures.
"""

from __future__ import annotations

import numpy as np

import oracle
from drift_b200.multispin import Lattice
from drift_b200.observables import blocked


def dense_couplings(lat: Lattice) -> np.ndarray:
    i, j, Jv = lat.couplings()
    J = np.zeros((lat.n, lat.n))
    np.add.at(J, (i, j), Jv)
    np.add.at(J, (j, i), Jv)
    return J


def unpack_natural(words: np.ndarray, lat: Lattice) -> np.ndarray:
    """(R, n) spins +-1 in natural site order from [W][N] words in colour-split order."""
    W = words.shape[0]
    bits = (words[:, None, :] >> np.arange(32, dtype=np.uint32)[None, :, None]) & 1
    s = (1 - 2 * bits.astype(np.int8)).reshape(32 * W, lat.n)
    return s[:, lat.q_of_site]


def test_lattice_dense_couplings_give_the_lattice_energy():
    lat = Lattice.edwards_anderson(2, 4, 3)
    J = dense_couplings(lat)
    s = np.random.default_rng(0).choice([-1.0, 1.0], size=(5, lat.n))
    assert np.allclose(-0.5 * np.einsum("ri,ij,rj->r", s, J, s), lat.energy(s))


def test_multispin_oracle_chain_samples_the_boltzmann_distribution():
    lat = Lattice.edwards_anderson(2, 4, 3)
    betas = 0.2 * 15.0 ** (np.arange(32) / 31)  # beta 0.2 .. 3.0
    ex = oracle.exact(dense_couplings(lat), np.zeros(lat.n), betas)
    st = None
    E, M = [], []
    for t in range(3000):
        st = oracle.ms_run(2, 4, lat.jneg, betas, n_rounds=1, sweeps_per_round=2, seed=6, state=st, round_offset=t)
        assert np.array_equal(lat.energy(unpack_natural(st.words, lat)).astype(np.int64), st.energy)
        s = unpack_natural(st.words, lat)
        E.append(st.energy[st.slot_of_rung].astype(np.float64))
        M.append(np.abs(s.mean(axis=1))[st.slot_of_rung])
    mE, sE = blocked(np.array(E))
    mM, sM = blocked(np.array(M))
    # a cold rung can sit in its ground state for the whole run (blocked error 0); the error of the
    # mean of that many independent samples, from the exact variance, is the floor of the error
    n_kept = len(E) - int(len(E) * 0.1)
    floor = np.sqrt(np.maximum(ex.mean_e2 - ex.mean_e ** 2, 0.0) / n_kept)
    assert np.all(np.abs(mE - ex.mean_e) <= 3.0 * np.maximum(sE, floor) + 1e-9), (mE, ex.mean_e, sE)
    floor_m = np.sqrt(np.maximum(ex.mean_m2 - ex.mean_absm ** 2, 0.0) / n_kept)
    assert np.all(np.abs(mM - ex.mean_absm) <= 3.0 * np.maximum(sM, floor_m) + 1e-9), (mM, ex.mean_absm, sM)
    assert st.best_energy.min() == ex.e_min
