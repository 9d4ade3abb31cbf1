"""Statistics of the chain (CPU): on the C1 companion instance (G(20, 0.3), +-1 couplings, with a
+-1 field), the oracle's chain and the reference CPU PT (oracle/ref_pt.py) each reproduce the exact
Boltzmann averages of exact enumeration: per-rung mean energy and |m| within 3 sigma (blocked
standard errors), site magnetisations (marginals) by an aggregate chi-square, and the exact ground
energy."""

from __future__ import annotations

import numpy as np

import oracle
from oracle import ref_pt

from drift_b200.engine import HostProblem
from drift_b200.instances import gnp_pm
from drift_b200.observables import blocked

R = 8
BETAS = 1.0 / (1.0 / 3.0 * 30.0 ** (np.arange(R) / (R - 1)))  # rung 0 coldest: the reference's ladder order


def model():
    return gnp_pm(20, 0.3, 2, field=1)


def check_against_exact(E, absm, spins, ex, z=3.0):
    mE, sE = blocked(E)
    mM, sM = blocked(absm)
    assert np.all(np.abs(mE - ex.mean_e) <= z * sE + 1e-9), (mE, ex.mean_e, sE)
    assert np.all(np.abs(mM - ex.mean_absm) <= z * sM + 1e-9), (mM, ex.mean_absm, sM)
    if spins is not None:
        mS, sS = blocked(spins.astype(np.float64))
        keep = sS > 0
        chi2 = (((mS - ex.site_mag) / np.where(keep, sS, 1.0)) ** 2)[keep].sum()
        dof = keep.sum()
        assert chi2 < dof + 4 * np.sqrt(2 * dof), (chi2, dof)


def test_oracle_chain_matches_exact_enumeration():
    m = model()
    hp = HostProblem.from_model(m)
    prob = oracle.OracleProblem(hp.n, hp.row_ptr, hp.col_idx, hp.weight, hp.h, hp.color_ptr, hp.color_spins)
    ex = oracle.exact(m.J, m.h, BETAS, site_mag=True)
    T = 3000
    E = np.zeros((T, R))
    M = np.zeros((T, R))
    S = np.zeros((T, R, m.n), np.int8)
    st = None
    for t in range(T):
        st = oracle.pt_run(prob, BETAS, n_rounds=1, sweeps_per_round=5, seed=3, state=st, round_offset=t)
        sl = st.slot_of_rung
        E[t] = st.energy[sl]
        S[t] = st.spins[sl]
        M[t] = np.abs(S[t].astype(np.float64).mean(axis=1))
    check_against_exact(E, M, S, ex)
    assert st.best_energy.min() == round(ex.e_min)


def test_reference_cpu_pt_matches_exact_enumeration():
    m = model()
    ex = oracle.exact(m.J, m.h, BETAS, site_mag=True)
    out = ref_pt.parallel_tempering(m, n_replicas=R, T_min=1.0 / 3.0, T_max=10.0, n_rounds=800, sweeps_per_round=5,
                                    seed=4, record=True, record_spins=True)
    check_against_exact(out["rung_energy"], out["rung_absm"], out["rung_spins"], ex)
    assert abs(out["best_E"] - ex.e_min) < 1e-9
