"""Whole two-site DMRG ground-state runs on the device hot path vs exact answers.

Workload of the plain fDMRG configuration: random-field Ising chain, open, J=1, h_i ~ U[0.5, 1.5]
(splitmix64 fields), MPO D=3, real FP64, random product-state start, two-site sweeps x10,
chi_max=64, SVD truncation limit 1e-12, eigensolver tolerance 1e-12.  Energies must agree with exact
diagonalisation / free fermions to 1e-10; the half-chain entanglement entropy with ED to 1e-8.
"""
import numpy as np
import pytest

import dmrg_b200 as hb
from oracle import physics as ph

pytestmark = pytest.mark.gpu


def test_fdmrg_L8_exact(cuda, physics):
    case = physics["ed"][0]  # L=8, ED energy and entropy
    r = hb.fdmrg(case["h"], chi_max=16, sweeps=4)
    assert abs(r["energy"] - case["E0"]) < 1e-10
    assert abs(r["entropy_mid"] - case["S_half"]) < 1e-8
    assert r["unconverged_solves"] == 0


def test_fdmrg_L12_vs_ed(cuda, physics):
    case = physics["ed"][2]
    r = hb.fdmrg(case["h"], chi_max=64, sweeps=6)
    assert abs(r["energy"] - case["E0"]) < 1e-10
    assert abs(r["entropy_mid"] - case["S_half"]) < 1e-8


def test_fdmrg_L16_chi64_ten_sweeps(cuda, physics):
    """The plain fDMRG configuration: L=16, chi_max=64, 10 sweeps; vs free fermions and ED."""
    case = physics["free_fermion"][0]  # L=16
    hs = np.array(case["h"])
    r = hb.fdmrg(hs, chi_max=64, sweeps=10, trunc_lim=1e-12, eig_tol=1e-12, seed=3)
    assert abs(r["energy"] - case["E0"]) < 1e-10
    e_ed, s_ed = ph.ed_ground(hs)
    assert abs(r["energy"] - e_ed) < 1e-10
    assert abs(r["entropy_mid"] - s_ed) < 1e-8
    # energies converge monotonically (variational) over the sweeps
    es = r["energy_per_sweep"]
    assert all(es[i + 1] <= es[i] + 1e-12 for i in range(len(es) - 1))
