"""Excited-state DMRG (folded spectrum, MPO squared with energy shift) on the device hot path.

The mid-spectrum configuration targets energy density 0.5 of the spectral width; its FP64 variance must reach
1e-10, the converged energy must be an exact eigenvalue (ED), and a run with mixed-precision matvecs
(split-BF16 + FP64 refinement) must give the same energy and variance as the all-FP64 run.
"""
import numpy as np
import pytest

import dmrg_b200 as hb
from oracle import physics as ph

pytestmark = pytest.mark.gpu


def spectrum(h):
    H = ph.ising_hamiltonian_sparse(h).toarray()
    return np.linalg.eigvalsh(H)


# The chain's spectrum is symmetric (E <-> -E), so energy density 0.5 falls exactly between the pairs +-E_k, whose
# folded eigenvalues (E_k - E_t)^2 coincide; a variance minimiser then has no unique answer.  As the reference moves
# its target off the symmetric point (energy_spectrum_shift, settings.h:427), the target is offset by 0.01, a
# fraction of the level spacing at L=10.
OFFSET = 0.01


@pytest.mark.parametrize("density", [0.5, 0.3])
def test_xdmrg_finds_eigenstate_near_target(cuda, density):
    h = ph.random_fields(4242, 10)
    lev = ph.free_fermion_levels(h)
    emin, emax = -lev.sum(), lev.sum()
    et = emin + density * (emax - emin) + OFFSET
    r = hb.xdmrg(h, et, chi_max=32, sweeps=12, eig_tol=1e-12, seed=1)
    w = spectrum(h)
    assert r["variance"] < 1e-10, r
    assert np.min(np.abs(w - r["energy"])) < 1e-9
    # a state near the target (among the 8 eigenvalues closest to it)
    assert np.sum(np.abs(w - et) < abs(r["energy"] - et) - 1e-12) < 8


def test_xdmrg_mixed_matches_fp64(cuda):
    h = ph.random_fields(4242, 10)
    lev = ph.free_fermion_levels(h)
    et = -lev.sum() + 0.3 * 2 * lev.sum() + OFFSET  # energy density 0.3 of the spectral width
    r64 = hb.xdmrg(h, et, chi_max=32, sweeps=12, eig_tol=1e-12, seed=1)
    rmx = hb.xdmrg(h, et, chi_max=32, sweeps=12, eig_tol=1e-12, seed=1, precision=hb.PREC_MIXED)
    assert r64["variance"] < 1e-10 and rmx["variance"] < 1e-10
    assert abs(r64["energy"] - rmx["energy"]) < 1e-9
    assert rmx["num_mv_mixed"] > 0
    # the converged energy is an eigenvalue of H: E0 + 2 * (sum of a subset of Lambda_k)
    w = spectrum(h)
    assert np.min(np.abs(w - r64["energy"])) < 1e-9


def test_xdmrg_block_jacobi_mid_spectrum_L12(cuda):
    """Energy density 0.5 (+ the offset) at L=12 with chi_max=64 (exact at the middle bond), the local solves
    preconditioned with 128-row Jacobi blocks (the reference's eigs_jcb_min_blocksize) and up to 60000 matvecs: the
    variance falls below 1e-10 at an exact eigenvalue."""
    h = ph.random_fields(4242, 12)
    lev = ph.free_fermion_levels(h)
    et = 0.0 + 1e-3  # energy density 0.5: E_min + 0.5 (E_max - E_min) = 0 for the symmetric spectrum
    r = hb.xdmrg(h, et, chi_max=64, sweeps=7, eig_tol=1e-12, seed=1, jcb_blocksize=128, eig_max_matvecs=60000)
    assert r["variance"] < 1e-10, r
    e = np.array([0.0])
    for x in lev:
        e = np.concatenate([e, e + 2 * x])
    w = -lev.sum() + e
    assert np.min(np.abs(w - r["energy"])) < 1e-9
    # mixed precision: split-BF16 products while the folded eigenvalue is resolvable, FP64 once it sits within the
    # BF16 operator's error of zero; the same eigenstate as the FP64 run
    rm = hb.xdmrg(h, et, chi_max=64, sweeps=7, eig_tol=1e-12, seed=1, jcb_blocksize=128, eig_max_matvecs=60000, precision=hb.PREC_MIXED)
    assert rm["variance"] < 1e-10, rm
    assert abs(rm["energy"] - r["energy"]) < 1e-9
    assert rm["num_mv_mixed"] > 0

