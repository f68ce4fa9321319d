"""Entanglement of the chain's excited eigenstates from the free-fermion solution (TEST INFRASTRUCTURE: checks the
oracle's Majorana-mode restatement against exact diagonalisation, then uses it to size the mid-spectrum problem).

The excited-state configuration (L=32, energy density 0.5, chi_max=512, variance <= 1e-10) asks for an eigenstate
that a bond dimension of 512 represents to a discarded weight of about 1e-11; the last test records how far the
eigenstates near that energy are from it."""
import numpy as np

from oracle import physics as ph


def test_mode_energies_and_schmidt_weights_match_ed():
    h = ph.random_fields(77, 8)
    eps, W = ph.free_fermion_modes(h)
    assert np.allclose(np.sort(eps), 2 * ph.free_fermion_levels(h), atol=1e-12)
    H = ph.ising_hamiltonian_sparse(h).toarray()
    w, v = np.linalg.eigh(H)
    E0 = -eps.sum() / 2
    rng = np.random.default_rng(5)
    for _ in range(6):
        occ = rng.integers(0, 2, 8)
        E = E0 + float(np.dot(eps, occ))
        j = int(np.argmin(np.abs(w - E)))
        assert abs(w[j] - E) < 1e-10
        if min(abs(w[j] - w[jj]) for jj in range(len(w)) if jj != j) < 1e-8:
            continue  # a degenerate level: its eigenvector is not unique
        # sites [0, 4) are the low bits of the basis index (ising_hamiltonian_sparse)
        s = np.linalg.svd(v[:, j].reshape(16, 16), compute_uv=False)
        p_ed = np.sort(s * s)[::-1]
        p_ff = ph.free_fermion_schmidt(eps, W, occ, 4)
        assert np.allclose(p_ed, p_ff[:16], atol=1e-10)


def test_mid_spectrum_eigenstates_at_L32_need_more_than_chi_512():
    """Among eigenstates within 1.0 of the middle of the spectrum (energy density 0.5 +- 0.6 %), none sampled has a
    middle-bond Schmidt spectrum that 512 values hold to a discarded weight of 1e-11."""
    h = ph.random_fields(0, 32)
    eps, W = ph.free_fermion_modes(h)
    E0 = -eps.sum() / 2
    rng = np.random.default_rng(1)
    need = []
    for _ in range(1500):
        occ = rng.integers(0, 2, 32)
        if abs(E0 + float(np.dot(eps, occ))) > 1.0:
            continue
        need.append(ph.bond_dimension_for_weight(ph.free_fermion_schmidt(eps, W, occ, 16), 1e-11))
    assert len(need) > 40
    assert min(need) > 512, min(need)
