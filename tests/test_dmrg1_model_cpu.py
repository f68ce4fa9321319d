"""Host model of the one-site DMRG sweep with forward subspace expansion (oracle.ref_numpy.dmrg1_expansion_model, the
device driver's index maps): from a random product state the expansion alone grows the bonds, and the sweep reaches
the exact ground energy (free fermions) of the random-field Ising chain; with a vanishing mixing factor it cannot
leave the product state."""

from oracle import physics as ph
from oracle import ref_numpy as rn


def test_one_site_expansion_model_reaches_the_ground_state():
    h = ph.random_fields(3, 8)
    E, chis = rn.dmrg1_expansion_model(ph.ising_mpos(h), chi_max=16, sweeps=6)
    assert abs(E[-1] - ph.free_fermion_ground(h)) < 1e-10
    assert max(chis) == 16


def test_one_site_model_without_expansion_stays_a_product_state():
    h = ph.random_fields(3, 8)
    E, chis = rn.dmrg1_expansion_model(ph.ising_mpos(h), chi_max=16, sweeps=4, alpha0=1e-300)
    assert max(chis) == 1
    assert E[-1] > ph.free_fermion_ground(h) + 1e-3
