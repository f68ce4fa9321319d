"""Host model of the block-Jacobi inversion kernel (oracle.ref_numpy.gauss_jordan_inverse, the kernel's step order):
the inverse of Hermitian, indefinite and pivot-needing blocks, real and complex, and the floored-pivot count of a
singular block."""
import numpy as np
import pytest

from oracle import ref_numpy as rn


@pytest.mark.parametrize("cplx", [False, True])
@pytest.mark.parametrize("bs", [1, 2, 7, 64])
def test_gauss_jordan_inverse_of_hermitian_blocks(cplx, bs):
    rng = np.random.default_rng(bs + 10 * cplx)
    X = rng.standard_normal((bs, bs)) + (1j * rng.standard_normal((bs, bs)) if cplx else 0)
    H = X + X.conj().T  # indefinite: needs pivoting
    inv, floored = rn.gauss_jordan_inverse(H)
    assert floored == 0
    assert np.linalg.norm(inv @ H - np.eye(bs)) < 1e-10 * max(1.0, np.linalg.cond(H) * 1e-4)


def test_zero_leading_entry_needs_a_row_interchange():
    A = np.array([[0.0, 2.0, 1.0], [3.0, 0.0, 1.0], [1.0, 1.0, 0.0]])
    inv, floored = rn.gauss_jordan_inverse(A)
    assert floored == 0
    assert np.allclose(inv, np.linalg.inv(A), atol=1e-14)


def test_singular_block_floors_its_pivot():
    A = np.array([[1.0, 2.0], [2.0, 4.0]])
    inv, floored = rn.gauss_jordan_inverse(A)
    assert floored == 1
    assert np.all(np.isfinite(inv))
