"""Dense small-problem path: get_matrix (matvec_mpo.cpp:313-332) vs the oracle's literal restatement, and the
device Hermitian eigendecomposition vs LAPACK (numpy eigh, the ?syevr/?heevd family the reference calls)."""
import numpy as np
import pytest
import torch

import dmrg_b200 as hb
import oracle
from oracle import physics as ph

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("chi,chiR,D,spin,c", [(4, 3, 3, 4, False), (5, 6, 3, 4, True), (6, 6, 9, 4, False), (8, 5, 3, 2, True)])
def test_get_matrix_vs_oracle(cuda, chi, chiR, D, spin, c):
    th, W, L, R = ph.heff_inputs(chi, D=D, cplx=c, seed=chi * 31 + D, chiR=chiR, spin=spin)
    op = hb.MatVecMPOS([W], L, R, cplx=c)
    n = op.rows()
    M = hb.to_host(op.get_matrix(), (n, n))
    ref = oracle.get_matrix(th.shape, W, L, R)
    assert np.linalg.norm(M - ref) <= 1e-13 * np.linalg.norm(ref)
    # consistent with the operator: M^T x = MultAx(x)
    x = hb.to_device(th)
    y = torch.empty_like(x)
    op.MultAx(x, y)
    torch.cuda.synchronize()
    assert np.linalg.norm(M.T @ th.ravel(order="F") - y.cpu().numpy()) <= 1e-12 * np.linalg.norm(y.cpu().numpy())
    op.close()


@pytest.mark.parametrize("n,c", [(1, False), (7, False), (64, True), (200, False), (513, True)])
def test_dense_eig_random_hermitian(cuda, n, c):
    rng = np.random.default_rng(n)
    X = rng.standard_normal((n, n)) + (1j * rng.standard_normal((n, n)) if c else 0)
    A = np.asfortranarray(0.5 * (X + X.conj().T))
    ev, V = hb.dense_eig(hb.to_device(A), n)
    torch.cuda.synchronize()
    ev = ev.cpu().numpy()
    V = hb.to_host(V, (n, n))
    ref = np.linalg.eigvalsh(A)
    nrm = np.max(np.abs(ref))
    assert np.all(np.diff(ev) >= -1e-12 * nrm)
    assert np.max(np.abs(ev - ref)) <= 1e-12 * nrm * max(1.0, np.sqrt(n) / 4)
    assert np.linalg.norm(V.conj().T @ V - np.eye(n)) <= 1e-13 * n
    assert np.linalg.norm(A @ V - V * ev) <= 1e-12 * nrm * n


def test_dense_eig_degenerate_and_indefinite(cuda):
    """Repeated eigenvalues of both signs (a shifted SVD would mix +-lambda without the positive shift)."""
    rng = np.random.default_rng(9)
    Q, _ = np.linalg.qr(rng.standard_normal((40, 40)))
    lam = np.array([-3.0] * 5 + [3.0] * 5 + list(np.linspace(-2, 2, 30)))
    A = np.asfortranarray((Q * lam) @ Q.T)
    ev, V = hb.dense_eig(hb.to_device(A), 40)
    ev = ev.cpu().numpy()
    V = hb.to_host(V, (40, 40))
    assert np.max(np.abs(ev - np.sort(lam))) < 1e-13 * 3 * 40
    assert np.linalg.norm(A @ V - V * ev) < 1e-12 * 3 * 40


@pytest.mark.parametrize("c", [False, True])
def test_dense_path_ground_state_matches_davidson(cuda, c):
    """Dense path on a small H_eff (problem size 4*12*12 = 576 <= eig_max_size): the lowest eigenvalue of
    get_matrix equals the iterative solver's."""
    th, W, L, R = ph.heff_inputs(12, D=3, cplx=c, seed=77)
    op = hb.MatVecMPOS([W], L, R, cplx=c)
    n = op.rows()
    ev, V = hb.dense_eig(op.get_matrix(), n)
    e_it, res = op.eigs(tol=1e-12, mixed=False)
    assert abs(ev[0].item() - e_it) < 1e-10 * max(1.0, abs(e_it))
    op.close()
