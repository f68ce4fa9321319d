"""Device Davidson eigensolver vs dense diagonalisation / ARPACK (scipy eigsh, the reference's Lib::ARPACK family)."""
import numpy as np
import pytest
import scipy.sparse.linalg as sla
import torch

import dmrg_b200 as hb
from oracle import physics as ph
from oracle import ref_numpy as rn

pytestmark = pytest.mark.gpu


def dense(th, W, L, R):
    H = np.einsum("axm,mnst,byn->txysab", L, W, R)
    n = th.size
    return H.reshape(n, n, order="F")


@pytest.mark.parametrize("c", [False, True])
@pytest.mark.parametrize("ritz", ["SA", "LA"])
def test_eigs_small_vs_dense(cuda, c, ritz):
    th, W, L, R = ph.heff_inputs(7, D=3, cplx=c, seed=21, chiR=6)
    H = dense(th, W, L, R)
    assert np.linalg.norm(H - H.conj().T) < 1e-12 * np.linalg.norm(H)
    w = np.linalg.eigvalsh(H)
    op = hb.MatVecMPOS([W], L, R, cplx=c)
    x = torch.empty(op.rows(), dtype=torch.complex128 if c else torch.float64, device="cuda")
    e, res = op.eigs(x_out=x, ritz=ritz, tol=1e-12)
    want = w[0] if ritz == "SA" else w[-1]
    assert res["converged"] == 1
    assert abs(e - want) < 1e-10 * max(1.0, abs(want))
    xv = x.cpu().numpy()
    assert np.linalg.norm(H @ xv - e * xv) < 1e-9 * np.max(np.abs(w))
    op.close()


@pytest.mark.parametrize("chi,chiR,c", [(6, 6, False), (7, 5, True), (16, 16, False), (12, 10, True)])
def test_eigs_target_interior(cuda, chi, chiR, c):
    """Closest-to-target interior eigenpairs: at rows() <= 2048 the dense path (get_matrix + the device dense
    eigensolver), as the reference switches to a dense solver for small problems; eigenvalue and eigenvector."""
    th, W, L, R = ph.heff_inputs(chi, D=3, cplx=c, seed=5 + chi, chiR=chiR)
    H = dense(th, W, L, R)
    w = np.linalg.eigvalsh(H)
    target = 0.5 * (w[0] + w[-1]) + 0.01
    op = hb.MatVecMPOS([W], L, R, cplx=c)
    x = torch.empty(th.size, dtype=torch.complex128 if c else torch.float64, device="cuda")
    e, res = op.eigs(x_out=x, ritz="TARGET", target=target, tol=1e-11, max_basis=64, min_basis=16)
    want = w[np.argmin(np.abs(w - target))]
    assert res["converged"] == 1
    assert abs(e - want) < 1e-9 * np.max(np.abs(w))
    xv = x.cpu().numpy()
    assert abs(np.linalg.norm(xv) - 1) < 1e-12
    assert np.linalg.norm(H @ xv - e * xv) < 1e-9 * np.max(np.abs(w))
    op.close()


@pytest.mark.parametrize("chi,c", [(32, False), (48, True), (96, False)])
def test_eigs_vs_arpack(cuda, chi, c):
    th, W, L, R = ph.heff_inputs(chi, D=3, cplx=c, seed=chi)
    n = th.size
    shape = th.shape

    def mv(v):
        return rn.matvec_blas(np.asfortranarray(v.reshape(shape, order="F")), W, L, R).ravel(order="F")

    A = sla.LinearOperator((n, n), matvec=mv, dtype=np.complex128 if c else np.float64)
    w_ref = sla.eigsh(A, k=1, which="SA", tol=1e-13, ncv=40)[0][0]
    op = hb.MatVecMPOS([W], L, R, cplx=c)
    e, res = op.eigs(ritz="SA", tol=1e-12, mixed=False)
    assert res["converged"] == 1
    assert abs(e - w_ref) < 1e-10 * max(1.0, abs(w_ref))
    assert res["num_mv"] == res["num_mv_fp64"]
    op.close()


def test_eigs_start_vector_and_nan_input(cuda):
    th, W, L, R = ph.heff_inputs(8, D=3, cplx=False, seed=2)
    op = hb.MatVecMPOS([W], L, R)
    x0 = hb.to_device(th)
    e1, r1 = op.eigs(x0=x0, tol=1e-12)
    e2, r2 = op.eigs(tol=1e-12)
    assert abs(e1 - e2) < 1e-10
    bad = x0.clone()
    bad[3] = float("nan")
    with pytest.raises(hb.HeffError) as err:
        op.eigs(x0=bad, tol=1e-12)
    assert err.value.code == 2  # HEFF_NAN_INPUT
    # the device still works after the rejected solve
    e3, _ = op.eigs(x0=x0, tol=1e-12)
    assert abs(e3 - e1) < 1e-10
    op.close()


def test_eigs_not_converged_status(cuda):
    th, W, L, R = ph.heff_inputs(16, D=3, cplx=False, seed=4)
    op = hb.MatVecMPOS([W], L, R)
    e, res = op.eigs(tol=1e-14, max_matvecs=3, mixed=False)
    assert res["converged"] == 0 and res["num_mv"] <= 4
    op.close()
