"""Jacobi preconditioner: device diagonal of H_eff vs the restatement of get_diagonal_new (matvec_mpos.cpp:300-407)
and the dense H_eff, MultPc (matvec_mpos.cpp:1349-1364), and the preconditioned Davidson vs dense / Krylov solves
and inside the excited-state sweep (H^2, where the reference turns the preconditioner on)."""
import numpy as np
import pytest
import torch

import dmrg_b200 as hb
from oracle import physics as ph
from oracle import ref_numpy as rn

pytestmark = pytest.mark.gpu


def dense(th, W, L, R):
    H = np.einsum("axm,mnst,byn->txysab", L, W, R)
    return H.reshape(th.size, th.size, order="F")


@pytest.mark.parametrize("chi,chiR,D,spin,c", [(5, 4, 3, 4, False), (7, 9, 3, 4, True), (16, 16, 9, 4, False), (33, 17, 9, 4, True),
                                               (12, 12, 3, 2, False), (40, 40, 3, 4, True)])
def test_diagonal_vs_restatement(cuda, chi, chiR, D, spin, c):
    th, W, L, R = ph.heff_inputs(chi, D=D, cplx=c, seed=chi * 7 + D, chiR=chiR, spin=spin)
    op = hb.MatVecMPOS([W], L, R, cplx=c)
    d = op.diagonal().cpu().numpy()
    torch.cuda.synchronize()
    ref = rn.diagonal_einsum(th.shape, W, L, R)
    assert np.linalg.norm(d - ref) <= 1e-13 * np.linalg.norm(ref)
    if th.size <= 600:
        assert np.linalg.norm(d - np.diag(dense(th, W, L, R))) <= 1e-13 * np.linalg.norm(ref)
    op.close()


def test_diagonal_of_merged_two_site_operator(cuda):
    """Two one-site MPOs merged by the operator (matvec_mpos.cpp:104-119): diagonal of the merged H_eff."""
    from oracle import clib

    rng = np.random.default_rng(3)
    WA, WB = clib.mpo_ising(1.0, 0.6), clib.mpo_ising(1.0, 1.4)
    chi = 10
    L, R = ph.hermitian_env(rng, chi, 3, False), ph.hermitian_env(rng, chi, 3, False)
    op = hb.MatVecMPOS([WA, WB], L, R)
    d = op.diagonal().cpu().numpy()
    ref = rn.diagonal_einsum((4, chi, chi), clib.mpo_merge(WA, WB), L, R)
    assert np.linalg.norm(d - ref) <= 1e-13 * np.linalg.norm(ref)
    op.close()


@pytest.mark.parametrize("c", [False, True])
def test_multpc(cuda, c):
    th, W, L, R = ph.heff_inputs(20, D=3, cplx=c, seed=4)
    op = hb.MatVecMPOS([W], L, R, cplx=c)
    x = hb.to_device(th)
    y = torch.empty_like(x)
    shift = -3.25
    op.MultPc(x, y, shift)
    torch.cuda.synchronize()
    ref = rn.multpc(th.ravel(order="F"), rn.diagonal_einsum(th.shape, W, L, R), shift)
    assert np.linalg.norm(y.cpu().numpy() - ref) <= 1e-13 * np.linalg.norm(ref)
    with pytest.raises(hb.HeffError):
        op.MultPc(x, y, float("nan"))
    op.close()


@pytest.mark.parametrize("c", [False, True])
def test_preconditioned_eigs_vs_dense(cuda, c):
    th, W, L, R = ph.heff_inputs(7, D=3, cplx=c, seed=21, chiR=6)
    w = np.linalg.eigvalsh(dense(th, W, L, R))
    op = hb.MatVecMPOS([W], L, R, cplx=c)
    e, res = op.eigs(ritz="SA", tol=1e-12, mixed=False, precond=1)
    assert res["converged"] == 1
    assert abs(e - w[0]) < 1e-10 * max(1.0, abs(w[0]))
    e2, res2 = op.eigs(ritz="LA", tol=1e-12, mixed=False, precond=1)
    assert abs(e2 - w[-1]) < 1e-10 * max(1.0, abs(w[-1]))
    op.close()


# D = 3 only: with random Hermitian environments and the squared MPO (D = 9) the low end of the spectrum is so
# clustered, and the diagonal so flat next to it, that any restarted GD (preconditioned or not) needs thousands of
# matvecs where the Krylov expansion does not; that comparison is not a parity question.
@pytest.mark.parametrize("chi,D,c", [(64, 3, False), (48, 3, True), (128, 3, False)])
def test_preconditioned_eigs_matches_krylov(cuda, chi, D, c):
    th, W, L, R = ph.heff_inputs(chi, D=D, cplx=c, seed=chi + D)
    op = hb.MatVecMPOS([W], L, R, cplx=c)
    x0 = hb.to_device(th)
    e_k, r_k = op.eigs(x0=x0, ritz="SA", tol=1e-12, mixed=False, precond=0)
    e_p, r_p = op.eigs(x0=x0, ritz="SA", tol=1e-12, mixed=False, precond=1)
    assert r_k["converged"] == 1 and r_p["converged"] == 1
    assert abs(e_k - e_p) < 1e-10 * max(1.0, abs(e_k))
    op.close()


def test_xdmrg_with_jacobi_preconditioner(cuda):
    """Folded-spectrum sweep with the preconditioned solver: same eigenstate and variance as the Krylov solver."""
    h = ph.random_fields(4242, 10)
    lev = ph.free_fermion_levels(h)
    et = -lev.sum() + 0.3 * 2 * lev.sum()
    r0 = hb.xdmrg(h, et, chi_max=32, sweeps=12, eig_tol=1e-12, seed=1)
    r1 = hb.xdmrg(h, et, chi_max=32, sweeps=12, eig_tol=1e-12, seed=1, precond=1)
    assert r0["variance"] < 1e-10 and r1["variance"] < 1e-10
    assert abs(r0["energy"] - r1["energy"]) < 1e-9
    print(f"xDMRG matvecs: Krylov {r0['num_mv']}, Jacobi-preconditioned {r1['num_mv']}")


def block_inverse_apply(H, x, bs, shift):
    """Reference for block Jacobi: y_blk = (H[blk, blk] - shift I)^-1 x_blk over consecutive blocks of bs rows
    (CalcPc / MultPc, matvec_mpos.cpp:1087-1240, 1349-1416), by a dense solve per block."""
    n = H.shape[0]
    y = np.zeros_like(x)
    for off in range(0, n, bs):
        e = min(bs, n - off)
        B = H[off:off + e, off:off + e] - shift * np.eye(e)
        y[off:off + e] = np.linalg.solve(B, x[off:off + e])
    return y


@pytest.mark.parametrize("chi,chiR,D,c,bs", [(5, 4, 3, False, 2), (7, 9, 3, True, 7), (9, 8, 9, False, 64), (8, 9, 3, True, 128),
                                             (10, 9, 9, False, 128), (11, 10, 3, False, 200), (9, 10, 9, True, 100)])
def test_block_jacobi_vs_dense_solve(cuda, chi, chiR, D, c, bs):
    """Blocks of every size class: a few rows, a shared-memory block (bs^2 entries within 200 KB) and blocks inverted
    in global memory (real 200, complex 128/100); n = 4 chi chiR is never a multiple of bs, so the last block is short."""
    th, W, L, R = ph.heff_inputs(chi, D=D, cplx=c, seed=chi * 31 + bs, chiR=chiR)
    H = dense(th, W, L, R)  # the matrix MultAx applies: y = H x
    op = hb.MatVecMPOS([W], L, R, cplx=c)
    op.set_jacobi_blocksize(bs)
    x = th.ravel(order="F")
    y = torch.empty(x.size, dtype=torch.complex128 if c else torch.float64, device="cuda")
    shift = -0.75
    op.MultPc(hb.to_device(th), y, shift)
    ref = block_inverse_apply(H, x, bs, shift)
    assert np.linalg.norm(y.cpu().numpy() - ref) <= 1e-11 * np.linalg.norm(ref)
    assert op.jacobi_singular() == 0
    # the blocks are formed at the first shift and reused, like readyCalcPc; a rebind-free second call with another
    # shift gives the same result
    y2 = torch.empty_like(y)
    op.MultPc(hb.to_device(th), y2, 5.0)
    assert torch.equal(y, y2)
    # a new block size takes effect at the next call (formed at that call's shift)
    op.set_jacobi_blocksize(3)
    op.MultPc(hb.to_device(th), y2, 1.5)
    ref3 = block_inverse_apply(H, x, 3, 1.5)
    assert np.linalg.norm(y2.cpu().numpy() - ref3) <= 1e-11 * np.linalg.norm(ref3)
    op.close()


def test_block_jacobi_of_whole_operator_is_the_inverse(cuda):
    """One block covering every row: MultPc is the dense inverse (H - shift)^-1, so A MultPc(x) = x."""
    th, W, L, R = ph.heff_inputs(6, D=3, cplx=False, seed=5, chiR=5)
    n = th.size
    H = dense(th, W, L, R)
    op = hb.MatVecMPOS([W], L, R)
    op.set_jacobi_blocksize(n)
    x = hb.to_device(th)
    y = torch.empty_like(x)
    op.MultPc(x, y, 0.3)
    z = (H - 0.3 * np.eye(n)) @ y.cpu().numpy()
    assert np.linalg.norm(z - th.ravel(order="F")) <= 1e-11 * np.linalg.norm(th)
    with pytest.raises(hb.HeffError):
        op.set_jacobi_blocksize(0)
    op.close()


@pytest.mark.parametrize("c", [False, True])
def test_block_jacobi_eigs_vs_dense(cuda, c):
    """The preconditioned Davidson with block-Jacobi expansion vectors converges to the dense eigenvalues.  The blocks are
    formed at the shift of the first MultPc (readyCalcPc), so the caller sets it the way PRIMME's preconditioner shift
    is set for a smallest-eigenvalue solve: at a lower bound of the spectrum (here w[0] - 1; in the folded spectrum the
    operator is positive semidefinite and the bound is 0), where every block B - shift I is positive definite."""
    th, W, L, R = ph.heff_inputs(8, D=3, cplx=c, seed=22, chiR=7)
    w = np.linalg.eigvalsh(dense(th, W, L, R))
    x = hb.to_device(th)
    y = torch.empty_like(x)
    for bs in (1, 16, 64):
        op = hb.MatVecMPOS([W], L, R, cplx=c)
        op.set_jacobi_blocksize(bs)
        if bs > 1:
            op.MultPc(x, y, float(w[0] - 1.0))  # forms the blocks at the lower bound
        e, res = op.eigs(ritz="SA", tol=1e-12, mixed=False, precond=1)
        assert res["converged"] == 1, (bs, res)
        assert abs(e - w[0]) < 1e-10 * max(1.0, abs(w[0])), bs
        op.close()
