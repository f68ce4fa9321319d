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
