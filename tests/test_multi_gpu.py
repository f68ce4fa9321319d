"""Multi-MPO matvec (site MPOs applied one at a time, contraction_tblis.cpp:307-420) on the device vs the oracle's
literal restatement, and the operator over more than 5 sites (matvec_mpos.cpp:104-123): MultAx, eigensolve,
preconditioner diagonal, and the refusals the reference has too (no get_matrix for unmerged MPOs)."""
import numpy as np
import pytest
import torch

import dmrg_b200 as hb
import oracle
from oracle import clib
from oracle import ref_numpy as rn

pytestmark = pytest.mark.gpu


def chain(nsites, c, seed, ising=False):
    rng = np.random.default_rng(seed)
    g = (lambda *s: rng.standard_normal(s) + 1j * rng.standard_normal(s)) if c else (lambda *s: rng.standard_normal(s))
    if ising:
        mpos = [clib.mpo_ising(1.0, 0.5 + 0.1 * i) for i in range(nsites)]
        mpos = [np.asfortranarray(W.astype(np.complex128) if c else W) for W in mpos]
    else:
        Ds = [int(x) for x in rng.integers(2, 5, nsites + 1)]
        mpos = [np.asfortranarray(g(Ds[i], Ds[i + 1], 2, 2)) for i in range(nsites)]
    return mpos, g


def herm_env(g, chi, D):
    X = g(chi, chi, D)
    return np.asfortranarray(0.5 * (X + np.conj(np.transpose(X, (1, 0, 2)))))


@pytest.mark.parametrize("nsites,chiL,chiR,c", [(1, 9, 7, False), (2, 16, 16, True), (3, 12, 20, False), (6, 8, 8, False), (6, 10, 6, True),
                                                (7, 6, 5, False)])
def test_multi_matvec_vs_literal(cuda, nsites, chiL, chiR, c):
    mpos, g = chain(nsites, c, seed=nsites * 10 + chiL)
    th = np.asfortranarray(g(2 ** nsites, chiL, chiR))
    L = np.asfortranarray(g(chiL, chiL, mpos[0].shape[0]))
    R = np.asfortranarray(g(chiR, chiR, mpos[-1].shape[1]))
    dev = [hb.to_device(W) for W in mpos]
    x = hb.to_device(th)
    y = torch.empty_like(x)
    hb.matrix_vector_product_multi(y, x, th.shape, dev, [W.shape for W in mpos], hb.to_device(L), L.shape, hb.to_device(R), R.shape)
    torch.cuda.synchronize()
    ref = rn.matvec_multi_literal(th, mpos, L, R)
    got = hb.to_host(y, th.shape)
    assert np.linalg.norm(got - ref) <= 1e-12 * np.linalg.norm(ref)


def test_operator_over_six_sites(cuda):
    """Ising chain of 6 sites inside Hermitian environments: MultAx == merged-MPO oracle, the lowest eigenvalue
    from the device solver == dense diagonalisation, diagonal == restatement; get_matrix and mixed refused."""
    mpos, g = chain(6, False, seed=3, ising=True)
    chi = 4
    L, R = herm_env(g, chi, 3), herm_env(g, chi, 3)
    W = mpos[0]
    for Wi in mpos[1:]:
        W = oracle.mpo_merge(W, Wi)
    op = hb.MatVecMPOS(mpos, L, R)
    assert op.rows() == 64 * chi * chi
    th = np.asfortranarray(np.random.default_rng(1).standard_normal((64, chi, chi)))
    x = hb.to_device(th)
    y = torch.empty_like(x)
    op.MultAx(x, y)
    torch.cuda.synchronize()
    ref = rn.matvec_einsum(th, W, L, R)
    assert np.linalg.norm(hb.to_host(y, th.shape) - ref) <= 1e-12 * np.linalg.norm(ref)
    H = np.einsum("axm,mnst,byn->txysab", L, W, R).reshape(th.size, th.size, order="F")
    w = np.linalg.eigvalsh(0.5 * (H + H.T))
    e, res = op.eigs(tol=1e-12, mixed=False)
    assert res["converged"] == 1 and abs(e - w[0]) < 1e-10 * max(1.0, abs(w[0]))
    d = op.diagonal().cpu().numpy()
    dref = rn.diagonal_einsum(th.shape, W, L, R)
    assert np.linalg.norm(d - dref) <= 1e-13 * np.linalg.norm(dref)
    with pytest.raises(hb.HeffError):
        op.get_matrix()
    with pytest.raises(hb.HeffError):
        op.set_precision(hb.PREC_MIXED)
    op.close()
    with pytest.raises(hb.HeffError):
        hb.MatVecMPOS(mpos, L, R, precision=hb.PREC_MIXED)
