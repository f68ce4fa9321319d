"""H_eff matvec parity: CUDA path (through the C ABI) vs the CPU oracle.

Tolerance: ||y_gpu - y_oracle|| / ||y_oracle|| <= 1e-12 (FP64 path), the parity bound for the
FP64 matvec against the reference's Eigen contraction sequence.
"""
import numpy as np
import pytest
import torch

import dmrg_b200 as hb
import oracle
from oracle import physics as ph
from oracle import ref_numpy as rn

from conftest import relerr

pytestmark = pytest.mark.gpu
TOL = 1e-12


def gpu_matvec(th, W, L, R):
    d = [hb.to_device(a) for a in (th, W, L, R)]
    res = torch.empty_like(d[0])
    hb.matrix_vector_product(res, d[0], th.shape, d[1], W.shape, d[2], L.shape, d[3], R.shape)
    torch.cuda.synchronize()
    return hb.to_host(res, th.shape)


@pytest.mark.parametrize("i", range(10))
def test_matvec_golden(cuda, golden, i):
    g = lambda k: golden[f"mv{i}_{k}"]
    y = gpu_matvec(g("mps"), g("mpo"), g("envL"), g("envR"))
    assert relerr(y, g("res")) < TOL


SMALL = [
    # spin, chiL, chiR, D, complex
    (4, 1, 1, 1, False), (4, 2, 3, 3, False), (4, 7, 5, 3, False), (4, 5, 7, 3, True),
    (2, 13, 11, 3, False), (2, 11, 13, 9, True), (4, 17, 33, 9, False), (4, 33, 17, 3, True),
    (4, 31, 31, 3, False), (4, 64, 64, 9, True), (2, 129, 65, 3, False), (4, 130, 2, 3, True),
]


@pytest.mark.parametrize("S,cL,cR,D,c", SMALL)
def test_matvec_vs_c_oracle(cuda, S, cL, cR, D, c):
    th, W, L, R = ph.heff_inputs(cL, D=D, cplx=c, seed=cL * 131 + cR, chiR=cR, spin=S)
    if D == 1:
        W = np.asfortranarray(np.random.default_rng(5).standard_normal((1, 1, S, S)))
    y = gpu_matvec(th, W, L, R)
    y_ref = oracle.matvec(th, W, L, R)  # branch chosen like the reference (chiL >= chiR -> envL first)
    assert relerr(y, y_ref) < TOL


@pytest.mark.parametrize("chi", [128, 256, 512])
@pytest.mark.parametrize("D", [3, 9])
@pytest.mark.parametrize("c", [False, True])
def test_matvec_large_vs_blas_oracle(cuda, chi, D, c):
    th, W, L, R = ph.heff_inputs(chi, D=D, cplx=c, seed=chi + D)
    y = gpu_matvec(th, W, L, R)
    y_ref = rn.matvec_blas(th, W, L, R)
    assert relerr(y, y_ref) < TOL


def test_matvec_linearity_full_size(cuda):
    """chi=1024 complex: H(a x1 + b x2) == a H x1 + b H x2 (size-independent property)."""
    chi = 1024
    th, W, L, R = ph.heff_inputs(chi, D=3, cplx=True, seed=3)
    op = hb.MatVecMPOS([W], L, R)
    n = op.rows()
    g = torch.Generator(device="cuda").manual_seed(1)
    x1 = torch.randn(n, dtype=torch.complex128, device="cuda", generator=g)
    x2 = torch.randn(n, dtype=torch.complex128, device="cuda", generator=g)
    a, b = 0.3 - 1.1j, 2.0 + 0.25j
    y1, y2, y3 = (torch.empty_like(x1) for _ in range(3))
    op.MultAx(x1, y1)
    op.MultAx(x2, y2)
    op.MultAx(a * x1 + b * x2, y3)
    err = torch.linalg.norm(y3 - (a * y1 + b * y2)) / torch.linalg.norm(y3)
    assert float(err) < 1e-13
    # Hermitian envs and Hermitian MPO slices -> H_eff Hermitian: <x1|H x2> == conj(<x2|H x1>)
    lhs = torch.vdot(x1, y2)
    rhs = torch.vdot(x2, y1).conj()
    assert abs(complex(lhs - rhs)) / abs(complex(lhs)) < 1e-12
    op.close()


def test_operator_multax_forms(cuda):
    th, W, L, R = ph.heff_inputs(24, D=3, cplx=False, seed=9, chiR=20)
    op = hb.MatVecMPOS([W], L, R)
    assert op.rows() == 4 * 24 * 20 and op.shape_mps == (4, 24, 20)
    y_ref = oracle.matvec(th, W, L, R)
    # ARPACK form MultAx(x, y)
    x = hb.to_device(th)
    y = torch.empty_like(x)
    op.MultAx(x, y)
    torch.cuda.synchronize()
    assert relerr(hb.to_host(y, th.shape), y_ref) < TOL
    # PRIMME form: blockSize columns with leading dims > rows
    n = op.rows()
    ld = n + 7
    X = torch.zeros(3 * ld, dtype=torch.float64, device="cuda")
    Y = torch.zeros(3 * ld, dtype=torch.float64, device="cuda")
    cols = [th, 2.0 * th, np.asfortranarray(np.random.default_rng(2).standard_normal(th.shape))]
    for k, c in enumerate(cols):
        X[k * ld:k * ld + n] = hb.to_device(c)
    op.MultAx_block(X, ld, Y, ld, 3)
    torch.cuda.synchronize()
    for k, c in enumerate(cols):
        assert relerr(hb.to_host(Y[k * ld:k * ld + n], th.shape), oracle.matvec(c, W, L, R)) < TOL
    # host-buffer form
    assert relerr(op.MultAx_host(th), y_ref) < TOL
    assert op.num_mv == 5
    op.close()


def test_operator_merges_site_mpos(cuda):
    """Two one-site MPOs are merged like matvec_mpos.cpp:104-119 before the matvec."""
    rng = np.random.default_rng(4)
    WA = oracle.mpo_ising(1.0, 0.7)
    WB = oracle.mpo_ising(1.0, 1.2)
    L = ph.hermitian_env(rng, 9, 3, True)
    R = ph.hermitian_env(rng, 6, 3, True)
    th = np.asfortranarray(rng.standard_normal((4, 9, 6)) + 1j * rng.standard_normal((4, 9, 6)))
    op = hb.MatVecMPOS([WA, WB], L, R, cplx=True)
    y = op.MultAx_host(th)
    y_ref = oracle.matvec(th, oracle.mpo_merge(WA, WB).astype(complex), L, R)
    assert relerr(y, y_ref) < TOL
    op.close()


def test_expval_golden(cuda, golden):
    for i in range(10):
        g = lambda k: golden[f"mv{i}_{k}"]
        d = [hb.to_device(g(k)) for k in ("mps", "mpo", "envL", "envR")]
        e = hb.expectation_value(d[0], g("mps").shape, d[1], g("mpo").shape, d[2], g("envL").shape, d[3], g("envR").shape)
        ref = complex(g("expval")[0])
        scale = np.linalg.norm(g("mps")) * np.linalg.norm(g("res"))
        assert abs(e - ref) <= 1e-13 * scale


def test_matvec_rejects_bad_shapes(cuda):
    th, W, L, R = ph.heff_inputs(6, D=3, cplx=False, seed=1)
    d = [hb.to_device(a) for a in (th, W, L, R)]
    res = torch.empty_like(d[0])
    with pytest.raises(hb.HeffError) as e:
        hb.matrix_vector_product(res, d[0], (4, 6, 7), d[1], W.shape, d[2], L.shape, d[3], R.shape)
    assert e.value.code == 1
    with pytest.raises(hb.HeffError) as e:
        hb.matrix_vector_product(d[0], d[0], th.shape, d[1], W.shape, d[2], L.shape, d[3], R.shape)
    assert e.value.code == 7
    # the device keeps working after rejected calls
    hb.matrix_vector_product(res, d[0], th.shape, d[1], W.shape, d[2], L.shape, d[3], R.shape)
    torch.cuda.synchronize()
    assert relerr(hb.to_host(res, th.shape), oracle.matvec(th, W, L, R)) < TOL


@pytest.mark.parametrize("chiL,chiR,c", [(512, 512, False), (400, 371, True), (1400, 200, False)])
def test_host_buffer_matvec_overlapped_path(cuda, chiL, chiR, c):
    """MultAx with host buffers of >= 8 MB takes the overlapped path (slabbed copies on a copy stream, two compute
    streams).  Its slab GEMMs run every tile whole, while the device-pointer MultAx may split the tiles of a last
    partial wave along K, so the two agree to rounding (1e-14 relative); each path is bit-identical call after call,
    with pageable and pinned buffers."""
    th, W, L, R = ph.heff_inputs(chiL, D=3, cplx=c, seed=chiL + chiR, chiR=chiR)
    assert th.nbytes >= 8 << 20
    op = hb.MatVecMPOS([W], L, R, cplx=c)
    x = hb.to_device(th)
    y = torch.empty_like(x)
    op.MultAx(x, y)
    torch.cuda.synchronize()
    y_dev = y.cpu().numpy()
    y_first = None
    for _ in range(2):
        y_host = op.MultAx_host(th).ravel(order="F")
        if y_first is None:
            y_first = y_host
        assert np.array_equal(y_host, y_first)
        assert relerr(y_host, y_dev) < 1e-14
        op.MultAx(x, y)  # interleaved device-pointer call on the same operator
        torch.cuda.synchronize()
        assert np.array_equal(y.cpu().numpy(), y_dev)
    # pinned buffers through the C ABI
    xp = torch.from_numpy(np.ascontiguousarray(th.ravel(order="F"))).pin_memory()
    yp = torch.empty_like(xp).pin_memory()
    hb.check(hb.lib().heff_op_multax_host(op.handle, hb.ptr(xp), hb.ptr(yp)), "multax_host")
    assert np.array_equal(yp.numpy(), y_first)
    assert relerr(y_dev.reshape(th.shape, order="F"), rn.matvec_blas(th, W, L, R)) < TOL
    op.close()
