"""FP64-accurate GEMM on the INT8 tensor cores (heff_gemm_i8_emu): digit planes, exact INT32 level sums, FP64
recombination.

Tolerances (normwise relative error against the FP64 product of the same inputs): 7 slices carry 48 bits
relative to each row's power-of-two scale, which for Gaussian data (row max ~4x the rms, scale up to 2x the
max) gives ~1e-14; the bar is 5e-13, well inside the 1e-12 matvec parity bar.  8 slices: 1e-15 (the FP64
reference's own rounding is of the same order).  4 slices (27 bits) must be visibly worse: above 1e-10.
"""
import ctypes

import numpy as np
import pytest
import torch

import dmrg_b200 as hb

pytestmark = pytest.mark.gpu

F64, C128 = 0, 1


def emu(A, B, ns=0):
    M, K = A.shape
    N = B.shape[0]
    cplx = A.is_complex()
    C = torch.full((N, M), float("nan"), device="cuda", dtype=A.dtype)  # column-major M x N == row-major N x M
    rc = hb.lib().heff_gemm_i8_emu(C128 if cplx else F64, hb.ptr(A), hb.ptr(B), hb.ptr(C), M, N, K, ns,
                                   ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    return rc, C.T


def rel(C, ref):
    return float(torch.linalg.norm(C - ref) / torch.linalg.norm(ref))


def rnd(shape, g, cplx):
    if cplx:
        return torch.complex(torch.randn(*shape, device="cuda", dtype=torch.float64, generator=g),
                             torch.randn(*shape, device="cuda", dtype=torch.float64, generator=g)).contiguous()
    return torch.randn(*shape, device="cuda", dtype=torch.float64, generator=g).contiguous()


# (128,256,128): one tile; (200,300,136) ragged M, N, K; (64,40,8): K below one k-block; (1536,4096,2048): 192 tiles on
# 148 SMs (several tiles per CTA, both TMEM buffers, 7 levels each); (1100,3000,4000): ragged edges, long K
@pytest.mark.parametrize("M,N,K", [(128, 256, 128), (200, 300, 136), (64, 40, 8), (1000, 700, 1024), (1536, 4096, 2048), (1100, 3000, 4000)])
@pytest.mark.parametrize("cplx", [False, True])
@pytest.mark.parametrize("bn", [0, 1, 128, 192, 256])
def test_i8_emu_gemm_vs_fp64(cuda, M, N, K, cplx, bn):
    g = torch.Generator(device="cuda").manual_seed(M * 7 + N * 3 + K + cplx)
    A, B = rnd((M, K), g, cplx), rnd((N, K), g, cplx)
    prev = hb.lib().heff_i8_set_tile_width(bn)
    try:
        rc, C = emu(A, B)
    finally:
        hb.lib().heff_i8_set_tile_width(prev)
    assert rc == 0, hb.lib().heff_last_error()
    ref = A @ B.T
    e = rel(C, ref)
    assert e < 5e-13, e


@pytest.mark.parametrize("ns,lo,hi", [(8, 0.0, 2e-15), (4, 1e-10, 1e-6)])
def test_i8_emu_slice_count(cuda, ns, lo, hi):
    g = torch.Generator(device="cuda").manual_seed(ns)
    A, B = rnd((300, 512), g, True), rnd((260, 512), g, True)
    rc, C = emu(A, B, ns)
    assert rc == 0, hb.lib().heff_last_error()
    e = rel(C, A @ B.T)
    assert lo <= e < hi, e


def test_i8_emu_row_scales(cuda):
    """Rows spread over 2^-300 .. 2^300 keep their own relative accuracy (one power-of-two scale per row)."""
    g = torch.Generator(device="cuda").manual_seed(5)
    M, N, K = 256, 512, 384
    A, B = rnd((M, K), g, False), rnd((N, K), g, False)
    ea = torch.randint(-300, 300, (M, 1), device="cuda", generator=g).double()
    eb = torch.randint(-300, 300, (N, 1), device="cuda", generator=g).double()
    A, B = (A * torch.exp2(ea)).contiguous(), (B * torch.exp2(eb)).contiguous()
    rc, C = emu(A, B)
    assert rc == 0, hb.lib().heff_last_error()
    ref = A @ B.T
    scale = torch.exp2(ea) * torch.exp2(eb).T  # the natural size of each entry
    e = float(((C - ref) / scale).abs().max() / ((ref / scale).abs().max()))
    assert e < 1e-13, e


def test_i8_emu_zero_rows_and_exact_integers(cuda):
    """Zero rows give exact zeros; small-integer operands are reproduced exactly (every digit product is exact)."""
    g = torch.Generator(device="cuda").manual_seed(9)
    A = torch.randint(-50, 50, (200, 100), device="cuda", generator=g).double()
    B = torch.randint(-50, 50, (150, 100), device="cuda", generator=g).double()
    A[17] = 0.0
    B[3] = 0.0
    rc, C = emu(A.contiguous(), B.contiguous())
    assert rc == 0, hb.lib().heff_last_error()
    assert torch.equal(C, A @ B.T)
    assert bool((C[17] == 0).all()) and bool((C[:, 3] == 0).all())


@pytest.mark.parametrize("cplx", [False, True])
def test_i8_emu_tile_widths_bitwise_equal(cuda, cplx):
    """128-wide tiles (level sum in TMEM) and 192/256-wide tiles (level sum in C) do the same FP64 operations."""
    g = torch.Generator(device="cuda").manual_seed(21)
    A, B = rnd((700, 520), g, cplx), rnd((900, 520), g, cplx)
    outs = []
    prev = hb.lib().heff_i8_set_tile_width(0)
    try:
        for bn in (128, 192, 256, 1):
            hb.lib().heff_i8_set_tile_width(bn)
            n0 = hb.lib().heff_i8_tuned_shapes()
            rc, C = emu(A, B)
            assert rc == 0, hb.lib().heff_last_error()
            if bn == 1:  # the autotuner timed this shape (its three trial runs rewrote C with identical bytes)
                assert hb.lib().heff_i8_tuned_shapes() >= n0
            outs.append(C.clone())
    finally:
        hb.lib().heff_i8_set_tile_width(prev)
    assert all(torch.equal(outs[0], o) for o in outs[1:])
    assert rel(outs[0], A @ B.T) < 5e-13


def test_i8_emu_rejects_nonfinite(cuda):
    A = torch.randn(64, 32, device="cuda", dtype=torch.float64)
    B = torch.randn(48, 32, device="cuda", dtype=torch.float64)
    A[5, 7] = float("nan")
    rc, C = emu(A, B)
    assert rc == 2  # HEFF_NAN_INPUT
    assert bool(torch.isnan(C).all())  # no finite garbage: the product is NaN, as an FP64 product would be
    A[5, 7] = float("inf")
    rc, C = emu(A, B)
    assert rc == 2 and bool(torch.isnan(C).all())
    A[5, 7] = 1.0
    rc, C = emu(A, B)  # a clean call after the bad ones
    assert rc == 0 and rel(C, A @ B.T) < 5e-13


def test_i8_emu_rejects_long_k(cuda):
    A = torch.zeros(16, 80000, device="cuda", dtype=torch.float64)
    rc, _ = emu(A, A)
    assert rc == 1  # HEFF_BAD_SHAPE: the INT32 level sums could overflow


# ---- the INT8 engine inside the H_eff matvec and the eigensolver ----
from oracle import physics as ph  # noqa: E402
from oracle import ref_numpy as rn  # noqa: E402

from conftest import relerr  # noqa: E402


@pytest.mark.parametrize("S,cL,cR,D,c", [(4, 64, 64, 3, False), (4, 64, 64, 3, True), (4, 37, 53, 9, False), (2, 100, 77, 9, True),
                                         (4, 5, 3, 3, True), (4, 256, 256, 3, False), (4, 300, 200, 9, True)])
def test_int8_engine_matvec_vs_oracle(cuda, S, cL, cR, D, c):
    """FP64-accurate matvec on the INT8 engine meets the FP64 parity bar (1e-12 relative) against the oracle."""
    th, W, L, R = ph.heff_inputs(cL, D=D, cplx=c, seed=cL + cR, chiR=cR, spin=S)
    op = hb.MatVecMPOS([W], L, R, cplx=c)
    op.set_fp64_engine(hb.FP64_INT8)
    y = op.MultAx_host(th)
    code = ctypes.c_int(-1)
    assert hb.lib().heff_op_device_error(op.handle, ctypes.byref(code)) == 0 and code.value == 0
    op.close()
    e = relerr(y, rn.matvec_blas(th, W, L, R))
    assert e < 1e-12, e


def test_int8_engine_matches_dmma_at_chi1024(cuda):
    """Full-size complex matvec: the two engines agree to the FP64 bar (size-independent check, no oracle)."""
    th, W, L, R = ph.heff_inputs(1024, D=3, cplx=True, seed=3)
    op = hb.MatVecMPOS([W], L, R)
    x = hb.to_device(th)
    y64, y8, y8b = torch.empty_like(x), torch.empty_like(x), torch.empty_like(x)
    op.MultAx(x, y64)
    op.set_fp64_engine(hb.FP64_INT8)
    op.MultAx(x, y8)
    op.MultAx(x, y8b)
    op.close()
    assert torch.equal(y8, y8b)  # deterministic
    assert float(torch.linalg.norm(y8 - y64) / torch.linalg.norm(y64)) < 1e-12


@pytest.mark.parametrize("chi,c", [(48, False), (40, True)])
def test_int8_engine_eigensolve(cuda, chi, c):
    """Plain FP64 and mixed eigensolves with the INT8 engine reach the DMMA solve's eigenvalue to 1e-10."""
    th, W, L, R = ph.heff_inputs(chi, D=3, cplx=c, seed=chi + 1)
    op = hb.MatVecMPOS([W], L, R, cplx=c)
    e64, r64 = op.eigs(tol=1e-12, mixed=False)
    op8 = hb.MatVecMPOS([W], L, R, cplx=c)
    op8.set_fp64_engine(hb.FP64_INT8)
    e8, r8 = op8.eigs(tol=1e-12, mixed=False)
    opm = hb.MatVecMPOS([W], L, R, cplx=c, precision=hb.PREC_MIXED)
    opm.set_fp64_engine(hb.FP64_INT8)
    em, rm = opm.eigs(tol=1e-12, mixed=True)
    assert r64["converged"] == 1 and r8["converged"] == 1 and rm["converged"] == 1
    assert abs(e8 - e64) < 1e-10 * max(1.0, abs(e64))
    assert abs(em - e64) < 1e-10 * max(1.0, abs(e64))
    for o in (op, op8, opm):
        o.close()


def test_int8_engine_slices_and_invalid_args(cuda):
    th, W, L, R = ph.heff_inputs(64, D=3, cplx=False, seed=2)
    op = hb.MatVecMPOS([W], L, R)
    ref = rn.matvec_blas(th, W, L, R)
    errs = {}
    for ns in (4, 7, 8):
        op.set_fp64_engine(hb.FP64_INT8, ns)
        errs[ns] = relerr(op.MultAx_host(th), ref)
    assert errs[8] < errs[7] < 1e-12 < errs[4]
    assert hb.lib().heff_op_set_fp64_engine(op.handle, 2, 0) == 7  # HEFF_BAD_ARG
    assert hb.lib().heff_op_set_fp64_engine(op.handle, 1, 9) == 7
    op.close()


@pytest.mark.parametrize("c", [False, True])
def test_int8_engine_nonfinite_input_gives_nan(cuda, c):
    """A NaN in theta makes the INT8-engine matvec NaN (like the DMMA path) instead of a finite wrong answer; the next
    clean matvec is correct again, and the operator's device status records the event (5)."""
    th, W, L, R = ph.heff_inputs(40, D=3, cplx=c, seed=8)
    op = hb.MatVecMPOS([W], L, R, cplx=c)
    op.set_fp64_engine(hb.FP64_INT8)
    bad = th.copy()
    bad[1, 3, 5] = np.nan
    y = op.MultAx_host(bad)
    assert np.isnan(y).any()
    y2 = op.MultAx_host(th)
    assert relerr(y2, rn.matvec_blas(th, W, L, R)) < 1e-12
    code = ctypes.c_int(-1)
    assert hb.lib().heff_op_device_error(op.handle, ctypes.byref(code)) == 0 and code.value == 5
    op.close()
