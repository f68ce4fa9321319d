"""Mixed-precision path: the tcgen05 BF16 GEMM, the split-BF16 matvec, and mixed eigensolves with FP64 refinement.

Tolerances: the BF16 GEMM (exact bf16 inputs, FP32 accumulation) matches an FP64 product of the same
bf16 values to 1e-5 relative; the split-BF16 matvec (two-part splits, three products) matches the
FP64 oracle to 1e-4 relative; eigenvalues from mixed solves with FP64 refinement match the FP64 solve to
1e-10 (the north-star bar |dE| <= 1e-10).
"""
import ctypes

import pytest
import torch

import dmrg_b200 as hb
from oracle import physics as ph
from oracle import ref_numpy as rn

from conftest import relerr

pytestmark = pytest.mark.gpu


# (1536, 4096, 2048): 192 tiles on 148 SMs -> one whole wave and 44 tiles split in K (several units per CTA, both
# TMEM accumulators, the ordered reduction of partial tiles); (1100, 3000, 4000): split tiles with ragged M, N, K edges
@pytest.mark.parametrize("M,N,K", [(128, 256, 64), (128, 256, 512), (200, 300, 136), (1000, 700, 1024), (64, 40, 8), (1536, 4096, 2048),
                                   (1100, 3000, 4000)])
def test_bf16_gemm_vs_fp64(cuda, M, N, K):
    g = torch.Generator(device="cuda").manual_seed(M + N + K)
    A = torch.randn(M, K, device="cuda", generator=g).to(torch.bfloat16).contiguous()
    B = torch.randn(N, K, device="cuda", generator=g).to(torch.bfloat16).contiguous()
    C = torch.full((N, M), float("nan"), device="cuda", dtype=torch.float32)  # column-major M x N == row-major N x M
    rc = hb.lib().heff_gemm_bf16_f32(hb.ptr(A), hb.ptr(B), hb.ptr(C), M, N, K, ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == 0, hb.lib().heff_last_error()
    ref = (A.double() @ B.double().T).T  # N x M
    err = torch.linalg.norm(C.double() - ref) / torch.linalg.norm(ref)
    assert float(err) < 1e-5


def mixed_matvec(th, W, L, R, cplx):
    op = hb.MatVecMPOS([W], L, R, cplx=cplx, precision=hb.PREC_MIXED)
    y = op.MultAx_host(th)
    code = ctypes.c_int(-1)
    assert hb.lib().heff_op_device_error(op.handle, ctypes.byref(code)) == 0
    assert code.value == 0
    op.close()
    return y


@pytest.mark.parametrize("S,cL,cR,D,c", [(4, 64, 64, 3, False), (4, 64, 64, 3, True), (4, 37, 53, 9, False), (2, 100, 77, 9, True),
                                         (4, 5, 3, 3, True), (4, 256, 256, 3, False), (4, 300, 200, 9, True)])
def test_mixed_matvec_vs_oracle(cuda, S, cL, cR, D, c):
    th, W, L, R = ph.heff_inputs(cL, D=D, cplx=c, seed=cL + cR, chiR=cR, spin=S)
    y = mixed_matvec(th, W, L, R, c)
    y_ref = rn.matvec_blas(th, W, L, R)
    e = relerr(y, y_ref)
    assert e < 1e-4, e
    assert e > 1e-12  # it really is the reduced-precision path


def test_mixed_matvec_full_size_linearity(cuda):
    chi = 1024
    th, W, L, R = ph.heff_inputs(chi, D=3, cplx=True, seed=3)
    op64 = hb.MatVecMPOS([W], L, R)
    opm = hb.MatVecMPOS([W], L, R, precision=hb.PREC_MIXED)
    x = hb.to_device(th)
    y64, ym = torch.empty_like(x), torch.empty_like(x)
    op64.MultAx(x, y64)
    opm.MultAx(x, ym)
    err = float(torch.linalg.norm(ym - y64) / torch.linalg.norm(y64))
    assert err < 1e-4
    op64.close()
    opm.close()


@pytest.mark.parametrize("chi,c", [(24, False), (40, True), (64, False)])
def test_mixed_eigensolve_refined_to_fp64(cuda, chi, c):
    th, W, L, R = ph.heff_inputs(chi, D=3, cplx=c, seed=chi + 1)
    op = hb.MatVecMPOS([W], L, R, cplx=c)
    e64, r64 = op.eigs(tol=1e-12, mixed=False)
    opm = hb.MatVecMPOS([W], L, R, cplx=c, precision=hb.PREC_MIXED)
    em, rm = opm.eigs(tol=1e-12, mixed=True)
    assert rm["converged"] == 1 and r64["converged"] == 1
    assert abs(em - e64) < 1e-10 * max(1.0, abs(e64))
    assert rm["num_mv_mixed"] > 0
    assert rm["num_mv_fp64"] < r64["num_mv_fp64"]
    op.close()
    opm.close()
