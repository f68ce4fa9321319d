"""Parity at the precision-microbenchmark grid: the standalone two-site H_eff matvec at
chi in {1024, 2048} x D in {3, 9} x {real, complex}, FP64 on the DMMA engine and on the
INT8 engine, against the BLAS restatement of the reference's contraction sequence
(contraction_tblis.cpp:277-290); the environment update at chi=1024, D in {3, 9}
(EnvBase.cpp:109-112, 146-149) against its BLAS restatement.

These are the shapes bench.py measures, so the benchmarked kernels are the ones pinned here.
Tolerance: ||y_gpu - y_oracle|| / ||y_oracle|| <= 1e-12 (the FP64 matvec bar).
"""
import gc

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


@pytest.mark.parametrize("chi", [1024, 2048])
@pytest.mark.parametrize("D", [3, 9])
@pytest.mark.parametrize("c", [False, True])
def test_matvec_grid_vs_blas_oracle(cuda, chi, D, c):
    th, W, L, R = ph.heff_inputs(chi, D=D, cplx=c, seed=10 * chi + D + (1 if c else 0))
    y_ref = rn.matvec_blas(th, W, L, R)
    op = hb.MatVecMPOS([W], L, R, cplx=c)
    del L, R
    gc.collect()
    x = hb.to_device(th)
    y = torch.empty_like(x)
    op.MultAx(x, y)
    torch.cuda.synchronize()
    err = relerr(hb.to_host(y, th.shape), y_ref)
    assert err < TOL, f"DMMA engine: {err:.3e}"
    # the same operator on the INT8 engine (FP64-accurate GEMMs from int8 digit planes)
    op.set_fp64_engine(hb.FP64_INT8)
    y.fill_(float("nan"))
    op.MultAx(x, y)
    torch.cuda.synchronize()
    assert op.device_error() == 0
    err8 = relerr(hb.to_host(y, th.shape), y_ref)
    assert err8 < TOL, f"INT8 engine: {err8:.3e}"
    op.close()
    del x, y
    torch.cuda.empty_cache()


@pytest.mark.parametrize("D", [3, 9])
@pytest.mark.parametrize("c", [False, True])
def test_env_update_chi1024_vs_blas_oracle(cuda, D, c):
    chi = 1024
    rng = np.random.default_rng(100 + D)
    M = np.asfortranarray(rng.standard_normal((2, chi, chi)) + (1j * rng.standard_normal((2, chi, chi)) if c else 0))
    W = oracle.mpo_ising(1.0, 0.8)
    if D == 9:
        W = oracle.mpo_square(W)
    W = W.astype(complex if c else float)
    for side in ("L", "R"):
        E = ph.hermitian_env(rng, chi, D, c)
        dE, dM, dW = (hb.to_device(a) for a in (E, M, W))
        out = torch.empty(chi * chi * D, dtype=dE.dtype, device="cuda")
        hb.env_update(side, out, dE, E.shape, dM, M.shape, dW, W.shape)
        torch.cuda.synchronize()
        err = relerr(hb.to_host(out, (chi, chi, D)), rn.env_update_blas(side, E, M, W))
        assert err < TOL, f"side {side}: {err:.3e}"
