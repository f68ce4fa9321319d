"""The INT8 engine (FP64-accurate matvecs emulated on the INT8 tensor cores) inside whole calculations: fDMRG and
xDMRG sweeps on fixed-capacity operators that are rebound at every bond, the overlapped ensemble, and the server.

Bar: the same energies as the DMMA engine to 1e-10 (xDMRG: 1e-9, the bar of its mixed-precision test), variance
below 1e-10, ensemble results identical alone and overlapped.
"""
import numpy as np
import pytest
import torch

import dmrg_b200 as hb
from oracle import physics as ph

pytestmark = pytest.mark.gpu


def test_fdmrg_int8_engine_matches_dmma(cuda):
    h = ph.random_fields(77, 12)
    r64 = hb.fdmrg(h, chi_max=64, sweeps=6, seed=2)
    r8 = hb.fdmrg(h, chi_max=64, sweeps=6, seed=2, fp64_engine=hb.FP64_INT8)
    assert abs(r8["energy"] - r64["energy"]) < 1e-10 * abs(r64["energy"])
    assert abs(r8["entropy_mid"] - r64["entropy_mid"]) < 1e-8
    assert r8["unconverged_solves"] == 0


def test_xdmrg_int8_engine_matches_dmma(cuda):
    h = ph.random_fields(4242, 10)
    lev = ph.free_fermion_levels(h)
    et = -lev.sum() + 0.3 * 2 * lev.sum()
    r64 = hb.xdmrg(h, et, chi_max=32, sweeps=12, eig_tol=1e-12, seed=1)
    r8 = hb.xdmrg(h, et, chi_max=32, sweeps=12, eig_tol=1e-12, seed=1, fp64_engine=hb.FP64_INT8)
    assert r8["variance"] < 1e-10
    assert abs(r8["energy"] - r64["energy"]) < 1e-9


def test_ensemble_int8_engine_alone_vs_overlapped(cuda):
    reals = [(ph.random_fields(500 + i, L), 2 ** (L // 2), i) for i, L in enumerate((8, 10, 12, 8, 10, 12))]
    r1, st1, _ = hb.ensemble(reals, nthreads=1, sweeps=4, fp64_engine=hb.FP64_INT8)
    r4, st4, _ = hb.ensemble(reals, nthreads=4, sweeps=4, fp64_engine=hb.FP64_INT8)
    rd, std, _ = hb.ensemble(reals, nthreads=4, sweeps=4)
    assert all(s == 0 for s in st1 + st4 + std)
    for a, b, c in zip(r1, r4, rd):
        assert a["energy"] == b["energy"]  # the same kernels with fixed-order reductions, alone or overlapped
        assert abs(a["energy"] - c["energy"]) < 1e-10 * abs(c["energy"])


def test_server_int8_engine_request(cuda):
    chi = 48
    W = ph.ising_two_site_mpo(0.8, 1.2).astype(np.float64)
    envL = hb.make_env(chi, 3, False, seed=5)
    envR = hb.make_env(chi, 3, False, seed=6)
    Lh, Rh = hb.to_host(envL, (chi, chi, 3)), hb.to_host(envR, (chi, chi, 3))
    op = hb.MatVecMPOS([W], Lh, Rh)
    e_direct, _ = op.eigs(tol=1e-12, mixed=False)
    op.close()
    torch.cuda.synchronize()
    req64 = hb.EigServer.request(W, envL, envR, 4, chi, chi, False, tol=1e-12)
    req8 = hb.EigServer.request(W, envL, envR, 4, chi, chi, False, tol=1e-12, fp64_engine=hb.FP64_INT8)
    assert hb.EigServer.request_bytes(req8[0]) > hb.EigServer.request_bytes(req64[0])  # the digit planes are budgeted
    srv = hb.EigServer(max_inflight=2)
    r = srv.wait(srv.submit(req8), timeout=120)
    srv.close()
    assert r["status"] == 0
    assert abs(r["eigval"] - e_direct) < 1e-10 * abs(e_direct)
