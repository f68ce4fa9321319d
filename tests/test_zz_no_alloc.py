"""heff_matvec_d_noalloc: the matvec entry point that allocates no device memory.

It serves callers that cannot let a library call cudaMalloc (for instance a
process that has already divided all device memory among its own pools, or one
that cannot afford the device-wide synchronisation of cudaMalloc/cudaFree).  Its
scratch lives in one fixed 32 MiB array inside the library that every call
shares.  This file is collected last (test_zz_*) so that a run stopping at the
first failure has already run every other test; it passes alone in a fresh
process as well as after the rest of the suite.
"""
import ctypes

import numpy as np
import pytest
import torch

import dmrg_b200 as hb
from oracle import physics as ph

from conftest import relerr

pytestmark = pytest.mark.gpu
TOL = 1e-12  # the FP64 matvec tolerance used by every parity test


def _noalloc():
    f = hb.lib().heff_matvec_d_noalloc
    P, D = ctypes.c_void_p, ctypes.POINTER(ctypes.c_int64)
    f.argtypes = [P, P, D, P, D, P, D, P, D, P]
    f.restype = ctypes.c_int
    return f


def _call(fn, th, W, L, R):
    d = [hb.to_device(a) for a in (th, W, L, R)]
    res = torch.full_like(d[0], float("nan"))
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = fn(hb.ptr(res), hb.ptr(d[0]), hb.dims(th.shape), hb.ptr(d[1]), hb.dims(W.shape), hb.ptr(d[2]), hb.dims(L.shape), hb.ptr(d[3]),
            hb.dims(R.shape), stream)
    torch.cuda.synchronize()
    return rc, hb.to_host(res, th.shape)


def test_noalloc_matches_allocating_entry_point_twice(cuda):
    noalloc = _noalloc()
    alloc = hb.lib().heff_matvec_d
    # two calls in a row with different shapes: the second must not depend on what the first left behind
    for chiL, chiR, D, seed in ((256, 256, 3, 1), (120, 161, 9, 2)):
        th, W, L, R = ph.heff_inputs(chiL, D=D, cplx=False, seed=seed, chiR=chiR)
        rc, y_na = _call(noalloc, th, W, L, R)
        assert rc == 0, hb.lib().heff_last_error()
        rc2, y_ref = _call(alloc, th, W, L, R)
        assert rc2 == 0
        assert np.all(np.isfinite(y_na))
        assert relerr(y_na, y_ref) < TOL


def test_noalloc_rejects_oversize(cuda):
    noalloc = _noalloc()
    chi = 1024  # needs ~248 MB of scratch, above the fixed 32 MiB array
    x = torch.zeros(4 * chi * chi, dtype=torch.float64, device="cuda")
    y = torch.zeros_like(x)
    env = torch.zeros(chi * chi * 3, dtype=torch.float64, device="cuda")
    W = torch.zeros(3 * 3 * 4 * 4, dtype=torch.float64, device="cuda")
    rc = noalloc(hb.ptr(y), hb.ptr(x), hb.dims((4, chi, chi)), hb.ptr(W), hb.dims((3, 3, 4, 4)), hb.ptr(env), hb.dims((chi, chi, 3)), hb.ptr(env),
                 hb.dims((chi, chi, 3)), ctypes.c_void_p(0))
    assert rc == 1  # HEFF_BAD_SHAPE
    assert b"scratch" in hb.lib().heff_last_error()
