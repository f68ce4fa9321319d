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
from oracle import ref_numpy as rn

from conftest import relerr

pytestmark = pytest.mark.gpu
TOL = 1e-12  # the FP64 matvec tolerance used by every parity test
SCRATCH_BYTES = 32 << 20  # size of the library's fixed scratch array


def _noalloc():
    f = hb.lib().heff_matvec_d_noalloc
    P, D = ctypes.c_void_p, ctypes.POINTER(ctypes.c_int64)
    f.argtypes = [P, P, D, P, D, P, D, P, D, P]
    f.restype = ctypes.c_int
    return f


def _scratch_bytes(S, cL, cR, DL, DR):
    """Scratch of one real matvec as the library lays it out: x' | T1 | T2 | R', each padded to 32 doubles."""
    pad = lambda n: (n + 31) // 32 * 32
    return 8 * (pad(S * cL * cR) + pad(DL * S * cL * cR) + pad(DR * S * cL * cR) + pad(cR * cR * DR))


def _upload(th, W, L, R):
    d = [hb.to_device(a) for a in (th, W, L, R)]
    return d, torch.full_like(d[0], float("nan"))


def _launch(fn, d, res, shapes):
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    th, W, L, R = shapes
    return fn(hb.ptr(res), hb.ptr(d[0]), hb.dims(th), hb.ptr(d[1]), hb.dims(W), hb.ptr(d[2]), hb.dims(L), hb.ptr(d[3]), hb.dims(R), stream)


def _call(fn, th, W, L, R):
    d, res = _upload(th, W, L, R)
    rc = _launch(fn, d, res, (th.shape, W.shape, L.shape, R.shape))
    torch.cuda.synchronize()
    return rc, hb.to_host(res, th.shape)


def test_noalloc_matches_allocating_entry_point_twice(cuda):
    """Calls in a row against the oracle and the allocating entry point.  The first call is the largest in every
    dimension and its mps is scaled by 1e100, so the shared array is left full of huge values: a later call that
    read any element it had not written itself would visibly break parity."""
    noalloc = _noalloc()
    alloc = hb.lib().heff_matvec_d
    cases = [  # spin, chiL, chiR, D, seed, scale
        (4, 220, 200, 9, 1, 1e100),  # norms of ~1e105-sized vectors stay finite in FP64
        (2, 150, 131, 3, 2, 1.0),
        (4, 97, 180, 3, 3, 1.0),
    ]
    for S, chiL, chiR, D, seed, scale in cases:
        assert _scratch_bytes(S, chiL, chiR, D, D) <= SCRATCH_BYTES
        th, W, L, R = ph.heff_inputs(chiL, D=D, cplx=False, seed=seed, chiR=chiR, spin=S)
        th = np.asfortranarray(th * scale)
        rc, y_na = _call(noalloc, th, W, L, R)
        assert rc == 0, hb.lib().heff_last_error()
        assert np.all(np.isfinite(y_na)) and np.isfinite(np.linalg.norm(y_na))
        assert relerr(y_na, rn.matvec_blas(th, W, L, R)) < TOL
        rc2, y_ref = _call(alloc, th, W, L, R)
        assert rc2 == 0
        assert relerr(y_na, y_ref) < TOL


def test_noalloc_leaves_free_device_memory_unchanged(cuda):
    """The call itself takes no device memory: free memory (cudaMemGetInfo) is the same before and after two calls.
    One call first, untimed, because the CUDA runtime may load the library's kernels on first use."""
    noalloc = _noalloc()
    th, W, L, R = ph.heff_inputs(200, D=3, cplx=False, seed=11, chiR=190)
    d, res = _upload(th, W, L, R)
    shapes = (th.shape, W.shape, L.shape, R.shape)
    assert _launch(noalloc, d, res, shapes) == 0
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(2):
        assert _launch(noalloc, d, res, shapes) == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    assert relerr(hb.to_host(res, th.shape), rn.matvec_blas(th, W, L, R)) < TOL


def test_noalloc_size_limit_boundary(cuda):
    """The largest square real two-site D=3 shape whose scratch fits the array runs; one bond more is rejected."""
    noalloc = _noalloc()
    chi = 1
    while _scratch_bytes(4, chi + 1, chi + 1, 3, 3) <= SCRATCH_BYTES:
        chi += 1
    assert _scratch_bytes(4, chi, chi, 3, 3) <= SCRATCH_BYTES < _scratch_bytes(4, chi + 1, chi + 1, 3, 3)
    th, W, L, R = ph.heff_inputs(chi, D=3, cplx=False, seed=chi)
    rc, y = _call(noalloc, th, W, L, R)
    assert rc == 0, hb.lib().heff_last_error()
    assert relerr(y, rn.matvec_blas(th, W, L, R)) < TOL
    big = chi + 1
    x = torch.zeros(4 * big * big, dtype=torch.float64, device="cuda")
    yb = torch.zeros_like(x)
    env = torch.zeros(big * big * 3, dtype=torch.float64, device="cuda")
    Wd = torch.zeros(3 * 3 * 4 * 4, dtype=torch.float64, device="cuda")
    rc = noalloc(hb.ptr(yb), hb.ptr(x), hb.dims((4, big, big)), hb.ptr(Wd), hb.dims((3, 3, 4, 4)), hb.ptr(env), hb.dims((big, big, 3)),
                 hb.ptr(env), hb.dims((big, big, 3)), ctypes.c_void_p(0))
    assert rc == 1  # HEFF_BAD_SHAPE
    assert b"scratch" in hb.lib().heff_last_error()


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
