"""Admission estimate of the eigensolve server (heff_request_bytes): pure host arithmetic, checked without a GPU.

The server admits a request only while the device memory its in-flight requests hold stays within the budget, so
the estimate must cover every buffer the request allocates: operator copies and matvec scratch always, the split
BF16 operands for mixed precision, the INT8 digit planes for the INT8 engine, and the eigensolver basis.
"""
import ctypes


import dmrg_b200 as hb
from dmrg_b200._sigs import Request


def req(chi, D=3, cplx=False, precision=hb.PREC_FP64, engine=hb.FP64_DMMA):
    r = Request()
    r.dtype = hb.C128 if cplx else hb.F64
    r.spin, r.chiL, r.chiR, r.mpoL, r.mpoR = 4, chi, chi, D, D
    r.precision = int(precision)
    r.fp64_engine = int(engine)
    return r


def nbytes(r, basis=24):
    return int(hb.lib().heff_request_bytes(ctypes.byref(r), basis))


def test_estimate_covers_the_operator_and_the_basis():
    for chi, D, c in [(64, 3, False), (256, 9, True), (1024, 3, True)]:
        es = 16 if c else 8
        n = 4 * chi * chi
        floor = es * (chi * chi * D + chi * chi * D + n * (1 + 2 * D)) + es * n * 2 * 25
        assert nbytes(req(chi, D, c)) >= floor


def test_estimate_grows_with_chi_and_basis():
    sizes = [nbytes(req(chi)) for chi in (32, 64, 128, 256, 512)]
    assert all(a < b for a, b in zip(sizes, sizes[1:]))
    assert nbytes(req(256), 48) > nbytes(req(256), 24)


def test_mixed_and_int8_requests_budget_their_buffers():
    for c in (False, True):
        base = nbytes(req(512, cplx=c))
        mixed = nbytes(req(512, cplx=c, precision=hb.PREC_MIXED))
        int8 = nbytes(req(512, cplx=c, engine=hb.FP64_INT8))
        assert mixed > base and int8 > base
        # 7 digit planes of L, x', T2 and R' (one byte per real entry, complex embedded at twice the width)
        cf = 2 if c else 1
        planes = 7 * cf * (512 * 3 * 512 + cf * 4 * 512 * 512 + 4 * 512 * 3 * 512 + cf * 512 * 3 * 512)
        assert int8 - base >= planes


def test_null_request_is_zero():
    assert hb.lib().heff_request_bytes(None, 24) == 0


def test_int8_tile_width_knob():
    """heff_i8_set_tile_width accepts 0 (cost model), 1 (autotuner, the default), 128, 192 or 256, returns the previous
    setting, rejects the rest."""
    L = hb.lib()
    prev = L.heff_i8_set_tile_width(0)
    try:
        assert prev in (0, 1, 128, 192, 256)
        assert L.heff_i8_set_tile_width(192) == 0
        assert L.heff_i8_set_tile_width(128) == 192
        assert L.heff_i8_set_tile_width(100) == -1
        assert L.heff_i8_set_tile_width(160) == -1
        assert L.heff_i8_set_tile_width(2) == -1
        assert L.heff_i8_set_tile_width(1) == 128
        assert L.heff_i8_set_tile_width(0) == 1
        assert L.heff_i8_tuned_shapes() >= 0
    finally:
        L.heff_i8_set_tile_width(prev)


def test_gemm_tail_split_knob():
    """heff_gemm_set_tail_split accepts 0 (off), 1 (automatic) or a piece count 2..16, returns the previous mode,
    rejects the rest."""
    L = hb.lib()
    prev = L.heff_gemm_set_tail_split(1)
    try:
        assert 0 <= prev <= 16
        assert L.heff_gemm_set_tail_split(0) == 1
        assert L.heff_gemm_set_tail_split(4) == 0
        assert L.heff_gemm_set_tail_split(17) == -1
        assert L.heff_gemm_set_tail_split(-1) == -1
        assert L.heff_gemm_set_tail_split(1) == 4
    finally:
        L.heff_gemm_set_tail_split(prev)
