"""CPU model of the INT8 engine's arithmetic (the scheme of dmrg_b200/csrc/gemm_i8.cuh), run in numpy.

Each step mirrors the kernels: the per-row power-of-two scale taken from the exponent bits (z_set_scale), the
round-half-even digits with exact FP64 remainders (z_digits16), the level sums of equal-weight digit products
(one INT32 accumulation per level, folded over K), the FP64 recombination smallest level first, and the complex
real embedding ([re | im] rows on the A side, [re | -im] / [im | re] row pairs on the B side).

Bars: the digits reproduce every entry to 2^-7s of its row scale (half a unit of the last digit); the level sums stay inside INT32 under the
bound the library checks (4096 * slices * K' < 2^31); the product matches FP64 to 5e-13 at 7 slices (1e-15 at 8)
and is clearly worse at 4.
"""
import numpy as np
import pytest


def row_scales(A):
    """(64 / sigma_r, sigma_r) per row, sigma_r the smallest power of two above max |A[r, :]| (at least 2^-1016)."""
    mx = np.max(np.abs(A), axis=1)
    E = ((mx.view(np.uint64) >> np.uint64(52)) & np.uint64(0x7FF)).astype(np.int64) + 1
    E[mx == 0] = 1023
    E = np.clip(E, 7, 2045)
    inv = ((2052 - E).astype(np.uint64) << np.uint64(52)).view(np.float64)
    sig = (E.astype(np.uint64) << np.uint64(52)).view(np.float64)
    return inv, sig


def digits(A, ns):
    inv, sig = row_scales(A)
    y = A * inv[:, None]  # exact (power of two)
    assert np.all(np.abs(y) <= 64.0)
    out = np.empty((ns,) + A.shape, dtype=np.int64)
    for t in range(ns):
        d = np.rint(y)  # round half to even, like __double2int_rn
        r = y - d
        assert np.all(np.abs(r) <= 0.5)
        y = r * 128.0
        out[t] = d
    assert np.all(np.abs(out) <= 64)
    return out, sig


def emu_gemm(A, B, ns):
    """C = A B^T from digit planes; also returns the largest |level sum| seen."""
    DA, sa = digits(A, ns)
    DB, sb = digits(B, ns)
    C = np.zeros((A.shape[0], B.shape[0]))
    smax = 0
    for g in range(ns - 1, -1, -1):  # smallest level first, as the epilogue sums them
        S = sum(DA[i] @ DB[g - i].T for i in range(g + 1))  # one K-folded integer GEMM per level
        smax = max(smax, int(np.max(np.abs(S))))
        C = C + S.astype(np.float64) * (2.0 ** (-12 - 7 * g)) * sa[:, None] * sb[None, :]
    return C, smax


def test_digit_planes_reproduce_entries():
    rng = np.random.default_rng(1)
    A = rng.standard_normal((40, 70)) * np.exp2(rng.integers(-40, 40, (40, 1)))
    for ns in (4, 7, 8):
        D, sig = digits(A, ns)
        w = 2.0 ** (-6 - 7 * np.arange(ns))
        rec = np.tensordot(w, D.astype(np.float64), axes=1) * sig[:, None]
        assert np.max(np.abs(rec - A) / sig[:, None]) <= 2.0 ** (-7 * ns)


@pytest.mark.parametrize("ns,hi", [(8, 1e-15), (7, 5e-13)])
def test_level_sums_match_fp64(ns, hi):
    rng = np.random.default_rng(ns)
    A, B = rng.standard_normal((50, 300)), rng.standard_normal((60, 300))
    C, smax = emu_gemm(A, B, ns)
    ref = A @ B.T
    assert np.linalg.norm(C - ref) / np.linalg.norm(ref) < hi
    assert smax < 2 ** 31


def test_four_slices_are_visibly_worse():
    rng = np.random.default_rng(4)
    A, B = rng.standard_normal((30, 200)), rng.standard_normal((20, 200))
    C, _ = emu_gemm(A, B, 4)
    assert np.linalg.norm(C - A @ B.T) / np.linalg.norm(A @ B.T) > 1e-10


def test_int32_bound_worst_case():
    """Every digit at +64: a level folds (g + 1) K' products of 4096; the library admits K' only while
    4096 * slices * K' < 2^31, which keeps the largest level inside INT32."""
    ns = 7
    kx = (2 ** 31 - 1) // (4096 * ns)
    assert 4096 * ns * kx < 2 ** 31 and 4096 * ns * (kx + 1) >= 2 ** 31
    assert 4096 * ns * kx <= 2 ** 31 - 1  # the top level (g = ns - 1) at its largest


def test_complex_embedding():
    rng = np.random.default_rng(7)
    A = rng.standard_normal((20, 64)) + 1j * rng.standard_normal((20, 64))
    B = rng.standard_normal((24, 64)) + 1j * rng.standard_normal((24, 64))
    Ae = np.hstack([A.real, A.imag])                        # A' rows [re | im]
    Be = np.empty((2 * B.shape[0], 128))
    Be[0::2] = np.hstack([B.real, -B.imag])                 # B' rows 2n = [re | -im]
    Be[1::2] = np.hstack([B.imag, B.real])                  #        2n+1 = [im | re]
    Ce, _ = emu_gemm(Ae, Be, 7)
    C = Ce[:, 0::2] + 1j * Ce[:, 1::2]
    ref = A @ B.T  # no conjugation
    assert np.linalg.norm(C - ref) / np.linalg.norm(ref) < 5e-13


def test_zero_rows_and_tiny_rows():
    A = np.zeros((3, 16))
    A[1] = 1e-310  # subnormal: scale floored at 2^-1016, digits still exact
    A[2, 3] = -2.5
    B = np.ones((2, 16))
    C, _ = emu_gemm(A, B, 7)
    assert np.all(C[0] == 0.0)
    assert np.allclose(C[2], -2.5)
    assert np.allclose(C[1], 16 * 1e-310, rtol=1e-6, atol=0)
