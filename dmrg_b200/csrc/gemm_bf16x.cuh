// BF16 GEMM on the sm_100a 5th-generation tensor cores (tcgen05.mma kind::f16, FP32 accumulators in
// TMEM), operands staged by TMA (cp.async.bulk.tensor, 128-byte swizzle) in a 4-stage mbarrier ring.
//
//   C[m, n] = sum_k A[m, k] * B[n, k]        A: M x K,  B: N x K, both K-contiguous ("K-major") bf16
//
// Used by the mixed-precision matvec: every FP64 operand is split into BF16 parts (x ~ x_hi + x_mid)
// and the split products are folded into the K dimension (A' = [a_hi | a_hi | a_mid],
// B' = [b_hi | b_mid | b_hi] gives a_hi b_hi + a_hi b_mid + a_mid b_hi in one GEMM).
//
// CTA: 192 threads = warp 0 TMA producer, warp 1 TMEM allocator + MMA issuer, warps 2-5 epilogue
// (tcgen05.ld 32x32b: warp w reads TMEM lanes 32*(w%4) .. +31).  Tile 128 x 256 x 64.  Persistent: one CTA
// per SM walks its share of the tiles with two TMEM accumulators (512 columns), so the epilogue of a tile
// overlaps the MMAs of the next.  Every mbarrier wait is bounded: on timeout the kernel raises *err, skips its
// remaining work, still frees its TMEM and returns.  No cluster multicast anywhere.
#pragma once
#include <cuda.h>

#include "heff_common.cuh"

namespace heff {

constexpr int X_BM = 128, X_BN = 256, X_BK = 64, X_STAGES = 4, X_THREADS = 192;
constexpr int X_A_BYTES     = X_BM * X_BK * 2;  // 16 KB
constexpr int X_B_BYTES     = X_BN * X_BK * 2;  // 32 KB
constexpr int X_STAGE_BYTES = X_A_BYTES + X_B_BYTES;
constexpr int X_SMEM_BYTES  = X_STAGES * X_STAGE_BYTES + 1024 /*align*/ + 256 /*barriers*/;

enum XEpilogue : int {
    X_OUT_F32     = 0,  // C float, column-major C[m + ldc*n]
    X_OUT_F64     = 1,  // C double, column-major
    X_OUT_C128    = 2,  // C complex double interleaved: column n < n_half -> re of (m, n), else im of (m, n - n_half)
    X_OUT_F32_ACC = 3   // C float, C[m + ldc*n] += acc
};

struct XGemmArgs {
    int   M, N, K;  // K = extended (split) K, multiple of 64 after padding
    void *C;
    int64_t ldc;
    int     mode;
    int     n_half;
    int    *err;  // device error flag (set to a nonzero code on a wait timeout)
};

// Builds a 2D K-major bf16 tensor map over rows x kcols (row pitch ld_elems) with box {64, box_rows}.
int make_tmap_bf16(CUtensorMap *map, const void *base, int64_t rows, int64_t kcols, int64_t ld_elems, int box_rows);

// Launch one BF16 GEMM.  tmA covers A (M x K, box rows 128), tmB covers B (N x K, box rows 256).
int gemm_bf16x(const CUtensorMap &tmA, const CUtensorMap &tmB, const XGemmArgs &args, cudaStream_t s);

}  // namespace heff
