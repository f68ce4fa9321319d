// FP64-accurate GEMM on the sm_100a INT8 tensor cores (tcgen05.mma kind::i8, exact INT32 accumulation in
// TMEM), by error-free digit splitting (the Ozaki scheme, Ozaki/Ogita/Oishi/Rump, Numer. Algorithms 59
// (2012); integer form: Ootomo/Ozaki/Yokota, IJHPCA 2024):
//
//   every row r of an operand is scaled by a power of two sigma_r > max_k |v[r,k]| and written as signed
//   digits  v[r,k] = sigma_r * 2^-6 * sum_t d_t[r,k] 2^(-7t)  (+ a remainder of at most 2^-7s sigma_r, half a
//   unit of the last digit),
//   d_0 = rint(64 x), d_t = rint(128 * remainder): |d_t| <= 64 fits int8 and every step is exact in FP64.
//
//   C[m,n] = fa[m] fb[n] sum_{g < s} 2^(-7g) S_g[m,n],   S_g = sum_{t+u=g} D^A_t (D^B_u)^T   (INT32, exact)
//
// The digit products of one level g are folded into the GEMM's K dimension (K' = (g+1) K: slice pairs
// (t, g-t) one after the other), so a level is one accumulation in TMEM; levels beyond s-1 are dropped
// (they are below 2^-(7s-1) of the leading term).  The epilogue turns each level's INT32 tile into FP64
// exactly (an integer times powers of two) and sums the levels smallest first (in TMEM for 128-wide tiles,
// else in C, which stays in L2 between a tile's levels).  With s = 7 the products carry 48 bits relative to
// sigma_a sigma_b, i.e. normwise errors of a few 2^-48 -- the same order as an FP64 GEMM's K-dependent bound.
// A non-finite operand entry raises the operand's bad word in the slicer; the GEMM then writes NaN.
//
// Complex operands use a real embedding: A' rows [re | im], B' rows 2n = [re | -im] and 2n+1 = [im | re],
// so C'[m, 2n] = Re C[m, n] and C'[m, 2n+1] = Im C[m, n] with one real GEMM of K' = 2K.
//
// CTA: 192 threads = warp 0 TMA producer, warp 1 TMEM allocator + MMA issuer, warps 2-5 epilogue.  Tile
// 128 x BN (BN = 128, 192 or 256), k-block 128 bytes, 4-6-stage ring, two TMEM accumulators; persistent (one
// CTA per SM) over the (tile, level) units.  Every mbarrier wait is bounded; on timeout *err is raised, the
// CTA skips its remaining work, frees its TMEM and returns.  No cluster multicast.
#pragma once
#include <cuda.h>

#include "heff_common.cuh"

namespace heff {

constexpr int Z_BM = 128, Z_BK = 128, Z_THREADS = 192;
constexpr int Z_A_BYTES = Z_BM * Z_BK;  // 16 KB
// Tile width BN in {128, 192, 256} (chosen per shape to fill the last wave): the ring takes as many stages of
// A (16 KB) + B (BN x 128 B) as fit in 210 KB.  At BN = 128 the FP64 sum over levels stays in TMEM (two INT32
// accumulators in columns [0, 256), the FP64 partial as b32 pairs in [256, 512)) and C is written once; at the
// wider tiles TMEM holds only the two accumulators and the levels are summed in C (L2-resident).
template<int BN>
struct ZCfg {
    static constexpr int  STAGE      = Z_A_BYTES + BN * Z_BK;
    static constexpr int  STAGES     = (210 * 1024) / STAGE;  // 4, 5, 6
    static constexpr int  SMEM       = STAGES * STAGE + 1024 /*align*/ + 256 /*barriers*/;
    static constexpr bool TMEM_SUM   = BN == 128;
    static constexpr int  TMEM_COLS  = 512;
    static constexpr int  PART_COL   = 2 * BN;  // first column of the FP64 partial (TMEM_SUM)
};
constexpr int Z_MAX_SLICES  = 8;
constexpr int Z_DEFAULT_SLICES = 7;

// Digit planes of one operand: planes[t * rows * kx + r * kx + k], t < nslice; kx a multiple of 16 bytes.
struct ZPlanes {
    int8_t  *planes = nullptr;
    int64_t  rows = 0, kx = 0;
    int      nslice = 0;
    double  *inv = nullptr;  // per source row: 64 / sigma_r (the first digit's scale)
    double  *fac = nullptr;  // per source row: sigma_r times the operand's extra factor (2^-12 on the A side)
    unsigned long long *rmax = nullptr;  // per source row: bits of max |v| (M-major sources); kept zero between uses
};

struct ZGemmArgs {
    int           M, N, K;  // C' rows (A rows), C' columns (B' rows), K' (bytes of a plane row)
    int           nslice;
    const double *fa, *fb;  // per A row; per B source row (complex: B' rows 2n, 2n+1 share fb[n])
    void         *C;
    int64_t       ldc;      // column-major C: real C[m + ldc n]; complex C[m + ldc (n'/2)] (re, im) from B' rows n', n'+1
    int           cplx;
    int          *err;           // sticky status: 1-4 a pipeline wait timed out, 5 an input was non-finite
    const int    *bad_a, *bad_b;  // the operands' bad words (raised by their slicers); either set: C is NaN
};

// 3D tensor map over digit planes {kx, rows, nslice}, box {128, box_rows, 1}, 128-byte swizzle.
int make_tmap_planes(CUtensorMap *map, const ZPlanes &p, int box_rows);
// Tile width for a C' of M x N over K' (fewest waves on the device's SMs, weighted by measured per-MAC costs).
int z_choose_bn(int64_t M, int64_t N, int64_t K);

// The slicers raise *bad (an int the caller clears) for a non-finite entry or one of magnitude >= 2^1022.
// Row scales of a K-major source src[r * ld + k] (k < K): inv, fac (fac = sigma * extra).
template<bool CPLX>
int z_scale_kmajor(const typename Scalar<CPLX>::T *src, int64_t rows, int64_t K, int64_t ld, double extra, ZPlanes &p, int *bad, cudaStream_t s);
// Row scales of an M-major source src[r + ld * k] (uses p.rmax, left zeroed).
template<bool CPLX>
int z_scale_mmajor(const typename Scalar<CPLX>::T *src, int64_t rows, int64_t K, int64_t ld, double extra, ZPlanes &p, int *bad, cudaStream_t s);
// Digit planes from a K-major source.  bmode (complex only): rows 2r = [re | -im], 2r+1 = [im | re];
// otherwise row r = [re | im] (complex) or [v] (real); each half is round16(K) wide.
template<bool CPLX>
int z_slice_kmajor(const typename Scalar<CPLX>::T *src, int64_t rows, int64_t K, int64_t ld, bool bmode, const ZPlanes &p, int *bad, cudaStream_t s);
// Digit planes (A-mode) from an M-major source src[r + ld * k].
template<bool CPLX>
int z_slice_mmajor(const typename Scalar<CPLX>::T *src, int64_t rows, int64_t K, int64_t ld, const ZPlanes &p, int *bad, cudaStream_t s);

// Plane row pitch for K source columns: round16(K), doubled for complex.
inline int64_t z_kx(int64_t K, bool cplx) { return ((K + 15) / 16 * 16) * (cplx ? 2 : 1); }
// Largest K' for which no level sum can overflow INT32 (|d| <= 64, s slices folded per level).
inline bool z_k_ok(int64_t kx, int nslice) { return kx > 0 && (int64_t)4096 * nslice * kx < ((int64_t)1 << 31); }

// C = (A planes)(B planes)^T combined as described above; builds the tensor maps for the chosen tile width.
int gemm_i8_ozaki(const ZPlanes &A, const ZPlanes &B, const ZGemmArgs &args, cudaStream_t s);

}  // namespace heff
