// FP64-accurate GEMM on the INT8 tensor cores (see gemm_i8.cuh): digit-plane slicers, row scales and the
// persistent tcgen05 kind::i8 kernel with the level-combining FP64 epilogue.
#include <algorithm>
#include <atomic>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>

#include "gemm_i8.cuh"
#include "runtime.cuh"
#include "tcgen05.cuh"

namespace heff {

using namespace tc;

// ---------------------------------------------------------------------------------------------------------
// Row scales and digit planes
// ---------------------------------------------------------------------------------------------------------

__device__ __forceinline__ double z_re(double v) { return v; }
__device__ __forceinline__ double z_im(double) { return 0.0; }
__device__ __forceinline__ double z_re(double2 v) { return v.x; }
__device__ __forceinline__ double z_im(double2 v) { return v.y; }

// sigma_r = 2^(Es - 1023), the smallest power of two above the row maximum mx (>= 0), at least 2^-1016 (an
// all-zero row takes sigma = 1).  inv = 64 / sigma_r and fac = sigma_r * extra are exact powers of two.  A
// maximum of 2^1022 or more (or inf) is out of range: the operand's bad word is raised and the row clamped
// (the GEMM then writes NaN, as an FP64 product of such an input would).
__device__ __forceinline__ void z_set_scale(double mx, double extra, double *inv, double *fac, int *bad) {
    const unsigned long long b = (unsigned long long)__double_as_longlong(mx);
    int                      Es = mx == 0.0 ? 1023 : (int)((b >> 52) & 0x7ff) + 1;
    if(Es < 7) Es = 7;
    if(Es > 2045) {
        atomicExch(bad, 1);
        Es = 2045;
    }
    *inv = __longlong_as_double((long long)((unsigned long long)(2052 - Es) << 52));
    *fac = __longlong_as_double((long long)((unsigned long long)Es << 52)) * extra;
}

// one warp per row of a K-major source
template<bool CPLX>
__global__ void z_scale_k_kernel(const typename Scalar<CPLX>::T *__restrict__ src, int64_t rows, int64_t K, int64_t ld, double extra,
                                 double *__restrict__ inv, double *__restrict__ fac, int *bad) {
    const int     lane = threadIdx.x & 31;
    const int64_t nw   = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for(int64_t r = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < rows; r += nw) {
        const typename Scalar<CPLX>::T *row = src + r * ld;
        double                          m   = 0.0;
        for(int64_t k = lane; k < K; k += 32) {
            const auto v = row[k];
            m            = fmax(m, fabs(z_re(v)));
            if(CPLX) m = fmax(m, fabs(z_im(v)));
        }
#pragma unroll
        for(int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
        if(lane == 0) z_set_scale(m, extra, inv + r, fac + r, bad);
    }
}

// M-major source src[r + ld k]: thread per row over one chunk of k; partial maxima meet in rmax (as the bit
// patterns of non-negative doubles, which order like the values)
template<bool CPLX>
__global__ void z_rowmax_m_kernel(const typename Scalar<CPLX>::T *__restrict__ src, int64_t rows, int64_t K, int64_t ld, int64_t kchunk,
                                  unsigned long long *rmax) {
    const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if(r >= rows) return;
    const int64_t k0 = (int64_t)blockIdx.y * kchunk, k1 = min(K, k0 + kchunk);
    double        m  = 0.0;
    for(int64_t k = k0; k < k1; k++) {
        const auto v = src[r + ld * k];
        m            = fmax(m, fabs(z_re(v)));
        if(CPLX) m = fmax(m, fabs(z_im(v)));
    }
    if(m > 0.0) atomicMax(rmax + r, (unsigned long long)__double_as_longlong(m));
}
__global__ void z_rowmax_fin_kernel(unsigned long long *rmax, int64_t rows, double extra, double *inv, double *fac, int *bad) {
    for(int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += (int64_t)gridDim.x * blockDim.x) {
        const double m = __longlong_as_double((long long)rmax[r]);
        rmax[r]        = 0ull;  // ready for the next use
        z_set_scale(m, extra, inv + r, fac + r, bad);
    }
}

// Digits of 16 scaled values y (|y| <= 64) for slice t: byte j of w = rint(y_j); y_j <- 128 (y_j - rint(y_j)).
// Both steps are exact in FP64 (|y - rint y| <= 1/2 lies on y's own grid), so after s slices the value is
// reproduced to half a unit of the last digit, 2^-7s of the row scale.
__device__ __forceinline__ void z_digits16(double (&y)[16], uint32_t (&w)[4], uint32_t (&wn)[4]) {
#pragma unroll
    for(int q = 0; q < 4; q++) {
        w[q] = 0u, wn[q] = 0u;
#pragma unroll
        for(int j = 0; j < 4; j++) {
            const int d = __double2int_rn(y[4 * q + j]);
            y[4 * q + j] = (y[4 * q + j] - (double)d) * 128.0;
            w[q] |= ((uint32_t)d & 0xffu) << (8 * j);
            wn[q] |= ((uint32_t)(-d) & 0xffu) << (8 * j);
        }
    }
}
__device__ __forceinline__ void z_st16(int8_t *p, const uint32_t (&w)[4]) { *reinterpret_cast<uint4 *>(p) = make_uint4(w[0], w[1], w[2], w[3]); }

__device__ __forceinline__ bool z_bad16(const double (&y)[16]) {
    bool bad = false;
#pragma unroll
    for(int j = 0; j < 16; j++) bad |= !(fabs(y[j]) <= 64.0);  // NaN, inf or beyond the row scale
    return bad;
}

// Writes the ns digit planes of a 16-column group g of source row r (yr, yi already scaled by 64 / sigma_r).
template<bool CPLX, bool BMODE>
__device__ __forceinline__ void z_emit(double (&yr)[16], double (&yi)[16], int8_t *planes, int64_t plane, int64_t kx, int64_t Kh, int64_t r,
                                       int64_t g, int ns, int *bad) {
    if(z_bad16(yr) || (CPLX && z_bad16(yi))) atomicExch(bad, 1);
    for(int t = 0; t < ns; t++) {
        uint32_t wr[4], wnr[4], wi[4], wni[4];
        z_digits16(yr, wr, wnr);
        int8_t *base = planes + t * plane;
        if constexpr(!CPLX) {
            z_st16(base + r * kx + g * 16, wr);
        } else {
            z_digits16(yi, wi, wni);
            if constexpr(!BMODE) {  // [re | im]
                z_st16(base + r * kx + g * 16, wr);
                z_st16(base + r * kx + Kh + g * 16, wi);
            } else {  // 2r: [re | -im], 2r + 1: [im | re]
                z_st16(base + (2 * r) * kx + g * 16, wr);
                z_st16(base + (2 * r) * kx + Kh + g * 16, wni);
                z_st16(base + (2 * r + 1) * kx + g * 16, wi);
                z_st16(base + (2 * r + 1) * kx + Kh + g * 16, wr);
            }
        }
    }
}

// K-major source: thread per (row, 16-column group), groups of a row on consecutive threads
template<bool CPLX, bool BMODE>
__global__ void __launch_bounds__(256) z_slice_k_kernel(const typename Scalar<CPLX>::T *__restrict__ src, int64_t rows, int64_t K, int64_t ld,
                                                         const double *__restrict__ inv, int8_t *__restrict__ planes, int64_t prow, int64_t kx, int ns,
                                                         int *bad) {
    const int64_t ng = (K + 15) / 16, Kh = ng * 16, tot = rows * ng, plane = prow * kx;
    for(int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < tot; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t g = e % ng, r = e / ng;
        const double  sc = inv[r];
        double        yr[16], yi[16];
        const auto   *row = src + r * ld + g * 16;
#pragma unroll
        for(int j = 0; j < 16; j++) {
            yr[j] = yi[j] = 0.0;
            if(g * 16 + j < K) {
                const auto v = row[j];
                yr[j]        = z_re(v) * sc;
                yi[j]        = z_im(v) * sc;
            }
        }
        z_emit<CPLX, BMODE>(yr, yi, planes, plane, kx, Kh, r, g, ns, bad);
    }
}

// M-major source src[r + ld k]: one CTA per tile of 32 rows x 64 columns, read along the rows (coalesced) into
// shared memory, then one thread per (row, 16-column group) emits the digits, so a warp writes 64 contiguous
// bytes per row and plane.
constexpr int ZM_TR = 32, ZM_TK = 64, ZM_THREADS = ZM_TR * ZM_TK / 16;
template<bool CPLX>
__global__ void __launch_bounds__(ZM_THREADS) z_slice_m_kernel(const typename Scalar<CPLX>::T *__restrict__ src, int64_t rows, int64_t K,
                                                                int64_t ld, const double *__restrict__ inv, int8_t *__restrict__ planes, int64_t kx,
                                                                int ns, int *bad) {
    using T = typename Scalar<CPLX>::T;
    __shared__ T  tile[ZM_TK][ZM_TR + 1];
    const int64_t ng = (K + 15) / 16, Kh = ng * 16, plane = rows * kx;
    const int64_t r0 = (int64_t)blockIdx.x * ZM_TR, k0 = (int64_t)blockIdx.y * ZM_TK;
    for(int idx = threadIdx.x; idx < ZM_TR * ZM_TK; idx += ZM_THREADS) {
        const int     rl = idx % ZM_TR, kl = idx / ZM_TR;
        const int64_t r = r0 + rl, k = k0 + kl;
        T             v;
        if constexpr(CPLX)
            v = make_double2(0.0, 0.0);
        else
            v = 0.0;
        if(r < rows && k < K) v = src[r + ld * k];
        tile[kl][rl] = v;
    }
    __syncthreads();
    const int     rl = threadIdx.x / (ZM_TK / 16), gl = threadIdx.x % (ZM_TK / 16);
    const int64_t r = r0 + rl, g = k0 / 16 + gl;
    if(r >= rows || g >= ng) return;
    const double sc = inv[r];
    double       yr[16], yi[16];
#pragma unroll
    for(int j = 0; j < 16; j++) {
        const T v = tile[16 * gl + j][rl];
        yr[j]     = z_re(v) * sc;
        yi[j]     = z_im(v) * sc;
    }
    z_emit<CPLX, false>(yr, yi, planes, plane, kx, Kh, r, g, ns, bad);
}

static int z_grid(int64_t n, int per_block = 256) {
    const int64_t g = (n + per_block - 1) / per_block, cap = (int64_t)device_sm_count() * 16;
    return (int)(g < 1 ? 1 : (g < cap ? g : cap));
}

template<bool CPLX>
int z_scale_kmajor(const typename Scalar<CPLX>::T *src, int64_t rows, int64_t K, int64_t ld, double extra, ZPlanes &p, int *bad, cudaStream_t s) {
    if(rows <= 0) return HEFF_OK;
    z_scale_k_kernel<CPLX><<<z_grid(rows * 32), 256, 0, s>>>(src, rows, K, ld, extra, p.inv, p.fac, bad);
    HEFF_LAUNCH_CHECK();
    return HEFF_OK;
}

template<bool CPLX>
int z_scale_mmajor(const typename Scalar<CPLX>::T *src, int64_t rows, int64_t K, int64_t ld, double extra, ZPlanes &p, int *bad, cudaStream_t s) {
    if(rows <= 0) return HEFF_OK;
    const int64_t rb      = cdiv(rows, 256);
    const int64_t nchunks = std::max<int64_t>(1, std::min<int64_t>(std::min<int64_t>(K, 65535), (int64_t)device_sm_count() * 8 / rb));
    const int64_t kchunk  = cdiv(K, nchunks);
    if(rb > 0x7fffffff) return HEFF_BAD_SHAPE;
    z_rowmax_m_kernel<CPLX><<<dim3((unsigned)rb, (unsigned)cdiv(K, kchunk)), 256, 0, s>>>(src, rows, K, ld, kchunk, p.rmax);
    HEFF_LAUNCH_CHECK();
    z_rowmax_fin_kernel<<<z_grid(rows), 256, 0, s>>>(p.rmax, rows, extra, p.inv, p.fac, bad);
    HEFF_LAUNCH_CHECK();
    return HEFF_OK;
}

template<bool CPLX>
int z_slice_kmajor(const typename Scalar<CPLX>::T *src, int64_t rows, int64_t K, int64_t ld, bool bmode, const ZPlanes &p, int *bad, cudaStream_t s) {
    if(rows <= 0) return HEFF_OK;
    const int64_t tot = rows * cdiv(K, 16);
    if(CPLX && bmode)
        z_slice_k_kernel<CPLX, true><<<z_grid(tot), 256, 0, s>>>(src, rows, K, ld, p.inv, p.planes, p.rows, p.kx, p.nslice, bad);
    else
        z_slice_k_kernel<CPLX, false><<<z_grid(tot), 256, 0, s>>>(src, rows, K, ld, p.inv, p.planes, p.rows, p.kx, p.nslice, bad);
    HEFF_LAUNCH_CHECK();
    return HEFF_OK;
}

template<bool CPLX>
int z_slice_mmajor(const typename Scalar<CPLX>::T *src, int64_t rows, int64_t K, int64_t ld, const ZPlanes &p, int *bad, cudaStream_t s) {
    if(rows <= 0) return HEFF_OK;
    const int64_t gx = cdiv(rows, ZM_TR), gy = cdiv(K, ZM_TK);
    if(gx > 0x7fffffff || gy > 65535) return HEFF_BAD_SHAPE;
    z_slice_m_kernel<CPLX><<<dim3((unsigned)gx, (unsigned)gy), ZM_THREADS, 0, s>>>(src, rows, K, ld, p.inv, p.planes, p.kx, p.nslice, bad);
    HEFF_LAUNCH_CHECK();
    return HEFF_OK;
}

template int z_scale_kmajor<false>(const double *, int64_t, int64_t, int64_t, double, ZPlanes &, int *, cudaStream_t);
template int z_scale_kmajor<true>(const double2 *, int64_t, int64_t, int64_t, double, ZPlanes &, int *, cudaStream_t);
template int z_scale_mmajor<false>(const double *, int64_t, int64_t, int64_t, double, ZPlanes &, int *, cudaStream_t);
template int z_scale_mmajor<true>(const double2 *, int64_t, int64_t, int64_t, double, ZPlanes &, int *, cudaStream_t);
template int z_slice_kmajor<false>(const double *, int64_t, int64_t, int64_t, bool, const ZPlanes &, int *, cudaStream_t);
template int z_slice_kmajor<true>(const double2 *, int64_t, int64_t, int64_t, bool, const ZPlanes &, int *, cudaStream_t);
template int z_slice_mmajor<false>(const double *, int64_t, int64_t, int64_t, const ZPlanes &, int *, cudaStream_t);
template int z_slice_mmajor<true>(const double2 *, int64_t, int64_t, int64_t, const ZPlanes &, int *, cudaStream_t);

// ---------------------------------------------------------------------------------------------------------
// tcgen05 kind::i8 GEMM over (tile, level) units
// ---------------------------------------------------------------------------------------------------------

// kind::i8 instruction descriptor: D = S32, A = B = signed 8-bit, both K-major, M = 128, N = BN
template<int BN>
constexpr uint32_t z_idesc() {
    return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(Z_BM >> 4) << 24);
}

template<int BN>
__device__ __forceinline__ void umma_i8(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(z_idesc<BN>()), "r"(accumulate)
        : "memory");
}

constexpr int Z_GROUP_M = 8;

template<int BN>
__device__ __forceinline__ void z_tile_mn(const ZGemmArgs &p, int tile, int &m0, int &n0) {
    const int num_m = (p.M + Z_BM - 1) / Z_BM, num_n = (p.N + BN - 1) / BN;
    const int per_group = Z_GROUP_M * num_n;
    const int first_m   = (tile / per_group) * Z_GROUP_M;
    const int gsize     = min(num_m - first_m, Z_GROUP_M);
    m0                  = (first_m + (tile % per_group) % gsize) * Z_BM;
    n0                  = ((tile % per_group) / gsize) * BN;
}

// Level g of tile (m0, n0) from TMEM columns [col0, col0 + BN) into C: the first level processed (g = s-1)
// stores, the others add.  All loads of a 32-column chunk are issued before its stores.
__device__ __forceinline__ double z_nan() { return __longlong_as_double(0x7ff8000000000000ll); }

template<int BN>
__device__ __forceinline__ void z_epilogue(const ZGemmArgs &p, uint32_t tmem_row, int row, int n0, int g, bool poison) {
    const bool first = g == p.nslice - 1;
    double     lv    = 1.0;
    for(int i = 0; i < g; i++) lv *= 0.0078125;  // 2^-7g, exact
    const double ra = row < p.M ? (poison ? z_nan() : p.fa[row] * lv) : 0.0;
    for(int c = 0; c < BN; c += 32) {
        uint32_t r[32];
        tmem_ld32(tmem_row + (uint32_t)c, r);
        if(row >= p.M) continue;
        if(!p.cplx) {
            double *C = reinterpret_cast<double *>(p.C) + row;
#pragma unroll
            for(int h = 0; h < 32; h += 16) {
                double old[16], f[16];
#pragma unroll
                for(int jj = 0; jj < 16; jj++) {
                    const int n = n0 + c + h + jj;
                    f[jj] = old[jj] = 0.0;
                    if(n < p.N) {
                        f[jj] = __ldg(p.fb + n);
                        if(!first) old[jj] = C[p.ldc * n];
                    }
                }
#pragma unroll
                for(int jj = 0; jj < 16; jj++) {
                    const int n = n0 + c + h + jj;
                    if(n < p.N) C[p.ldc * n] = old[jj] + (double)(int)r[h + jj] * (ra * f[jj]);  // the product is exact
                }
            }
        } else {
            double2 *C = reinterpret_cast<double2 *>(p.C) + row;
            double2  old[16];
            double   f[16];
#pragma unroll
            for(int jj = 0; jj < 16; jj++) {
                const int n = n0 + c + 2 * jj;  // even; n + 1 < N whenever n < N
                f[jj] = 0.0, old[jj] = make_double2(0.0, 0.0);
                if(n < p.N) {
                    f[jj] = __ldg(p.fb + (n >> 1));
                    if(!first) old[jj] = C[p.ldc * (n >> 1)];
                }
            }
#pragma unroll
            for(int jj = 0; jj < 16; jj++) {
                const int n = n0 + c + 2 * jj;
                if(n < p.N) {
                    const double s = ra * f[jj];
                    C[p.ldc * (n >> 1)] = make_double2(old[jj].x + (double)(int)r[2 * jj] * s, old[jj].y + (double)(int)r[2 * jj + 1] * s);
                }
            }
        }
    }
}

// Level g of tile (m0, n0) with the FP64 sum over levels kept in TMEM (TMEM_SUM tiles): INT32 accumulator at
// tacc, FP64 partial at tpart (column pairs lo, hi); the same FP64 operations in the same order as z_epilogue,
// so both give identical results.  The last level (g = 0) writes C once.
template<int BN>
__device__ __forceinline__ void z_epilogue_tsum(const ZGemmArgs &p, uint32_t tacc, uint32_t tpart, int row, int n0, int g, bool poison) {
    const bool first = g == p.nslice - 1, last = g == 0;
    double     lv    = 1.0;
    for(int i = 0; i < g; i++) lv *= 0.0078125;  // 2^-7g, exact
    const double ra = row < p.M ? (poison ? z_nan() : p.fa[row] * lv) : 0.0;
    for(int c = 0; c < BN; c += 32) {
        uint32_t r[32];
        tmem_ld32(tacc + (uint32_t)c, r);
#pragma unroll
        for(int h = 0; h < 32; h += 16) {  // 16 columns = 32 partial words per pass
            double   v[16];
            uint32_t w[32];
            if(!first) tmem_ld32(tpart + (uint32_t)(2 * (c + h)), w);
#pragma unroll
            for(int jj = 0; jj < 16; jj++) {
                const int    n  = n0 + c + h + jj;
                const int    nb = p.cplx ? (n >> 1) : n;
                const double f  = n < p.N ? __ldg(p.fb + nb) : 0.0;
                const double x  = (double)(int)r[h + jj] * (ra * f);  // exact
                v[jj]           = first ? x : __hiloint2double((int)w[2 * jj + 1], (int)w[2 * jj]) + x;
            }
            if(!last) {
#pragma unroll
                for(int jj = 0; jj < 16; jj++) {
                    w[2 * jj]     = (uint32_t)__double2loint(v[jj]);
                    w[2 * jj + 1] = (uint32_t)__double2hiint(v[jj]);
                }
                tmem_st32(tpart + (uint32_t)(2 * (c + h)), w);
            } else if(row < p.M) {
                if(!p.cplx) {
                    double *C = reinterpret_cast<double *>(p.C) + row;
#pragma unroll
                    for(int jj = 0; jj < 16; jj++) {
                        const int n = n0 + c + h + jj;
                        if(n < p.N) C[p.ldc * n] = v[jj];
                    }
                } else {
                    double2 *C = reinterpret_cast<double2 *>(p.C) + row;
#pragma unroll
                    for(int jj = 0; jj < 16; jj += 2) {
                        const int n = n0 + c + h + jj;
                        if(n < p.N) C[p.ldc * (n >> 1)] = make_double2(v[jj], v[jj + 1]);
                    }
                }
            }
        }
    }
    if(!last) tmem_wait_st();
}

// Persistent CTA (one per SM) over units (tile t, level g), t = blockIdx.x, blockIdx.x + gridDim.x, ...,
// g = s-1 .. 0; unit j of the CTA accumulates in TMEM buffer (j & 1).
//   warp 0 lane 0: TMA producer: unit (t, g) streams k-blocks of slice pairs (i, g - i), i = 0..g
//   warp 1 lane 0: MMA issuer
//   warps 2-5:     epilogue of unit j while the MMAs of unit j+1 run in the other buffer
template<int BN>
__global__ void __launch_bounds__(Z_THREADS, 1)
    gemm_i8_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, const ZGemmArgs p) {
    extern __shared__ __align__(1024) unsigned char zsm_raw[];
    unsigned char *smem = reinterpret_cast<unsigned char *>((reinterpret_cast<uintptr_t>(zsm_raw) + 1023) & ~uintptr_t(1023));
    using Cfg                = ZCfg<BN>;
    uint64_t      *full      = reinterpret_cast<uint64_t *>(smem + Cfg::STAGES * Cfg::STAGE);
    uint64_t      *empty     = full + Cfg::STAGES;
    uint64_t      *acc_full  = empty + Cfg::STAGES;  // [2]
    uint64_t      *acc_empty = acc_full + 2;      // [2]
    uint32_t      *tmem_slot = reinterpret_cast<uint32_t *>(acc_empty + 2);
    int           *s_fail    = reinterpret_cast<int *>(tmem_slot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ntiles = ((p.M + Z_BM - 1) / Z_BM) * ((p.N + BN - 1) / BN);
    const int KBs    = (p.K + Z_BK - 1) / Z_BK;  // k-blocks per slice
    const int ns     = p.nslice;

    if(threadIdx.x == 0) {
        for(int s = 0; s < Cfg::STAGES; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for(int b = 0; b < 2; b++) {
            mbar_init(&acc_full[b], 1);
            mbar_init(&acc_empty[b], 128);
        }
        *s_fail = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if(warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(saddr(tmem_slot)), "r"(Cfg::TMEM_COLS) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem_base = *tmem_slot;

    if(warp == 0) {
        if(lane == 0) {  // TMA producer
            int  it = 0;
            bool ok = true;
            for(int t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
                int m0, n0;
                z_tile_mn<BN>(p, t, m0, n0);
                for(int g = ns - 1; g >= 0 && ok; g--) {
                    const int nkb = (g + 1) * KBs;
                    for(int kb = 0; kb < nkb; kb++, it++) {
                        const int      st = it % Cfg::STAGES;
                        const uint32_t ph = (it / Cfg::STAGES) & 1;
                        if(!mbar_wait(&empty[st], ph ^ 1)) {
                            atomicExch(p.err, 1);
                            ok = false;
                            break;
                        }
                        const int      i  = kb / KBs;  // A slice i, B slice g - i
                        const int      k0 = (kb - i * KBs) * Z_BK;
                        unsigned char *a = smem + st * Cfg::STAGE, *b = a + Z_A_BYTES;
                        mbar_expect_tx(&full[st], Cfg::STAGE);
                        tma_load_3d(&tmA, &full[st], a, k0, m0, i);
                        tma_load_3d(&tmB, &full[st], b, k0, n0, g - i);
                    }
                }
            }
        }
    } else if(warp == 1) {
        if(lane == 0) {  // MMA issuer
            int  it = 0, j = 0;
            bool ok = true;
            for(int t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
                for(int g = ns - 1; g >= 0 && ok; g--, j++) {
                    const int      buf = j & 1;
                    const uint32_t acc = tmem_base + (uint32_t)(buf * BN);
                    if(!mbar_wait(&acc_empty[buf], ((j >> 1) & 1) ^ 1)) {  // the epilogue drained this buffer
                        atomicExch(p.err, 4);
                        ok = false;
                        break;
                    }
                    fence_after();
                    const int nkb = (g + 1) * KBs;
                    for(int kb = 0; kb < nkb; kb++, it++) {
                        const int      st = it % Cfg::STAGES;
                        const uint32_t ph = (it / Cfg::STAGES) & 1;
                        if(!mbar_wait(&full[st], ph)) {
                            atomicExch(p.err, 2);
                            ok = false;
                            break;
                        }
                        fence_after();
                        const uint32_t a = saddr(smem + st * Cfg::STAGE), b = a + Z_A_BYTES;
#pragma unroll
                        for(int k = 0; k < Z_BK / 32; k++) umma_i8<BN>(acc, sdesc_sw128(a + 32 * k), sdesc_sw128(b + 32 * k), (kb | k) != 0);
                        umma_commit(&empty[st]);
                    }
                    if(ok) umma_commit(&acc_full[buf]);  // fires when every MMA of this unit has completed
                }
            }
        }
    } else {
        // epilogue: warps 2..5 -> TMEM lane quarters 2,3,0,1
        const int  q      = warp & 3;
        int        j      = 0;
        bool       stop   = false;
        const bool poison = (*p.bad_a | *p.bad_b) != 0;  // raised by the slicers, which ran before this kernel
        if(poison && threadIdx.x == 64) atomicExch(p.err, 5);
        for(int t = blockIdx.x; t < ntiles && !stop; t += gridDim.x) {
            int m0, n0;
            z_tile_mn<BN>(p, t, m0, n0);
            for(int g = ns - 1; g >= 0; g--, j++) {
                const int buf = j & 1;
                if(!mbar_wait(&acc_full[buf], (j >> 1) & 1)) {
                    atomicExch(p.err, 3);
                    atomicOr(s_fail, 1);
                }
                epi_bar();  // every epilogue warp takes the same decision
                if(*s_fail) {
                    stop = true;
                    break;
                }
                fence_after();
                const uint32_t trow = tmem_base + ((uint32_t)(q * 32) << 16);
                if constexpr(ZCfg<BN>::TMEM_SUM)
                    z_epilogue_tsum<BN>(p, trow + (uint32_t)(buf * BN), trow + (uint32_t)ZCfg<BN>::PART_COL, m0 + q * 32 + lane, n0, g, poison);
                else
                    z_epilogue<BN>(p, trow + (uint32_t)(buf * BN), m0 + q * 32 + lane, n0, g, poison);
                fence_before();
                mbar_arrive(&acc_empty[buf]);  // TMEM buffer free for the unit after next
                epi_bar();                     // *s_fail is read by all before the next wait may set it
            }
        }
    }
    fence_before();
    __syncthreads();
    if(warp == 1) {
        fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base), "r"(Cfg::TMEM_COLS) : "memory");
    }
}

typedef CUresult (*PFN_encodeTiledZ)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *, const cuuint64_t *,
                                     const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle, CUtensorMapL2promotion,
                                     CUtensorMapFloatOOBfill);

static PFN_encodeTiledZ encode_fn_z() {
    static PFN_encodeTiledZ fn = nullptr;
    if(!fn) {
        void                            *q = nullptr;
        cudaDriverEntryPointQueryResult r;
        if(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &q, cudaEnableDefault, &r) == cudaSuccess && r == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_encodeTiledZ>(q);
    }
    return fn;
}

int make_tmap_planes(CUtensorMap *map, const ZPlanes &p, int box_rows) {
    PFN_encodeTiledZ fn = encode_fn_z();
    if(!fn) {
        set_last_error_msg("cuTensorMapEncodeTiled is not available from the driver");
        return HEFF_CUDA_ERROR;
    }
    if(((uintptr_t)p.planes & 15) || p.kx % 16 || p.rows <= 0 || p.nslice <= 0 || p.nslice > Z_MAX_SLICES) return HEFF_BAD_ARG;
    std::memset(map, 0, sizeof(*map));
    cuuint64_t dims[3]    = {(cuuint64_t)p.kx, (cuuint64_t)p.rows, (cuuint64_t)p.nslice};
    cuuint64_t strides[2] = {(cuuint64_t)p.kx, (cuuint64_t)(p.kx * p.rows)};
    cuuint32_t box[3]     = {(cuuint32_t)Z_BK, (cuuint32_t)box_rows, 1};
    cuuint32_t estr[3]    = {1, 1, 1};
    CUresult   r = fn(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, p.planes, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                      CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if(r != CUDA_SUCCESS) {
        set_last_error_msg("cuTensorMapEncodeTiled failed for digit planes (%d)", (int)r);
        return HEFF_CUDA_ERROR;
    }
    return HEFF_OK;
}

// Tile-width override (0 = automatic); initialised from the environment variable HEFF_I8_BN.
static std::atomic<int> g_force_bn{-1};

static int z_forced_bn() {
    int f = g_force_bn.load();
    if(f < 0) {
        const char *e = getenv("HEFF_I8_BN");
        const int   v = e ? atoi(e) : 1;
        int         expect = -1;
        g_force_bn.compare_exchange_strong(expect, (v == 0 || v == 1 || v == 128 || v == 192 || v == 256) ? v : 1);
        f = g_force_bn.load();
    }
    return f;
}

int z_choose_bn(int64_t M, int64_t N, int64_t K) {
    if(const int forced = z_forced_bn(); forced >= 128) return forced;
    // cost = waves x width x per-MAC weight.  The weights are measured (B200, 7 slices, the matvec GEMMs of
    // chi=1024, real and complex): with few k-blocks per slice the levels are short and summing them in C
    // costs more than the 128-wide tile's extra operand traffic; with long K the widest tile is best.
    const int64_t sms  = device_sm_count();
    const int64_t kbs  = cdiv(K, Z_BK);
    const int     bn[3] = {256, 192, 128};
    const double  w[3]  = {1.0, kbs <= 16 ? 0.95 : 1.06, kbs <= 8 ? 0.85 : 1.3};
    int           best = 256;
    double        bc   = 1e300;
    for(int i = 0; i < 3; i++) {
        const int64_t tiles = cdiv(M, Z_BM) * cdiv(N, bn[i]);
        const double  c     = (double)cdiv(tiles, sms) * bn[i] * w[i];
        if(c < bc * 0.999) bc = c, best = bn[i];
    }
    return best;
}

template<int BN>
static int z_launch(const CUtensorMap &tA, const CUtensorMap &tB, const ZGemmArgs &a, cudaStream_t s) {
    static int attr_done[64] = {0};
    int        dev           = 0;
    HEFF_CUDA(cudaGetDevice(&dev));
    if(dev < 0 || dev >= 64 || !attr_done[dev]) {
        HEFF_CUDA(cudaFuncSetAttribute(gemm_i8_kernel<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, ZCfg<BN>::SMEM));
        if(dev >= 0 && dev < 64) attr_done[dev] = 1;
    }
    const int64_t tiles = cdiv(a.M, Z_BM) * cdiv(a.N, BN);
    if(tiles > 0x7fffffff) return HEFF_BAD_SHAPE;
    const int grid = (int)std::min<int64_t>(tiles, device_sm_count());
    gemm_i8_kernel<BN><<<(unsigned)grid, Z_THREADS, ZCfg<BN>::SMEM, s>>>(tA, tB, a);
    HEFF_LAUNCH_CHECK();
    return HEFF_OK;
}

static int z_launch_bn(int bn, const ZPlanes &A, const ZPlanes &B, const ZGemmArgs &a, cudaStream_t s) {
    CUtensorMap tA, tB;
    HEFF_TRY(make_tmap_planes(&tA, A, Z_BM));
    HEFF_TRY(make_tmap_planes(&tB, B, bn));
    if(bn == 256) return z_launch<256>(tA, tB, a, s);
    if(bn == 192) return z_launch<192>(tA, tB, a, s);
    return z_launch<128>(tA, tB, a, s);
}

// Autotuned tile width (the default, heff_i8_set_tile_width(1)): the first GEMM of each shape (device, M, N, K,
// slices) runs once with the model's width to warm up, then once with each width under CUDA events on its own
// stream; the fastest width is cached for the shape.  Every width sums the same exact level products in the same
// order, so the extra runs rewrite C with identical bytes and the choice never changes a result.
struct ZTuneKey {
    int     dev, ns;
    int64_t M, N, K;
    bool    operator<(const ZTuneKey &o) const { return std::tie(dev, ns, M, N, K) < std::tie(o.dev, o.ns, o.M, o.N, o.K); }
};
static std::mutex                  g_tune_mu;
static std::map<ZTuneKey, int>     g_tune;

static int z_tuned_bn(const ZPlanes &A, const ZPlanes &B, const ZGemmArgs &a, cudaStream_t s, int *bn_out) {
    int dev = 0;
    HEFF_CUDA(cudaGetDevice(&dev));
    const ZTuneKey key{dev, a.nslice, a.M, a.N, a.K};
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        auto                        it = g_tune.find(key);
        if(it != g_tune.end()) {
            *bn_out = it->second;
            return HEFF_OK;
        }
    }
    const int   cand[3] = {128, 192, 256};
    cudaEvent_t ev[4];
    for(auto &e : ev) HEFF_CUDA(cudaEventCreate(&e));
    int rc = z_launch_bn(z_choose_bn(a.M, a.N, a.K), A, B, a, s);  // warm-up (attributes, caches)
    for(int i = 0; i < 3 && rc == HEFF_OK; i++) {
        if(cudaEventRecord(ev[i], s) != cudaSuccess) rc = HEFF_CUDA_ERROR;
        if(rc == HEFF_OK) rc = z_launch_bn(cand[i], A, B, a, s);
    }
    if(rc == HEFF_OK && cudaEventRecord(ev[3], s) != cudaSuccess) rc = HEFF_CUDA_ERROR;
    if(rc == HEFF_OK && cudaEventSynchronize(ev[3]) != cudaSuccess) rc = HEFF_CUDA_ERROR;
    int best = z_choose_bn(a.M, a.N, a.K);
    if(rc == HEFF_OK) {
        float bt = 0;
        for(int i = 0; i < 3; i++) {
            float ms = 0;
            if(cudaEventElapsedTime(&ms, ev[i], ev[i + 1]) != cudaSuccess) continue;
            if(i == 0 || ms < bt) bt = ms, best = cand[i];
        }
    }
    for(auto &e : ev) cudaEventDestroy(e);
    HEFF_TRY(rc);
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        g_tune[key] = best;
    }
    *bn_out = best;
    return HEFF_OK;
}

int gemm_i8_ozaki(const ZPlanes &A, const ZPlanes &B, const ZGemmArgs &a, cudaStream_t s) {
    if(a.M <= 0 || a.N <= 0) return HEFF_OK;
    if(a.K <= 0 || a.K % 16 || a.nslice < 1 || a.nslice > Z_MAX_SLICES || !z_k_ok(a.K, a.nslice) || (a.cplx && a.N % 2)) return HEFF_BAD_ARG;
    if(A.kx != a.K || B.kx != a.K || A.rows < a.M || B.rows < a.N || A.nslice < a.nslice || B.nslice < a.nslice) return HEFF_BAD_ARG;
    if(!a.err || !a.bad_a || !a.bad_b) return HEFF_BAD_ARG;
    int bn = 0;
    if(z_forced_bn() == 1)
        HEFF_TRY(z_tuned_bn(A, B, a, s, &bn));
    else
        bn = z_choose_bn(a.M, a.N, a.K);
    return z_launch_bn(bn, A, B, a, s);
}

int z_tuned_count() {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    return (int)g_tune.size();
}

// ---------------------------------------------------------------------------------------------------------
// Standalone entry point: C = A B^T from FP64 / complex operands
// ---------------------------------------------------------------------------------------------------------

template<bool CPLX>
static int gemm_emu_impl(const void *Av, const void *Bv, void *C, int64_t M, int64_t N, int64_t K, int ns, cudaStream_t s) {
    using T             = typename Scalar<CPLX>::T;
    const int     cf    = CPLX ? 2 : 1;
    const int64_t kx    = z_kx(K, CPLX);
    if(!z_k_ok(kx, ns)) {
        set_last_error_msg("heff_gemm_i8_emu: K = %lld too large for exact INT32 level sums with %d slices", (long long)K, ns);
        return HEFF_BAD_SHAPE;
    }
    if(M > 0x7fffffff || cf * N > 0x7fffffff) return HEFF_BAD_SHAPE;
    auto          up    = [](size_t b) { return (b + 255) / 256 * 256; };
    const size_t  bPA   = up((size_t)ns * M * kx), bPB = up((size_t)ns * cf * N * kx);
    const size_t  bS    = up(sizeof(double) * (size_t)(2 * M + 2 * N)), bE = 256;
    unsigned char *w    = nullptr;
    HEFF_TRY(stream_workspace(s, bPA + bPB + bS + bE, reinterpret_cast<void **>(&w)));
    ZPlanes pa, pb;
    pa.planes = reinterpret_cast<int8_t *>(w), pa.rows = M, pa.kx = kx, pa.nslice = ns;
    pb.planes = reinterpret_cast<int8_t *>(w + bPA), pb.rows = cf * N, pb.kx = kx, pb.nslice = ns;
    double *sc = reinterpret_cast<double *>(w + bPA + bPB);
    pa.inv = sc, pa.fac = sc + M, pb.inv = sc + 2 * M, pb.fac = sc + 2 * M + N;
    int *err = reinterpret_cast<int *>(w + bPA + bPB + bS);  // err, bad word of A, bad word of B
    HEFF_CUDA(cudaMemsetAsync(err, 0, 3 * sizeof(int), s));
    const T *A = reinterpret_cast<const T *>(Av), *B = reinterpret_cast<const T *>(Bv);
    HEFF_TRY(z_scale_kmajor<CPLX>(A, M, K, K, 1.0 / 4096.0, pa, err + 1, s));
    HEFF_TRY(z_scale_kmajor<CPLX>(B, N, K, K, 1.0, pb, err + 2, s));
    HEFF_TRY(z_slice_kmajor<CPLX>(A, M, K, K, false, pa, err + 1, s));
    HEFF_TRY(z_slice_kmajor<CPLX>(B, N, K, K, true, pb, err + 2, s));
    ZGemmArgs g{};
    g.M = (int)M, g.N = (int)(cf * N), g.K = (int)kx, g.nslice = ns, g.fa = pa.fac, g.fb = pb.fac, g.C = C, g.ldc = M, g.cplx = CPLX, g.err = err;
    g.bad_a = err + 1, g.bad_b = err + 2;
    HEFF_TRY(gemm_i8_ozaki(pa, pb, g, s));
    int h = 0;
    HEFF_CUDA(cudaMemcpyAsync(&h, err, sizeof(int), cudaMemcpyDeviceToHost, s));
    HEFF_CUDA(cudaStreamSynchronize(s));
    if(h == 5) {
        set_last_error_msg("heff_gemm_i8_emu: non-finite input or an entry of magnitude >= 2^1022");
        return HEFF_NAN_INPUT;
    }
    if(h) {
        set_last_error_msg("heff_gemm_i8_emu: pipeline wait timed out (code %d)", h);
        return HEFF_TIMEOUT;
    }
    return HEFF_OK;
}

}  // namespace heff

using namespace heff;

extern "C" int heff_gemm_i8_emu(int dtype, const void *A, const void *B, void *C, int64_t M, int64_t N, int64_t K, int nslices, void *stream) {
    if(!A || !B || !C || M <= 0 || N <= 0 || K <= 0) return HEFF_BAD_ARG;
    if(nslices == 0) nslices = Z_DEFAULT_SLICES;
    if(nslices < 1 || nslices > Z_MAX_SLICES) return HEFF_BAD_ARG;
    if(dtype == HEFF_F64) return gemm_emu_impl<false>(A, B, C, M, N, K, nslices, (cudaStream_t)stream);
    if(dtype == HEFF_C128) return gemm_emu_impl<true>(A, B, C, M, N, K, nslices, (cudaStream_t)stream);
    return HEFF_BAD_ARG;
}

extern "C" int heff_i8_tuned_shapes(void) { return heff::z_tuned_count(); }

extern "C" int heff_i8_set_tile_width(int bn) {
    if(bn != 0 && bn != 1 && bn != 128 && bn != 192 && bn != 256) return -1;
    const int prev = z_forced_bn();
    g_force_bn.store(bn);
    return prev;
}
