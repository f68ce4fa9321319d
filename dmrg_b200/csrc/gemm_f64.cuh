// FP64 / complex128 batched GEMM on the sm_100a FP64 tensor pipe (DMMA, mma.sync.m16n8k4.f64).
//
// tcgen05.mma has no f64 kind, so the FP64 tensor path on Blackwell is the warp-level DMMA
// instruction.  Operands are staged global -> shared through a multistage cp.async pipeline
// (16-byte copies where the layout allows, zero-fill at the edges), fragments are read from
// padded shared tiles whose leading dimensions make every fragment load bank-conflict free.
//
//   C[b] = alpha * op(A[b]) * op(B[b]) + beta * C[b]      (column-major, BLAS conventions)
//   op(A) = A (M x K, m contiguous)   or  A^T (A stored K x M, k contiguous)   [TA]
//   op(B) = B (K x N, k contiguous)   or  B^T (B stored N x K, n contiguous)   [TB]
//   complex: 3 real DMMAs per fragment pair (3M / Gauss): t1 = ar br, t2 = ai bi, t3 = (ar + ai)(br + bi)
//   accumulated over K, then Re = t1 - t2, Im = t3 - t1 - t2 (normwise error a small constant times the 4M
//   product's, eps sqrt(K) |A| |B|); optional conjugation of A (CJA).  Measured on the matvec's GEMMs
//   (chi=1024): 3.21 ms with 4 DMMAs, 2.69 ms with 3, 2.63 ms with 3 and BK = 32.
#pragma once
#include "heff_common.cuh"

namespace heff {

struct GemmArgs {
    int         M, N, K, batch;
    const void *A;
    int64_t     lda, sA;
    const void *B;
    int64_t     ldb, sB;
    void       *C;
    int64_t     ldc, sC;
    double2     alpha, beta;  // real GEMMs use .x
    // Optional scratch for the tail split (set by the caller; nullptr or too small: no split).  When the
    // tiles do not fill whole waves of the device, the tiles of the last partial wave are split along K
    // into `split` pieces that write partial tiles to `part`; a second kernel sums the pieces in piece
    // order (deterministic) and applies alpha/beta.  Set by the launcher: split, nfull, part.
    void       *split_ws;
    size_t      split_ws_bytes;
    int         split, nfull;
    void       *part;
};

template<bool CPLX>
struct GemmTile;
template<>
struct GemmTile<false> {
    static constexpr int BM = 128, BN = 128, BK = 32, WM = 64, WN = 32, STAGES = 3;  // 212 KB of stages: one barrier per 8 k-steps
    static constexpr int PAD_MN = 4;  // leading dim == 4 (mod 16) doubles: conflict-free 8-byte fragment loads
    static constexpr int PAD_K  = 4;
};
template<>
struct GemmTile<true> {
    static constexpr int BM = 64, BN = 64, BK = 32, WM = 32, WN = 16, STAGES = 3;
    static constexpr int PAD_MN = 2;  // leading dim == 2 (mod 8) elements: conflict-free 16-byte loads, m/n-major tile
    static constexpr int PAD_K  = 4;  // leading dim == 4 (mod 8) elements: conflict-free 16-byte loads, k-major tile
};

template<bool CPLX, bool TA, bool TB>
struct GemmSmem {
    using G                  = GemmTile<CPLX>;
    using T                  = typename Scalar<CPLX>::T;
    static constexpr int LDA = TA ? (G::BK + G::PAD_K) : (G::BM + G::PAD_MN);  // row length of the A tile
    static constexpr int LDB = TB ? (G::BN + G::PAD_MN) : (G::BK + G::PAD_K);
    static constexpr int A_ELEMS = TA ? G::BM * LDA : G::BK * LDA;
    static constexpr int B_ELEMS = TB ? G::BK * LDB : G::BN * LDB;
    static constexpr int STAGE   = A_ELEMS + B_ELEMS;
    static constexpr size_t BYTES = (size_t)STAGE * G::STAGES * sizeof(T);
};

constexpr int GROUP_M = 16;  // row panels per rasterisation group

// Grouped rasterisation: consecutive tile ids walk GROUP_M row panels for every column panel, so the
// CTAs resident at one time share their A and B panels in L2 instead of re-reading them from HBM.
template<int BM, int BN>
__device__ __forceinline__ void gemm_raster(int pid, int M, int N, int &tile_m, int &tile_n) {
    const int num_m = (M + BM - 1) / BM, num_n = (N + BN - 1) / BN;
    const int per_group = GROUP_M * num_n;
    const int first_m   = (pid / per_group) * GROUP_M;
    const int gsize     = min(num_m - first_m, GROUP_M);
    tile_m              = first_m + (pid % per_group) % gsize;
    tile_n              = (pid % per_group) / gsize;
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

template<int BYTES>
__device__ __forceinline__ void cp_async(uint32_t dst, const void *src, bool valid) {
    const int n = valid ? BYTES : 0;  // src-size 0 -> destination is zero-filled, nothing is read
    if constexpr(BYTES == 16)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(src), "r"(n));
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(dst), "l"(src), "r"(n));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template<int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

__device__ __forceinline__ void dmma(double (&c)[4], double a0, double a1, double b0) {
    asm volatile("mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};\n"
                 : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
                 : "d"(a0), "d"(a1), "d"(b0));
}

// One 256-thread CTA computes a BM x BN tile of C.  VEC = elements per cp.async (2 doubles or 1).
template<bool CPLX, bool TA, bool TB, bool CJA, int VEC>
__global__ void __launch_bounds__(256, 1) gemm_f64_kernel(const GemmArgs p) {
    using G  = GemmTile<CPLX>;
    using SM = GemmSmem<CPLX, TA, TB>;
    using T  = typename Scalar<CPLX>::T;
    constexpr int BM = G::BM, BN = G::BN, BK = G::BK, WM = G::WM, WN = G::WN, ST = G::STAGES;
    constexpr int MT = WM / 16, NT = WN / 8;  // mma tiles per warp
    constexpr int CPB = CPLX ? 16 : 8 * VEC;  // bytes per copy
    constexpr int EPC = CPLX ? 1 : VEC;       // elements per copy
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *smem = reinterpret_cast<T *>(smem_raw);

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, t = lane & 3;
    const int wm0 = (warp % (BM / WM)) * WM, wn0 = (warp / (BM / WM)) * WN;
    const int M = p.M, N = p.N, K = p.K;
    const int KT = (K + BK - 1) / BK;
    // Tail split: CTAs past the first nfull tiles each take one K-range piece of a tail tile.
    int tile_id = blockIdx.x, kt0 = 0, kt1 = KT, unit = -1;
    if(p.split > 1 && tile_id >= p.nfull) {
        unit            = tile_id - p.nfull;
        const int piece = unit % p.split;
        tile_id         = p.nfull + unit / p.split;
        kt0             = (int)((int64_t)KT * piece / p.split);
        kt1             = (int)((int64_t)KT * (piece + 1) / p.split);
    }
    int tile_m, tile_n;
    gemm_raster<BM, BN>(tile_id, M, N, tile_m, tile_n);
    const int m0 = tile_m * BM, n0 = tile_n * BN;
    const int bz = blockIdx.z;
    const T  *A  = reinterpret_cast<const T *>(p.A) + (int64_t)bz * p.sA;
    const T  *B  = reinterpret_cast<const T *>(p.B) + (int64_t)bz * p.sB;
    T        *C  = reinterpret_cast<T *>(p.C) + (int64_t)bz * p.sC;

    auto load_stage = [&](int stage, int kt) {
        T        *As = smem + stage * SM::STAGE;
        T        *Bs = As + SM::A_ELEMS;
        const int k0 = kt * BK;
        // A tile
        constexpr int A_CHUNKS = BM * BK / EPC;
#pragma unroll
        for(int c = tid; c < A_CHUNKS; c += 256) {
            int mm, kk;
            if constexpr(!TA) {
                kk = c / (BM / EPC);
                mm = (c % (BM / EPC)) * EPC;
            } else {
                mm = c / (BK / EPC);
                kk = (c % (BK / EPC)) * EPC;
            }
            const int  gm = m0 + mm, gk = k0 + kk;
            const bool v  = (gm < M) && (gk < K);
            const T   *src = v ? (TA ? A + gk + (int64_t)gm * p.lda : A + gm + (int64_t)gk * p.lda) : A;
            T         *dst = TA ? As + mm * SM::LDA + kk : As + kk * SM::LDA + mm;
            cp_async<CPB>(smem_u32(dst), src, v);
        }
        constexpr int B_CHUNKS = BN * BK / EPC;
#pragma unroll
        for(int c = tid; c < B_CHUNKS; c += 256) {
            int nn, kk;
            if constexpr(!TB) {
                nn = c / (BK / EPC);
                kk = (c % (BK / EPC)) * EPC;
            } else {
                kk = c / (BN / EPC);
                nn = (c % (BN / EPC)) * EPC;
            }
            const int  gn = n0 + nn, gk = k0 + kk;
            const bool v  = (gn < N) && (gk < K);
            const T   *src = v ? (TB ? B + gn + (int64_t)gk * p.ldb : B + gk + (int64_t)gn * p.ldb) : B;
            T         *dst = TB ? Bs + kk * SM::LDB + nn : Bs + nn * SM::LDB + kk;
            cp_async<CPB>(smem_u32(dst), src, v);
        }
    };

    double acc[MT][NT][CPLX ? 3 : 1][4];  // complex: t1, t2, t3 of the 3M product
#pragma unroll
    for(int i = 0; i < MT; i++)
#pragma unroll
        for(int j = 0; j < NT; j++)
#pragma unroll
            for(int c = 0; c < (CPLX ? 3 : 1); c++)
#pragma unroll
                for(int r = 0; r < 4; r++) acc[i][j][c][r] = 0.0;

#pragma unroll
    for(int s = 0; s < ST - 1; s++) {
        if(kt0 + s < kt1) load_stage(s, kt0 + s);
        cp_async_commit();
    }

    for(int kt = kt0; kt < kt1; kt++) {
        const int it = kt - kt0;  // pipeline slot counter
        cp_async_wait<ST - 2>();
        __syncthreads();
        {
            const int nk = kt + ST - 1;
            if(nk < kt1) load_stage((it + ST - 1) % ST, nk);
            cp_async_commit();
        }
        const T *As = smem + (it % ST) * SM::STAGE;
        const T *Bs = As + SM::A_ELEMS;
#pragma unroll
        for(int k4 = 0; k4 < BK; k4 += 4) {
            T a[MT][2], b[NT];
#pragma unroll
            for(int i = 0; i < MT; i++) {
                const int mr = wm0 + i * 16 + g;
                if constexpr(TA) {
                    a[i][0] = As[mr * SM::LDA + k4 + t];
                    a[i][1] = As[(mr + 8) * SM::LDA + k4 + t];
                } else {
                    a[i][0] = As[(k4 + t) * SM::LDA + mr];
                    a[i][1] = As[(k4 + t) * SM::LDA + mr + 8];
                }
            }
#pragma unroll
            for(int j = 0; j < NT; j++) {
                const int nc = wn0 + j * 8 + g;
                if constexpr(TB)
                    b[j] = Bs[(k4 + t) * SM::LDB + nc];
                else
                    b[j] = Bs[nc * SM::LDB + k4 + t];
            }
#pragma unroll
            for(int i = 0; i < MT; i++)
#pragma unroll
                for(int j = 0; j < NT; j++) {
                    if constexpr(!CPLX) {
                        dmma(acc[i][j][0], a[i][0], a[i][1], b[j]);
                    } else {
                        const double ai0 = CJA ? -a[i][0].y : a[i][0].y, ai1 = CJA ? -a[i][1].y : a[i][1].y;
                        dmma(acc[i][j][0], a[i][0].x, a[i][1].x, b[j].x);                       // t1 += ar br
                        dmma(acc[i][j][1], ai0, ai1, b[j].y);                                   // t2 += ai bi
                        dmma(acc[i][j][2], a[i][0].x + ai0, a[i][1].x + ai1, b[j].x + b[j].y);  // t3 += (ar+ai)(br+bi)
                    }
                }
        }
    }
    cp_async_wait<0>();

    if(unit >= 0) {
        // Tail piece: the raw partial tile, element (i, j, r) of thread tid at [(i NT + j) 4 + r] * 256 + tid
        // (coalesced), summed by gemm_split_reduce_kernel.
        T *P = reinterpret_cast<T *>(p.part) + (size_t)unit * (BM * BN);
#pragma unroll
        for(int i = 0; i < MT; i++)
#pragma unroll
            for(int j = 0; j < NT; j++)
#pragma unroll
                for(int r = 0; r < 4; r++) {
                    const int e = (i * NT + j) * 4 + r;
                    if constexpr(!CPLX) {
                        P[e * 256 + tid] = acc[i][j][0][r];
                    } else {
                        const double t1 = acc[i][j][0][r], t2 = acc[i][j][1][r], t3 = acc[i][j][2][r];
                        P[e * 256 + tid] = make_double2(t1 - t2, t3 - t1 - t2);
                    }
                }
        return;
    }

    // Epilogue: C = alpha*acc + beta*C (C is not read when beta == 0).
    const bool use_beta = (p.beta.x != 0.0) || (p.beta.y != 0.0);
#pragma unroll
    for(int i = 0; i < MT; i++)
#pragma unroll
        for(int j = 0; j < NT; j++)
#pragma unroll
            for(int r = 0; r < 4; r++) {
                const int gm = m0 + wm0 + i * 16 + g + ((r >> 1) << 3);
                const int gn = n0 + wn0 + j * 8 + 2 * t + (r & 1);
                if(gm < M && gn < N) {
                    T *cp = C + gm + (int64_t)gn * p.ldc;
                    if constexpr(!CPLX) {
                        double v = p.alpha.x * acc[i][j][0][r];
                        if(use_beta) v += p.beta.x * (*cp);
                        *cp = v;
                    } else {
                        const double t1 = acc[i][j][0][r], t2 = acc[i][j][1][r], t3 = acc[i][j][2][r];
                        double2      v  = cmul(p.alpha, make_double2(t1 - t2, t3 - t1 - t2));
                        if(use_beta) v = cadd(v, cmul(p.beta, *cp));
                        *cp = v;
                    }
                }
            }
}

// Second pass of the tail split: sums each tail tile's `split` partial pieces in piece order (the same order on
// every run) and writes C = alpha * sum + beta * C with the GEMM kernel's thread mapping.  Grid: (tail tiles,
// EPT / EPB); each thread takes EPB of its tile elements and issues all EPB * split loads before any addition,
// so the pass runs at memory bandwidth instead of one load latency per partial.
constexpr int SPLIT_MAX = 16;
template<bool CPLX>
struct SplitReduce {
    using G                 = GemmTile<CPLX>;
    static constexpr int MT = G::WM / 16, NT = G::WN / 8;
    static constexpr int EPT = MT * NT * 4;   // tile elements per thread
    static constexpr int EPB = CPLX ? 2 : 4;  // elements per thread per CTA of the reduction
};
template<bool CPLX>
__global__ void __launch_bounds__(256) gemm_split_reduce_kernel(const GemmArgs p) {
    using G  = GemmTile<CPLX>;
    using T  = typename Scalar<CPLX>::T;
    using SR = SplitReduce<CPLX>;
    constexpr int BM = G::BM, BN = G::BN, WM = G::WM, WN = G::WN, NT = SR::NT, EPB = SR::EPB;
    const int     tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int     g = lane >> 2, t = lane & 3;
    const int     wm0 = (warp % (BM / WM)) * WM, wn0 = (warp / (BM / WM)) * WN;
    const int     tail = blockIdx.x, e0 = blockIdx.y * EPB;
    int           tile_m, tile_n;
    gemm_raster<BM, BN>(p.nfull + tail, p.M, p.N, tile_m, tile_n);
    const int     m0 = tile_m * BM, n0 = tile_n * BN;
    const T      *P  = reinterpret_cast<const T *>(p.part) + (size_t)tail * p.split * (BM * BN);
    T            *C  = reinterpret_cast<T *>(p.C);
    const bool    use_beta = (p.beta.x != 0.0) || (p.beta.y != 0.0);
    const int     ns = p.split < SPLIT_MAX ? p.split : SPLIT_MAX;
    T             w[EPB][SPLIT_MAX];
#pragma unroll
    for(int q = 0; q < SPLIT_MAX; q++)
#pragma unroll
        for(int u = 0; u < EPB; u++)
            if(q < ns) w[u][q] = P[(size_t)q * (BM * BN) + (e0 + u) * 256 + tid];
#pragma unroll
    for(int u = 0; u < EPB; u++) {
        const int e = e0 + u, r = e & 3, j = (e >> 2) % NT, i = (e >> 2) / NT;
        T         v = w[u][0];
#pragma unroll
        for(int q = 1; q < SPLIT_MAX; q++)
            if(q < ns) {
                if constexpr(!CPLX)
                    v += w[u][q];
                else
                    v = cadd(v, w[u][q]);
            }
        const int gm = m0 + wm0 + i * 16 + g + ((r >> 1) << 3);
        const int gn = n0 + wn0 + j * 8 + 2 * t + (r & 1);
        if(gm < p.M && gn < p.N) {
            T *cp = C + gm + (int64_t)gn * p.ldc;
            if constexpr(!CPLX) {
                double o = p.alpha.x * v;
                if(use_beta) o += p.beta.x * (*cp);
                *cp = o;
            } else {
                double2 o = cmul(p.alpha, v);
                if(use_beta) o = cadd(o, cmul(p.beta, *cp));
                *cp = o;
            }
        }
    }
}

// Tail-split plan for a GEMM of `tiles` tiles of KT k-tiles on `slots` co-resident CTAs: the number of K pieces
// (1 = no split) that minimises (whole waves + the pieces' rounds / split) plus the split's own cost, the
// reduction launch and the partial tiles' HBM round trip measured against one tile's time `tile_s`; pieces
// keep >= 4 k-tiles and their partials (unit_bytes each) fit `max_units`.
struct SplitPlan {
    int split = 1, nfull = 0;
};
SplitPlan gemm_split_plan(int64_t tiles, int KT, int64_t slots, int64_t max_units, double tile_s, double unit_bytes);

// Bytes of tail-split scratch that let every GEMM of a matvec-sized problem pick its best split: at most
// 4 * (co-resident CTAs) partial tiles of the larger (real) tile.
size_t gemm_split_ws_bytes();

// Host launcher.  Returns HEFF_OK or a status code; never synchronises.
template<bool CPLX>
int gemm_f64(bool ta, bool tb, bool cja, const GemmArgs &args, cudaStream_t stream);
bool gemm_fn_known(const void *f);  // a DMMA GEMM or split-reduction kernel (single GemmArgs parameter)

}  // namespace heff
