// Mixed-precision H_eff matvec: split-BF16 operands on tcgen05 tensor cores with FP32 accumulation.
//
// Same contraction order as the FP64 path (matvec.cuh):
//   G1  T1[(a',m),(s,b)]   = sum_a L[a,(a',m)] x[s,a,b]              BF16 GEMM, K = chiL
//   MIX T2[(s',a'),(b,n)]  = sum_{m,s} W[m,n,s,s'] T1[(a',m),(s,b)]  FP64 arithmetic on FP32 inputs
//   G2  y[(s',a'),b']      = sum_{(b,n)} T2[(s',a'),(b,n)] R[b,b',n]  BF16 GEMM, K = chiR*D, FP64 output
// Each FP64 operand v is split into v_hi = bf16(v), v_mid = bf16(v - v_hi) (16 significant bits) and the
// three leading split products are folded into the GEMM's K dimension (segments):
//   real:    A' = [a_h | a_h | a_m]                    B' = [b_h | b_m | b_h]
//   complex: A' = [ar_h | ar_h | ar_m | ai_h | ai_h | ai_m]
//            B' rows of Re(C): [br_h | br_m | br_h | -bi_h | -bi_m | -bi_h],  rows of Im(C): [bi_h | bi_m | bi_h | br_h | br_m | br_h]
// so one K-major BF16 GEMM per stage computes the product to ~2^-16 relative accuracy (FP32 accumulation
// adds ~sqrt(K) 2^-24).  The eigensolver uses this path for its inner iterations and restores FP64
// accuracy by refinement with the FP64 matvec.  The environment operands (L, R') are split once per
// operator; x and T2 are split per matvec.
#include <cstdlib>
#include <algorithm>
#include <cuda_bf16.h>

#include "gemm_bf16x.cuh"
#include "matvec.cuh"
#include "op.cuh"
#include "runtime.cuh"
#include "wlist.cuh"

namespace heff {

struct MixedState {
    int            cplx, nseg;
    int64_t        M1, N1, K1, Kp1, Kx1;  // GEMM1: rows (a',m), cols (s,b), K = a
    int64_t        M2, N2, K2, Kp2, Kx2;  // GEMM2: rows (s',a'), cols b', K = (b,n)
    __nv_bfloat16 *A1 = nullptr, *B1 = nullptr, *A2 = nullptr, *B2 = nullptr;
    float         *T1  = nullptr;
    int           *err = nullptr;
    unsigned char *wl  = nullptr;  // the MPO's nonzero list (wlist.cuh layout)
    int            wl_bytes = 0;
    CUtensorMap    tA1, tB1, tA2, tB2;
    // every buffer above is carved from one pooled allocation that persists across rebinds (grown, never shrunk)
    void          *pool  = nullptr;
    size_t         cap   = 0;
    bool           stale = true;  // the split operands belong to other environments (set by a rebind)
};

__device__ __forceinline__ void split2(double v, __nv_bfloat16 &h, __nv_bfloat16 &m) {
    h = __double2bfloat16(v);
    m = __double2bfloat16(v - (double)__bfloat162float(h));
}

// Segment tables.  A: (component, part); B for Re rows and Im rows: (component, part, sign).
struct SegA {
    int comp, part;
};
struct SegB {
    int comp, part, sign;
};
__constant__ SegA c_segA_real[3] = {{0, 0}, {0, 0}, {0, 1}};
__constant__ SegB c_segB_real[3] = {{0, 0, 1}, {0, 1, 1}, {0, 0, 1}};
__constant__ SegA c_segA_cplx[6] = {{0, 0}, {0, 0}, {0, 1}, {1, 0}, {1, 0}, {1, 1}};
__constant__ SegB c_segB_re[6]   = {{0, 0, 1}, {0, 1, 1}, {0, 0, 1}, {1, 0, -1}, {1, 1, -1}, {1, 0, -1}};
__constant__ SegB c_segB_im[6]   = {{1, 0, 1}, {1, 1, 1}, {1, 0, 1}, {0, 0, 1}, {0, 1, 1}, {0, 0, 1}};

// Writes the A'-segments of one value pair (re, im) at row base `dst` (column k of each segment).
template<bool CPLX>
__device__ __forceinline__ void put_A(__nv_bfloat16 *dst, int64_t Kp, int64_t k, double re, double im) {
    __nv_bfloat16 rh, rm, ih, imm;
    split2(re, rh, rm);
    if constexpr(!CPLX) {
        dst[k]          = rh;
        dst[Kp + k]     = rh;
        dst[2 * Kp + k] = rm;
    } else {
        split2(im, ih, imm);
        dst[k]          = rh;
        dst[Kp + k]     = rh;
        dst[2 * Kp + k] = rm;
        dst[3 * Kp + k] = ih;
        dst[4 * Kp + k] = ih;
        dst[5 * Kp + k] = imm;
    }
}
// B'-segments: Re-output row at dst_re, Im-output row at dst_im (complex only).
template<bool CPLX>
__device__ __forceinline__ void put_B(__nv_bfloat16 *dst_re, __nv_bfloat16 *dst_im, int64_t Kp, int64_t k, double re, double im) {
    __nv_bfloat16 rh, rm;
    split2(re, rh, rm);
    if constexpr(!CPLX) {
        dst_re[k]          = rh;
        dst_re[Kp + k]     = rm;
        dst_re[2 * Kp + k] = rh;
    } else {
        __nv_bfloat16 ih, imm, nih, nim;
        split2(im, ih, imm);
        split2(-im, nih, nim);
        dst_re[k]          = rh;
        dst_re[Kp + k]     = rm;
        dst_re[2 * Kp + k] = rh;
        dst_re[3 * Kp + k] = nih;
        dst_re[4 * Kp + k] = nim;
        dst_re[5 * Kp + k] = nih;
        dst_im[k]          = ih;
        dst_im[Kp + k]     = imm;
        dst_im[2 * Kp + k] = ih;
        dst_im[3 * Kp + k] = rh;
        dst_im[4 * Kp + k] = rm;
        dst_im[5 * Kp + k] = rh;
    }
}

__device__ __forceinline__ double re_of(double v) { return v; }
__device__ __forceinline__ double im_of(double) { return 0.0; }
__device__ __forceinline__ double re_of(double2 v) { return v.x; }
__device__ __forceinline__ double im_of(double2 v) { return v.y; }

// A1'[r][seg*Kp1 + a] from L[a + cL*r]   (r = a' + cL*m)
template<bool CPLX>
__global__ void split_L_kernel(const typename Scalar<CPLX>::T *__restrict__ L, __nv_bfloat16 *__restrict__ A1, int64_t cL, int64_t M1, int64_t Kp1,
                               int64_t Kx1) {
    const int64_t tot = cL * M1;
    for(int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < tot; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t a = e % cL, r = e / cL;
        const auto    v = L[e];
        put_A<CPLX>(A1 + r * Kx1, Kp1, a, re_of(v), im_of(v));
    }
}
// B2'[b'][seg*Kp2 + k] from R'[k + K2*b'] (k = b + cR*n); complex: Im rows at b' + cR
template<bool CPLX>
__global__ void split_R_kernel(const typename Scalar<CPLX>::T *__restrict__ Rp, __nv_bfloat16 *__restrict__ B2, int64_t K2, int64_t cR, int64_t Kp2,
                               int64_t Kx2) {
    const int64_t tot = K2 * cR;
    for(int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < tot; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t k = e % K2, bp = e / K2;
        const auto    v = Rp[e];
        put_B<CPLX>(B2 + bp * Kx2, CPLX ? B2 + (bp + cR) * Kx2 : nullptr, Kp2, k, re_of(v), im_of(v));
    }
}
// B1'[(s + S b)][seg*Kp1 + a] from x[s + S*(a + cL*b)]; complex: Im rows at + N1.
// One block per (slab of ta values of a, one b): the S * ta inputs are a contiguous run of x (read
// coalesced into shared memory), and every output row segment is ta consecutive bf16.
template<bool CPLX>
__global__ void __launch_bounds__(256) split_x_kernel(const typename Scalar<CPLX>::T *__restrict__ x, __nv_bfloat16 *__restrict__ B1, int64_t S,
                                                      int64_t cL, int64_t N1, int64_t Kp1, int64_t Kx1, int ta) {
    using T = typename Scalar<CPLX>::T;
    extern __shared__ __align__(16) unsigned char sx_smem[];
    T            *sx  = reinterpret_cast<T *>(sx_smem);  // [S][ta]
    const int64_t a0  = (int64_t)blockIdx.x * ta, b = blockIdx.y;
    const int     na  = (int)(cL - a0 < (int64_t)ta ? cL - a0 : (int64_t)ta);
    const T      *src = x + S * (a0 + cL * b);  // x[s + S (a0 + j + cL b)] for j < na: contiguous
    for(int e = threadIdx.x; e < S * na; e += blockDim.x) sx[(e % S) * ta + e / S] = src[e];
    __syncthreads();
    for(int e = threadIdx.x; e < S * na; e += blockDim.x) {
        const int     s = e / na, j = e % na;
        const int64_t n = s + S * b;
        const T       v = sx[s * ta + j];
        put_B<CPLX>(B1 + n * Kx1, CPLX ? B1 + (n + N1) * Kx1 : nullptr, Kp1, a0 + j, re_of(v), im_of(v));
    }
}

// Two adjacent outputs k, k+1 (k even, Kp even) of every A'-segment as bf16 pairs (4-byte stores).
template<bool CPLX>
__device__ __forceinline__ void put_A_pair(__nv_bfloat16 *dst, int64_t Kp, int64_t k, double re0, double im0, double re1, double im1) {
    __nv_bfloat16 h0, m0, h1, m1;
    auto          st2 = [&](int64_t off, __nv_bfloat16 a, __nv_bfloat16 b) {
        *reinterpret_cast<__nv_bfloat162 *>(dst + off) = __halves2bfloat162(a, b);
    };
    split2(re0, h0, m0);
    split2(re1, h1, m1);
    st2(k, h0, h1);
    st2(Kp + k, h0, h1);
    st2(2 * Kp + k, m0, m1);
    if constexpr(CPLX) {
        split2(im0, h0, m0);
        split2(im1, h1, m1);
        st2(3 * Kp + k, h0, h1);
        st2(4 * Kp + k, h0, h1);
        st2(5 * Kp + k, m0, m1);
    }
}

// MIX: tile of TA a' x 64 b, 32*TA threads.  Load phase a'-fastest (coalesced T1 reads) into shared memory;
// compute phase: each thread two adjacent b, so the split T2 segments are written as bf16 pairs, contiguous
// along k = b + cR*n across the warp.  Staged rows of 64 b are padded to 66 floats: the a'-fastest stores hit
// distinct banks and the float2 reads of the compute phase are aligned and conflict-free.
constexpr int MX_TB = 64, MX_ROW = MX_TB + 2;
template<int TA>
constexpr int mx_sstr() {
    return TA * MX_ROW;  // floats per staged (m, s) slice
}
template<bool CPLX, int TA>
__global__ void __launch_bounds__(32 * TA) mix_mixed_kernel(const float *__restrict__ T1, const unsigned char *__restrict__ wl, int wl_bytes,
                                                           __nv_bfloat16 *__restrict__ A2, int S, int cL, int cR, int DL, int DR, int64_t M1,
                                                           int64_t N1, int64_t Kp2, int64_t Kx2) {
    using T                 = typename Scalar<CPLX>::T;
    constexpr int SSTR      = mx_sstr<TA>();
    constexpr int NTHREADS  = 32 * TA;
    extern __shared__ __align__(16) unsigned char mxs[];
    float *sRe = reinterpret_cast<float *>(mxs);
    const int NP = DL * S;
    float *sIm = sRe + NP * SSTR;
    unsigned char *lmem = reinterpret_cast<unsigned char *>(sIm + (CPLX ? NP * SSTR : 0));
    // the MPO's nonzero list (built once per operator) lands in shared memory with the T1 tile, under the same barrier
    for(int i = threadIdx.x; i < wl_bytes / 16; i += NTHREADS) reinterpret_cast<uint4 *>(lmem)[i] = reinterpret_cast<const uint4 *>(wl)[i];
    const int a0 = blockIdx.x * TA, b0 = blockIdx.y * MX_TB;
    if((cL & 3) == 0 && a0 + TA <= cL) {
        // 16-byte loads of 4 consecutive a' (T1's rows are a'-contiguous and 16-byte aligned when cL % 4 == 0), four
        // per thread in flight before their shared-memory stores; lanes run a'-quads fastest, then 8 b
        constexpr int Q = TA / 4, NB = 4;
        const int     items = Q * MX_TB * NP;
        for(int it0 = threadIdx.x; it0 < items; it0 += NTHREADS * NB) {
            float4 vr[NB], vi[NB];
#pragma unroll
            for(int u = 0; u < NB; u++) {
                const int it = it0 + u * NTHREADS;
                vr[u] = vi[u] = make_float4(0.f, 0.f, 0.f, 0.f);
                if(it < items) {
                    const int q = it % Q, rest = it / Q, bl = rest % MX_TB, ms = rest / MX_TB, m = ms / S, s = ms % S, b = b0 + bl;
                    if(b < cR) {
                        const int64_t idx = (a0 + 4 * q + (int64_t)cL * m) + M1 * (s + (int64_t)S * b);
                        vr[u]             = *reinterpret_cast<const float4 *>(T1 + idx);
                        if(CPLX) vi[u] = *reinterpret_cast<const float4 *>(T1 + idx + M1 * N1);
                    }
                }
            }
#pragma unroll
            for(int u = 0; u < NB; u++) {
                const int it = it0 + u * NTHREADS;
                if(it < items) {
                    const int q = it % Q, rest = it / Q, bl = rest % MX_TB, ms = rest / MX_TB;
                    float    *d = sRe + ms * SSTR + (4 * q) * MX_ROW + bl;
                    d[0]        = vr[u].x;
                    d[MX_ROW]   = vr[u].y;
                    d[2 * MX_ROW] = vr[u].z;
                    d[3 * MX_ROW] = vr[u].w;
                    if(CPLX) {
                        float *e = sIm + ms * SSTR + (4 * q) * MX_ROW + bl;
                        e[0]          = vi[u].x;
                        e[MX_ROW]     = vi[u].y;
                        e[2 * MX_ROW] = vi[u].z;
                        e[3 * MX_ROW] = vi[u].w;
                    }
                }
            }
        }
    } else {
        // a'-fastest loads (coalesced along T1's rows), 8 in flight per thread, two halves of the b range
        const int al = threadIdx.x % TA, bl = threadIdx.x / TA;  // bl < 32
        const int ap = a0 + al;
        for(int h = 0; h < 2; h++) {
            const int  b  = b0 + bl + 32 * h;
            const bool ok = ap < cL && b < cR;
            for(int ms0 = 0; ms0 < NP; ms0 += 8) {
                float vr[8], vi[8];
#pragma unroll
                for(int u = 0; u < 8; u++) {
                    const int ms = ms0 + u, m = ms / S, s = ms % S;
                    vr[u] = vi[u] = 0.f;
                    if(ok && ms < NP) {
                        const int64_t idx = (ap + (int64_t)cL * m) + M1 * (s + (int64_t)S * b);
                        vr[u]             = T1[idx];
                        if(CPLX) vi[u] = T1[idx + M1 * N1];
                    }
                }
#pragma unroll
                for(int u = 0; u < 8; u++)
                    if(ms0 + u < NP) {
                        sRe[(ms0 + u) * SSTR + al * MX_ROW + bl + 32 * h] = vr[u];
                        if(CPLX) sIm[(ms0 + u) * SSTR + al * MX_ROW + bl + 32 * h] = vi[u];
                    }
            }
        }
    }
    __syncthreads();
    int   *off;
    short *idx;
    T     *wv;
    wlist_views(lmem, DL, DR, S, off, idx, wv);
    const int bp = threadIdx.x % 32, al = threadIdx.x / 32;
    const int ap = a0 + al, b = b0 + 2 * bp;
    if(ap >= cL || b >= cR) return;
    const bool second = b + 1 < cR;
    const bool paired = second && (cR % 2 == 0);  // k = b + cR*n even for every n
    const int  me     = al * MX_ROW + 2 * bp;
    for(int n = 0; n < DR; n++)
        for(int sp = 0; sp < S; sp++) {
            const int o   = n * S + sp;
            double    re0 = 0, im0 = 0, re1 = 0, im1 = 0;
            for(int e = off[o]; e < off[o + 1]; e++) {
                const T      w    = wv[e];
                const int    slot = idx[e] * SSTR + me;
                const float2 xr   = *reinterpret_cast<const float2 *>(sRe + slot);
                if constexpr(CPLX) {
                    const float2 xi = *reinterpret_cast<const float2 *>(sIm + slot);
                    re0 += w.x * xr.x - w.y * xi.x;
                    im0 += w.x * xi.x + w.y * xr.x;
                    re1 += w.x * xr.y - w.y * xi.y;
                    im1 += w.x * xi.y + w.y * xr.y;
                } else {
                    re0 += w * xr.x;
                    re1 += w * xr.y;
                }
            }
            const int64_t row = sp + (int64_t)S * ap, k = b + (int64_t)cR * n;
            if(paired) {
                put_A_pair<CPLX>(A2 + row * Kx2, Kp2, k, re0, im0, re1, im1);
            } else {
                put_A<CPLX>(A2 + row * Kx2, Kp2, k, re0, im0);
                if(second) put_A<CPLX>(A2 + row * Kx2, Kp2, k + 1, re1, im1);
            }
        }
}

// Tile height: 16 a' when the staging fits in ~100 KB (two or more CTAs per SM), else 8; the environment variable
// HEFF_MIX_TA (8 or 16) overrides it for measurements.
static int mx_ta(int64_t NP, int cf) {
    static const int forced = [] {
        const char *e = getenv("HEFF_MIX_TA");
        const int   v = e ? atoi(e) : 0;
        return (v == 8 || v == 16) ? v : 0;
    }();
    if(forced == 8) return 8;
    if(forced == 16 && (size_t)cf * 4 * NP * mx_sstr<16>() <= 200 * 1024) return 16;
    return (size_t)cf * 4 * NP * mx_sstr<16>() <= 100 * 1024 ? 16 : 8;
}
static size_t mx_smem(int64_t NP, int cf, int ta, int wl_bytes) {
    return (size_t)cf * 4 * NP * (ta == 16 ? mx_sstr<16>() : mx_sstr<8>()) + (size_t)wl_bytes;
}

static int g1(int64_t n) {
    int64_t g = (n + 255) / 256, cap = (int64_t)device_sm_count() * 16;
    return (int)(g < 1 ? 1 : (g < cap ? g : cap));
}
static int64_t r64(int64_t v) { return (v + 63) / 64 * 64; }

// Byte sizes of the split operands, the FP32 T1 and the flags of one operator shape, each rounded to 256 bytes
// (in carve order: A1, B1, A2, B2, T1, err, wl).
struct MixedSizes {
    size_t b[7];
    size_t total() const {
        size_t t = 0;
        for(size_t v : b) t += v;
        return t;
    }
};
static size_t up256m(size_t v) { return (v + 255) / 256 * 256; }
static MixedSizes mixed_sizes(int64_t S, int64_t cL, int64_t cR, int64_t DL, int64_t DR, bool cplx) {
    const int64_t nseg = cplx ? 6 : 3, cf = cplx ? 2 : 1;
    const int64_t M1 = cL * DL, N1 = S * cR, Kx1 = nseg * r64(cL);
    const int64_t M2 = S * cL, N2 = cR, Kx2 = nseg * r64(cR * DR);
    MixedSizes    z;
    z.b[0] = up256m(2 * (size_t)M1 * Kx1);
    z.b[1] = up256m(2 * (size_t)(cf * N1) * Kx1);
    z.b[2] = up256m(2 * (size_t)M2 * Kx2);
    z.b[3] = up256m(2 * (size_t)(cf * N2) * Kx2);
    z.b[4] = up256m(4 * (size_t)M1 * (cf * N1));
    z.b[5] = 256;
    z.b[6] = up256m(wlist_bytes((int)DL, (int)DR, (int)S, cplx ? 16 : 8));
    return z;
}

size_t mixed_bytes(int64_t S, int64_t cL, int64_t cR, int64_t DL, int64_t DR, bool cplx) { return mixed_sizes(S, cL, cR, DL, DR, cplx).total(); }

static void mixed_destroy(heff_op *op) {
    MixedState *m = reinterpret_cast<MixedState *>(op->mixed);
    if(!m) return;
    if(m->pool) cudaFree(m->pool);
    delete m;
    op->mixed = nullptr;
}

void mixed_invalidate(heff_op *op) {
    if(op->mixed) reinterpret_cast<MixedState *>(op->mixed)->stale = true;
}

size_t mixed_held_bytes(const heff_op *op) { return op->mixed ? reinterpret_cast<const MixedState *>(op->mixed)->cap : 0; }

static MixedState *mixed_state(heff_op *op) {
    if(!op->mixed) {
        op->mixed        = new MixedState();
        op->destroy_hook = mixed_destroy;
    }
    return reinterpret_cast<MixedState *>(op->mixed);
}

// Grows the pooled buffer to at least `bytes` (stream-synchronised free of the old one; nothing when it is
// large enough already).
static int mixed_grow(heff_op *op, MixedState *m, size_t bytes) {
    if(m->cap >= bytes) return HEFF_OK;
    if(m->pool) {
        HEFF_CUDA(cudaStreamSynchronize(op->stream));
        cudaFree(m->pool);
        m->pool = nullptr;
        m->cap  = 0;
    }
    cudaError_t e = cudaMalloc(&m->pool, bytes);
    if(e != cudaSuccess) {
        m->pool = nullptr;
        set_last_cuda_error(e, "mixed-precision buffers", __FILE__, __LINE__);
        return HEFF_OOM;
    }
    m->cap   = bytes;
    m->stale = true;
    return HEFF_OK;
}

int mixed_reserve(heff_op *op, size_t bytes) { return mixed_grow(op, mixed_state(op), bytes); }

// Lays the split operands of the operator's current shape out in the pooled buffer (grown when needed), splits
// L and R' into them and builds the tensor maps.  Runs on the first mixed matvec after a create or a rebind.
template<bool CPLX>
static int mixed_setup(heff_op *op) {
    using T         = typename Scalar<CPLX>::T;
    const auto &d   = op->d;
    MixedState *m   = mixed_state(op);
    m->cplx         = CPLX;
    m->nseg         = CPLX ? 6 : 3;
    const int cf    = CPLX ? 2 : 1;
    m->M1           = d.cL * d.DL;
    m->N1           = d.S * d.cR;
    m->K1           = d.cL;
    m->Kp1          = r64(m->K1);
    m->Kx1          = m->nseg * m->Kp1;
    m->M2           = d.S * d.cL;
    m->N2           = d.cR;
    m->K2           = d.cR * d.DR;
    m->Kp2          = r64(m->K2);
    m->Kx2          = m->nseg * m->Kp2;
    const MixedSizes z = mixed_sizes(d.S, d.cL, d.cR, d.DL, d.DR, CPLX);
    HEFF_TRY(mixed_grow(op, m, z.total()));
    unsigned char *p = reinterpret_cast<unsigned char *>(m->pool);
    void         **dst[7] = {(void **)&m->A1, (void **)&m->B1, (void **)&m->A2, (void **)&m->B2, (void **)&m->T1, (void **)&m->err, (void **)&m->wl};
    for(int i = 0; i < 7; i++) {
        *dst[i] = p;
        p += z.b[i];
    }
    cudaStream_t s = op->stream;
    // K padding of every segment must read zero: the split operands (and the padding the kernels never write) are
    // cleared whenever the layout is (re)built, since the pool may hold another shape's values
    HEFF_CUDA(cudaMemsetAsync(m->pool, 0, z.b[0] + z.b[1] + z.b[2] + z.b[3], s));
    HEFF_CUDA(cudaMemsetAsync(m->err, 0, sizeof(int), s));
    split_L_kernel<CPLX><<<g1(m->K1 * m->M1), 256, 0, s>>>(reinterpret_cast<const T *>(op->L), m->A1, d.cL, m->M1, m->Kp1, m->Kx1);
    HEFF_LAUNCH_CHECK();
    split_R_kernel<CPLX><<<g1(m->K2 * m->N2), 256, 0, s>>>(reinterpret_cast<const T *>(op->Rp), m->B2, m->K2, d.cR, m->Kp2, m->Kx2);
    HEFF_LAUNCH_CHECK();
    HEFF_TRY(make_tmap_bf16(&m->tA1, m->A1, m->M1, m->Kx1, m->Kx1, X_BM));
    HEFF_TRY(make_tmap_bf16(&m->tB1, m->B1, cf * m->N1, m->Kx1, m->Kx1, X_BN));
    HEFF_TRY(make_tmap_bf16(&m->tA2, m->A2, m->M2, m->Kx2, m->Kx2, X_BM));
    HEFF_TRY(make_tmap_bf16(&m->tB2, m->B2, cf * m->N2, m->Kx2, m->Kx2, X_BN));

    m->wl_bytes = (int)wlist_bytes((int)d.DL, (int)d.DR, (int)d.S, sizeof(T));
    wlist_global_kernel<T><<<1, 32, 0, s>>>(reinterpret_cast<const T *>(op->W), (int)d.DL, (int)d.DR, (int)d.S, m->wl);
    HEFF_LAUNCH_CHECK();
    const int    ta       = mx_ta(d.DL * d.S, cf);
    const size_t mix_smem = mx_smem(d.DL * d.S, cf, ta, m->wl_bytes);
    if(mix_smem > 200 * 1024) return HEFF_BAD_SHAPE;
    HEFF_CUDA(cudaFuncSetAttribute(mix_mixed_kernel<CPLX, 16>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    HEFF_CUDA(cudaFuncSetAttribute(mix_mixed_kernel<CPLX, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    m->stale = false;
    return HEFF_OK;
}

template<bool CPLX>
static int mixed_apply_impl(heff_op *op, const void *x, void *y) {
    using T = typename Scalar<CPLX>::T;
    if(!op->mixed || reinterpret_cast<MixedState *>(op->mixed)->stale) HEFF_TRY(mixed_setup<CPLX>(op));
    MixedState  *m  = reinterpret_cast<MixedState *>(op->mixed);
    const auto  &d  = op->d;
    cudaStream_t s  = op->stream;
    const int    cf = CPLX ? 2 : 1;
    // slab width: 256 values of a, fewer for large merged spins so the tile stays within 48 KB
    const int ta = (int)std::max<int64_t>(32, std::min<int64_t>(256, (int64_t)(48 * 1024 / (sizeof(T) * d.S)) / 32 * 32));
    if(d.cR > 65535 || (size_t)d.S * ta * sizeof(T) > 48 * 1024) return HEFF_BAD_SHAPE;
    split_x_kernel<CPLX><<<dim3((unsigned)cdiv(d.cL, ta), (unsigned)d.cR), 256, (size_t)d.S * ta * sizeof(T), s>>>(
        reinterpret_cast<const T *>(x), m->B1, d.S, d.cL, m->N1, m->Kp1, m->Kx1, ta);
    HEFF_LAUNCH_CHECK();
    XGemmArgs g1a{};
    g1a.M = (int)m->M1, g1a.N = (int)(cf * m->N1), g1a.K = (int)m->Kx1, g1a.C = m->T1, g1a.ldc = m->M1, g1a.mode = X_OUT_F32, g1a.err = m->err;
    HEFF_TRY(gemm_bf16x(m->tA1, m->tB1, g1a, s));
    const int    mta      = mx_ta(d.DL * d.S, cf);
    const size_t mix_smem = mx_smem(d.DL * d.S, cf, mta, m->wl_bytes);
    if(d.cR / MX_TB + 1 > 65535) return HEFF_BAD_SHAPE;
    dim3 grid((unsigned)cdiv(d.cL, mta), (unsigned)cdiv(d.cR, MX_TB));
    if(mta == 16)
        mix_mixed_kernel<CPLX, 16><<<grid, 32 * 16, mix_smem, s>>>(m->T1, m->wl, m->wl_bytes, m->A2, (int)d.S, (int)d.cL, (int)d.cR, (int)d.DL,
                                                                  (int)d.DR, m->M1, m->N1, m->Kp2, m->Kx2);
    else
        mix_mixed_kernel<CPLX, 8><<<grid, 32 * 8, mix_smem, s>>>(m->T1, m->wl, m->wl_bytes, m->A2, (int)d.S, (int)d.cL, (int)d.cR, (int)d.DL,
                                                                (int)d.DR, m->M1, m->N1, m->Kp2, m->Kx2);
    HEFF_LAUNCH_CHECK();
    XGemmArgs g2{};
    g2.M = (int)m->M2, g2.N = (int)(cf * m->N2), g2.K = (int)m->Kx2, g2.C = y, g2.ldc = m->M2, g2.err = m->err;
    g2.mode   = CPLX ? X_OUT_C128 : X_OUT_F64;
    g2.n_half = (int)m->N2;
    HEFF_TRY(gemm_bf16x(m->tA2, m->tB2, g2, s));
    op->num_mv++;
    return HEFF_OK;
}

int mixed_apply(heff_op *op, const void *x, void *y) {
    if(x == y) return HEFF_BAD_ARG;
    return op->cplx ? mixed_apply_impl<true>(op, x, y) : mixed_apply_impl<false>(op, x, y);
}

int mixed_error_flag(heff_op *op, int *flag) {
    *flag = 0;
    MixedState *m = reinterpret_cast<MixedState *>(op->mixed);
    if(!m) return HEFF_OK;
    HEFF_CUDA(cudaMemcpyAsync(flag, m->err, sizeof(int), cudaMemcpyDeviceToHost, op->stream));
    HEFF_CUDA(cudaStreamSynchronize(op->stream));
    return HEFF_OK;
}

}  // namespace heff
