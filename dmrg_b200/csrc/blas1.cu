// Tall-skinny vector kernels for the eigensolver (see blas1.cuh).  All reductions run in a fixed
// order (per-block partial sums, then one block), so results do not depend on scheduling: the same
// eigensolve gives bit-identical output alone or next to other work on the device.
#include "blas1.cuh"

namespace heff {

__device__ __forceinline__ double cj_mul_re(double a, double b) { return a * b; }
template<class T>
struct VOps;
template<>
struct VOps<double> {
    static __device__ __forceinline__ void dot_acc(double &re, double &im, double v, double t) { re = fma(v, t, re); }
    static __device__ __forceinline__ double axpy(double acc, double v, double h) { return fma(v, h, acc); }
    static __device__ __forceinline__ double zero() { return 0.0; }
    static __device__ __forceinline__ double scale(double x, double a) { return x * a; }
    static __device__ __forceinline__ double make(double re, double) { return re; }
    static __device__ __forceinline__ double addscaled(double y, double a, double x) { return fma(a, x, y); }
};
template<>
struct VOps<double2> {
    static __device__ __forceinline__ void dot_acc(double &re, double &im, double2 v, double2 t) {
        re = fma(v.x, t.x, fma(v.y, t.y, re));  // conj(v) * t
        im = fma(v.x, t.y, fma(-v.y, t.x, im));
    }
    static __device__ __forceinline__ double2 axpy(double2 acc, double2 v, double2 h) {
        return make_double2(fma(v.x, h.x, fma(-v.y, h.y, acc.x)), fma(v.x, h.y, fma(v.y, h.x, acc.y)));
    }
    static __device__ __forceinline__ double2 zero() { return make_double2(0, 0); }
    static __device__ __forceinline__ double2 scale(double2 x, double a) { return make_double2(x.x * a, x.y * a); }
    static __device__ __forceinline__ double2 make(double re, double im) { return make_double2(re, im); }
    static __device__ __forceinline__ double2 addscaled(double2 y, double a, double2 x) { return make_double2(fma(a, x.x, y.x), fma(a, x.y, y.y)); }
};

// Partial sums of h[j] = sum_i conj(V[i,j]) t[i], MD_G columns per pass: every thread streams rows
// (coalesced across the warp, one load per column per row) into MD_G register accumulators, then the
// block reduces them.  partials[(j * nb + blk) * 2 + {0,1}] (column-major over blocks for the final pass).
constexpr int MD_G = 8;
template<class T>
__global__ void __launch_bounds__(256) multi_dot_partial(const T *__restrict__ V, int64_t ldv, int64_t n, int k, const T *__restrict__ t,
                                                        double *__restrict__ partials) {
    constexpr bool CPLX = sizeof(T) == 16;
    __shared__ double sre[8][MD_G], sim[8][MD_G];
    const int         lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int         nb   = gridDim.x;
    for(int j0 = 0; j0 < k; j0 += MD_G) {
        const int jn = min(MD_G, k - j0);
        double    re[MD_G], im[MD_G];
#pragma unroll
        for(int q = 0; q < MD_G; q++) re[q] = im[q] = 0.0;
        const T *Vj = V + ldv * j0;
        for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
            const T tv = t[i];
            if(jn == MD_G) {
#pragma unroll
                for(int q = 0; q < MD_G; q++) VOps<T>::dot_acc(re[q], im[q], Vj[i + ldv * q], tv);
            } else {
                for(int q = 0; q < jn; q++) VOps<T>::dot_acc(re[q], im[q], Vj[i + ldv * q], tv);
            }
        }
#pragma unroll
        for(int q = 0; q < MD_G; q++) {
            double a = re[q], b = im[q];
            for(int o = 16; o > 0; o >>= 1) {
                a += __shfl_xor_sync(0xffffffffu, a, o);
                if(CPLX) b += __shfl_xor_sync(0xffffffffu, b, o);
            }
            if(lane == 0) {
                sre[warp][q] = a;
                sim[warp][q] = b;
            }
        }
        __syncthreads();
        if(threadIdx.x < jn) {
            double a = 0, b = 0;
            for(int w = 0; w < 8; w++) {
                a += sre[w][threadIdx.x];
                b += sim[w][threadIdx.x];
            }
            const int64_t j = j0 + threadIdx.x;
            partials[(j * nb + blockIdx.x) * 2 + 0] = a;
            partials[(j * nb + blockIdx.x) * 2 + 1] = b;
        }
        __syncthreads();
    }
}

// One block per column: fixed-order tree reduction of the nb partial sums.
template<class T>
__global__ void __launch_bounds__(256) multi_dot_final(const double *__restrict__ partials, int nb, int k, T *__restrict__ h) {
    __shared__ double sa[256], sb[256];
    const int         j = blockIdx.x;
    double            a = 0, b = 0;
    for(int blk = threadIdx.x; blk < nb; blk += blockDim.x) {
        a += partials[((int64_t)j * nb + blk) * 2 + 0];
        b += partials[((int64_t)j * nb + blk) * 2 + 1];
    }
    sa[threadIdx.x] = a;
    sb[threadIdx.x] = b;
    __syncthreads();
    for(int w = 128; w > 0; w >>= 1) {
        if(threadIdx.x < w) {
            sa[threadIdx.x] += sa[threadIdx.x + w];
            sb[threadIdx.x] += sb[threadIdx.x + w];
        }
        __syncthreads();
    }
    if(threadIdx.x == 0) h[j] = VOps<T>::make(sa[0], sb[0]);
}

template<class T>
__global__ void multi_axpy_kernel(const T *__restrict__ V, int64_t ldv, int64_t n, int k, const T *__restrict__ h, double alpha, T *__restrict__ t) {
    extern __shared__ __align__(16) unsigned char hsm[];
    T *sh = reinterpret_cast<T *>(hsm);
    for(int j = threadIdx.x; j < k; j += blockDim.x) sh[j] = h[j];
    __syncthreads();
    for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        T acc = VOps<T>::zero();
        for(int j = 0; j < k; j++) acc = VOps<T>::axpy(acc, V[i + ldv * j], sh[j]);
        t[i] = VOps<T>::addscaled(t[i], alpha, acc);
    }
}

template<class T>
__global__ void combine_kernel(const T *__restrict__ V, int64_t ldv, int64_t n, int k, const T *__restrict__ c, T *__restrict__ x) {
    extern __shared__ __align__(16) unsigned char csm[];
    T *sc = reinterpret_cast<T *>(csm);
    for(int j = threadIdx.x; j < k; j += blockDim.x) sc[j] = c[j];
    __syncthreads();
    for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        T acc = VOps<T>::zero();
        for(int j = 0; j < k; j++) acc = VOps<T>::axpy(acc, V[i + ldv * j], sc[j]);
        x[i] = acc;
    }
}

template<class T>
__global__ void scale_kernel(T *__restrict__ x, int64_t n, const double *__restrict__ a, bool inv_sqrt) {
    const double v = inv_sqrt ? (a[0] > 0 ? rsqrt(a[0]) : 0.0) : a[0];
    for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) x[i] = VOps<T>::scale(x[i], v);
}

template<class T>
__global__ void residual_kernel(const T *__restrict__ ax, const T *__restrict__ x, double theta, T *__restrict__ r, int64_t n) {
    for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        r[i] = VOps<T>::addscaled(ax[i], -theta, x[i]);
}

static int grid_for(int64_t n, int cap_per_sm = 8) {
    int64_t g = (n + 255) / 256, cap = (int64_t)device_sm_count() * cap_per_sm;
    return (int)(g < 1 ? 1 : (g < cap ? g : cap));
}

template<bool CPLX>
int multi_dot(const typename Scalar<CPLX>::T *V, int64_t ldv, int64_t n, int k, const typename Scalar<CPLX>::T *t, typename Scalar<CPLX>::T *h,
              double *partials, cudaStream_t s) {
    using T = typename Scalar<CPLX>::T;
    if(k <= 0) return HEFF_OK;
    if(k > MD_MAXK) return HEFF_BAD_ARG;
    const int nb = (int)std::min<int64_t>(std::min<int64_t>(MD_BLOCKS, 4 * (int64_t)device_sm_count()), std::max<int64_t>(1, (n + 255) / 256));
    multi_dot_partial<T><<<nb, 256, 0, s>>>(V, ldv, n, k, t, partials);
    HEFF_LAUNCH_CHECK();
    multi_dot_final<T><<<k, 256, 0, s>>>(partials, nb, k, h);
    HEFF_LAUNCH_CHECK();
    return HEFF_OK;
}

template<bool CPLX>
int multi_axpy(const typename Scalar<CPLX>::T *V, int64_t ldv, int64_t n, int k, const typename Scalar<CPLX>::T *h, double alpha,
               typename Scalar<CPLX>::T *t, cudaStream_t s) {
    using T = typename Scalar<CPLX>::T;
    if(k <= 0) return HEFF_OK;
    multi_axpy_kernel<T><<<grid_for(n), 256, sizeof(T) * k, s>>>(V, ldv, n, k, h, alpha, t);
    HEFF_LAUNCH_CHECK();
    return HEFF_OK;
}

template<bool CPLX>
int combine(const typename Scalar<CPLX>::T *V, int64_t ldv, int64_t n, int k, const typename Scalar<CPLX>::T *c, typename Scalar<CPLX>::T *x,
            cudaStream_t s) {
    using T = typename Scalar<CPLX>::T;
    combine_kernel<T><<<grid_for(n), 256, sizeof(T) * std::max(k, 1), s>>>(V, ldv, n, k, c, x);
    HEFF_LAUNCH_CHECK();
    return HEFF_OK;
}

template<bool CPLX>
int scale_dev(typename Scalar<CPLX>::T *x, int64_t n, const double *a, bool inv_sqrt, cudaStream_t s) {
    scale_kernel<typename Scalar<CPLX>::T><<<grid_for(n), 256, 0, s>>>(x, n, a, inv_sqrt);
    HEFF_LAUNCH_CHECK();
    return HEFF_OK;
}

template<bool CPLX>
int residual(const typename Scalar<CPLX>::T *ax, const typename Scalar<CPLX>::T *x, double theta, typename Scalar<CPLX>::T *r, int64_t n,
             cudaStream_t s) {
    residual_kernel<typename Scalar<CPLX>::T><<<grid_for(n), 256, 0, s>>>(ax, x, theta, r, n);
    HEFF_LAUNCH_CHECK();
    return HEFF_OK;
}

// ---------------------------------------------------------------------------------------------------------
// Device-side classical Gram-Schmidt with a conditional second pass (DGKS) and normalisation, for the
// Krylov expansion of the eigensolver: no host decision between the passes, so the next matvec can be
// enqueued before the host reads the coefficients.
//
// State st[] (doubles): [0] ||w||^2, [1] second pass needed (0/1), [2] ||w'||^2 after pass 1, [3] beta^2,
// h1 at st + ORTH_H1 (re, im pairs), h2 at st + ORTH_H2.  Host-visible result hres (T): hres[j] = h1 + h2
// (j < k), hres[k] = beta, hres[k+1] = (||w||^2, second pass flag).
constexpr int ORTH_H1 = 8;
constexpr int ORTH_H2 = 8 + 2 * (MD_MAXK + 2);

template<class T>
__device__ __forceinline__ T orth_make(double re, double im) {
    return VOps<T>::make(re, im);
}

// pass 0: h1[j] = <V_j, w>, ||w||^2;  pass 1 (only when st[1] != 0): h2[j] = <V_j, v>, ||v||^2.
// Partial sums per block, then the last block to finish reduces them in block order (deterministic).
template<class T>
__global__ void __launch_bounds__(256) orth_dot_kernel(const T *__restrict__ V, int64_t ldv, int64_t n, int k, const T *__restrict__ t,
                                                      double *__restrict__ partials, unsigned *__restrict__ counter, double *__restrict__ st,
                                                      T *__restrict__ hres, int pass) {
    constexpr bool CPLX = sizeof(T) == 16;
    if(pass == 1 && st[1] == 0.0) return;  // uniform over the grid
    __shared__ double sre[8][MD_G], sim[8][MD_G];
    __shared__ bool   s_last;
    const int         lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int         nb = gridDim.x, kk = k + 1;  // column k is t itself
    for(int j0 = 0; j0 < kk; j0 += MD_G) {
        const int jn = min(MD_G, kk - j0);
        double    re[MD_G], im[MD_G];
#pragma unroll
        for(int q = 0; q < MD_G; q++) re[q] = im[q] = 0.0;
        for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
            const T tv = t[i];
#pragma unroll
            for(int q = 0; q < MD_G; q++) {
                const int j = j0 + q;
                if(q < jn) VOps<T>::dot_acc(re[q], im[q], j < k ? V[i + ldv * j] : tv, tv);
            }
        }
#pragma unroll
        for(int q = 0; q < MD_G; q++) {
            double a = re[q], b = im[q];
            for(int o = 16; o > 0; o >>= 1) {
                a += __shfl_xor_sync(0xffffffffu, a, o);
                if(CPLX) b += __shfl_xor_sync(0xffffffffu, b, o);
            }
            if(lane == 0) {
                sre[warp][q] = a;
                sim[warp][q] = b;
            }
        }
        __syncthreads();
        if(threadIdx.x < jn) {
            double a = 0, b = 0;
            for(int w = 0; w < 8; w++) {
                a += sre[w][threadIdx.x];
                b += sim[w][threadIdx.x];
            }
            const int64_t j = j0 + threadIdx.x;
            partials[(j * nb + blockIdx.x) * 2 + 0] = a;
            partials[(j * nb + blockIdx.x) * 2 + 1] = b;
        }
        __syncthreads();
    }
    __threadfence();
    if(threadIdx.x == 0) s_last = atomicAdd(counter, 1u) == (unsigned)(nb - 1);
    __syncthreads();
    if(!s_last) return;
    __threadfence();
    double *h = st + (pass == 0 ? ORTH_H1 : ORTH_H2);
    // one warp per column: lanes take blocks lane, lane+32, ... in order, then a fixed shuffle tree
    for(int j = warp; j < kk; j += 8) {
        double a = 0, b = 0;
        for(int blk = lane; blk < nb; blk += 32) {
            a += __ldcg(&partials[((int64_t)j * nb + blk) * 2 + 0]);
            b += __ldcg(&partials[((int64_t)j * nb + blk) * 2 + 1]);
        }
        for(int o = 16; o > 0; o >>= 1) {
            a += __shfl_xor_sync(0xffffffffu, a, o);
            b += __shfl_xor_sync(0xffffffffu, b, o);
        }
        if(lane == 0) {
            h[2 * j]     = a;
            h[2 * j + 1] = CPLX ? b : 0.0;
        }
    }
    __syncthreads();
    if(threadIdx.x == 0) {
        double hn2 = 0;
        for(int j = 0; j < k; j++) hn2 += h[2 * j] * h[2 * j] + h[2 * j + 1] * h[2 * j + 1];
        const double nrm2 = h[2 * k];
        if(pass == 0) {
            st[0] = nrm2;
            st[3] = nrm2 - hn2;
            st[1] = (nrm2 - hn2 > 0.5 * nrm2) ? 0.0 : 1.0;  // severe cancellation: orthogonalise again
        } else {
            st[2] = nrm2;
            st[3] = nrm2 - hn2;
        }
        *counter = 0u;  // ready for the next launch
    }
    __syncthreads();
    // host-visible coefficients and beta (block 0 of the last pass that ran writes them)
    const double beta2 = st[3];
    for(int j = threadIdx.x; j < k; j += blockDim.x) {
        double re = st[ORTH_H1 + 2 * j], im = st[ORTH_H1 + 2 * j + 1];
        if(pass == 1) {
            re += st[ORTH_H2 + 2 * j];
            im += st[ORTH_H2 + 2 * j + 1];
        }
        hres[j] = orth_make<T>(re, im);
    }
    if(threadIdx.x == 0) {
        hres[k]     = orth_make<T>(sqrt(fmax(beta2, 0.0)), 0.0);
        hres[k + 1] = orth_make<T>(st[0], st[1]);
    }
}

// out = (in - V h) * s, with h = h1 (pass 0) or h2 (pass 1, skipped unless st[1] != 0) and s = 1 / beta when
// this is the last pass (no second pass needed, or pass 1), else 1.  A vanishing beta (invariant subspace)
// writes zeros (the host stops before using the vector).
template<class T>
__global__ void orth_axpy_kernel(const T *__restrict__ V, int64_t ldv, int64_t n, int k, const T *in, T *out, const double *__restrict__ st,
                                 int pass) {
    if(pass == 1 && st[1] == 0.0) return;
    extern __shared__ __align__(16) unsigned char osm[];
    T            *sh   = reinterpret_cast<T *>(osm);
    const double *h    = st + (pass == 0 ? ORTH_H1 : ORTH_H2);
    for(int j = threadIdx.x; j < k; j += blockDim.x) sh[j] = orth_make<T>(h[2 * j], h[2 * j + 1]);
    const bool   last  = pass == 1 || st[1] == 0.0;
    const double beta2 = st[3];
    const double s     = !last ? 1.0 : (beta2 > 1e-300 ? 1.0 / sqrt(beta2) : 0.0);
    __syncthreads();
    for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        T acc = VOps<T>::zero();
        for(int j = 0; j < k; j++) acc = VOps<T>::axpy(acc, V[i + ldv * j], sh[j]);
        out[i] = VOps<T>::scale(VOps<T>::addscaled(in[i], -1.0, acc), s);
    }
}

// ---- Fast path of orth_cgs2 for k <= 24 and 16-byte rows (real: two rows per double2; complex: one element).
// Every thread first loads its row of all k basis columns (16-byte loads, all in flight together), then does
// the arithmetic: the loads-first order and the 16-byte width are what bring these HBM-bound passes near the
// copy bandwidth.  Three modes, each ending in the same deterministic last-block reduction as orth_dot_kernel:
//   MODE 0: h1 = V^H w, ||w||^2                                    (decides the second pass, as orth_dot pass 0)
//   MODE 1: v = (w - V h1) s1 with s1 = 1/beta1 unless a second pass follows; in the same sweep over V,
//           h2 = V^H v and ||v||^2 (used only when the second pass runs)
//   MODE 2: v = (v - V h2) / beta  (launched always, returns at once unless the second pass is needed)
template<bool CPLX, int KM, int MODE>
__global__ void __launch_bounds__(256, 1) orth_fast_kernel(const double2 *V, int64_t ldu, int64_t nu, int k, const double2 *in, double2 *out,
                                                           double *__restrict__ partials, unsigned *__restrict__ counter, double *__restrict__ st,
                                                           typename Scalar<CPLX>::T *__restrict__ hres) {
    using T = typename Scalar<CPLX>::T;
    if(MODE == 2 && st[1] == 0.0) return;  // uniform over the grid
    __shared__ double sre[8][KM + 1], sim[8][KM + 1];
    __shared__ double shr[KM], shi[KM];
    __shared__ bool   s_last;
    const int         lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nb = gridDim.x;
    if(MODE != 0) {
        const double *h = st + (MODE == 1 ? ORTH_H1 : ORTH_H2);
        for(int j = threadIdx.x; j < KM; j += blockDim.x) {
            shr[j] = j < k ? h[2 * j] : 0.0;
            shi[j] = j < k ? h[2 * j + 1] : 0.0;
        }
    }
    double scale = 1.0;
    if(MODE == 1) scale = st[1] != 0.0 ? 1.0 : (st[3] > 1e-300 ? 1.0 / sqrt(st[3]) : 0.0);
    if(MODE == 2) scale = st[3] > 1e-300 ? 1.0 / sqrt(st[3]) : 0.0;
    __syncthreads();
    double are[KM + 1], aim[KM + 1];
#pragma unroll
    for(int j = 0; j <= KM; j++) are[j] = aim[j] = 0.0;
    for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nu; i += (int64_t)gridDim.x * blockDim.x) {
        double2 v[KM];
#pragma unroll
        for(int j = 0; j < KM; j++) v[j] = V[i + ldu * (j < k ? j : 0)];
        double2 r = in[i];
        if(MODE != 0) {
            double ax = 0, ay = 0;
#pragma unroll
            for(int j = 0; j < KM; j++) {
                if constexpr(CPLX) {
                    ax = fma(v[j].x, shr[j], fma(-v[j].y, shi[j], ax));
                    ay = fma(v[j].x, shi[j], fma(v[j].y, shr[j], ay));
                } else {
                    ax = fma(v[j].x, shr[j], ax);
                    ay = fma(v[j].y, shr[j], ay);
                }
            }
            r = make_double2((r.x - ax) * scale, (r.y - ay) * scale);
            out[i] = r;
        }
        if(MODE != 2) {
#pragma unroll
            for(int j = 0; j < KM; j++)
                if(j < k) {
                    if constexpr(CPLX) {
                        are[j] = fma(v[j].x, r.x, fma(v[j].y, r.y, are[j]));  // conj(v) r
                        aim[j] = fma(v[j].x, r.y, fma(-v[j].y, r.x, aim[j]));
                    } else {
                        are[j] = fma(v[j].x, r.x, fma(v[j].y, r.y, are[j]));
                    }
                }
            are[KM] = fma(r.x, r.x, fma(r.y, r.y, are[KM]));
        }
    }
    if(MODE == 2) return;
    // block partial sums (column j < k, and the norm in slot k), fixed order
#pragma unroll
    for(int j = 0; j <= KM; j++) {
        double a = are[j], b = aim[j];
        for(int o = 16; o > 0; o >>= 1) {
            a += __shfl_xor_sync(0xffffffffu, a, o);
            if(CPLX) b += __shfl_xor_sync(0xffffffffu, b, o);
        }
        if(lane == 0) sre[warp][j] = a, sim[warp][j] = b;
    }
    __syncthreads();
    for(int j = threadIdx.x; j <= k; j += blockDim.x) {
        const int src = j < k ? j : KM;
        double    a = 0, b = 0;
        for(int w = 0; w < 8; w++) a += sre[w][src], b += sim[w][src];
        partials[((int64_t)j * nb + blockIdx.x) * 2 + 0] = a;
        partials[((int64_t)j * nb + blockIdx.x) * 2 + 1] = b;
    }
    __threadfence();
    __syncthreads();
    if(threadIdx.x == 0) s_last = atomicAdd(counter, 1u) == (unsigned)(nb - 1);
    __syncthreads();
    if(!s_last) return;
    __threadfence();
    double *h = st + (MODE == 0 ? ORTH_H1 : ORTH_H2);
    for(int j = warp; j <= k; j += 8) {
        double a = 0, b = 0;
        for(int blk = lane; blk < nb; blk += 32) {
            a += __ldcg(&partials[((int64_t)j * nb + blk) * 2 + 0]);
            b += __ldcg(&partials[((int64_t)j * nb + blk) * 2 + 1]);
        }
        for(int o = 16; o > 0; o >>= 1) {
            a += __shfl_xor_sync(0xffffffffu, a, o);
            b += __shfl_xor_sync(0xffffffffu, b, o);
        }
        if(lane == 0) h[2 * j] = a, h[2 * j + 1] = CPLX ? b : 0.0;
    }
    __syncthreads();
    const bool second = MODE == 1 && st[1] != 0.0;
    if(threadIdx.x == 0) {
        double hn2 = 0;
        for(int j = 0; j < k; j++) hn2 += h[2 * j] * h[2 * j] + h[2 * j + 1] * h[2 * j + 1];
        const double nrm2 = h[2 * k];
        if(MODE == 0) {
            st[0] = nrm2;
            st[3] = nrm2 - hn2;
            st[1] = (nrm2 - hn2 > 0.5 * nrm2) ? 0.0 : 1.0;  // severe cancellation: orthogonalise again
        } else if(second) {
            st[2] = nrm2;
            st[3] = nrm2 - hn2;
        }
        *counter = 0u;
    }
    __syncthreads();
    if(MODE == 0 || second) {
        for(int j = threadIdx.x; j < k; j += blockDim.x) {
            double re = st[ORTH_H1 + 2 * j], im = st[ORTH_H1 + 2 * j + 1];
            if(second) re += st[ORTH_H2 + 2 * j], im += st[ORTH_H2 + 2 * j + 1];
            hres[j] = orth_make<T>(re, im);
        }
        if(threadIdx.x == 0) {
            hres[k]     = orth_make<T>(sqrt(fmax(st[3], 0.0)), 0.0);
            hres[k + 1] = orth_make<T>(st[0], st[1]);
        }
    }
}

template<bool CPLX, int KM>
static int orth_fast(const double2 *V, int64_t ldu, int64_t nu, int k, const double2 *w, double2 *v, double *partials, unsigned *counter, double *st,
                     typename Scalar<CPLX>::T *hres, cudaStream_t s) {
    const int nb = (int)std::min<int64_t>(std::min<int64_t>(MD_BLOCKS, 4 * (int64_t)device_sm_count()), std::max<int64_t>(1, (nu + 255) / 256));
    orth_fast_kernel<CPLX, KM, 0><<<nb, 256, 0, s>>>(V, ldu, nu, k, w, nullptr, partials, counter, st, hres);
    HEFF_LAUNCH_CHECK();
    orth_fast_kernel<CPLX, KM, 1><<<nb, 256, 0, s>>>(V, ldu, nu, k, w, v, partials, counter, st, hres);
    HEFF_LAUNCH_CHECK();
    orth_fast_kernel<CPLX, KM, 2><<<nb, 256, 0, s>>>(V, ldu, nu, k, v, v, partials, counter, st, hres);
    HEFF_LAUNCH_CHECK();
    return HEFF_OK;
}

template<bool CPLX>
int orth_cgs2(const typename Scalar<CPLX>::T *V, int64_t ldv, int64_t n, int k, const typename Scalar<CPLX>::T *w, typename Scalar<CPLX>::T *v,
              double *partials, unsigned *counter, double *st, typename Scalar<CPLX>::T *hres, cudaStream_t s) {
    using T = typename Scalar<CPLX>::T;
    if(k <= 0 || k + 1 > 2 * MD_MAXK || k > MD_MAXK) return HEFF_BAD_ARG;
    // fast path: 16-byte rows (complex always; real when the rows pair up on 16-byte boundaries)
    const bool rows16 = CPLX || (n % 2 == 0 && ldv % 2 == 0 && ((uintptr_t)V & 15) == 0 && ((uintptr_t)w & 15) == 0 && ((uintptr_t)v & 15) == 0);
    if(k <= 24 && rows16) {
        const double2 *V2  = reinterpret_cast<const double2 *>(V);
        const int64_t  ldu = CPLX ? ldv : ldv / 2, nu = CPLX ? n : n / 2;
        const double2 *w2  = reinterpret_cast<const double2 *>(w);
        double2       *v2  = reinterpret_cast<double2 *>(v);
        if(k <= 8) return orth_fast<CPLX, 8>(V2, ldu, nu, k, w2, v2, partials, counter, st, hres, s);
        if(k <= 16) return orth_fast<CPLX, 16>(V2, ldu, nu, k, w2, v2, partials, counter, st, hres, s);
        return orth_fast<CPLX, 24>(V2, ldu, nu, k, w2, v2, partials, counter, st, hres, s);
    }
    const int nb = (int)std::min<int64_t>(std::min<int64_t>(MD_BLOCKS, 4 * (int64_t)device_sm_count()), std::max<int64_t>(1, (n + 255) / 256));
    orth_dot_kernel<T><<<nb, 256, 0, s>>>(V, ldv, n, k, w, partials, counter, st, hres, 0);
    HEFF_LAUNCH_CHECK();
    orth_axpy_kernel<T><<<grid_for(n), 256, sizeof(T) * k, s>>>(V, ldv, n, k, w, v, st, 0);
    HEFF_LAUNCH_CHECK();
    orth_dot_kernel<T><<<nb, 256, 0, s>>>(V, ldv, n, k, v, partials, counter, st, hres, 1);
    HEFF_LAUNCH_CHECK();
    orth_axpy_kernel<T><<<grid_for(n), 256, sizeof(T) * k, s>>>(V, ldv, n, k, v, v, st, 1);
    HEFF_LAUNCH_CHECK();
    return HEFF_OK;
}

// ---- Device-side CG for the Jacobi-Davidson correction equation ------------------------------------------------
//   (I - u u^H)(H - theta)(I - u u^H) d = -r0,   r0 and the iterates orthogonal to u (u normalised).
// All scalars live in cs[] on the device, so an iteration needs no host round trip; once CG stops (converged,
// or an indefinite direction) cs[CG_DONE] turns the remaining kernels into no-ops.  Reductions: per-block
// partial sums, then the last block to finish sums them in block order (deterministic).
enum { CG_RHO = 0, CG_RHO0, CG_ALPHA, CG_BETA, CG_CRE, CG_CIM, CG_DONE, CG_TOL2, CG_THETA, CG_SIZE };

// Fixed-order reduction of NV per-thread doubles over the grid; true in the last block, with the sums in out[].
template<int NV>
__device__ bool grid_reduce_last(double (&v)[NV], double *__restrict__ partials, unsigned *__restrict__ counter, double (&out)[NV]) {
    __shared__ double sred[8][NV];
    __shared__ double sout[NV];
    __shared__ bool   s_last;
    const int         lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nb = gridDim.x;
#pragma unroll
    for(int j = 0; j < NV; j++) {
        double a = v[j];
        for(int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
        if(lane == 0) sred[warp][j] = a;
    }
    __syncthreads();
    if(threadIdx.x < NV) {
        double a = 0;
        for(int w = 0; w < (int)(blockDim.x >> 5); w++) a += sred[w][threadIdx.x];
        partials[(int64_t)threadIdx.x * nb + blockIdx.x] = a;
    }
    __threadfence();
    __syncthreads();
    if(threadIdx.x == 0) s_last = atomicAdd(counter, 1u) == (unsigned)(nb - 1);
    __syncthreads();
    if(!s_last) return false;
    __threadfence();
    for(int j = warp; j < NV; j += (int)(blockDim.x >> 5)) {
        double a = 0;
        for(int blk = lane; blk < nb; blk += 32) a += __ldcg(&partials[(int64_t)j * nb + blk]);
        for(int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
        if(lane == 0) sout[j] = a;
    }
    __syncthreads();
    if(threadIdx.x == 0) *counter = 0u;
#pragma unroll
    for(int j = 0; j < NV; j++) out[j] = sout[j];
    return true;
}

// d = 0, r = p = -r0; scalars
template<class T>
__global__ void cg_init_kernel(T *__restrict__ d, T *__restrict__ r, T *__restrict__ p, const T *__restrict__ r0, int64_t n, double *__restrict__ cs,
                               double rho0, double theta, double tol2) {
    for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const T v = VOps<T>::scale(r0[i], -1.0);
        d[i]      = VOps<T>::zero();
        r[i]      = v;
        p[i]      = v;
    }
    if(blockIdx.x == 0 && threadIdx.x == 0) {
        cs[CG_RHO] = rho0, cs[CG_RHO0] = rho0, cs[CG_TOL2] = tol2, cs[CG_THETA] = theta;
        cs[CG_DONE] = rho0 > 0 ? 0.0 : 1.0;
    }
}

__device__ __forceinline__ void cj_acc(double &re, double &im, double a, double b) { re = fma(a, b, re); }
__device__ __forceinline__ void cj_acc(double &re, double &im, double2 a, double2 b) {
    re = fma(a.x, b.x, fma(a.y, b.y, re));  // conj(a) b
    im = fma(a.x, b.y, fma(-a.y, b.x, im));
}

// q = z - theta p;  c = u^H q, pq = Re(p^H (q - c u)) = Re(p^H q - (p^H u) c);  alpha = rho / pq (done if pq <= 0)
template<class T>
__global__ void __launch_bounds__(256) cg_a_kernel(const T *__restrict__ z, const T *__restrict__ p, const T *__restrict__ u, T *__restrict__ q,
                                                  int64_t n, double *__restrict__ cs, double *__restrict__ partials, unsigned *__restrict__ counter) {
    if(cs[CG_DONE] != 0.0) return;
    const double theta = cs[CG_THETA];
    double       v[6]  = {0, 0, 0, 0, 0, 0};  // u^H q, p^H q, p^H u (re, im)
    for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const T zi = z[i], pi = p[i], ui = u[i];
        const T qi = VOps<T>::addscaled(zi, -theta, pi);
        q[i]       = qi;
        cj_acc(v[0], v[1], ui, qi);
        cj_acc(v[2], v[3], pi, qi);
        cj_acc(v[4], v[5], pi, ui);
    }
    double s[6];
    if(!grid_reduce_last<6>(v, partials, counter, s)) return;
    if(threadIdx.x == 0) {
        const double cre = s[0], cim = s[1];
        const double pq  = s[2] - (s[4] * cre - s[5] * cim);  // Re(p^H q - (p^H u) c)
        cs[CG_CRE] = cre, cs[CG_CIM] = cim;
        if(!(pq > 0)) {
            cs[CG_DONE] = 1.0;  // indefinite direction: keep what we have
        } else {
            cs[CG_ALPHA] = cs[CG_RHO] / pq;
        }
    }
}

// q <- q - c u;  d += alpha p;  r -= alpha q;  rho' = |r|^2;  done when rho' <= tol^2 rho0;  beta = rho'/rho
template<class T>
__global__ void __launch_bounds__(256) cg_b_kernel(const T *__restrict__ q, const T *__restrict__ u, const T *__restrict__ p, T *__restrict__ d,
                                                  T *__restrict__ r, int64_t n, double *__restrict__ cs, double *__restrict__ partials,
                                                  unsigned *__restrict__ counter) {
    if(cs[CG_DONE] != 0.0) return;
    const double alpha = cs[CG_ALPHA];
    const T      c     = VOps<T>::make(cs[CG_CRE], cs[CG_CIM]);
    double       v[1]  = {0};
    for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const T ui = u[i], pi = p[i], di = d[i], ri = r[i];
        const T qp = VOps<T>::addscaled(q[i], -1.0, VOps<T>::axpy(VOps<T>::zero(), ui, c));  // q - c u
        d[i]       = VOps<T>::addscaled(di, alpha, pi);
        const T rn = VOps<T>::addscaled(ri, -alpha, qp);
        r[i]       = rn;
        double im  = 0;
        cj_acc(v[0], im, rn, rn);
    }
    double s[1];
    if(!grid_reduce_last<1>(v, partials, counter, s)) return;
    if(threadIdx.x == 0) {
        const double rho_new = s[0];
        if(rho_new <= cs[CG_TOL2] * cs[CG_RHO0]) cs[CG_DONE] = 1.0;
        cs[CG_BETA] = rho_new / cs[CG_RHO];
        cs[CG_RHO]  = rho_new;
    }
}

// p = r + beta p
template<class T>
__global__ void cg_c_kernel(const T *__restrict__ r, T *__restrict__ p, int64_t n, const double *__restrict__ cs) {
    if(cs[CG_DONE] != 0.0) return;
    const double beta = cs[CG_BETA];
    for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        p[i] = VOps<T>::addscaled(r[i], beta, p[i]);
}

template<bool CPLX>
int cg_init(typename Scalar<CPLX>::T *d, typename Scalar<CPLX>::T *r, typename Scalar<CPLX>::T *p, const typename Scalar<CPLX>::T *r0, int64_t n,
            double *cs, double rho0, double theta, double tol2, cudaStream_t s) {
    cg_init_kernel<typename Scalar<CPLX>::T><<<grid_for(n), 256, 0, s>>>(d, r, p, r0, n, cs, rho0, theta, tol2);
    HEFF_LAUNCH_CHECK();
    return HEFF_OK;
}

template<bool CPLX>
int cg_step(const typename Scalar<CPLX>::T *z, typename Scalar<CPLX>::T *p, const typename Scalar<CPLX>::T *u, typename Scalar<CPLX>::T *q,
            typename Scalar<CPLX>::T *d, typename Scalar<CPLX>::T *r, int64_t n, double *cs, double *partials, unsigned *counter, cudaStream_t s) {
    using T      = typename Scalar<CPLX>::T;
    const int nb = (int)std::min<int64_t>(std::min<int64_t>(MD_BLOCKS, 4 * (int64_t)device_sm_count()), std::max<int64_t>(1, (n + 255) / 256));
    cg_a_kernel<T><<<nb, 256, 0, s>>>(z, p, u, q, n, cs, partials, counter);
    HEFF_LAUNCH_CHECK();
    cg_b_kernel<T><<<nb, 256, 0, s>>>(q, u, p, d, r, n, cs, partials, counter);
    HEFF_LAUNCH_CHECK();
    cg_c_kernel<T><<<grid_for(n), 256, 0, s>>>(r, p, n, cs);
    HEFF_LAUNCH_CHECK();
    return HEFF_OK;
}

#define INST(C)                                                                                                                              \
    template int multi_dot<C>(const Scalar<C>::T *, int64_t, int64_t, int, const Scalar<C>::T *, Scalar<C>::T *, double *, cudaStream_t);   \
    template int multi_axpy<C>(const Scalar<C>::T *, int64_t, int64_t, int, const Scalar<C>::T *, double, Scalar<C>::T *, cudaStream_t);   \
    template int combine<C>(const Scalar<C>::T *, int64_t, int64_t, int, const Scalar<C>::T *, Scalar<C>::T *, cudaStream_t);              \
    template int scale_dev<C>(Scalar<C>::T *, int64_t, const double *, bool, cudaStream_t);                                             \
    template int residual<C>(const Scalar<C>::T *, const Scalar<C>::T *, double, Scalar<C>::T *, int64_t, cudaStream_t);                  \
    template int cg_init<C>(Scalar<C>::T *, Scalar<C>::T *, Scalar<C>::T *, const Scalar<C>::T *, int64_t, double *, double, double, double,      \
                            cudaStream_t);                                                                                               \
    template int cg_step<C>(const Scalar<C>::T *, Scalar<C>::T *, const Scalar<C>::T *, Scalar<C>::T *, Scalar<C>::T *, Scalar<C>::T *, int64_t, \
                            double *, double *, unsigned *, cudaStream_t);                                                               \
    template int orth_cgs2<C>(const Scalar<C>::T *, int64_t, int64_t, int, const Scalar<C>::T *, Scalar<C>::T *, double *, unsigned *,     \
                              double *, Scalar<C>::T *, cudaStream_t);
INST(false)
INST(true)
#undef INST

}  // namespace heff
