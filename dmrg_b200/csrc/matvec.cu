// H_eff * theta: layout kernels, MPO mixing kernel, matvec driver, expectation value,
// and the stateless C entry points heff_matvec_{d,z} / heff_expval_{d,z}.
#include <algorithm>
#include "matvec.cuh"
#include "runtime.cuh"
#include "wlist.cuh"

namespace heff {

int check_matvec_dims(const int64_t md[3], const int64_t wd[4], const int64_t ld[3], const int64_t rd[3], MatvecDims &d) {
    if(!md || !wd || !ld || !rd) return HEFF_BAD_ARG;
    d = MatvecDims{md[0], md[1], md[2], wd[0], wd[1]};
    // contraction_tblis.cpp:230-234
    if(md[1] != ld[0] || md[2] != rd[0] || md[0] != wd[2] || ld[2] != wd[0] || rd[2] != wd[1]) {
        set_last_error_msg("matvec: dimension mismatch mps [%lld,%lld,%lld] mpo [%lld,%lld,%lld,%lld] envL [%lld,%lld,%lld] envR [%lld,%lld,%lld]",
                           (long long)md[0], (long long)md[1], (long long)md[2], (long long)wd[0], (long long)wd[1], (long long)wd[2],
                           (long long)wd[3], (long long)ld[0], (long long)ld[1], (long long)ld[2], (long long)rd[0], (long long)rd[1],
                           (long long)rd[2]);
        return HEFF_BAD_SHAPE;
    }
    if(wd[3] != wd[2] || ld[1] != ld[0] || rd[1] != rd[0]) {
        set_last_error_msg("matvec: mpo must be [mL,mR,d,d] and envs [chi,chi,m]");
        return HEFF_BAD_SHAPE;
    }
    if(d.S <= 0 || d.cL <= 0 || d.cR <= 0 || d.DL <= 0 || d.DR <= 0) return HEFF_BAD_SHAPE;
    if(d.S > 64 || d.DL * d.S > 256 || d.DR * d.S > 256) {
        set_last_error_msg("matvec: spin*mpo bond dimension above 256 is not supported");
        return HEFF_BAD_SHAPE;
    }
    if(d.cL > (1 << 20) || d.cR > (1 << 20)) return HEFF_BAD_SHAPE;
    return HEFF_OK;
}

// x'[a + cL*(s + S*b)] = x[s + S*(a + cL*b)]   (output-linear: coalesced writes)
template<class T>
__global__ void permute_mps_kernel(const T *__restrict__ x, T *__restrict__ xp, int64_t S, int64_t cL, int64_t n) {
    for(int64_t o = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; o < n; o += (int64_t)gridDim.x * blockDim.x) {
        const int64_t a = o % cL, r = o / cL, s = r % S, b = r / S;
        xp[o]           = x[s + S * (a + cL * b)];
    }
}

// x'[o] for o in [o0, o1) (the x' columns (s,b) of a slab of b)
template<class T>
__global__ void permute_mps_range_kernel(const T *__restrict__ x, T *__restrict__ xp, int64_t S, int64_t cL, int64_t o0, int64_t o1) {
    for(int64_t o = o0 + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; o < o1; o += (int64_t)gridDim.x * blockDim.x) {
        const int64_t a = o % cL, r = o / cL, s = r % S, b = r / S;
        xp[o]           = x[s + S * (a + cL * b)];
    }
}

// R'[b + cR*n + cR*DR*b'] = R[b + cR*(b' + cR*n)]
template<class T>
__global__ void permute_R_kernel(const T *__restrict__ R, T *__restrict__ Rp, int64_t cR, int64_t DR, int64_t n) {
    for(int64_t o = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; o < n; o += (int64_t)gridDim.x * blockDim.x) {
        const int64_t b = o % cR, r = o / cR, nn = r % DR, bp = r / DR;
        Rp[o]           = R[b + cR * (bp + cR * nn)];
    }
}

__device__ __forceinline__ bool is_zero(double w) { return w == 0.0; }
__device__ __forceinline__ bool is_zero(double2 w) { return w.x == 0.0 && w.y == 0.0; }
__device__ __forceinline__ double fma_s(double w, double v, double acc) { return fma(w, v, acc); }
__device__ __forceinline__ double2 fma_s(double2 w, double2 v, double2 acc) {
    return make_double2(fma(w.x, v.x, fma(-w.y, v.y, acc.x)), fma(w.x, v.y, fma(w.y, v.x, acc.y)));
}
__device__ __forceinline__ void zero(double &v) { v = 0.0; }
__device__ __forceinline__ void zero(double2 &v) { v = make_double2(0.0, 0.0); }

// T2[(s' + S a') + S cL (b + cR n)] = sum_{m,s} W[m + DL(n + DR(s + S s'))] T1[(a' + cL m) + cL DL (s + S b)]
// One CTA: 128 consecutive a' at one b.  W, its nonzero list (wlist.cuh) and the CTA's T1 column block are
// staged in shared memory; each output runs only over the nonzero MPO entries.
constexpr int MIX_THREADS = 128;
template<class T>
__global__ void __launch_bounds__(MIX_THREADS) mix_kernel(const T *__restrict__ T1, T *__restrict__ T2, const T *__restrict__ W, int S, int cL,
                                                         int cR, int DL, int DR, int b0) {
    extern __shared__ __align__(16) unsigned char mix_smem[];
    T        *sW  = reinterpret_cast<T *>(mix_smem);
    const int nW  = DL * DR * S * S;
    T        *sIn = sW + nW;
    unsigned char *lmem = reinterpret_cast<unsigned char *>(sIn + (size_t)DL * S * MIX_THREADS);
    for(int i = threadIdx.x; i < nW; i += blockDim.x) sW[i] = W[i];
    const int     b   = b0 + blockIdx.y;  // columns b0 .. b0 + gridDim.y - 1
    const int     ap  = blockIdx.x * MIX_THREADS + threadIdx.x;
    const bool    act = ap < cL;
    const int64_t cLD = (int64_t)cL * DL;
    // 8 loads in flight per thread before their shared-memory stores (slot ms = m*S + s)
    const int NP = DL * S;
    for(int ms0 = 0; ms0 < NP; ms0 += 8) {
        T v[8];
#pragma unroll
        for(int u = 0; u < 8; u++) {
            const int ms = ms0 + u, m = ms / S, s = ms % S;
            zero(v[u]);
            if(act && ms < NP) v[u] = T1[(ap + (int64_t)cL * m) + cLD * (s + (int64_t)S * b)];
        }
#pragma unroll
        for(int u = 0; u < 8; u++)
            if(ms0 + u < NP) sIn[(ms0 + u) * MIX_THREADS + threadIdx.x] = v[u];
    }
    __syncthreads();
    int   *off;
    short *idx;
    T     *wv;
    build_wlist(sW, DL, DR, S, lmem, off, idx, wv);
    if(!act) return;
    for(int n = 0; n < DR; n++) {
        T *out = T2 + ((int64_t)S * ap) + (int64_t)S * cL * (b + (int64_t)cR * n);
        for(int sp = 0; sp < S; sp++) {
            const int o = n * S + sp;
            T         acc;
            zero(acc);
            for(int e = off[o]; e < off[o + 1]; e++) acc = fma_s(wv[e], sIn[idx[e] * MIX_THREADS + threadIdx.x], acc);
            out[sp] = acc;
        }
    }
}

static int grid_1d(int64_t n) {
    int64_t g = (n + 255) / 256;
    int64_t cap = (int64_t)device_sm_count() * 16;
    return (int)(g < cap ? (g > 0 ? g : 1) : cap);
}

template<bool CPLX>
int permute_R(const typename Scalar<CPLX>::T *R, typename Scalar<CPLX>::T *Rp, const MatvecDims &d, cudaStream_t s) {
    const int64_t n = d.size_Rp();
    permute_R_kernel<<<grid_1d(n), 256, 0, s>>>(R, Rp, d.cR, d.DR, n);
    HEFF_LAUNCH_CHECK();
    return HEFF_OK;
}

template<bool CPLX>
static int launch_mix(const MatvecDims &d, const typename Scalar<CPLX>::T *T1, typename Scalar<CPLX>::T *T2, const typename Scalar<CPLX>::T *W,
                      cudaStream_t s, int64_t b0 = 0, int64_t nb = -1) {
    using T           = typename Scalar<CPLX>::T;
    const size_t smem = sizeof(T) * ((size_t)d.DL * d.DR * d.S * d.S + (size_t)d.DL * d.S * MIX_THREADS) +
                        wlist_bytes((int)d.DL, (int)d.DR, (int)d.S, sizeof(T));
    if(smem > 200 * 1024) return HEFF_BAD_SHAPE;
    static int attr_done[64] = {0};
    int        dev           = 0;
    HEFF_CUDA(cudaGetDevice(&dev));
    if(dev < 0 || dev >= 64 || !attr_done[dev]) {
        HEFF_CUDA(cudaFuncSetAttribute(mix_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
        if(dev >= 0 && dev < 64) attr_done[dev] = 1;
    }
    if(nb < 0) nb = d.cR;
    if(nb > 65535) return HEFF_BAD_SHAPE;
    if(nb == 0) return HEFF_OK;
    dim3 grid((unsigned)cdiv(d.cL, MIX_THREADS), (unsigned)nb);
    mix_kernel<T><<<grid, MIX_THREADS, smem, s>>>(T1, T2, W, (int)d.S, (int)d.cL, (int)d.cR, (int)d.DL, (int)d.DR, (int)b0);
    HEFF_LAUNCH_CHECK();
    return HEFF_OK;
}

template<bool CPLX>
int matvec_fp64(const MatvecDims &d, const typename Scalar<CPLX>::T *x, typename Scalar<CPLX>::T *y, const typename Scalar<CPLX>::T *L,
                const typename Scalar<CPLX>::T *Rp, const typename Scalar<CPLX>::T *W, const MatvecScratch<CPLX> &ws, cudaStream_t s,
                cudaEvent_t *ev) {
    const int64_t n = d.size_mps();
    if(ev) HEFF_CUDA(cudaEventRecord(ev[0], s));
    permute_mps_kernel<<<grid_1d(n), 256, 0, s>>>(x, ws.xp, d.S, d.cL, n);
    HEFF_LAUNCH_CHECK();
    count_launches(2);  // the permutation and the MPO mix below (the GEMM launcher counts its own kernels)
    if(ev) HEFF_CUDA(cudaEventRecord(ev[1], s));
    GemmArgs g1{};
    g1.M     = (int)(d.cL * d.DL);
    g1.N     = (int)(d.S * d.cR);
    g1.K     = (int)d.cL;
    g1.batch = 1;
    g1.A     = L;
    g1.lda   = d.cL;
    g1.B     = ws.xp;
    g1.ldb   = d.cL;
    g1.C     = ws.T1;
    g1.ldc   = d.cL * d.DL;
    g1.alpha = make_double2(1.0, 0.0);
    g1.beta  = make_double2(0.0, 0.0);
    g1.split_ws       = ws.split_ws;
    g1.split_ws_bytes = ws.split_bytes;
    HEFF_TRY(gemm_f64<CPLX>(/*ta=*/true, /*tb=*/false, false, g1, s));
    if(ev) HEFF_CUDA(cudaEventRecord(ev[2], s));
    HEFF_TRY(launch_mix<CPLX>(d, ws.T1, ws.T2, W, s));
    if(ev) HEFF_CUDA(cudaEventRecord(ev[3], s));
    GemmArgs g2{};
    g2.M     = (int)(d.S * d.cL);
    g2.N     = (int)d.cR;
    g2.K     = (int)(d.cR * d.DR);
    g2.batch = 1;
    g2.A     = ws.T2;
    g2.lda   = d.S * d.cL;
    g2.B     = Rp;
    g2.ldb   = d.cR * d.DR;
    g2.C     = y;
    g2.ldc   = d.S * d.cL;
    g2.alpha = make_double2(1.0, 0.0);
    g2.beta  = make_double2(0.0, 0.0);
    g2.split_ws       = ws.split_ws;
    g2.split_ws_bytes = ws.split_bytes;
    HEFF_TRY(gemm_f64<CPLX>(false, false, false, g2, s));
    if(ev) HEFF_CUDA(cudaEventRecord(ev[4], s));
    return HEFF_OK;
}

// First two stages of the matvec with alpha folded into GEMM 1 and the mix written to `out`:
//   out[s' + S (a' + cL (b + cR n))] = alpha * sum_{a,m,s} L[a,a',m] x[s,a,b] W[m,n,s,s']
// which is the L-side subspace-expansion term P of EnvBase::get_expansion_term (EnvBase.cpp:303-333).
template<bool CPLX>
int matvec_left_stages(const MatvecDims &d, const typename Scalar<CPLX>::T *x, const typename Scalar<CPLX>::T *L, const typename Scalar<CPLX>::T *W,
                       typename Scalar<CPLX>::T *out, typename Scalar<CPLX>::T *xp, typename Scalar<CPLX>::T *T1, double alpha, cudaStream_t s) {
    const int64_t n = d.size_mps();
    permute_mps_kernel<<<grid_1d(n), 256, 0, s>>>(x, xp, d.S, d.cL, n);
    HEFF_LAUNCH_CHECK();
    GemmArgs g1{};
    g1.M     = (int)(d.cL * d.DL);
    g1.N     = (int)(d.S * d.cR);
    g1.K     = (int)d.cL;
    g1.batch = 1;
    g1.A     = L;
    g1.lda   = d.cL;
    g1.B     = xp;
    g1.ldb   = d.cL;
    g1.C     = T1;
    g1.ldc   = d.cL * d.DL;
    g1.alpha = make_double2(alpha, 0.0);
    g1.beta  = make_double2(0.0, 0.0);
    HEFF_TRY(gemm_f64<CPLX>(/*ta=*/true, /*tb=*/false, false, g1, s));
    return launch_mix<CPLX>(d, T1, out, W, s);
}

// y = H_eff x with x and y in HOST memory, copies overlapped with the computation.  The slab of theta with
// columns b in [b0, b1) is contiguous (theta[s + S(a + cL b)]), and GEMM 1 and the mix of that slab need
// nothing else: slab c is copied in on the copy stream and processed on compute stream c % 2 as soon as it
// has landed.  GEMM 2's output columns b' are independent: slab c' of y is computed on stream c' % 2 once
// every mix is done and copied out right after.  Two compute streams let a slab's GEMM fill the tail wave of
// the previous one.  Synchronises before returning.
template<bool CPLX>
int matvec_fp64_host(const MatvecDims &d, const typename Scalar<CPLX>::T *xh, typename Scalar<CPLX>::T *yh, const typename Scalar<CPLX>::T *L,
                     const typename Scalar<CPLX>::T *Rp, const typename Scalar<CPLX>::T *W, const MatvecScratch<CPLX> &ws, typename Scalar<CPLX>::T *dx,
                     typename Scalar<CPLX>::T *dy, const HostPipe &hp) {
    using T               = typename Scalar<CPLX>::T;
    const int         nin = (int)std::min<int64_t>(hp.n_in, d.cR), nout = (int)std::min<int64_t>(hp.n_out, d.cR);
    cudaStream_t      cs[2] = {hp.s, hp.aux};
    const int64_t     colx = d.S * d.cL;  // elements per b column of theta / y
    auto              slab = [&](int c, int nc, int64_t &b0, int64_t &b1) {
        b0 = d.cR * c / nc;
        b1 = d.cR * (c + 1) / nc;
    };
    // everything queued on the caller's stream before this call precedes the copies into dx
    HEFF_CUDA(cudaEventRecord(hp.ev[0], hp.s));
    HEFF_CUDA(cudaStreamWaitEvent(hp.copy, hp.ev[0], 0));
    HEFF_CUDA(cudaStreamWaitEvent(hp.aux, hp.ev[0], 0));
    for(int c = 0; c < nin; c++) {
        int64_t b0, b1;
        slab(c, nin, b0, b1);
        if(b1 == b0) continue;
        HEFF_CUDA(cudaMemcpyAsync(dx + colx * b0, xh + colx * b0, sizeof(T) * colx * (b1 - b0), cudaMemcpyHostToDevice, hp.copy));
        HEFF_CUDA(cudaEventRecord(hp.ev[1 + c], hp.copy));
        cudaStream_t s = cs[c & 1];
        HEFF_CUDA(cudaStreamWaitEvent(s, hp.ev[1 + c], 0));
        const int64_t o0 = d.cL * d.S * b0, o1 = d.cL * d.S * b1;
        permute_mps_range_kernel<<<grid_1d(o1 - o0), 256, 0, s>>>(dx, ws.xp, d.S, d.cL, o0, o1);
        HEFF_LAUNCH_CHECK();
        GemmArgs g1{};
        g1.M = (int)(d.cL * d.DL), g1.N = (int)(d.S * (b1 - b0)), g1.K = (int)d.cL, g1.batch = 1;
        g1.A = L, g1.lda = d.cL, g1.B = ws.xp + o0, g1.ldb = d.cL, g1.C = ws.T1 + d.cL * d.DL * d.S * b0, g1.ldc = d.cL * d.DL;
        g1.alpha = make_double2(1.0, 0.0), g1.beta = make_double2(0.0, 0.0);
        HEFF_TRY(gemm_f64<CPLX>(/*ta=*/true, /*tb=*/false, false, g1, s));
        HEFF_TRY(launch_mix<CPLX>(d, ws.T1, ws.T2, W, s, b0, b1 - b0));
    }
    // every mix (both streams) before any GEMM 2 slab
    HEFF_CUDA(cudaEventRecord(hp.ev[HostPipe::MAXS + 1], hp.aux));
    HEFF_CUDA(cudaStreamWaitEvent(hp.s, hp.ev[HostPipe::MAXS + 1], 0));
    HEFF_CUDA(cudaEventRecord(hp.ev[HostPipe::MAXS + 2], hp.s));
    HEFF_CUDA(cudaStreamWaitEvent(hp.aux, hp.ev[HostPipe::MAXS + 2], 0));
    for(int c = 0; c < nout; c++) {
        int64_t b0, b1;
        slab(c, nout, b0, b1);
        if(b1 == b0) continue;
        cudaStream_t s = cs[c & 1];
        GemmArgs     g2{};
        g2.M = (int)(d.S * d.cL), g2.N = (int)(b1 - b0), g2.K = (int)(d.cR * d.DR), g2.batch = 1;
        g2.A = ws.T2, g2.lda = d.S * d.cL, g2.B = Rp + d.cR * d.DR * b0, g2.ldb = d.cR * d.DR, g2.C = dy + colx * b0, g2.ldc = d.S * d.cL;
        g2.alpha = make_double2(1.0, 0.0), g2.beta = make_double2(0.0, 0.0);
        HEFF_TRY(gemm_f64<CPLX>(false, false, false, g2, s));
        HEFF_CUDA(cudaEventRecord(hp.ev[HostPipe::MAXS + 3 + c], s));
        HEFF_CUDA(cudaStreamWaitEvent(hp.copy, hp.ev[HostPipe::MAXS + 3 + c], 0));
        HEFF_CUDA(cudaMemcpyAsync(yh + colx * b0, dy + colx * b0, sizeof(T) * colx * (b1 - b0), cudaMemcpyDeviceToHost, hp.copy));
    }
    // the caller's stream resumes after the last copy out; the host waits for it
    HEFF_CUDA(cudaEventRecord(hp.ev[2 * HostPipe::MAXS + 3], hp.copy));
    HEFF_CUDA(cudaStreamWaitEvent(hp.s, hp.ev[2 * HostPipe::MAXS + 3], 0));
    HEFF_CUDA(cudaStreamSynchronize(hp.s));
    return HEFF_OK;
}

// ---- deterministic dot product ----
constexpr int DOT_BLOCKS = 1024;
template<bool CPLX>
__global__ void dot_partial_kernel(const typename Scalar<CPLX>::T *__restrict__ x, const typename Scalar<CPLX>::T *__restrict__ y, int64_t n,
                                   double *partials) {
    __shared__ double sre[256], sim[256];
    double            re = 0, im = 0;
    for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        if constexpr(CPLX) {
            double2 a = x[i], b = y[i];
            re += a.x * b.x + a.y * b.y;  // conj(a) * b
            im += a.x * b.y - a.y * b.x;
        } else {
            re += x[i] * y[i];
        }
    }
    sre[threadIdx.x] = re;
    sim[threadIdx.x] = im;
    __syncthreads();
    for(int w = 128; w > 0; w >>= 1) {
        if(threadIdx.x < w) {
            sre[threadIdx.x] += sre[threadIdx.x + w];
            sim[threadIdx.x] += sim[threadIdx.x + w];
        }
        __syncthreads();
    }
    if(threadIdx.x == 0) {
        partials[blockIdx.x]              = sre[0];
        partials[DOT_BLOCKS + blockIdx.x] = sim[0];
    }
}
template<bool CPLX>
__global__ void dot_final_kernel(const double *partials, int nb, typename Scalar<CPLX>::T *out) {
    __shared__ double sre[256], sim[256];
    double            re = 0, im = 0;
    for(int i = threadIdx.x; i < nb; i += 256) {
        re += partials[i];
        im += partials[DOT_BLOCKS + i];
    }
    sre[threadIdx.x] = re;
    sim[threadIdx.x] = im;
    __syncthreads();
    for(int w = 128; w > 0; w >>= 1) {
        if(threadIdx.x < w) {
            sre[threadIdx.x] += sre[threadIdx.x + w];
            sim[threadIdx.x] += sim[threadIdx.x + w];
        }
        __syncthreads();
    }
    if(threadIdx.x == 0) {
        if constexpr(CPLX)
            *out = make_double2(sre[0], sim[0]);
        else
            *out = sre[0];
    }
}

template<bool CPLX>
int dot_device(const typename Scalar<CPLX>::T *x, const typename Scalar<CPLX>::T *y, int64_t n, typename Scalar<CPLX>::T *out, double *partials,
               cudaStream_t s) {
    int nb = (int)std::min<int64_t>(DOT_BLOCKS, std::max<int64_t>(1, (n + 255) / 256));
    dot_partial_kernel<CPLX><<<nb, 256, 0, s>>>(x, y, n, partials);
    HEFF_LAUNCH_CHECK();
    dot_final_kernel<CPLX><<<1, 256, 0, s>>>(partials, nb, out);
    HEFF_LAUNCH_CHECK();
    return HEFF_OK;
}

const void *permute_kernel_fn(bool cplx) {
    return cplx ? reinterpret_cast<const void *>(permute_mps_kernel<double2>) : reinterpret_cast<const void *>(permute_mps_kernel<double>);
}

template<bool CPLX>
int permute_mps(const MatvecDims &d, const typename Scalar<CPLX>::T *x, typename Scalar<CPLX>::T *xp, cudaStream_t s) {
    const int64_t n = d.size_mps();
    permute_mps_kernel<<<grid_1d(n), 256, 0, s>>>(x, xp, d.S, d.cL, n);
    HEFF_LAUNCH_CHECK();
    return HEFF_OK;
}
template<bool CPLX>
int mix_fp64(const MatvecDims &d, const typename Scalar<CPLX>::T *T1, typename Scalar<CPLX>::T *T2, const typename Scalar<CPLX>::T *W, cudaStream_t s) {
    return launch_mix<CPLX>(d, T1, T2, W, s);
}
template int permute_mps<false>(const MatvecDims &, const double *, double *, cudaStream_t);
template int permute_mps<true>(const MatvecDims &, const double2 *, double2 *, cudaStream_t);
template int mix_fp64<false>(const MatvecDims &, const double *, double *, const double *, cudaStream_t);
template int mix_fp64<true>(const MatvecDims &, const double2 *, double2 *, const double2 *, cudaStream_t);
template int permute_R<false>(const double *, double *, const MatvecDims &, cudaStream_t);
template int permute_R<true>(const double2 *, double2 *, const MatvecDims &, cudaStream_t);
template int matvec_fp64<false>(const MatvecDims &, const double *, double *, const double *, const double *, const double *,
                                const MatvecScratch<false> &, cudaStream_t, cudaEvent_t *);
template int matvec_fp64<true>(const MatvecDims &, const double2 *, double2 *, const double2 *, const double2 *, const double2 *,
                               const MatvecScratch<true> &, cudaStream_t, cudaEvent_t *);
template int matvec_left_stages<false>(const MatvecDims &, const double *, const double *, const double *, double *, double *, double *, double,
                                       cudaStream_t);
template int matvec_left_stages<true>(const MatvecDims &, const double2 *, const double2 *, const double2 *, double2 *, double2 *, double2 *, double,
                                      cudaStream_t);
template int matvec_fp64_host<false>(const MatvecDims &, const double *, double *, const double *, const double *, const double *,
                                     const MatvecScratch<false> &, double *, double *, const HostPipe &);
template int matvec_fp64_host<true>(const MatvecDims &, const double2 *, double2 *, const double2 *, const double2 *, const double2 *,
                                    const MatvecScratch<true> &, double2 *, double2 *, const HostPipe &);
template int dot_device<false>(const double *, const double *, int64_t, double *, double *, cudaStream_t);
template int dot_device<true>(const double2 *, const double2 *, int64_t, double2 *, double *, cudaStream_t);

// ---- stateless entry points ----
template<bool CPLX>
static int matvec_stateless(void *res, const void *mps, const int64_t md[3], const void *mpo, const int64_t wd[4], const void *envL,
                            const int64_t ld[3], const void *envR, const int64_t rd[3], cudaStream_t s) {
    using T = typename Scalar<CPLX>::T;
    MatvecDims d;
    HEFF_TRY(check_matvec_dims(md, wd, ld, rd, d));
    if(!res || !mps || !mpo || !envL || !envR) return HEFF_BAD_ARG;
    if(res == mps) {
        set_last_error_msg("matvec: res must not alias mps");
        return HEFF_BAD_ARG;
    }
    const int64_t elems = MatvecScratch<CPLX>::elems(d) + MatvecScratch<CPLX>::pad(d.size_Rp());
    const size_t  split = matvec_split_bytes((size_t)elems * sizeof(T));
    void         *base  = nullptr;
    HEFF_TRY(stream_workspace(s, (size_t)elems * sizeof(T) + split, &base));
    MatvecScratch<CPLX> ws;
    T                  *Rp = ws.carve(reinterpret_cast<T *>(base), d);
    ws.split_ws           = reinterpret_cast<unsigned char *>(base) + (size_t)elems * sizeof(T);
    ws.split_bytes        = split;
    HEFF_TRY(permute_R<CPLX>(reinterpret_cast<const T *>(envR), Rp, d, s));
    return matvec_fp64<CPLX>(d, reinterpret_cast<const T *>(mps), reinterpret_cast<T *>(res), reinterpret_cast<const T *>(envL), Rp,
                             reinterpret_cast<const T *>(mpo), ws, s);
}

template<bool CPLX>
static int expval_stateless(double *result, const void *mps, const int64_t md[3], const void *mpo, const int64_t wd[4], const void *envL,
                            const int64_t ld[3], const void *envR, const int64_t rd[3], cudaStream_t s) {
    using T = typename Scalar<CPLX>::T;
    MatvecDims d;
    HEFF_TRY(check_matvec_dims(md, wd, ld, rd, d));
    if(!result || !mps || !mpo || !envL || !envR) return HEFF_BAD_ARG;
    const int64_t extra = MatvecScratch<CPLX>::pad(d.size_Rp()) + MatvecScratch<CPLX>::pad(d.size_mps()) + 1;
    const int64_t elems = MatvecScratch<CPLX>::elems(d) + extra;
    void         *base  = nullptr;
    HEFF_TRY(stream_workspace(s, (size_t)elems * sizeof(T) + 2 * DOT_BLOCKS * sizeof(double), &base));
    MatvecScratch<CPLX> ws;
    T      *Rp       = ws.carve(reinterpret_cast<T *>(base), d);
    T      *y        = Rp + MatvecScratch<CPLX>::pad(d.size_Rp());
    T      *dres     = y + d.size_mps();
    double *partials = reinterpret_cast<double *>(dres + 1);
    HEFF_TRY(permute_R<CPLX>(reinterpret_cast<const T *>(envR), Rp, d, s));
    HEFF_TRY(matvec_fp64<CPLX>(d, reinterpret_cast<const T *>(mps), y, reinterpret_cast<const T *>(envL), Rp, reinterpret_cast<const T *>(mpo),
                               ws, s));
    HEFF_TRY(dot_device<CPLX>(reinterpret_cast<const T *>(mps), y, d.size_mps(), dres, partials, s));
    T h;
    HEFF_CUDA(cudaMemcpyAsync(&h, dres, sizeof(T), cudaMemcpyDeviceToHost, s));
    HEFF_CUDA(cudaStreamSynchronize(s));
    if constexpr(CPLX) {
        result[0] = h.x;
        result[1] = h.y;
    } else {
        result[0] = h;
        result[1] = 0.0;
    }
    return HEFF_OK;
}

}  // namespace heff

using namespace heff;

extern "C" int heff_matvec_d(double *res, const double *mps, const int64_t mps_dims[3], const double *mpo, const int64_t mpo_dims[4],
                             const double *envL, const int64_t envL_dims[3], const double *envR, const int64_t envR_dims[3], void *stream) {
    return matvec_stateless<false>(res, mps, mps_dims, mpo, mpo_dims, envL, envL_dims, envR, envR_dims, (cudaStream_t)stream);
}
extern "C" int heff_matvec_z(heff_z *res, const heff_z *mps, const int64_t mps_dims[3], const heff_z *mpo, const int64_t mpo_dims[4],
                             const heff_z *envL, const int64_t envL_dims[3], const heff_z *envR, const int64_t envR_dims[3], void *stream) {
    return matvec_stateless<true>(res, mps, mps_dims, mpo, mpo_dims, envL, envL_dims, envR, envR_dims, (cudaStream_t)stream);
}
extern "C" int heff_expval_d(double *result, const double *mps, const int64_t mps_dims[3], const double *mpo, const int64_t mpo_dims[4],
                             const double *envL, const int64_t envL_dims[3], const double *envR, const int64_t envR_dims[3], void *stream) {
    return expval_stateless<false>(result, mps, mps_dims, mpo, mpo_dims, envL, envL_dims, envR, envR_dims, (cudaStream_t)stream);
}
extern "C" int heff_expval_z(double *result, const heff_z *mps, const int64_t mps_dims[3], const heff_z *mpo, const int64_t mpo_dims[4],
                             const heff_z *envL, const int64_t envL_dims[3], const heff_z *envR, const int64_t envR_dims[3], void *stream) {
    return expval_stateless<true>(result, mps, mps_dims, mpo, mpo_dims, envL, envL_dims, envR, envR_dims, (cudaStream_t)stream);
}
