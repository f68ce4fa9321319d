// L/R environment ("edge") update: EnvBase::build_block (source/tensors/site/env/EnvBase.cpp:67-151).
//
// L side (EnvBase.cpp:109-112):  L'[b,b',n] = sum M[s,a,b] L[a,a',m] conj(M)[s',a',b'] W[m,n,s,s']
//   E1  X_m[a,(s',b')]      = sum_a' L[a,a',m] Mc[a',(s',b')]          batched DMMA GEMM over m
//   E2  Y[(s,a),(b',n)]     = sum_{m,s'} W[m,n,s,s'] X_m[a,(s',b')]     mix kernel per (a,b')
//   E3  L'[b,(b',n)]        = sum_{(s,a)} M[(s,a),b] Y[(s,a),(b',n)]     DMMA GEMM (A = M read as K x M)
// R side (EnvBase.cpp:146-149):  R'[a,a',m] = sum M[s,a,b] R[b,b',n] conj(M)[s',a',b'] W[m,n,s,s']
//   E1  X_n[b,(s',a')]      = sum_b' R[b,b',n] conj(M)[(s',a'),b']      batched DMMA GEMM over n (B read transposed)
//   E2  Y[(s,b),(a',m)]     = sum_{n,s'} W[m,n,s,s'] X_n[b,(s',a')]     mix kernel per (b,a')
//   E3  R'[a,(a',m)]        = sum_{(s,b)} M2[(s,b),a] Y[(s,b),(a',m)]    DMMA GEMM, M2 = M with (a,b) swapped
// FLOPs per update (chiL = chiR = chi, d = 2): 8 D chi^3 + 8 D^2 chi^2 (x4 complex).
#include "env.cuh"
#include "matvec.cuh"
#include "runtime.cuh"

namespace heff {

__device__ __forceinline__ double conj_s(double v) { return v; }
__device__ __forceinline__ double2 conj_s(double2 v) { return make_double2(v.x, -v.y); }
__device__ __forceinline__ double fma_e(double w, double v, double acc) { return fma(w, v, acc); }
__device__ __forceinline__ double2 fma_e(double2 w, double2 v, double2 acc) {
    return make_double2(fma(w.x, v.x, fma(-w.y, v.y, acc.x)), fma(w.x, v.y, fma(w.y, v.x, acc.y)));
}
__device__ __forceinline__ bool nz(double w) { return w != 0.0; }
__device__ __forceinline__ bool nz(double2 w) { return w.x != 0.0 || w.y != 0.0; }
__device__ __forceinline__ void setz(double &v) { v = 0.0; }
__device__ __forceinline__ void setz(double2 &v) { v = make_double2(0.0, 0.0); }

// Mc[a' + cL*(s' + d*b')] = conj(M[s' + d*(a' + cL*b')])
template<class T>
__global__ void env_prep_L(const T *__restrict__ M, T *__restrict__ Mc, int64_t d, int64_t cL, int64_t n) {
    for(int64_t o = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; o < n; o += (int64_t)gridDim.x * blockDim.x) {
        const int64_t ap = o % cL, r = o / cL, sp = r % d, bp = r / d;
        Mc[o]            = conj_s(M[sp + d * (ap + cL * bp)]);
    }
}
// Mc[i] = conj(M[i]);  M2[s + d*(b + cR*a)] = M[s + d*(a + cL*b)]
template<class T>
__global__ void env_prep_R(const T *__restrict__ M, T *__restrict__ Mc, T *__restrict__ M2, int64_t d, int64_t cL, int64_t cR, int64_t n) {
    for(int64_t o = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; o < n; o += (int64_t)gridDim.x * blockDim.x) {
        Mc[o]           = conj_s(M[o]);
        const int64_t s = o % d, r = o / d, b = r % cR, a = r / cR;
        M2[o]           = M[s + d * (a + cL * b)];
    }
}

// Mix of both sides. One thread per (p, q): p runs over the contiguous index of X (a for L, b for R),
// q over the other point index (b' for L, a' for R).
//   in[k, s'] = X[p + P*(s' + d*q) + P*d*Q*k]      (k = m for L, n for R)
//   out[j, s] = Y[s + d*p + d*P*(q + Q*j)]         (j = n for L, m for R)
//   L: out[n,s] = sum_{m,s'} W[m,n,s,s'] in[m,s'];   R: out[m,s] = sum_{n,s'} W[m,n,s,s'] in[n,s']
template<class T, bool LEFT>
__global__ void env_mix_kernel(const T *__restrict__ X, T *__restrict__ Y, const T *__restrict__ W, int d, int P, int Q, int DL, int DR) {
    extern __shared__ __align__(16) unsigned char env_smem[];
    T        *sW = reinterpret_cast<T *>(env_smem);
    const int nW = DL * DR * d * d;
    for(int i = threadIdx.x; i < nW; i += blockDim.x) sW[i] = W[i];
    __syncthreads();
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    const int q = blockIdx.y;
    if(p >= P) return;
    const int     Kin = LEFT ? DL : DR, Kout = LEFT ? DR : DL;
    const int64_t PdQ = (int64_t)P * d * Q;
    for(int j = 0; j < Kout; j++) {
        for(int s = 0; s < d; s++) {
            T acc;
            setz(acc);
            for(int k = 0; k < Kin; k++)
                for(int sp = 0; sp < d; sp++) {
                    const int m = LEFT ? k : j, n = LEFT ? j : k;
                    const T   w = sW[m + DL * (n + DR * (s + d * sp))];
                    if(nz(w)) acc = fma_e(w, X[p + (int64_t)P * (sp + (int64_t)d * q) + PdQ * k], acc);
                }
            Y[s + (int64_t)d * p + (int64_t)d * P * (q + (int64_t)Q * j)] = acc;
        }
    }
}

static int grid1(int64_t n) {
    int64_t g = (n + 255) / 256, cap = (int64_t)device_sm_count() * 16;
    return (int)(g < 1 ? 1 : (g < cap ? g : cap));
}

int check_env_dims(int side, const int64_t ed[3], const int64_t md[3], const int64_t wd[4]) {
    // EnvBase.cpp:93-101 (L) and :130-138 (R)
    if(md[0] != wd[2] || wd[2] != wd[3]) {
        set_last_error_msg("env%c: mps dim 0 (%lld) != mpo dim 2 (%lld)", side == 0 ? 'L' : 'R', (long long)md[0], (long long)wd[2]);
        return HEFF_BAD_SHAPE;
    }
    if(side == 0 && (md[1] != ed[0] || ed[1] != ed[0] || wd[0] != ed[2])) {
        set_last_error_msg("envL: dimension mismatch mps [%lld,%lld,%lld] mpo [%lld,%lld] env [%lld,%lld,%lld]", (long long)md[0], (long long)md[1],
                           (long long)md[2], (long long)wd[0], (long long)wd[1], (long long)ed[0], (long long)ed[1], (long long)ed[2]);
        return HEFF_BAD_SHAPE;
    }
    if(side == 1 && (md[2] != ed[0] || ed[1] != ed[0] || wd[1] != ed[2])) {
        set_last_error_msg("envR: dimension mismatch mps [%lld,%lld,%lld] mpo [%lld,%lld] env [%lld,%lld,%lld]", (long long)md[0], (long long)md[1],
                           (long long)md[2], (long long)wd[0], (long long)wd[1], (long long)ed[0], (long long)ed[1], (long long)ed[2]);
        return HEFF_BAD_SHAPE;
    }
    for(int i = 0; i < 3; i++)
        if(md[i] <= 0 || ed[i] <= 0) return HEFF_BAD_SHAPE;
    if(wd[0] * wd[1] * wd[2] * wd[3] > 4096 || md[1] > (1 << 20) || md[2] > (1 << 20)) return HEFF_BAD_SHAPE;
    return HEFF_OK;
}

int64_t env_scratch_elems(const int64_t md[3], const int64_t wd[4]) {
    auto          pad = [](int64_t n) { return (n + 31) / 32 * 32; };
    const int64_t d = md[0], cL = md[1], cR = md[2], Dm = wd[0] > wd[1] ? wd[0] : wd[1];
    return 2 * pad(d * cL * cR) + 2 * pad(Dm * d * cL * cR);
}

// out = build_block(env, M, W); scratch holds env_scratch_elems() elements.
template<bool CPLX>
int env_update(int side, typename Scalar<CPLX>::T *out, const typename Scalar<CPLX>::T *E, const int64_t ed[3], const typename Scalar<CPLX>::T *M,
               const int64_t md[3], const typename Scalar<CPLX>::T *W, const int64_t wd[4], typename Scalar<CPLX>::T *scratch, cudaStream_t s,
               void *split_ws, size_t split_bytes) {
    using T = typename Scalar<CPLX>::T;
    HEFF_TRY(check_env_dims(side, ed, md, wd));
    auto          pad = [](int64_t n) { return (n + 31) / 32 * 32; };
    const int64_t d = md[0], cL = md[1], cR = md[2], DL = wd[0], DR = wd[1], Dm = DL > DR ? DL : DR;
    const int64_t nM  = d * cL * cR;
    T            *Mc  = scratch;
    T            *M2  = Mc + pad(nM);
    T            *X   = M2 + pad(nM);
    T            *Y   = X + pad(Dm * nM);
    const size_t  wsm = sizeof(T) * (size_t)(DL * DR * d * d);
    if(side == 0) {
        env_prep_L<<<grid1(nM), 256, 0, s>>>(M, Mc, d, cL, nM);
        HEFF_LAUNCH_CHECK();
        GemmArgs g{};
        g.M = (int)cL, g.N = (int)(d * cR), g.K = (int)cL, g.batch = (int)DL;
        g.A = E, g.lda = cL, g.sA = cL * cL;
        g.B = Mc, g.ldb = cL, g.sB = 0;
        g.C = X, g.ldc = cL, g.sC = cL * d * cR;
        g.alpha = make_double2(1, 0), g.beta = make_double2(0, 0);
        HEFF_TRY(gemm_f64<CPLX>(false, false, false, g, s));
        if(cR > 65535) return HEFF_BAD_SHAPE;
        dim3 grid((unsigned)cdiv(cL, 128), (unsigned)cR);
        env_mix_kernel<T, true><<<grid, 128, wsm, s>>>(X, Y, W, (int)d, (int)cL, (int)cR, (int)DL, (int)DR);
        HEFF_LAUNCH_CHECK();
        GemmArgs h{};
        h.M = (int)cR, h.N = (int)(cR * DR), h.K = (int)(d * cL), h.batch = 1;
        h.A = M, h.lda = d * cL, h.B = Y, h.ldb = d * cL, h.C = out, h.ldc = cR;
        h.alpha = make_double2(1, 0), h.beta = make_double2(0, 0);
        h.split_ws = split_ws, h.split_ws_bytes = split_bytes;
        HEFF_TRY(gemm_f64<CPLX>(true, false, false, h, s));
    } else {
        env_prep_R<<<grid1(nM), 256, 0, s>>>(M, Mc, M2, d, cL, cR, nM);
        HEFF_LAUNCH_CHECK();
        GemmArgs g{};
        g.M = (int)cR, g.N = (int)(d * cL), g.K = (int)cR, g.batch = (int)DR;
        g.A = E, g.lda = cR, g.sA = cR * cR;
        g.B = Mc, g.ldb = d * cL, g.sB = 0;  // conj(M) stored N x K: (s',a') contiguous, b' outer
        g.C = X, g.ldc = cR, g.sC = cR * d * cL;
        g.alpha = make_double2(1, 0), g.beta = make_double2(0, 0);
        HEFF_TRY(gemm_f64<CPLX>(false, true, false, g, s));
        if(cL > 65535) return HEFF_BAD_SHAPE;
        dim3 grid((unsigned)cdiv(cR, 128), (unsigned)cL);
        env_mix_kernel<T, false><<<grid, 128, wsm, s>>>(X, Y, W, (int)d, (int)cR, (int)cL, (int)DL, (int)DR);
        HEFF_LAUNCH_CHECK();
        GemmArgs h{};
        h.M = (int)cL, h.N = (int)(cL * DL), h.K = (int)(d * cR), h.batch = 1;
        h.A = M2, h.lda = d * cR, h.B = Y, h.ldb = d * cR, h.C = out, h.ldc = cL;
        h.alpha = make_double2(1, 0), h.beta = make_double2(0, 0);
        h.split_ws = split_ws, h.split_ws_bytes = split_bytes;
        HEFF_TRY(gemm_f64<CPLX>(true, false, false, h, s));
    }
    return HEFF_OK;
}

template int env_update<false>(int, double *, const double *, const int64_t *, const double *, const int64_t *, const double *, const int64_t *,
                               double *, cudaStream_t, void *, size_t);
template int env_update<true>(int, double2 *, const double2 *, const int64_t *, const double2 *, const int64_t *, const double2 *,
                              const int64_t *, double2 *, cudaStream_t, void *, size_t);

template<bool CPLX>
static int env_stateless(int side, void *out, const void *env, const int64_t ed[3], const void *mps, const int64_t md[3], const void *mpo,
                         const int64_t wd[4], cudaStream_t s) {
    using T = typename Scalar<CPLX>::T;
    if(!out || !env || !mps || !mpo || !ed || !md || !wd || (side != 0 && side != 1)) return HEFF_BAD_ARG;
    if(out == env || out == mps) {
        set_last_error_msg("env update: out must not alias env or mps");
        return HEFF_BAD_ARG;
    }
    HEFF_TRY(check_env_dims(side, ed, md, wd));
    void        *base  = nullptr;
    const size_t bytes = (size_t)env_scratch_elems(md, wd) * sizeof(T);
    const size_t split = matvec_split_bytes(bytes);
    HEFF_TRY(stream_workspace(s, bytes + split, &base));
    return env_update<CPLX>(side, reinterpret_cast<T *>(out), reinterpret_cast<const T *>(env), ed, reinterpret_cast<const T *>(mps), md,
                            reinterpret_cast<const T *>(mpo), wd, reinterpret_cast<T *>(base), s, reinterpret_cast<unsigned char *>(base) + bytes,
                            split);
}

}  // namespace heff

using namespace heff;

extern "C" int heff_env_update_d(int side, double *out, const double *env, const int64_t env_dims[3], const double *mps, const int64_t mps_dims[3],
                                 const double *mpo, const int64_t mpo_dims[4], void *stream) {
    return env_stateless<false>(side, out, env, env_dims, mps, mps_dims, mpo, mpo_dims, (cudaStream_t)stream);
}
extern "C" int heff_env_update_z(int side, heff_z *out, const heff_z *env, const int64_t env_dims[3], const heff_z *mps, const int64_t mps_dims[3],
                                 const heff_z *mpo, const int64_t mpo_dims[4], void *stream) {
    return env_stateless<true>(side, out, env, env_dims, mps, mps_dims, mpo, mpo_dims, (cudaStream_t)stream);
}
