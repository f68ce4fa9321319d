// Subspace-expansion term of one-site DMRG: EnvBase::get_expansion_term (source/tensors/site/env/EnvBase.cpp:303-364).
//
// L side (:311-333), env B [cL, cL, DL], mps M [S, cL, cR], mpo W [DL, DR, S, S]:
//   P[s', a', b + cR n] = alpha sum_{a,m,s} B[a,a',m] M[s,a,b] W[m,n,s,s']        P: [S, cL, cR*DR]
//   = the first two stages of the matvec with B as the left environment (permute, DMMA GEMM, MPO mix).
// R side (:335-357), env B [cR, cR, DR]:
//   Q[s', b', a, m] = alpha sum_{b,n,s} B[b,b',n] M[s,a,b] W[m,n,s,s']
//   stored in Q's memory order (the reference's shuffle {3,0,1,2} of [b',a,m,s'] followed by a reshape to
//   [S, cL*DL, cR], which keeps that order): P_flat[s' + S (b' + cR (a + cL m))].
//   X[(s + S a), (b' + cR n)] = alpha sum_b M[(s,a), b] B[b, (b',n)]              DMMA GEMM
//   P_flat[s' + S (b' + cR (a + cL m))] = sum_{n,s} W[m,n,s,s'] X[(s + S a), (b' + cR n)]   mix kernel
// alpha == 0 gives zeros (the reference returns a zeroed P); a NaN alpha is rejected (the reference throws).
#include <cmath>

#include "gemm_f64.cuh"
#include "matvec.cuh"
#include "runtime.cuh"

namespace heff {

__device__ __forceinline__ double ex_fma(double w, double v, double acc) { return fma(w, v, acc); }
__device__ __forceinline__ double2 ex_fma(double2 w, double2 v, double2 acc) {
    return make_double2(fma(w.x, v.x, fma(-w.y, v.y, acc.x)), fma(w.x, v.y, fma(w.y, v.x, acc.y)));
}
__device__ __forceinline__ bool ex_nz(double w) { return w != 0.0; }
__device__ __forceinline__ bool ex_nz(double2 w) { return w.x != 0.0 || w.y != 0.0; }

template<class T>
__global__ void expansion_mix_R(const T *__restrict__ X, const T *__restrict__ W, T *__restrict__ P, int S, int64_t cL, int64_t cR, int DL, int DR) {
    extern __shared__ __align__(16) unsigned char ex_smem[];
    T        *sW = reinterpret_cast<T *>(ex_smem);
    const int nW = DL * DR * S * S;
    for(int i = threadIdx.x; i < nW; i += blockDim.x) sW[i] = W[i];
    __syncthreads();
    const int64_t tot = (int64_t)S * cR * cL * DL, ldx = (int64_t)S * cL;
    for(int64_t o = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; o < tot; o += (int64_t)gridDim.x * blockDim.x) {
        const int64_t sp = o % S, r = o / S, bp = r % cR, r2 = r / cR, a = r2 % cL, m = r2 / cL;
        T             acc{};
        for(int nn = 0; nn < DR; nn++)
            for(int s = 0; s < S; s++) {
                const T w = sW[m + DL * (nn + DR * (s + S * sp))];
                if(ex_nz(w)) acc = ex_fma(w, X[(s + S * a) + ldx * (bp + cR * nn)], acc);
            }
        P[o] = acc;
    }
}

static int ex_grid(int64_t n) {
    const int64_t g = (n + 255) / 256, cap = (int64_t)device_sm_count() * 8;
    return (int)(g < 1 ? 1 : (g < cap ? g : cap));
}

int check_expansion_dims(int side, const int64_t ed[3], const int64_t md[3], const int64_t wd[4]) {
    for(int i = 0; i < 3; i++)
        if(ed[i] <= 0 || md[i] <= 0) return HEFF_BAD_SHAPE;
    for(int i = 0; i < 4; i++)
        if(wd[i] <= 0) return HEFF_BAD_SHAPE;
    if(wd[2] != md[0] || wd[3] != md[0] || ed[0] != ed[1]) return HEFF_BAD_SHAPE;
    if(side == 0 && (ed[0] != md[1] || ed[2] != wd[0])) return HEFF_BAD_SHAPE;
    if(side == 1 && (ed[0] != md[2] || ed[2] != wd[1])) return HEFF_BAD_SHAPE;
    if(side != 0 && side != 1) return HEFF_BAD_ARG;
    return HEFF_OK;
}

template<bool CPLX>
int expansion_term(int side, typename Scalar<CPLX>::T *P, const typename Scalar<CPLX>::T *B, const int64_t ed[3], const typename Scalar<CPLX>::T *M,
                   const int64_t md[3], const typename Scalar<CPLX>::T *W, const int64_t wd[4], double alpha, cudaStream_t s) {
    using T = typename Scalar<CPLX>::T;
    HEFF_TRY(check_expansion_dims(side, ed, md, wd));
    if(std::isnan(alpha)) {
        set_last_error_msg("expansion term: the mixing factor alpha is NaN");
        return HEFF_NAN_INPUT;
    }
    const int64_t S = md[0], cL = md[1], cR = md[2], DL = wd[0], DR = wd[1];
    const int64_t nP = side == 0 ? S * cL * cR * DR : S * cL * DL * cR;
    if(alpha == 0.0) {
        HEFF_CUDA(cudaMemsetAsync(P, 0, sizeof(T) * nP, s));
        return HEFF_OK;
    }
    auto pad = [](int64_t e) { return (e + 31) / 32 * 32; };
    if(side == 0) {
        const MatvecDims d{S, cL, cR, DL, DR};
        void            *base = nullptr;
        HEFF_TRY(stream_workspace(s, sizeof(T) * (size_t)(pad(d.size_mps()) + pad(d.size_T1())), &base));
        T *xp = reinterpret_cast<T *>(base), *T1 = xp + pad(d.size_mps());
        return matvec_left_stages<CPLX>(d, M, B, W, P, xp, T1, alpha, s);
    }
    const size_t smem = sizeof(T) * (size_t)(DL * DR * S * S);
    if(smem > 48 * 1024) return HEFF_BAD_SHAPE;
    void *base = nullptr;
    HEFF_TRY(stream_workspace(s, sizeof(T) * (size_t)pad(S * cL * cR * DR), &base));
    T       *X = reinterpret_cast<T *>(base);
    GemmArgs g{};
    g.M     = (int)(S * cL);
    g.N     = (int)(cR * DR);
    g.K     = (int)cR;
    g.batch = 1;
    g.A     = M;
    g.lda   = S * cL;
    g.B     = B;
    g.ldb   = cR;
    g.C     = X;
    g.ldc   = S * cL;
    g.alpha = make_double2(alpha, 0.0);
    g.beta  = make_double2(0.0, 0.0);
    HEFF_TRY(gemm_f64<CPLX>(false, false, false, g, s));
    expansion_mix_R<T><<<ex_grid(nP), 256, smem, s>>>(X, W, P, (int)S, cL, cR, (int)DL, (int)DR);
    HEFF_LAUNCH_CHECK();
    return HEFF_OK;
}

template int expansion_term<false>(int, double *, const double *, const int64_t[3], const double *, const int64_t[3], const double *,
                                   const int64_t[4], double, cudaStream_t);
template int expansion_term<true>(int, double2 *, const double2 *, const int64_t[3], const double2 *, const int64_t[3], const double2 *,
                                  const int64_t[4], double, cudaStream_t);

}  // namespace heff

using namespace heff;

extern "C" int heff_expansion_term_d(int side, double *P, const double *env, const int64_t env_dims[3], const double *mps, const int64_t mps_dims[3],
                                     const double *mpo, const int64_t mpo_dims[4], double alpha, void *stream) {
    if(!P || !env || !mps || !mpo || !env_dims || !mps_dims || !mpo_dims) return HEFF_BAD_ARG;
    return expansion_term<false>(side, P, env, env_dims, mps, mps_dims, mpo, mpo_dims, alpha, (cudaStream_t)stream);
}

extern "C" int heff_expansion_term_z(int side, heff_z *P, const heff_z *env, const int64_t env_dims[3], const heff_z *mps, const int64_t mps_dims[3],
                                     const heff_z *mpo, const int64_t mpo_dims[4], double alpha, void *stream) {
    if(!P || !env || !mps || !mpo || !env_dims || !mps_dims || !mpo_dims) return HEFF_BAD_ARG;
    return expansion_term<true>(side, reinterpret_cast<double2 *>(P), reinterpret_cast<const double2 *>(env), env_dims,
                                reinterpret_cast<const double2 *>(mps), mps_dims, reinterpret_cast<const double2 *>(mpo), mpo_dims, alpha,
                                (cudaStream_t)stream);
}
