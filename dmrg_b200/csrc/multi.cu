// H_eff matvec with a chain of site MPOs applied one at a time: the multi-MPO matrix_vector_product
// (source/tools/common/contraction/contraction_tblis.cpp:307-420), which the reference uses when a multisite
// operator has more than 5 sites (matvec_mpos.cpp:104-123) so that the merged MPO (D^2 prod(d_i)^2 entries)
// is never formed.
//
//   y[s',a',b'] = sum L[a,a',m0] W1[m0,m1,s1,s1'] ... WK[m_{K-1},mK,sK,sK'] R[b,b',mK] theta[s,a,b],
//   s = s1 + d1 (s2 + d2 (...)) (site 1 fastest, as the reference's reshapes and the two-site merge order).
//
// Stages (S = prod d_i; the physical multi-index is updated in place, site by site):
//   permute      x'[a, (s,b)]                                    (as the one-MPO matvec)
//   DMMA GEMM    T[(a',m0), (s,b)] = sum_a L[a,(a',m0)] x'[a,(s,b)]
//   site i       T'[(a',m_i), (..s_i'..,b)] = sum_{m_{i-1},s_i} W_i[m_{i-1},m_i,s_i,s_i'] T[(a',m_{i-1}), (..s_i..,b)]
//                (the last site writes the one-MPO matvec's T2 layout [(s',a'), (b,mK)])
//   DMMA GEMM    y[(s',a'), b'] = sum_{(b,mK)} T2[(s',a'),(b,mK)] R'[(b,mK), b']
// The sums differ from the reference's only in their order (it contracts the same indices in the same
// sequence, with Eigen's blocking).
#include <algorithm>
#include <vector>

#include "gemm_f64.cuh"
#include "matvec.cuh"
#include "multi.cuh"
#include "runtime.cuh"

namespace heff {

__device__ __forceinline__ double sm_fma(double w, double v, double acc) { return fma(w, v, acc); }
__device__ __forceinline__ double2 sm_fma(double2 w, double2 v, double2 acc) {
    return make_double2(fma(w.x, v.x, fma(-w.y, v.y, acc.x)), fma(w.x, v.y, fma(w.y, v.x, acc.y)));
}
__device__ __forceinline__ bool sm_nz(double w) { return w != 0.0; }
__device__ __forceinline__ bool sm_nz(double2 w) { return w.x != 0.0 || w.y != 0.0; }

// One thread per point (a', p, q, b), p < P = prod_{j<i} d_j, q < Q = S / (P d); a' fastest (coalesced).
template<class T, bool LAST>
__global__ void site_mix_kernel(const T *__restrict__ in, T *__restrict__ out, const T *__restrict__ W, int Din, int Dout, int d, int64_t cL,
                                int64_t cR, int64_t S, int64_t P) {
    extern __shared__ __align__(16) unsigned char sm_smem[];
    T        *sW = reinterpret_cast<T *>(sm_smem);
    const int nW = Din * Dout * d * d;
    for(int i = threadIdx.x; i < nW; i += blockDim.x) sW[i] = W[i];
    __syncthreads();
    const int64_t Q = S / (P * d), npts = cL * P * Q * cR;
    const int64_t ldi = cL * Din, ldo = cL * Dout;
    for(int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < npts; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t ap = e % cL, r = e / cL, p = r % P, r2 = r / P, q = r2 % Q, b = r2 / Q;
        for(int tp = 0; tp < d; tp++)
            for(int n = 0; n < Dout; n++) {
                T acc{};
                for(int t = 0; t < d; t++) {
                    const int64_t col = (p + P * (t + (int64_t)d * q)) + S * b;
                    for(int m = 0; m < Din; m++) {
                        const T w = sW[m + Din * (n + Dout * (t + d * tp))];
                        if(sm_nz(w)) acc = sm_fma(w, in[(ap + cL * m) + ldi * col], acc);
                    }
                }
                const int64_t sp = p + P * (tp + (int64_t)d * q);
                if(LAST)
                    out[(sp + S * ap) + S * cL * (b + cR * n)] = acc;
                else
                    out[(ap + cL * n) + ldo * (sp + S * b)] = acc;
            }
    }
}

static int mm_grid(int64_t n) {
    const int64_t g = (n + 255) / 256, cap = (int64_t)device_sm_count() * 8;
    return (int)(g < 1 ? 1 : (g < cap ? g : cap));
}

template<class T>
__global__ void mm_permute_kernel(const T *__restrict__ x, T *__restrict__ xp, int64_t S, int64_t cL, int64_t n) {
    // xp[a + cL (s + S b)] = x[s + S (a + cL b)]
    for(int64_t o = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; o < n; o += (int64_t)gridDim.x * blockDim.x) {
        const int64_t a = o % cL, r = o / cL, s = r % S, b = r / S;
        xp[o]           = x[s + S * (a + cL * b)];
    }
}

int check_multi_dims(const int64_t md[3], int nmpo, const int64_t *wd, const int64_t ld[3], const int64_t rd[3], MultiDims &out) {
    if(nmpo < 1 || nmpo > 64) return HEFF_BAD_ARG;
    int64_t S = 1, Dmax = 0;
    for(int i = 0; i < nmpo; i++) {
        const int64_t *w = wd + 4 * i;
        if(w[0] <= 0 || w[1] <= 0 || w[2] <= 0 || w[2] != w[3]) return HEFF_BAD_SHAPE;
        if(i > 0 && w[0] != wd[4 * (i - 1) + 1]) return HEFF_BAD_SHAPE;
        S *= w[2];
        Dmax = std::max(Dmax, std::max(w[0], w[1]));
    }
    // contraction_tblis.cpp:331-332 checks, plus square environments and matching bond dimensions
    if(md[0] != S || md[1] != ld[0] || md[2] != rd[0] || ld[0] != ld[1] || rd[0] != rd[1]) return HEFF_BAD_SHAPE;
    if(ld[2] != wd[0] || rd[2] != wd[4 * (nmpo - 1) + 1]) return HEFF_BAD_SHAPE;
    out.S = S, out.cL = md[1], out.cR = md[2], out.Dmax = Dmax, out.nmpo = nmpo;
    out.dims.assign(wd, wd + 4 * nmpo);
    return HEFF_OK;
}

int64_t multi_scratch_elems(const MultiDims &md) {
    auto          pad = [](int64_t e) { return (e + 31) / 32 * 32; };
    const int64_t n   = md.S * md.cL * md.cR;
    return pad(n) + 2 * pad(n * md.Dmax);
}

template<bool CPLX>
int matvec_multi(const MultiDims &md, const typename Scalar<CPLX>::T *x, typename Scalar<CPLX>::T *y, const typename Scalar<CPLX>::T *L,
                 const typename Scalar<CPLX>::T *Rp, const typename Scalar<CPLX>::T *const *W, typename Scalar<CPLX>::T *scratch, cudaStream_t s) {
    using T             = typename Scalar<CPLX>::T;
    auto          pad   = [](int64_t e) { return (e + 31) / 32 * 32; };
    const int64_t S = md.S, cL = md.cL, cR = md.cR, n = S * cL * cR;
    T            *xp    = scratch;
    T            *buf[2] = {xp + pad(n), xp + pad(n) + pad(n * md.Dmax)};
    const int64_t D0 = md.dims[0], DK = md.dims[4 * (md.nmpo - 1) + 1];
    mm_permute_kernel<T><<<mm_grid(n), 256, 0, s>>>(x, xp, S, cL, n);
    HEFF_LAUNCH_CHECK();
    GemmArgs g1{};
    g1.M = (int)(cL * D0), g1.N = (int)(S * cR), g1.K = (int)cL, g1.batch = 1;
    g1.A = L, g1.lda = cL, g1.B = xp, g1.ldb = cL, g1.C = buf[0], g1.ldc = cL * D0;
    g1.alpha = make_double2(1.0, 0.0), g1.beta = make_double2(0.0, 0.0);
    HEFF_TRY(gemm_f64<CPLX>(/*ta=*/true, /*tb=*/false, false, g1, s));
    int64_t P = 1;
    int     cur = 0;
    for(int i = 0; i < md.nmpo; i++) {
        const int64_t *w    = md.dims.data() + 4 * i;
        const bool     last = i == md.nmpo - 1;
        const size_t   smem = sizeof(T) * (size_t)(w[0] * w[1] * w[2] * w[3]);
        if(smem > 48 * 1024) return HEFF_BAD_SHAPE;
        const int64_t npts = cL * cR * S / w[2];
        if(last)
            site_mix_kernel<T, true><<<mm_grid(npts), 256, smem, s>>>(buf[cur], buf[cur ^ 1], W[i], (int)w[0], (int)w[1], (int)w[2], cL, cR, S, P);
        else
            site_mix_kernel<T, false><<<mm_grid(npts), 256, smem, s>>>(buf[cur], buf[cur ^ 1], W[i], (int)w[0], (int)w[1], (int)w[2], cL, cR, S, P);
        HEFF_LAUNCH_CHECK();
        cur ^= 1;
        P *= w[2];
    }
    GemmArgs g2{};
    g2.M = (int)(S * cL), g2.N = (int)cR, g2.K = (int)(cR * DK), g2.batch = 1;
    g2.A = buf[cur], g2.lda = S * cL, g2.B = Rp, g2.ldb = cR * DK, g2.C = y, g2.ldc = S * cL;
    g2.alpha = make_double2(1.0, 0.0), g2.beta = make_double2(0.0, 0.0);
    return gemm_f64<CPLX>(false, false, false, g2, s);
}

template int matvec_multi<false>(const MultiDims &, const double *, double *, const double *, const double *, const double *const *, double *,
                                 cudaStream_t);
template int matvec_multi<true>(const MultiDims &, const double2 *, double2 *, const double2 *, const double2 *, const double2 *const *, double2 *,
                                cudaStream_t);

// ---- stateless entry point: device buffers, unshuffled site MPOs W_i[m, n, s, s'] ----
template<bool CPLX>
static int multi_stateless(void *res, const void *mps, const int64_t md3[3], int nmpo, const void *const *mpos, const int64_t *mpo_dims,
                           const void *envL, const int64_t ld[3], const void *envR, const int64_t rd[3], cudaStream_t s) {
    using T = typename Scalar<CPLX>::T;
    if(!res || !mps || !mpos || !mpo_dims || !envL || !envR || !md3 || !ld || !rd) return HEFF_BAD_ARG;
    if(res == mps) {
        set_last_error_msg("matrix_vector_product: res must not alias mps");
        return HEFF_BAD_ARG;
    }
    MultiDims md;
    HEFF_TRY(check_multi_dims(md3, nmpo, mpo_dims, ld, rd, md));
    auto          pad  = [](int64_t e) { return (e + 31) / 32 * 32; };
    const int64_t DK   = mpo_dims[4 * (nmpo - 1) + 1];
    const int64_t nRp  = md.cR * md.cR * DK;
    void         *base = nullptr;
    HEFF_TRY(stream_workspace(s, sizeof(T) * (size_t)(multi_scratch_elems(md) + pad(nRp)), &base));
    T         *scr = reinterpret_cast<T *>(base);
    T         *Rp  = scr + multi_scratch_elems(md);
    MatvecDims dR{md.S, md.cL, md.cR, 1, DK};
    HEFF_TRY(permute_R<CPLX>(reinterpret_cast<const T *>(envR), Rp, dR, s));
    std::vector<const T *> W(nmpo);
    for(int i = 0; i < nmpo; i++) W[i] = reinterpret_cast<const T *>(mpos[i]);
    return matvec_multi<CPLX>(md, reinterpret_cast<const T *>(mps), reinterpret_cast<T *>(res), reinterpret_cast<const T *>(envL), Rp, W.data(), scr, s);
}

}  // namespace heff

using namespace heff;

extern "C" int heff_matvec_multi_d(double *res, const double *mps, const int64_t mps_dims[3], int nmpo, const double *const *mpos,
                                   const int64_t *mpo_dims, const double *envL, const int64_t envL_dims[3], const double *envR,
                                   const int64_t envR_dims[3], void *stream) {
    return multi_stateless<false>(res, mps, mps_dims, nmpo, reinterpret_cast<const void *const *>(mpos), mpo_dims, envL, envL_dims, envR, envR_dims,
                                  (cudaStream_t)stream);
}

extern "C" int heff_matvec_multi_z(heff_z *res, const heff_z *mps, const int64_t mps_dims[3], int nmpo, const heff_z *const *mpos,
                                   const int64_t *mpo_dims, const heff_z *envL, const int64_t envL_dims[3], const heff_z *envR,
                                   const int64_t envR_dims[3], void *stream) {
    return multi_stateless<true>(res, mps, mps_dims, nmpo, reinterpret_cast<const void *const *>(mpos), mpo_dims, envL, envL_dims, envR, envR_dims,
                                 (cudaStream_t)stream);
}
