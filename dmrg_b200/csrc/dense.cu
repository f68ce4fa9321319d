// Dense small-problem path: MatVecMPO(S)::get_tensor / get_matrix (source/math/eig/matvec/matvec_mpo.cpp:313-332,
// matvec_mpos.cpp:1570-1588) and the full Hermitian eigendecomposition the reference runs on it with LAPACK
// ?syevr / ?heevd (eig::solver::eig, used when the problem size is <= settings::precision::eig_max_size = 4096,
// AlgorithmFinite.cpp:318).
//
// get_matrix: M[(s,a,b), (s',a',b')] = sum_{m,n} L[a,a',m] W[m,n,s,s'] R[b,b',n]  (column-major, rows = input
// index of the matvec: the reference's shuffle {2,0,4,3,1,5} puts (s,a,b) first), one thread per entry.
//
// Eigendecomposition of a Hermitian M: with sigma = 1.01 * max_i sum_j |M_ij| + tiny (a Gershgorin bound on the
// spectral radius, with margin), A = M + sigma I is positive definite, its singular values are its eigenvalues
// and its left singular vectors are eigenvectors (distinct eigenvalues of A are distinct singular values, and a
// degenerate singular subspace is an eigenspace).  The one-sided Jacobi SVD of svd.cu gives them; then
// lambda_i = s_i - sigma in ascending order.  Absolute accuracy ~ eps (||M|| + sigma), the level of ?syevr.
#include <algorithm>
#include <cmath>
#include <vector>

#include "op.cuh"
#include "runtime.cuh"
#include "svd.cuh"

namespace heff {

__device__ __forceinline__ double dn_abs(double v) { return fabs(v); }
__device__ __forceinline__ double dn_abs(double2 v) { return hypot(v.x, v.y); }
__device__ __forceinline__ double dn_fma(double a, double b, double c) { return fma(a, b, c); }
__device__ __forceinline__ double2 dn_fma(double2 a, double2 b, double2 c) {
    return make_double2(fma(a.x, b.x, fma(-a.y, b.y, c.x)), fma(a.x, b.y, fma(a.y, b.x, c.y)));
}
__device__ __forceinline__ bool dn_nz(double v) { return v != 0.0; }
__device__ __forceinline__ bool dn_nz(double2 v) { return v.x != 0.0 || v.y != 0.0; }
__device__ __forceinline__ double dn_shift(double v, double s) { return v + s; }
__device__ __forceinline__ double2 dn_shift(double2 v, double s) { return make_double2(v.x + s, v.y); }

// L reference layout L[a + cL (a' + cL m)];  R permuted R'[b + cR n + cR DR b'] (matvec.cu)
template<class T>
__global__ void get_matrix_kernel(const T *__restrict__ L, const T *__restrict__ Rp, const T *__restrict__ W, int S, int64_t cL, int64_t cR, int DL,
                                  int DR, T *__restrict__ M) {
    extern __shared__ __align__(16) unsigned char dn_smem[];
    T        *sW = reinterpret_cast<T *>(dn_smem);
    const int nW = DL * DR * S * S;
    for(int i = threadIdx.x; i < nW; i += blockDim.x) sW[i] = W[i];
    __syncthreads();
    const int64_t N = (int64_t)S * cL * cR, tot = N * N;
    for(int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < tot; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t I = e % N, J = e / N;
        const int64_t s = I % S, a = (I / S) % cL, b = I / (S * cL);
        const int64_t sp = J % S, ap = (J / S) % cL, bp = J / (S * cL);
        T             acc{};
        for(int nn = 0; nn < DR; nn++) {
            const T r = Rp[b + cR * nn + cR * DR * bp];
            if(!dn_nz(r)) continue;
            T inner{};
            for(int m = 0; m < DL; m++) {
                const T w = sW[m + DL * (nn + DR * (s + S * sp))];
                if(dn_nz(w)) inner = dn_fma(L[a + cL * (ap + cL * (int64_t)m)], w, inner);
            }
            acc = dn_fma(inner, r, acc);
        }
        M[e] = acc;
    }
}

// Largest absolute row sum (Gershgorin radius bound), one block per row chunk, atomic max of non-negative doubles.
template<class T>
__global__ void row_abs_max_kernel(const T *__restrict__ A, int64_t lda, int64_t n, double *__restrict__ out) {
    for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double acc = 0;
        for(int64_t j = 0; j < n; j++) acc += dn_abs(A[i + lda * j]);
        atomicMax(reinterpret_cast<unsigned long long *>(out), (unsigned long long)__double_as_longlong(acc));
    }
}

template<class T>
__global__ void shift_copy_kernel(const T *__restrict__ A, int64_t lda, int64_t n, const double *__restrict__ gmax, T *__restrict__ B) {
    const double sigma = 1.01 * gmax[0] + 1e-300;
    for(int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n * n; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = e % n, j = e / n;
        B[e]            = i == j ? dn_shift(A[i + lda * j], sigma) : A[i + lda * j];
    }
}

// evals[i] = S[n-1-i] - sigma (ascending), evecs[:, i] = U[:, n-1-i]
template<class T>
__global__ void dense_eig_finish_kernel(const T *__restrict__ U, const double *__restrict__ Sv, const double *__restrict__ gmax, int64_t n,
                                        double *__restrict__ evals, T *__restrict__ evecs) {
    const double sigma = 1.01 * gmax[0] + 1e-300;
    for(int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n * n; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = e % n, c = e / n, src = n - 1 - c;
        evecs[e]        = U[r + n * src];
        if(r == 0) evals[c] = Sv[src] - sigma;
    }
}

static int dn_grid(int64_t n) {
    const int64_t g = (n + 255) / 256, cap = (int64_t)device_sm_count() * 16;
    return (int)(g < 1 ? 1 : (g < cap ? g : cap));
}

template<bool CPLX>
static int get_matrix_impl(heff_op *op, void *Mout) {
    using T = typename Scalar<CPLX>::T;
    if(op->sequential) {  // as MatVecMPOS::get_tensor, matvec_mpos.cpp:1587
        set_last_error_msg("get_matrix: not implemented for more than one (unmerged) MPO");
        return HEFF_BAD_ARG;
    }
    const MatvecDims &d = op->d;
    const size_t smem   = sizeof(T) * (size_t)(d.DL * d.DR * d.S * d.S);
    if(smem > 48 * 1024) return HEFF_BAD_SHAPE;
    const int64_t N = d.size_mps();
    get_matrix_kernel<T><<<dn_grid(N * N), 256, smem, op->stream>>>(reinterpret_cast<const T *>(op->L), reinterpret_cast<const T *>(op->Rp),
                                                                     reinterpret_cast<const T *>(op->W), (int)d.S, d.cL, d.cR, (int)d.DL, (int)d.DR,
                                                                     reinterpret_cast<T *>(Mout));
    HEFF_LAUNCH_CHECK();
    return HEFF_OK;
}

template<bool CPLX>
static int dense_eig_impl(int64_t n, const void *Av, int64_t lda, double *evals, void *evecs_v, cudaStream_t s) {
    using T       = typename Scalar<CPLX>::T;
    const T *A    = reinterpret_cast<const T *>(Av);
    T       *evec = reinterpret_cast<T *>(evecs_v);
    auto     pad  = [](int64_t e) { return (e + 31) / 32 * 32; };
    const int64_t es = sizeof(T), nn = pad(n * n);
    const size_t  need = (size_t)(es * 3 * nn + 8 * pad(n) + 256 + svd_scratch_bytes(n, n, es) + 256);
    void         *base = nullptr;
    HEFF_TRY(stream_workspace(s, need, &base));
    T      *B    = reinterpret_cast<T *>(base);
    T      *U    = B + nn;
    T      *VT   = U + nn;
    double *Sv   = reinterpret_cast<double *>(VT + nn);
    double *gmax = Sv + pad(n);
    void   *jscr = reinterpret_cast<char *>(gmax) + 256;
    HEFF_CUDA(cudaMemsetAsync(gmax, 0, sizeof(double), s));
    row_abs_max_kernel<T><<<dn_grid(n), 256, 0, s>>>(A, lda, n, gmax);
    HEFF_LAUNCH_CHECK();
    shift_copy_kernel<T><<<dn_grid(n * n), 256, 0, s>>>(A, lda, n, gmax, B);
    HEFF_LAUNCH_CHECK();
    int64_t rank = 0;
    double  te   = 0;
    HEFF_TRY(svd_truncated(B, n, n, n, 0, 0.0, U, Sv, VT, &rank, &te, jscr, nullptr, s));
    if(rank != n) {
        set_last_error_msg("dense eigensolver: shifted matrix lost rank (%lld of %lld)", (long long)rank, (long long)n);
        return HEFF_NOT_CONVERGED;
    }
    dense_eig_finish_kernel<T><<<dn_grid(n * n), 256, 0, s>>>(U, Sv, gmax, n, evals, evec);
    HEFF_LAUNCH_CHECK();
    return HEFF_OK;
}

}  // namespace heff

using namespace heff;

extern "C" int heff_op_get_matrix(heff_op *op, void *M_out) {
    if(!op || !M_out) return HEFF_BAD_ARG;
    return op->cplx ? get_matrix_impl<true>(op, M_out) : get_matrix_impl<false>(op, M_out);
}

extern "C" int heff_dense_eig(heff_dtype dtype, int64_t n, const void *A, int64_t lda, double *evals, void *evecs, void *stream) {
    if(!A || !evals || !evecs || n <= 0 || lda < n) return HEFF_BAD_ARG;
    if(n > 16384) return HEFF_BAD_SHAPE;
    if(dtype == HEFF_F64) return dense_eig_impl<false>(n, A, lda, evals, evecs, (cudaStream_t)stream);
    if(dtype == HEFF_C128) return dense_eig_impl<true>(n, A, lda, evals, evecs, (cudaStream_t)stream);
    return HEFF_BAD_ARG;
}
