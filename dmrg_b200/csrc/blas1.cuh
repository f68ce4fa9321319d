// Deterministic level-1/"tall-skinny" vector kernels for the eigensolver (FP64, real or complex):
//   multi_dot:  h[j]  = sum_i conj(V[i,j]) t[i]        (j < k)     two-pass, fixed reduction order
//   multi_axpy: t[i] += alpha * sum_j V[i,j] h[j]
//   combine:    x[i]  = sum_j V[i,j] c[j]
#pragma once
#include "heff_common.cuh"

namespace heff {

constexpr int MD_BLOCKS = 512;  // partial-sum rows of multi_dot
constexpr int MD_MAXK   = 128;  // max columns handled by one multi_dot call

template<bool CPLX>
int multi_dot(const typename Scalar<CPLX>::T *V, int64_t ldv, int64_t n, int k, const typename Scalar<CPLX>::T *t, typename Scalar<CPLX>::T *h,
              double *partials /* >= MD_BLOCKS * MD_MAXK * 2 doubles */, cudaStream_t s);
template<bool CPLX>
int multi_axpy(const typename Scalar<CPLX>::T *V, int64_t ldv, int64_t n, int k, const typename Scalar<CPLX>::T *h, double alpha,
               typename Scalar<CPLX>::T *t, cudaStream_t s);
template<bool CPLX>
int combine(const typename Scalar<CPLX>::T *V, int64_t ldv, int64_t n, int k, const typename Scalar<CPLX>::T *c, typename Scalar<CPLX>::T *x,
            cudaStream_t s);
// x *= a (real scalar a read from device memory: a = *scale_dev, or 1/sqrt(*scale_dev) when inv_sqrt)
template<bool CPLX>
int scale_dev(typename Scalar<CPLX>::T *x, int64_t n, const double *scale_dev, bool inv_sqrt, cudaStream_t s);
// y = x - theta*z  (residual), theta real on the host
template<bool CPLX>
int residual(const typename Scalar<CPLX>::T *ax, const typename Scalar<CPLX>::T *x, double theta, typename Scalar<CPLX>::T *r, int64_t n,
             cudaStream_t s);

// Krylov expansion step on the device: v = (w - V h) / beta with h = V^H w, a second classical Gram-Schmidt
// pass when ||w - V h||^2 <= 0.5 ||w||^2 (decided on the device), beta = ||v|| before normalisation.
// st: >= 8 + 4 (MD_MAXK + 2) doubles of state; counter: one zeroed unsigned (left zeroed); hres (device, k+2):
// hres[j] = h_j (j < k), hres[k] = beta, hres[k+1] = (||w||^2, 1 if the second pass ran).  w and v must differ.
template<bool CPLX>
int orth_cgs2(const typename Scalar<CPLX>::T *V, int64_t ldv, int64_t n, int k, const typename Scalar<CPLX>::T *w, typename Scalar<CPLX>::T *v,
              double *partials, unsigned *counter, double *st, typename Scalar<CPLX>::T *hres, cudaStream_t s);

// Device-side CG for the Jacobi-Davidson correction equation (I - uu^H)(H - theta)(I - uu^H) d = -r0 (see blas1.cu):
// cg_init sets d = 0, r = p = -r0 and the scalars in cs (>= 16 doubles); each cg_step, after the caller has
// formed z = H p, does the update with all scalars on the device.  cs[6] != 0 once CG has stopped (converged to
// rho <= tol2 rho0, or an indefinite direction); later steps are no-ops.  partials >= 6 * MD_BLOCKS doubles.
template<bool CPLX>
int cg_init(typename Scalar<CPLX>::T *d, typename Scalar<CPLX>::T *r, typename Scalar<CPLX>::T *p, const typename Scalar<CPLX>::T *r0, int64_t n,
            double *cs, double rho0, double theta, double tol2, cudaStream_t s);
template<bool CPLX>
int cg_step(const typename Scalar<CPLX>::T *z, typename Scalar<CPLX>::T *p, const typename Scalar<CPLX>::T *u, typename Scalar<CPLX>::T *q,
            typename Scalar<CPLX>::T *d, typename Scalar<CPLX>::T *r, int64_t n, double *cs, double *partials, unsigned *counter, cudaStream_t s);
constexpr int CG_DONE_SLOT = 6;

}  // namespace heff
