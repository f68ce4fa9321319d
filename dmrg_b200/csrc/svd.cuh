// Device SVD (one-sided block Jacobi, real and complex FP64) and the two-site Schmidt split; see svd.cu.
#pragma once
#include "heff_common.cuh"

namespace heff {
int64_t svd_scratch_bytes(int64_t m, int64_t n, int64_t esize = 8);
int64_t schmidt_scratch_bytes(int64_t dL, int64_t dR, int64_t cL, int64_t cR, int64_t rank_max, int64_t esize = 8);
int    &last_svd_sweeps();  // Jacobi sweeps of the calling thread's last SVD
int64_t truncation_rank(const double *S, int64_t n, int64_t rank_max, int64_t rank_min, double lim, double *trunc_err);
int     svd_truncated(const double *A, int64_t lda, int64_t m, int64_t n, int64_t rank_max, double trunc_lim, double *U, double *S, double *VT,
                      int64_t *rank, double *trunc_err, void *scratch, int *sweeps_out, cudaStream_t s);
int     svd_truncated(const double2 *A, int64_t lda, int64_t m, int64_t n, int64_t rank_max, double trunc_lim, double2 *U, double *S, double2 *VT,
                      int64_t *rank, double *trunc_err, void *scratch, int *sweeps_out, cudaStream_t s);
int     schmidt_split(const double *theta, int64_t dL, int64_t dR, int64_t cL, int64_t cR, int64_t rank_max, double trunc_lim, double *U, double *S,
                      double *V, int64_t *rank, double *trunc_err, void *scratch, cudaStream_t s);
int     schmidt_split(const double2 *theta, int64_t dL, int64_t dR, int64_t cL, int64_t cR, int64_t rank_max, double trunc_lim, double2 *U, double *S,
                      double2 *V, int64_t *rank, double *trunc_err, void *scratch, cudaStream_t s);
}  // namespace heff
