// Environment update (see env.cu).
#pragma once
#include "heff_common.cuh"

namespace heff {
int     check_env_dims(int side, const int64_t ed[3], const int64_t md[3], const int64_t wd[4]);
int64_t env_scratch_elems(const int64_t md[3], const int64_t wd[4]);
// out = build_block(env, M, W); scratch holds env_scratch_elems() elements; split_ws (optional, split_bytes) is
// the tail-split scratch of the final GEMM (GemmArgs).
template<bool CPLX>
int env_update(int side, typename Scalar<CPLX>::T *out, const typename Scalar<CPLX>::T *E, const int64_t ed[3], const typename Scalar<CPLX>::T *M,
               const int64_t md[3], const typename Scalar<CPLX>::T *W, const int64_t wd[4], typename Scalar<CPLX>::T *scratch, cudaStream_t s,
               void *split_ws = nullptr, size_t split_bytes = 0);
}  // namespace heff
