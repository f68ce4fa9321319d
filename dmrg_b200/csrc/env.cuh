// Environment update (see env.cu).
#pragma once
#include "heff_common.cuh"

namespace heff {
int     check_env_dims(int side, const int64_t ed[3], const int64_t md[3], const int64_t wd[4]);
int64_t env_scratch_elems(const int64_t md[3], const int64_t wd[4]);
template<bool CPLX>
int env_update(int side, typename Scalar<CPLX>::T *out, const typename Scalar<CPLX>::T *E, const int64_t ed[3], const typename Scalar<CPLX>::T *M,
               const int64_t md[3], const typename Scalar<CPLX>::T *W, const int64_t wd[4], typename Scalar<CPLX>::T *scratch, cudaStream_t s);
}  // namespace heff
