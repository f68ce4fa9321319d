// Multi-MPO H_eff matvec (site MPOs applied one at a time); see multi.cu.
#pragma once
#include <vector>

#include "heff_common.cuh"

namespace heff {

struct MultiDims {
    int64_t              S = 0, cL = 0, cR = 0, Dmax = 0;
    int                  nmpo = 0;
    std::vector<int64_t> dims;  // 4 per site MPO: [D_{i-1}, D_i, d_i, d_i]
};

int     check_multi_dims(const int64_t md[3], int nmpo, const int64_t *wd, const int64_t ld[3], const int64_t rd[3], MultiDims &out);
int64_t multi_scratch_elems(const MultiDims &md);
template<bool CPLX>
int matvec_multi(const MultiDims &md, const typename Scalar<CPLX>::T *x, typename Scalar<CPLX>::T *y, const typename Scalar<CPLX>::T *L,
                 const typename Scalar<CPLX>::T *Rp, const typename Scalar<CPLX>::T *const *W, typename Scalar<CPLX>::T *scratch, cudaStream_t s);

}  // namespace heff
