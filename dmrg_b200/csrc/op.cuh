// Internal definition of the heff_op operator object (opaque in include/heff.h).
#pragma once
#include "matvec.cuh"

struct heff_op {
    bool               cplx = false;
    heff::MatvecDims   d{};
    int64_t            mpo_dims[4] = {0, 0, 0, 0};
    heff_precision     precision   = HEFF_PREC_FP64;
    cudaStream_t       stream      = nullptr;
    void              *L = nullptr, *Rp = nullptr, *W = nullptr;  // device: envL (reference layout), R', merged W
    void              *scratch       = nullptr;                    // x' | T1 | T2
    size_t             scratch_bytes = 0;
    void              *stage_x       = nullptr;  // device staging for MultAx with host buffers
    int64_t            num_mv        = 0;
    // mixed-precision state (owned by the mixed path; null until first use)
    void              *mixed         = nullptr;
    int (*mixed_apply)(heff_op *, const void *, void *) = nullptr;
    void (*destroy_hook)(heff_op *)                     = nullptr;
};

namespace heff {
int op_apply(heff_op *op, const void *x, void *y);
}
