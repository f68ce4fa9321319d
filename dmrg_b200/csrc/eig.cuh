// Device eigensolver (see eig.cu).
#pragma once
#include "heff_common.cuh"

namespace heff {
int eigs(heff_op *op, const heff_eig_config *cfg, const void *x0, void *x_out, heff_eig_result *res);
int eig_reserve(heff_op *op, int64_t n_max, int max_basis, bool mixed);
}
