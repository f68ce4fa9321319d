// Minimal two-site DMRG sweep driver (see dmrg.cu).
#pragma once
#include "heff_common.cuh"

namespace heff {
int dmrg_run(const heff_dmrg_config &cfg, heff_dmrg_result &res, cudaStream_t s);
}
