// Shared definitions of the heff_b200 CUDA library (status codes, error plumbing, scalar traits).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/heff.h"

namespace heff {

// Status propagation: every internal routine returns an int status (HEFF_OK == 0).
#define HEFF_TRY(expr)                    \
    do {                                  \
        int _rc = (expr);                 \
        if(_rc != HEFF_OK) return _rc;    \
    } while(0)

#define HEFF_CUDA(expr)                                          \
    do {                                                         \
        cudaError_t _e = (expr);                                 \
        if(_e != cudaSuccess) {                                  \
            ::heff::set_last_cuda_error(_e, #expr, __FILE__, __LINE__); \
            return (_e == cudaErrorMemoryAllocation) ? HEFF_OOM : HEFF_CUDA_ERROR; \
        }                                                        \
    } while(0)

void set_last_cuda_error(cudaError_t e, const char *what, const char *file, int line);
void set_last_error_msg(const char *fmt, ...);

// Launch check: picks up launch-configuration errors without synchronising.
#define HEFF_LAUNCH_CHECK() HEFF_CUDA(cudaPeekAtLastError())

template<bool CPLX>
struct Scalar;
template<>
struct Scalar<false> {
    using T = double;
};
template<>
struct Scalar<true> {
    using T = double2;  // interleaved (re, im) == std::complex<double>
};

__host__ __device__ inline double2 cmul(double2 a, double2 b) { return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
__host__ __device__ inline double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__host__ __device__ inline double2 cconj(double2 a) { return make_double2(a.x, -a.y); }

inline int64_t cdiv(int64_t a, int64_t b) { return (a + b - 1) / b; }

int device_sm_count();

}  // namespace heff
