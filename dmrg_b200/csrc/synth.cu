// Seeded synthetic inputs generated on the device (for workloads too large to build on the host):
// environments [chi, chi, D] whose D-slices make H_eff Hermitian, and Gaussian start vectors.
//
// env[a, a', mu] = (g(a, a', mu) + conj(g(a', a, pair(mu)))) / 2 with g a counter-based Gaussian
// (splitmix64 hash -> Box-Muller).  pair(mu) = mu for an MPO whose slices are Hermitian (the Ising MPO,
// D = 3); for the uncompressed MPO squared (D = d0^2, slots mu = m + d0*m~) pair swaps (m, m~), which is
// the symmetry W2[(m~,m),(n~,n)] = W2[(m,m~),(n,n~)]^T of MpoSite.cpp:57-70, so
// env[., ., pair(mu)] = env[., ., mu]^dagger keeps sum_mu,nu L_mu (x) W_mu,nu (x) R_nu Hermitian.
#include <cmath>

#include "heff_common.cuh"

namespace heff {

__device__ __forceinline__ uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
__device__ __forceinline__ double u01(uint64_t key) { return ((double)(mix64(key) >> 11) + 0.5) * (1.0 / 9007199254740992.0); }
// standard normal pair for counter `c` under `seed`
__device__ __forceinline__ double2 gauss2(uint64_t seed, uint64_t c) {
    const double u1 = u01(seed ^ (0x9E3779B97F4A7C15ull * (2 * c + 1)));
    const double u2 = u01(seed ^ (0x9E3779B97F4A7C15ull * (2 * c + 2)));
    const double rr = sqrt(-2.0 * log(u1));
    double       sn, cs;
    sincospi(2.0 * u2, &sn, &cs);
    return make_double2(rr * cs, rr * sn);
}

template<bool CPLX>
__global__ void make_env_kernel(typename Scalar<CPLX>::T *out, int64_t chi, int64_t D, int64_t d0, uint64_t seed) {
    const int64_t tot = chi * chi * D;
    for(int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < tot; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t a = e % chi, r = e / chi, ap = r % chi, mu = r / chi;
        int64_t       pmu = mu;
        if(d0 > 1) pmu = (mu / d0) + d0 * (mu % d0);
        const double2 g1 = gauss2(seed, (uint64_t)(a + chi * (ap + chi * mu)));
        const double2 g2 = gauss2(seed, (uint64_t)(ap + chi * (a + chi * pmu)));
        if constexpr(CPLX)
            out[e] = make_double2(0.5 * (g1.x + g2.x), 0.5 * (g1.y - g2.y));
        else
            out[e] = 0.5 * (g1.x + g2.x);
    }
}

template<bool CPLX>
__global__ void make_vec_kernel(typename Scalar<CPLX>::T *out, int64_t n, uint64_t seed) {
    for(int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        const double2 g = gauss2(seed, (uint64_t)e);
        if constexpr(CPLX)
            out[e] = g;
        else
            out[e] = g.x;
    }
}

static int g1(int64_t n) {
    int64_t g = (n + 255) / 256, cap = (int64_t)device_sm_count() * 16;
    return (int)(g < 1 ? 1 : (g < cap ? g : cap));
}

}  // namespace heff

using namespace heff;

extern "C" int heff_make_env(int dtype, int64_t chi, int64_t D, int64_t swap_base, uint64_t seed, void *out, void *stream) {
    if(!out || chi <= 0 || D <= 0 || (swap_base > 1 && swap_base * swap_base != D)) return HEFF_BAD_ARG;
    const int64_t tot = chi * chi * D;
    if(dtype == HEFF_C128)
        make_env_kernel<true><<<g1(tot), 256, 0, (cudaStream_t)stream>>>(reinterpret_cast<double2 *>(out), chi, D, swap_base, seed);
    else
        make_env_kernel<false><<<g1(tot), 256, 0, (cudaStream_t)stream>>>(reinterpret_cast<double *>(out), chi, D, swap_base, seed);
    HEFF_LAUNCH_CHECK();
    return HEFF_OK;
}

extern "C" int heff_make_vector(int dtype, int64_t n, uint64_t seed, void *out, void *stream) {
    if(!out || n <= 0) return HEFF_BAD_ARG;
    if(dtype == HEFF_C128)
        make_vec_kernel<true><<<g1(n), 256, 0, (cudaStream_t)stream>>>(reinterpret_cast<double2 *>(out), n, seed);
    else
        make_vec_kernel<false><<<g1(n), 256, 0, (cudaStream_t)stream>>>(reinterpret_cast<double *>(out), n, seed);
    HEFF_LAUNCH_CHECK();
    return HEFF_OK;
}
