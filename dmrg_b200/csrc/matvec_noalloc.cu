// heff_matvec_d_noalloc: the real (fp64) H_eff matvec without any device allocation.
//
// Who needs it: a host program that has already divided the whole device memory among its own
// pools at start-up (a serving process that pins every byte for resident environments, or an
// application whose caching allocator owns the device) and does not permit a library to call
// cudaMalloc behind its back.  cudaMalloc/cudaFree also synchronise the device, which stalls the
// other streams of such a program.  heff_matvec_d takes its scratch from a workspace that grows
// with cudaMalloc; this entry point instead carves its scratch out of one fixed array compiled
// into the library.
//
// Limits and sharing:
//  * the array holds HEFF_NOALLOC_SCRATCH_BYTES (32 MiB); every GPU that loads the library
//    reserves that much until the process exits;
//  * a call whose scratch (x' + T1 + T2 + R', see matvec.cuh) exceeds it returns HEFF_BAD_SHAPE;
//  * every call on a device uses the same array, so calls that can run at the same time on the
//    GPU (different streams without ordering between them) race and corrupt each other; serialise them;
//  * the array keeps the previous call's contents; nothing in it needs to start at zero, since
//    every scratch element is written before it is read in each call;
//  * the first call on a device looks up the array's device address (cudaGetSymbolAddress, with
//    that device current) and caches it; make that first call before any stream capture.
#include <mutex>

#include "matvec.cuh"
#include "runtime.cuh"

#define HEFF_NOALLOC_SCRATCH_BYTES (32u << 20)

namespace heff {

static __device__ __align__(256) unsigned char g_noalloc_scratch[HEFF_NOALLOC_SCRATCH_BYTES];

static std::mutex g_noalloc_mutex;
static void      *g_noalloc_addr[64] = {nullptr};

// Device address of g_noalloc_scratch on the current device (host code must not use the symbol
// itself: in host code its name stands for a host-side shadow, not device memory).
static int noalloc_scratch(void **out) {
    int dev = 0;
    HEFF_CUDA(cudaGetDevice(&dev));
    if(dev < 0 || dev >= 64) return HEFF_NO_DEVICE;
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if(!g_noalloc_addr[dev]) {
        void       *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if(e != cudaSuccess || !p) {
            set_last_cuda_error(e, "cudaGetSymbolAddress(g_noalloc_scratch)", __FILE__, __LINE__);
            return HEFF_CUDA_ERROR;
        }
        g_noalloc_addr[dev] = p;
    }
    *out = g_noalloc_addr[dev];
    return HEFF_OK;
}

}  // namespace heff

using namespace heff;

extern "C" int heff_matvec_d_noalloc(double *res, const double *mps, const int64_t mps_dims[3], const double *mpo, const int64_t mpo_dims[4],
                                     const double *envL, const int64_t envL_dims[3], const double *envR, const int64_t envR_dims[3],
                                     void *stream) {
    MatvecDims d;
    HEFF_TRY(check_matvec_dims(mps_dims, mpo_dims, envL_dims, envR_dims, d));
    if(!res || !mps || !mpo || !envL || !envR) return HEFF_BAD_ARG;
    if(res == mps) {
        set_last_error_msg("matvec: res must not alias mps");
        return HEFF_BAD_ARG;
    }
    const int64_t elems = MatvecScratch<false>::elems(d) + MatvecScratch<false>::pad(d.size_Rp());
    const size_t  bytes = (size_t)elems * sizeof(double);
    if(bytes > HEFF_NOALLOC_SCRATCH_BYTES) {
        set_last_error_msg("heff_matvec_d_noalloc: needs %zu bytes of scratch for mps [%lld,%lld,%lld], mpo bond [%lld,%lld]; the fixed "
                           "scratch array holds %u bytes (use heff_matvec_d)",
                           bytes, (long long)d.S, (long long)d.cL, (long long)d.cR, (long long)d.DL, (long long)d.DR,
                           (unsigned)HEFF_NOALLOC_SCRATCH_BYTES);
        return HEFF_BAD_SHAPE;
    }
    void *base = nullptr;
    HEFF_TRY(noalloc_scratch(&base));
    cudaStream_t        s = (cudaStream_t)stream;
    MatvecScratch<false> ws;
    double              *Rp = ws.carve(reinterpret_cast<double *>(base), d);
    HEFF_TRY(permute_R<false>(envR, Rp, d, s));
    return matvec_fp64<false>(d, mps, res, envL, Rp, mpo, ws, s);
}
