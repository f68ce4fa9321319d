// Host-side dispatch of the DMMA GEMM template (gemm_f64.cuh).
#include "gemm_f64.cuh"

namespace heff {

template<bool CPLX, bool TA, bool TB, bool CJA, int VEC>
static int launch_gemm(const GemmArgs &a, cudaStream_t stream) {
    using G                  = GemmTile<CPLX>;
    using SM                 = GemmSmem<CPLX, TA, TB>;
    auto       kern = gemm_f64_kernel<CPLX, TA, TB, CJA, VEC>;
    static int attr_done[64] = {0};  // per instantiation and device; setting it twice is harmless
    int        dev           = 0;
    HEFF_CUDA(cudaGetDevice(&dev));
    if(dev < 0 || dev >= 64 || !attr_done[dev]) {
        HEFF_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SM::BYTES));
        if(dev >= 0 && dev < 64) attr_done[dev] = 1;
    }
    const int64_t tiles = cdiv(a.M, G::BM) * cdiv(a.N, G::BN);
    if(tiles > 0x7fffffffLL) return HEFF_BAD_SHAPE;
    dim3 grid((unsigned)tiles, 1u, (unsigned)a.batch);
    kern<<<grid, 256, SM::BYTES, stream>>>(a);
    HEFF_LAUNCH_CHECK();
    return HEFF_OK;
}

static bool aligned16(const void *p) { return ((uintptr_t)p & 15u) == 0; }

template<>
int gemm_f64<false>(bool ta, bool tb, bool cja, const GemmArgs &a, cudaStream_t s) {
    (void)cja;
    if(a.M <= 0 || a.N <= 0 || a.batch <= 0) return HEFF_OK;
    if(a.K <= 0) return HEFF_BAD_ARG;  // callers never form empty contractions
    if(a.batch > 65535 || cdiv(a.N, GemmTile<false>::BN) > 65535) return HEFF_BAD_SHAPE;
    // 16-byte copies need: 16B-aligned bases, even leading dims / batch strides, even contiguous extent.
    const bool v2 = aligned16(a.A) && aligned16(a.B) && (a.lda % 2 == 0) && (a.ldb % 2 == 0) && (a.sA % 2 == 0) && (a.sB % 2 == 0) &&
                    ((ta ? a.K : a.M) % 2 == 0) && ((tb ? a.N : a.K) % 2 == 0);
    if(v2) {
        if(!ta && !tb) return launch_gemm<false, false, false, false, 2>(a, s);
        if(ta && !tb) return launch_gemm<false, true, false, false, 2>(a, s);
        if(!ta && tb) return launch_gemm<false, false, true, false, 2>(a, s);
        return launch_gemm<false, true, true, false, 2>(a, s);
    }
    if(!ta && !tb) return launch_gemm<false, false, false, false, 1>(a, s);
    if(ta && !tb) return launch_gemm<false, true, false, false, 1>(a, s);
    if(!ta && tb) return launch_gemm<false, false, true, false, 1>(a, s);
    return launch_gemm<false, true, true, false, 1>(a, s);
}

template<>
int gemm_f64<true>(bool ta, bool tb, bool cja, const GemmArgs &a, cudaStream_t s) {
    if(a.M <= 0 || a.N <= 0 || a.batch <= 0) return HEFF_OK;
    if(a.K <= 0) return HEFF_BAD_ARG;
    if(a.batch > 65535 || cdiv(a.N, GemmTile<true>::BN) > 65535) return HEFF_BAD_SHAPE;
    if(!aligned16(a.A) || !aligned16(a.B)) return HEFF_BAD_ARG;  // complex128 buffers are always 16-byte aligned
    if(cja) {
        if(!ta && !tb) return launch_gemm<true, false, false, true, 1>(a, s);
        if(ta && !tb) return launch_gemm<true, true, false, true, 1>(a, s);
        if(!ta && tb) return launch_gemm<true, false, true, true, 1>(a, s);
        return launch_gemm<true, true, true, true, 1>(a, s);
    }
    if(!ta && !tb) return launch_gemm<true, false, false, false, 1>(a, s);
    if(ta && !tb) return launch_gemm<true, true, false, false, 1>(a, s);
    if(!ta && tb) return launch_gemm<true, false, true, false, 1>(a, s);
    return launch_gemm<true, true, true, false, 1>(a, s);
}

}  // namespace heff
