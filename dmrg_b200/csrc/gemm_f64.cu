// Host-side dispatch of the DMMA GEMM template (gemm_f64.cuh).
#include <algorithm>
#include <atomic>
#include <cstdlib>
#include <mutex>
#include <vector>

#include "gemm_f64.cuh"
#include "runtime.cuh"

namespace heff {

// Tail-split mode of the DMMA GEMMs: 0 off, 1 automatic (the cost model below), 2..16 that many pieces whenever
// the tiles leave a partial wave.  Initial value from the environment variable HEFF_GEMM_SPLIT (default 1).
static std::atomic<int> g_split_mode{-1};

static int split_mode() {
    int m = g_split_mode.load();
    if(m < 0) {
        const char *e      = getenv("HEFF_GEMM_SPLIT");
        const int   v      = e ? atoi(e) : 1;
        int         expect = -1;
        g_split_mode.compare_exchange_strong(expect, (v >= 0 && v <= 16) ? v : 1);
        m = g_split_mode.load();
    }
    return m;
}

SplitPlan gemm_split_plan(int64_t tiles, int KT, int64_t slots, int64_t max_units, double tile_s, double unit_bytes) {
    SplitPlan best;
    best.nfull = (int)tiles;
    const int mode = split_mode();
    if(mode == 0 || slots <= 0 || tiles <= 0 || tiles % slots == 0 || tile_s <= 0) return best;
    const int64_t waves = tiles / slots, rem = tiles % slots;
    if(mode >= 2) {  // forced piece count (when the pieces keep >= 1 k-tile and fit the scratch)
        if(KT >= mode && rem * mode <= max_units) {
            best.split = mode;
            best.nfull = (int)(tiles - rem);
        }
        return best;
    }
    // cost of a split in units of one whole tile's time: the reduction launch plus the partial tiles written
    // and read back at HBM speed (device-wide)
    constexpr double kLaunchS = 5e-6, kHbmBps = 6.0e12;
    double           best_cost = (double)waves + 1.0;
    for(int s = 2; s <= SPLIT_MAX; s++) {
        if(KT / s < 4) break;
        const int64_t units = rem * s;
        if(units > max_units) break;
        const double cost = (double)waves + (double)cdiv(units, slots) / s + (kLaunchS + 2.0 * unit_bytes * units / kHbmBps) / tile_s;
        if(cost < best_cost - 1e-9) {
            best_cost  = cost;
            best.split = s;
            best.nfull = (int)(tiles - rem);
        }
    }
    return best;
}

size_t gemm_split_ws_bytes() {
    // at most 4 partial tiles per co-resident CTA (the real kernel runs one 128x128 CTA per SM)
    return (size_t)4 * device_sm_count() * GemmTile<false>::BM * GemmTile<false>::BN * sizeof(double);
}

// Every DMMA GEMM kernel (and split reduction) this process has launched; a captured graph's kernel nodes are
// recognised by their function (their one parameter is a GemmArgs), so a replay can retarget their output.
static std::mutex               g_gemm_fn_mu;
static std::vector<const void *> g_gemm_fns;
static void gemm_fn_register(const void *f) {
    std::lock_guard<std::mutex> lk(g_gemm_fn_mu);
    if(std::find(g_gemm_fns.begin(), g_gemm_fns.end(), f) == g_gemm_fns.end()) g_gemm_fns.push_back(f);
}
bool gemm_fn_known(const void *f) {
    std::lock_guard<std::mutex> lk(g_gemm_fn_mu);
    return std::find(g_gemm_fns.begin(), g_gemm_fns.end(), f) != g_gemm_fns.end();
}

template<bool CPLX, bool TA, bool TB, bool CJA, int VEC>
static int launch_gemm(const GemmArgs &a_in, cudaStream_t stream) {
    using G                  = GemmTile<CPLX>;
    using SM                 = GemmSmem<CPLX, TA, TB>;
    using T                  = typename Scalar<CPLX>::T;
    auto       kern = gemm_f64_kernel<CPLX, TA, TB, CJA, VEC>;
    static int occ[64] = {0};  // per instantiation and device: co-resident CTAs per SM (0 = not set up yet)
    int        dev     = 0;
    HEFF_CUDA(cudaGetDevice(&dev));
    if(dev < 0 || dev >= 64 || !occ[dev]) {
        HEFF_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SM::BYTES));
        int n = 0;
        HEFF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kern, 256, SM::BYTES));
        if(dev >= 0 && dev < 64) occ[dev] = n > 0 ? n : 1;
    }
    const int     per_sm = (dev >= 0 && dev < 64) ? occ[dev] : 1;
    const int64_t tiles  = cdiv(a_in.M, G::BM) * cdiv(a_in.N, G::BN);
    if(tiles > 0x7fffffffLL) return HEFF_BAD_SHAPE;
    GemmArgs  a = a_in;
    SplitPlan sp;
    sp.nfull = (int)tiles;
    if(a.split_ws && a.batch == 1) {
        const int64_t tile_bytes = (int64_t)G::BM * G::BN * sizeof(T);
        // one whole tile's time on one SM: its DMMA work (3 real products per complex one) at ~30 TFLOP/s per device
        const double  sms    = (double)device_sm_count();
        const double  tile_s = (CPLX ? 3.0 : 1.0) * 2.0 * G::BM * G::BN * (double)a.K / (30e12 / sms) * per_sm;
        sp = gemm_split_plan(tiles, (int)cdiv(a.K, G::BK), (int64_t)device_sm_count() * per_sm, (int64_t)(a.split_ws_bytes / tile_bytes), tile_s,
                             (double)tile_bytes);
    }
    a.split = sp.split;
    a.nfull = sp.nfull;
    a.part  = sp.split > 1 ? a.split_ws : nullptr;
    const int64_t ctas = sp.nfull + (tiles - sp.nfull) * sp.split;
    if(ctas > 0x7fffffffLL) return HEFF_BAD_SHAPE;
    dim3 grid((unsigned)ctas, 1u, (unsigned)a.batch);
    gemm_fn_register(reinterpret_cast<const void *>(kern));
    kern<<<grid, 256, SM::BYTES, stream>>>(a);
    HEFF_LAUNCH_CHECK();
    count_launches(sp.split > 1 ? 2 : 1);
    if(sp.split > 1) {
        const dim3 rgrid((unsigned)(tiles - sp.nfull), (unsigned)(SplitReduce<CPLX>::EPT / SplitReduce<CPLX>::EPB));
        gemm_fn_register(reinterpret_cast<const void *>(gemm_split_reduce_kernel<CPLX>));
        gemm_split_reduce_kernel<CPLX><<<rgrid, 256, 0, stream>>>(a);
        HEFF_LAUNCH_CHECK();
    }
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

extern "C" int heff_gemm_set_tail_split(int mode) {
    if(mode < 0 || mode > heff::SPLIT_MAX) return -1;
    const int prev = heff::split_mode();
    heff::g_split_mode.store(mode);
    return prev;
}
