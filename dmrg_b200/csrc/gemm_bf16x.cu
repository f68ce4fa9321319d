// tcgen05 BF16 GEMM (see gemm_bf16x.cuh).
#include <algorithm>
#include <cstring>

#include "gemm_bf16x.cuh"
#include "tcgen05.cuh"
#include "runtime.cuh"

namespace heff {

using namespace tc;

// kind::f16 instruction descriptor: D=F32, A=B=BF16, both K-major, N=256, M=128
constexpr uint32_t X_IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(X_BN >> 3) << 17) | ((uint32_t)(X_BM >> 4) << 24);

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(X_IDESC), "r"(accumulate)
        : "memory");
}

constexpr int X_GROUP_M = 8;

__device__ __forceinline__ void x_tile_mn(const XGemmArgs &p, int tile, int &m0, int &n0) {
    const int num_m = (p.M + X_BM - 1) / X_BM, num_n = (p.N + X_BN - 1) / X_BN;
    const int per_group = X_GROUP_M * num_n;
    const int first_m   = (tile / per_group) * X_GROUP_M;
    const int gsize     = min(num_m - first_m, X_GROUP_M);
    m0                  = (first_m + (tile % per_group) % gsize) * X_BM;
    n0                  = ((tile % per_group) / gsize) * X_BN;
}

__device__ __forceinline__ void x_store(const XGemmArgs &p, int row, int n, float v) {
    if(p.mode == X_OUT_F32)
        reinterpret_cast<float *>(p.C)[row + p.ldc * n] = v;
    else if(p.mode == X_OUT_F32_ACC)
        reinterpret_cast<float *>(p.C)[row + p.ldc * n] += v;
    else if(p.mode == X_OUT_F64)
        reinterpret_cast<double *>(p.C)[row + p.ldc * n] = (double)v;
    else {
        const bool im = n >= p.n_half;
        const int  nn = im ? n - p.n_half : n;
        reinterpret_cast<double *>(p.C)[2 * (row + p.ldc * nn) + (im ? 1 : 0)] = (double)v;
    }
}

// Persistent CTA (one per SM): walks the tiles t = blockIdx.x, blockIdx.x + gridDim.x, ... (grouped order)
//   warp 0 lane 0: TMA producer over the k-blocks of all its tiles (one continuous smem ring)
//   warp 1 lane 0: MMA issuer into TMEM accumulator buffer (j & 1) for the CTA's j-th tile
//   warps 2-5:     epilogue of tile j from buffer (j & 1) while the MMAs of tile j+1 run in the other buffer
__global__ void __launch_bounds__(X_THREADS, 1)
    gemm_bf16x_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, const XGemmArgs p) {
    extern __shared__ __align__(1024) unsigned char xsm_raw[];
    unsigned char *smem = reinterpret_cast<unsigned char *>((reinterpret_cast<uintptr_t>(xsm_raw) + 1023) & ~uintptr_t(1023));
    uint64_t      *full      = reinterpret_cast<uint64_t *>(smem + X_STAGES * X_STAGE_BYTES);
    uint64_t      *empty     = full + X_STAGES;
    uint64_t      *acc_full  = empty + X_STAGES;  // [2]
    uint64_t      *acc_empty = acc_full + 2;      // [2]
    uint32_t      *tmem_slot = reinterpret_cast<uint32_t *>(acc_empty + 2);
    int           *s_fail    = reinterpret_cast<int *>(tmem_slot + 1);  // an epilogue wait timed out

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ntiles = ((p.M + X_BM - 1) / X_BM) * ((p.N + X_BN - 1) / X_BN);
    const int KB     = (p.K + X_BK - 1) / X_BK;

    if(threadIdx.x == 0) {
        for(int s = 0; s < X_STAGES; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for(int b = 0; b < 2; b++) {
            mbar_init(&acc_full[b], 1);
            mbar_init(&acc_empty[b], 128);
        }
        *s_fail = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if(warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(saddr(tmem_slot)), "r"(2 * X_BN) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem_base = *tmem_slot;

    if(warp == 0) {
        if(lane == 0) {  // TMA producer
            int  it = 0;
            bool ok = true;
            for(int t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
                int m0, n0;
                x_tile_mn(p, t, m0, n0);
                for(int kb = 0; kb < KB; kb++, it++) {
                    const int      st = it % X_STAGES;
                    const uint32_t ph = (it / X_STAGES) & 1;
                    if(!mbar_wait(&empty[st], ph ^ 1)) {
                        atomicExch(p.err, 1);
                        ok = false;
                        break;
                    }
                    unsigned char *a = smem + st * X_STAGE_BYTES, *b = a + X_A_BYTES;
                    mbar_expect_tx(&full[st], X_STAGE_BYTES);
                    tma_load_2d(&tmA, &full[st], a, kb * X_BK, m0);
                    tma_load_2d(&tmB, &full[st], b, kb * X_BK, n0);
                }
            }
        }
    } else if(warp == 1) {
        if(lane == 0) {  // MMA issuer
            int  it = 0, j = 0;
            bool ok = true;
            for(int t = blockIdx.x; t < ntiles && ok; t += gridDim.x, j++) {
                const int      buf = j & 1;
                const uint32_t acc = tmem_base + (uint32_t)(buf * X_BN);
                if(!mbar_wait(&acc_empty[buf], ((j >> 1) & 1) ^ 1)) {  // the epilogue drained this buffer
                    atomicExch(p.err, 4);
                    break;
                }
                fence_after();
                for(int kb = 0; kb < KB; kb++, it++) {
                    const int      st = it % X_STAGES;
                    const uint32_t ph = (it / X_STAGES) & 1;
                    if(!mbar_wait(&full[st], ph)) {
                        atomicExch(p.err, 2);
                        ok = false;
                        break;
                    }
                    fence_after();
                    const uint32_t a = saddr(smem + st * X_STAGE_BYTES), b = a + X_A_BYTES;
#pragma unroll
                    for(int k = 0; k < X_BK / 16; k++) umma_bf16(acc, sdesc_sw128(a + 32 * k), sdesc_sw128(b + 32 * k), (kb | k) != 0);
                    umma_commit(&empty[st]);
                }
                if(ok) umma_commit(&acc_full[buf]);  // fires when every MMA of this tile has completed
            }
        }
    } else {
        // epilogue: warps 2..5 -> TMEM lane quarters 2,3,0,1
        const int q = warp & 3;
        int       j = 0;
        for(int t = blockIdx.x; t < ntiles; t += gridDim.x, j++) {
            const int buf = j & 1;
            int       m0, n0;
            x_tile_mn(p, t, m0, n0);
            if(!mbar_wait(&acc_full[buf], (j >> 1) & 1)) {
                atomicExch(p.err, 3);
                atomicOr(s_fail, 1);
            }
            epi_bar();  // every epilogue warp takes the same decision
            if(*s_fail) break;
            fence_after();
            const int row = m0 + q * 32 + lane;
            for(int c = 0; c < X_BN; c += 32) {
                uint32_t r[32];
                tmem_ld32(tmem_base + ((uint32_t)(q * 32) << 16) + (uint32_t)(buf * X_BN + c), r);
                if(row < p.M) {
#pragma unroll
                    for(int jj = 0; jj < 32; jj++) {
                        const int n = n0 + c + jj;
                        if(n < p.N) x_store(p, row, n, __uint_as_float(r[jj]));
                    }
                }
            }
            fence_before();
            mbar_arrive(&acc_empty[buf]);  // TMEM buffer free for the tile after next
            epi_bar();                     // *s_fail is read by all before the next wait may set it
        }
    }
    fence_before();
    __syncthreads();
    if(warp == 1) {
        fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base), "r"(2 * X_BN) : "memory");
    }
}

typedef CUresult (*PFN_encodeTiled)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *, const cuuint64_t *,
                                    const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle, CUtensorMapL2promotion,
                                    CUtensorMapFloatOOBfill);

static PFN_encodeTiled encode_fn() {
    static PFN_encodeTiled fn = nullptr;
    if(!fn) {
        void                            *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess && q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_encodeTiled>(p);
    }
    return fn;
}

int make_tmap_bf16(CUtensorMap *map, const void *base, int64_t rows, int64_t kcols, int64_t ld_elems, int box_rows) {
    PFN_encodeTiled fn = encode_fn();
    if(!fn) {
        set_last_error_msg("cuTensorMapEncodeTiled is not available from the driver");
        return HEFF_CUDA_ERROR;
    }
    if(((uintptr_t)base & 15) || (ld_elems * 2) % 16 || kcols % 8) return HEFF_BAD_ARG;
    std::memset(map, 0, sizeof(*map));
    cuuint64_t dims[2]    = {(cuuint64_t)kcols, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)(ld_elems * 2)};
    cuuint32_t box[2]     = {(cuuint32_t)X_BK, (cuuint32_t)box_rows};
    cuuint32_t estr[2]    = {1, 1};
    CUresult   r = fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void *>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                      CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if(r != CUDA_SUCCESS) {
        set_last_error_msg("cuTensorMapEncodeTiled failed (%d)", (int)r);
        return HEFF_CUDA_ERROR;
    }
    return HEFF_OK;
}

int gemm_bf16x(const CUtensorMap &tmA, const CUtensorMap &tmB, const XGemmArgs &a, cudaStream_t s) {
    if(a.M <= 0 || a.N <= 0) return HEFF_OK;
    if(a.K <= 0 || a.K % 8) return HEFF_BAD_ARG;  // K tail beyond a multiple of 64 is zero-filled by TMA
    static int attr_done[64] = {0};
    int        dev           = 0;
    HEFF_CUDA(cudaGetDevice(&dev));
    if(dev < 0 || dev >= 64 || !attr_done[dev]) {
        HEFF_CUDA(cudaFuncSetAttribute(gemm_bf16x_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, X_SMEM_BYTES));
        if(dev >= 0 && dev < 64) attr_done[dev] = 1;
    }
    const int64_t tiles = cdiv(a.M, X_BM) * cdiv(a.N, X_BN);
    if(tiles > 0x7fffffff) return HEFF_BAD_SHAPE;
    const int grid = (int)std::min<int64_t>(tiles, device_sm_count());  // persistent: one CTA per SM
    gemm_bf16x_kernel<<<(unsigned)grid, X_THREADS, X_SMEM_BYTES, s>>>(tmA, tmB, a);
    HEFF_LAUNCH_CHECK();
    return HEFF_OK;
}

}  // namespace heff

using namespace heff;

extern "C" int heff_gemm_bf16_f32(const void *A, const void *B, float *C, int64_t M, int64_t N, int64_t K, void *stream) {
    if(!A || !B || !C || M <= 0 || N <= 0 || K <= 0) return HEFF_BAD_ARG;
    if(K % 8 || M > 0x7fffffff || N > 0x7fffffff || K > 0x7fffffff) {
        set_last_error_msg("heff_gemm_bf16_f32: K must be a multiple of 8");
        return HEFF_BAD_SHAPE;
    }
    CUtensorMap ta, tb;
    HEFF_TRY(make_tmap_bf16(&ta, A, M, K, K, X_BM));
    HEFF_TRY(make_tmap_bf16(&tb, B, N, K, K, X_BN));
    void *err = nullptr;
    HEFF_TRY(stream_workspace((cudaStream_t)stream, 256, &err));
    HEFF_CUDA(cudaMemsetAsync(err, 0, sizeof(int), (cudaStream_t)stream));
    XGemmArgs g{};
    g.M = (int)M, g.N = (int)N, g.K = (int)K, g.C = C, g.ldc = M, g.mode = X_OUT_F32, g.err = reinterpret_cast<int *>(err);
    HEFF_TRY(gemm_bf16x(ta, tb, g, (cudaStream_t)stream));
    int h = 0;
    HEFF_CUDA(cudaMemcpyAsync(&h, err, sizeof(int), cudaMemcpyDeviceToHost, (cudaStream_t)stream));
    HEFF_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
    if(h) {
        set_last_error_msg("heff_gemm_bf16_f32: pipeline wait timed out (code %d)", h);
        return HEFF_TIMEOUT;
    }
    return HEFF_OK;
}
