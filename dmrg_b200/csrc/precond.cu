// Jacobi (diagonal) preconditioner of the effective Hamiltonian.
//
// Diagonal: MatVecMPOS::get_diagonal_new / get_matrix_element (source/math/eig/matvec/matvec_mpos.cpp:300-407)
// at I == J: for I = s + S (a + cL b),
//     diag[I] = sum_{m,n} L[a, a, m] W[m, n, s, s] R[b, b, n],
// one thread per element (S cL cR DL DR multiply-adds in total, negligible next to one matvec).
// Application: the block-size-1 branch of MultPc (matvec_mpos.cpp:1349-1364),
//     y = x / (diag - shift),
// with the denominator kept at least 1e-10 max(|shift|, 1) in magnitude (the reference divides unguarded).
//
// Block Jacobi (jcbMaxBlockSize > 1; CalcPc and MultPc, matvec_mpos.cpp:1087-1240, 1349-1416): the flattened
// index range [0, n) is cut into consecutive blocks of `bs` indices (the last one shorter), each block
// B_k = H[blk, blk] - shift I is formed once, at the shift of the first MultPc after a (re)bind (the reference's
// readyCalcPc), and MultPc applies y_blk = B_k^-1 x_blk.  The reference factorises each block (LLT of +-B_k,
// falling back to LDLT and then LU) and solves; here every block is inverted explicitly on the device by
// Gauss-Jordan elimination with partial (row) pivoting -- the same operator B_k^-1 for any nonsingular block,
// and MultPc becomes one batched matrix-vector product.  A pivot below 1e-14 of the block's largest entry is
// replaced by that floor (counted in jcb_singular; the reference's LU would divide by it).
#include <algorithm>
#include <cmath>

#include "op.cuh"
#include "runtime.cuh"

namespace heff {

__device__ __forceinline__ double pc_mul(double a, double b) { return a * b; }
__device__ __forceinline__ double2 pc_mul(double2 a, double2 b) { return cmul(a, b); }
__device__ __forceinline__ double pc_add(double a, double b) { return a + b; }
__device__ __forceinline__ double2 pc_add(double2 a, double2 b) { return cadd(a, b); }
__device__ __forceinline__ double pc_re(double a) { return a; }
__device__ __forceinline__ double pc_re(double2 a) { return a.x; }
__device__ __forceinline__ double pc_scale(double a, double f) { return a * f; }
__device__ __forceinline__ double2 pc_scale(double2 a, double f) { return make_double2(a.x * f, a.y * f); }

// L in the reference layout L[a + cL (a' + cL m)]; R permuted R'[b + cR n + cR DR b'] (matvec.cu)
template<class T>
__global__ void diag_kernel(const T *__restrict__ L, const T *__restrict__ Rp, const T *__restrict__ W, int64_t S, int64_t cL, int64_t cR, int DL,
                            int DR, T *__restrict__ out) {
    const int64_t n = S * cL * cR;
    for(int64_t o = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; o < n; o += (int64_t)gridDim.x * blockDim.x) {
        const int64_t s = o % S, a = (o / S) % cL, b = o / (S * cL);
        T             acc{};
        for(int m = 0; m < DL; m++) {
            const T l = L[a + cL * (a + cL * (int64_t)m)];
            T       inner{};
            for(int nn = 0; nn < DR; nn++)
                inner = pc_add(inner, pc_mul(W[m + (int64_t)DL * (nn + (int64_t)DR * (s + S * s))], Rp[b + cR * nn + cR * DR * b]));
            acc = pc_add(acc, pc_mul(l, inner));
        }
        out[o] = acc;
    }
}

template<class T>
__global__ void multpc_kernel(const T *__restrict__ x, const T *__restrict__ diag, double shift, T *__restrict__ y, int64_t n) {
    const double floor_ = 1e-10 * fmax(fabs(shift), 1.0);
    for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double den = pc_re(diag[i]) - shift;
        if(fabs(den) < floor_) den = den < 0 ? -floor_ : floor_;
        y[i] = pc_scale(x[i], 1.0 / den);
    }
}

static int pc_grid(int64_t n) {
    const int64_t g = (n + 255) / 256, cap = (int64_t)device_sm_count() * 8;
    return (int)(g < 1 ? 1 : (g < cap ? g : cap));
}

__device__ __forceinline__ double pc_abs(double a) { return fabs(a); }
__device__ __forceinline__ double pc_abs(double2 a) { return hypot(a.x, a.y); }
__device__ __forceinline__ double pc_inv(double a) { return 1.0 / a; }
__device__ __forceinline__ double2 pc_inv(double2 a) {
    const double d = a.x * a.x + a.y * a.y;
    return make_double2(a.x / d, -a.y / d);
}
__device__ __forceinline__ double pc_sub(double a, double b) { return a - b; }
__device__ __forceinline__ double2 pc_sub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double pc_real(double v) { return v; }
template<class T>
__device__ __forceinline__ T pc_from_real(double v);
template<>
__device__ __forceinline__ double pc_from_real<double>(double v) { return v; }
template<>
__device__ __forceinline__ double2 pc_from_real<double2>(double v) { return make_double2(v, 0.0); }

// blocks[k][i + bs j] = H[k bs + i, k bs + j] - shift delta_ij (column-major per block); indices past n give the
// identity, so the padded tail of the last block inverts to itself and never touches a real entry.
template<class T>
__global__ void jcb_extract_kernel(const T *__restrict__ L, const T *__restrict__ Rp, const T *__restrict__ W, int64_t S, int64_t cL, int64_t cR,
                                   int DL, int DR, int64_t bs, int64_t nb, double shift, T *__restrict__ blocks) {
    const int64_t n = S * cL * cR, per = bs * bs, tot = nb * per;
    for(int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < tot; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t k = e / per, rem = e - k * per, i = rem % bs, j = rem / bs;
        const int64_t r = k * bs + i, c = k * bs + j;
        T             acc{};
        if(r >= n || c >= n) {
            acc = pc_from_real<T>(i == j ? 1.0 : 0.0);
        } else {
            // r = (s', a', b') (output), c = (s, a, b) (input): H[r, c] = sum_{m,n} L[a, a', m] W[m, n, s, s'] R[b, b', n]
            const int64_t s1 = r % S, a1 = (r / S) % cL, b1 = r / (S * cL);
            const int64_t s0 = c % S, a0 = (c / S) % cL, b0 = c / (S * cL);
            for(int m = 0; m < DL; m++) {
                const T l = L[a0 + cL * (a1 + cL * (int64_t)m)];
                T       inner{};
                for(int nn = 0; nn < DR; nn++)
                    inner = pc_add(inner, pc_mul(W[m + (int64_t)DL * (nn + (int64_t)DR * (s0 + S * s1))], Rp[b0 + cR * nn + cR * DR * b1]));
                acc = pc_add(acc, pc_mul(l, inner));
            }
            if(r == c) acc = pc_sub(acc, pc_from_real<T>(shift));
        }
        blocks[e] = acc;
    }
}

__host__ __device__ constexpr size_t jcb_r16(size_t b) { return (b + 15) / 16 * 16; }

// In-place Gauss-Jordan inversion with partial (row) pivoting of one bs x bs block per CTA (column-major), in
// shared memory when it fits (SMEM) or in the block's own global storage.  Row interchanges are undone at the end
// as column interchanges in reverse order.
template<class T, bool SMEM>
__global__ void __launch_bounds__(256) jcb_invert_kernel(T *__restrict__ blocks, int bs, int *__restrict__ singular) {
    extern __shared__ __align__(16) unsigned char jcb_smem[];
    // carve (every piece 16-byte aligned; jcb_smem_fixed gives the same total)
    const size_t o_perm = jcb_r16(sizeof(T) * bs), o_rv = o_perm + jcb_r16(sizeof(int) * bs), o_ri = o_rv + 64, o_sinv = o_ri + 32,
                 o_amax = o_sinv + 16, o_A = o_amax + 16;
    T        *f     = reinterpret_cast<T *>(jcb_smem);                 // bs: column k before the update
    int      *perm  = reinterpret_cast<int *>(jcb_smem + o_perm);      // bs: pivot row of each step
    double   *rv    = reinterpret_cast<double *>(jcb_smem + o_rv);     // 8 warps: |value| of the warp's best row
    int      *ri    = reinterpret_cast<int *>(jcb_smem + o_ri);        // 8 warps: its row
    T        *sinv  = reinterpret_cast<T *>(jcb_smem + o_sinv);        // inverse pivot
    double   *samax = reinterpret_cast<double *>(jcb_smem + o_amax);   // largest |entry| of the block
    T        *A     = SMEM ? reinterpret_cast<T *>(jcb_smem + o_A) : blocks + (int64_t)blockIdx.x * bs * bs;
    T        *G    = blocks + (int64_t)blockIdx.x * bs * bs;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int per = bs * bs;
    // load (shared-memory variant) and largest magnitude of the block (pivot floor)
    double amax = 0.0;
    for(int e = tid; e < per; e += 256) {
        const T v = G[e];
        if(SMEM) A[e] = v;
        amax = fmax(amax, pc_abs(v));
    }
    for(int o = 16; o; o >>= 1) amax = fmax(amax, __shfl_xor_sync(0xffffffffu, amax, o));
    if(lane == 0) rv[warp] = amax;
    __syncthreads();
    if(tid == 0) {
        double m = 0.0;
        for(int w = 0; w < 8; w++) m = fmax(m, rv[w]);
        samax[0] = m;
    }
    __syncthreads();
    const double floor_ = 1e-14 * (samax[0] > 0.0 ? samax[0] : 1.0);
    for(int k = 0; k < bs; k++) {
        // pivot: the largest |A(i, k)| for i >= k (lowest row on ties)
        double best = -1.0;
        int    bi   = k;
        for(int i = k + tid; i < bs; i += 256) {
            const double v = pc_abs(A[i + (int64_t)bs * k]);
            if(v > best) {
                best = v;
                bi   = i;
            }
        }
        for(int o = 16; o; o >>= 1) {
            const double ov = __shfl_xor_sync(0xffffffffu, best, o);
            const int    oi = __shfl_xor_sync(0xffffffffu, bi, o);
            if(ov > best || (ov == best && oi < bi)) {
                best = ov;
                bi   = oi;
            }
        }
        if(lane == 0) {
            rv[warp] = best;
            ri[warp] = bi;
        }
        __syncthreads();
        if(tid == 0) {
            double b = rv[0];
            int    p = ri[0];
            for(int w = 1; w < 8; w++)
                if(rv[w] > b || (rv[w] == b && ri[w] < p)) {
                    b = rv[w];
                    p = ri[w];
                }
            perm[k] = p;
        }
        __syncthreads();
        const int p = perm[k];
        if(p != k)
            for(int j = tid; j < bs; j += 256) {
                const T t             = A[k + (int64_t)bs * j];
                A[k + (int64_t)bs * j] = A[p + (int64_t)bs * j];
                A[p + (int64_t)bs * j] = t;
            }
        __syncthreads();
        for(int i = tid; i < bs; i += 256) f[i] = i == k ? T{} : A[i + (int64_t)bs * k];
        if(tid == 0) {
            T piv = A[k + (int64_t)bs * k];
            if(!(pc_abs(piv) >= floor_)) {  // (near-)singular block: floor the pivot, keep its sign
                const double sgn = pc_re(piv) < 0.0 ? -1.0 : 1.0;
                piv              = pc_from_real<T>(sgn * floor_);
                atomicAdd(singular, 1);
            }
            sinv[0] = pc_inv(piv);
        }
        __syncthreads();
        const T inv = sinv[0];
        for(int j = tid; j < bs; j += 256) A[k + (int64_t)bs * j] = j == k ? inv : pc_mul(A[k + (int64_t)bs * j], inv);
        __syncthreads();
        for(int e = tid; e < per; e += 256) {
            const int i = e % bs, j = e / bs;
            if(i == k) continue;
            const T aij = j == k ? T{} : A[e];
            A[e]        = pc_sub(aij, pc_mul(f[i], A[k + (int64_t)bs * j]));
        }
        __syncthreads();
    }
    for(int k = bs - 1; k >= 0; k--) {
        const int p = perm[k];
        if(p != k)
            for(int i = tid; i < bs; i += 256) {
                const T t             = A[i + (int64_t)bs * k];
                A[i + (int64_t)bs * k] = A[i + (int64_t)bs * p];
                A[i + (int64_t)bs * p] = t;
            }
        __syncthreads();
    }
    if(SMEM)
        for(int e = tid; e < per; e += 256) G[e] = A[e];
}

// y_blk = B_k^-1 x_blk, one CTA per block (the segment of x staged in shared memory; column-major inverse read
// coalesced along rows).
template<class T>
__global__ void __launch_bounds__(256) jcb_apply_kernel(const T *__restrict__ inv, const T *__restrict__ x, T *__restrict__ y, int bs, int64_t n) {
    extern __shared__ __align__(16) unsigned char jcb_smem[];
    T            *xs  = reinterpret_cast<T *>(jcb_smem);
    const int64_t off = (int64_t)blockIdx.x * bs;
    const int     ext = (int)(n - off < (int64_t)bs ? n - off : (int64_t)bs);
    for(int j = threadIdx.x; j < bs; j += 256) xs[j] = j < ext ? x[off + j] : T{};
    __syncthreads();
    const T *B = inv + (int64_t)blockIdx.x * bs * bs;
    for(int i = threadIdx.x; i < ext; i += 256) {
        T acc{};
        for(int j = 0; j < ext; j++) acc = pc_add(acc, pc_mul(B[i + (int64_t)bs * j], xs[j]));
        y[off + i] = acc;
    }
}

static size_t jcb_smem_fixed(int bs, size_t es) { return jcb_r16(es * bs) + jcb_r16(sizeof(int) * bs) + 64 + 32 + 16 + 16; }

// Forms and inverts the Jacobi blocks at `shift` (stream-ordered; the buffer grows on demand).
template<class T>
static int jcb_build(heff_op *op, double shift) {
    const MatvecDims &d  = op->d;
    const int64_t     n  = d.size_mps(), bs = op->jcb_block, nb = (n + bs - 1) / bs;
    const size_t      es = sizeof(T);
    const size_t need    = (size_t)nb * bs * bs * es + 256;
    if(op->jcb_bytes < need) {
        if(op->jcb) {
            HEFF_CUDA(cudaStreamSynchronize(op->stream));
            cudaFree(op->jcb);
            op->jcb       = nullptr;
            op->jcb_bytes = 0;
        }
        cudaError_t e = cudaMalloc(&op->jcb, need);
        if(e != cudaSuccess) {
            op->jcb = nullptr;
            set_last_cuda_error(e, "block-Jacobi preconditioner", __FILE__, __LINE__);
            return HEFF_OOM;
        }
        op->jcb_bytes = need;
    }
    T   *blocks = reinterpret_cast<T *>(reinterpret_cast<unsigned char *>(op->jcb) + 256);
    int *sing   = reinterpret_cast<int *>(op->jcb);
    HEFF_CUDA(cudaMemsetAsync(sing, 0, sizeof(int), op->stream));
    const int64_t tot = nb * bs * bs;
    const int64_t g   = std::min<int64_t>((tot + 255) / 256, (int64_t)device_sm_count() * 16);
    jcb_extract_kernel<T><<<(int)std::max<int64_t>(g, 1), 256, 0, op->stream>>>(reinterpret_cast<const T *>(op->L), reinterpret_cast<const T *>(op->Rp),
                                                                               reinterpret_cast<const T *>(op->W), d.S, d.cL, d.cR, (int)d.DL, (int)d.DR,
                                                                               bs, nb, shift, blocks);
    HEFF_LAUNCH_CHECK();
    const size_t fixed = jcb_smem_fixed((int)bs, es);
    const size_t full  = fixed + (size_t)bs * bs * es;
    if(nb > 0x7fffffffLL) return HEFF_BAD_SHAPE;
    if(full <= 200 * 1024) {
        HEFF_CUDA(cudaFuncSetAttribute(jcb_invert_kernel<T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)full));
        jcb_invert_kernel<T, true><<<(unsigned)nb, 256, full, op->stream>>>(blocks, (int)bs, sing);
    } else {
        jcb_invert_kernel<T, false><<<(unsigned)nb, 256, fixed, op->stream>>>(blocks, (int)bs, sing);
    }
    HEFF_LAUNCH_CHECK();
    op->jcb_ready = true;
    op->jcb_shift = shift;
    return HEFF_OK;
}

template<class T>
static int jcb_apply(heff_op *op, const void *x, void *y) {
    const int64_t n = op->d.size_mps(), bs = op->jcb_block, nb = (n + bs - 1) / bs;
    const T      *blocks = reinterpret_cast<const T *>(reinterpret_cast<const unsigned char *>(op->jcb) + 256);
    jcb_apply_kernel<T><<<(unsigned)nb, 256, (size_t)bs * sizeof(T), op->stream>>>(blocks, reinterpret_cast<const T *>(x), reinterpret_cast<T *>(y),
                                                                                   (int)bs, n);
    HEFF_LAUNCH_CHECK();
    return HEFF_OK;
}

int op_diagonal_ready(heff_op *op) {
    if(op->diag_ready) return HEFF_OK;
    if(!op->W) {
        set_last_error_msg("preconditioner diagonal: the site MPOs are too large to tabulate their s == s' part");
        return HEFF_BAD_SHAPE;
    }
    const MatvecDims &d  = op->d;
    const int64_t     n  = d.size_mps();
    const size_t      es = op->cplx ? 16 : 8;
    if(n > op->diag_cap) {
        if(op->diag) {
            HEFF_CUDA(cudaStreamSynchronize(op->stream));
            cudaFree(op->diag);
            op->diag     = nullptr;
            op->diag_cap = 0;
        }
        cudaError_t e = cudaMalloc(&op->diag, n * es);
        if(e != cudaSuccess) {
            set_last_cuda_error(e, "preconditioner diagonal", __FILE__, __LINE__);
            return HEFF_OOM;
        }
        op->diag_cap = n;
    }
    if(op->cplx)
        diag_kernel<double2><<<pc_grid(n), 256, 0, op->stream>>>(reinterpret_cast<const double2 *>(op->L), reinterpret_cast<const double2 *>(op->Rp),
                                                                  reinterpret_cast<const double2 *>(op->W), d.S, d.cL, d.cR, (int)d.DL, (int)d.DR,
                                                                  reinterpret_cast<double2 *>(op->diag));
    else
        diag_kernel<double><<<pc_grid(n), 256, 0, op->stream>>>(reinterpret_cast<const double *>(op->L), reinterpret_cast<const double *>(op->Rp),
                                                                 reinterpret_cast<const double *>(op->W), d.S, d.cL, d.cR, (int)d.DL, (int)d.DR,
                                                                 reinterpret_cast<double *>(op->diag));
    HEFF_LAUNCH_CHECK();
    op->diag_ready = true;
    return HEFF_OK;
}

int op_multpc(heff_op *op, const void *x, void *y, double shift) {
    if(op->jcb_block > 1) {
        if(!op->W || op->sequential) {
            set_last_error_msg("block-Jacobi preconditioner: the site MPOs are too large to tabulate");
            return HEFF_BAD_SHAPE;
        }
        if(!op->jcb_ready) HEFF_TRY(op->cplx ? jcb_build<double2>(op, shift) : jcb_build<double>(op, shift));
        return op->cplx ? jcb_apply<double2>(op, x, y) : jcb_apply<double>(op, x, y);
    }
    HEFF_TRY(op_diagonal_ready(op));
    const int64_t n = op->d.size_mps();
    if(op->cplx)
        multpc_kernel<double2><<<pc_grid(n), 256, 0, op->stream>>>(reinterpret_cast<const double2 *>(x), reinterpret_cast<const double2 *>(op->diag),
                                                                    shift, reinterpret_cast<double2 *>(y), n);
    else
        multpc_kernel<double><<<pc_grid(n), 256, 0, op->stream>>>(reinterpret_cast<const double *>(x), reinterpret_cast<const double *>(op->diag), shift,
                                                                   reinterpret_cast<double *>(y), n);
    HEFF_LAUNCH_CHECK();
    return HEFF_OK;
}

}  // namespace heff

using namespace heff;

extern "C" int heff_op_diagonal(heff_op *op, void *diag_out) {
    if(!op || !diag_out) return HEFF_BAD_ARG;
    HEFF_TRY(op_diagonal_ready(op));
    const size_t es = op->cplx ? 16 : 8;
    HEFF_CUDA(cudaMemcpyAsync(diag_out, op->diag, op->d.size_mps() * es, cudaMemcpyDeviceToDevice, op->stream));
    return HEFF_OK;
}

extern "C" int heff_op_set_jacobi_blocksize(heff_op *op, int64_t block_size) {
    if(!op || block_size < 1 || block_size > HEFF_JCB_MAX_BLOCK) return HEFF_BAD_ARG;
    if(block_size != op->jcb_block) op->jcb_ready = false;
    op->jcb_block = block_size;
    return HEFF_OK;
}

extern "C" int heff_op_jacobi_singular(heff_op *op, int *count) {
    if(!op || !count) return HEFF_BAD_ARG;
    *count = 0;
    if(op->jcb_block <= 1 || !op->jcb_ready) return HEFF_OK;
    HEFF_CUDA(cudaMemcpyAsync(count, op->jcb, sizeof(int), cudaMemcpyDeviceToHost, op->stream));
    HEFF_CUDA(cudaStreamSynchronize(op->stream));
    return HEFF_OK;
}

extern "C" int heff_op_multpc(heff_op *op, const void *x, void *y, double shift) {
    if(!op || !x || !y) return HEFF_BAD_ARG;
    if(!std::isfinite(shift)) return HEFF_NAN_INPUT;
    return op_multpc(op, x, y, shift);
}
