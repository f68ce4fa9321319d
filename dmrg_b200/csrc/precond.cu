// Jacobi (diagonal) preconditioner of the effective Hamiltonian.
//
// Diagonal: MatVecMPOS::get_diagonal_new / get_matrix_element (source/math/eig/matvec/matvec_mpos.cpp:300-407)
// at I == J: for I = s + S (a + cL b),
//     diag[I] = sum_{m,n} L[a, a, m] W[m, n, s, s] R[b, b, n],
// one thread per element (S cL cR DL DR multiply-adds in total, negligible next to one matvec).
// Application: the block-size-1 branch of MultPc (matvec_mpos.cpp:1349-1364),
//     y = x / (diag - shift),
// with the denominator kept at least 1e-10 max(|shift|, 1) in magnitude (the reference divides unguarded).
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

extern "C" int heff_op_multpc(heff_op *op, const void *x, void *y, double shift) {
    if(!op || !x || !y) return HEFF_BAD_ARG;
    if(!std::isfinite(shift)) return HEFF_NAN_INPUT;
    return op_multpc(op, x, y, shift);
}
