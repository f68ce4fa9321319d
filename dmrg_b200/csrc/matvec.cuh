// H_eff * theta on the GPU: layout kernels, the MPO mixing kernel and the matvec driver.
//
// Contraction order (one of the two orders of contraction_tblis.cpp:277-290; both cost
// 2*S*D*chiL*chiR*(chiL+chiR) + 2*S^2*DL*DR*chiL*chiR FLOPs, so one order serves both branches):
//   P   x'[a,(s,b)]         = theta[s,a,b]                                    (layout, O(S chi^2))
//   G1  T1[(a',m),(s,b)]    = sum_a  L[a,(a',m)] x'[a,(s,b)]                   (DMMA GEMM, K = chiL)
//   MIX T2[(s',a'),(b,n)]   = sum_{m,s} W[m,n,s,s'] T1[(a',m),(s,b)]           (CUDA cores, per (a',b))
//   G2  y[(s',a'),b']       = sum_{(b,n)} T2[(s',a'),(b,n)] R'[(b,n),b']       (DMMA GEMM, K = chiR*DR)
// with R'[(b,n),b'] = R[b,b',n] permuted once per operator.  y lands directly in the
// reference layout y[s' + S*(a' + chiL*b')].
#pragma once
#include "gemm_f64.cuh"

namespace heff {

struct MatvecDims {
    int64_t S, cL, cR, DL, DR;
    int64_t size_mps() const { return S * cL * cR; }
    int64_t size_T1() const { return DL * S * cL * cR; }
    int64_t size_T2() const { return DR * S * cL * cR; }
    int64_t size_Rp() const { return cR * cR * DR; }
};

// Validates reference-style dims (contraction_tblis.cpp:230-234 checks, plus the square-env shapes).
int check_matvec_dims(const int64_t md[3], const int64_t wd[4], const int64_t ld[3], const int64_t rd[3], MatvecDims &out);

template<bool CPLX>
int permute_R(const typename Scalar<CPLX>::T *R, typename Scalar<CPLX>::T *Rp, const MatvecDims &d, cudaStream_t s);

// Scratch layout for one matvec: x' | T1 | T2 (elements).
template<bool CPLX>
struct MatvecScratch {
    using T = typename Scalar<CPLX>::T;
    T *xp = nullptr, *T1 = nullptr, *T2 = nullptr;
    // optional tail-split scratch of the two GEMMs (nullptr: every tile runs whole; see GemmArgs)
    void  *split_ws    = nullptr;
    size_t split_bytes = 0;
    // sub-buffers start on 256-byte boundaries so the GEMMs can use 16-byte copies
    static int64_t pad(int64_t n) { return (n + 31) / 32 * 32; }
    static int64_t elems(const MatvecDims &d) { return pad(d.size_mps()) + pad(d.size_T1()) + pad(d.size_T2()); }
    T             *carve(T *base, const MatvecDims &d) {  // returns the first element after the scratch
        xp = base;
        T1 = xp + pad(d.size_mps());
        T2 = T1 + pad(d.size_T1());
        return T2 + pad(d.size_T2());
    }
};

// Host-side address of the matvec's input permutation kernel (its first parameter is the input vector): a captured
// matvec graph is retargeted to a new input through it.
const void *permute_kernel_fn(bool cplx);

// Tail-split scratch to reserve beside a matvec scratch of `scratch_bytes`: enough partial tiles for the best
// split of large GEMMs (gemm_split_ws_bytes), at least 16 MB so small-bond GEMMs with few tiles can split finely.
inline size_t matvec_split_bytes(size_t scratch_bytes) {
    const size_t cap = gemm_split_ws_bytes();
    const size_t want = scratch_bytes > ((size_t)16 << 20) ? scratch_bytes : ((size_t)16 << 20);
    return want < cap ? want : cap;
}

// Streams and events of the host-buffer matvec pipeline (matvec_fp64_host), owned by the operator.
struct HostPipe {
    static constexpr int MAXS = 16;  // slabs per side at most
    cudaStream_t         s = nullptr, aux = nullptr, copy = nullptr;
    cudaEvent_t          ev[2 * MAXS + 4] = {};
    int                  n_in = 8, n_out = 8;  // measured at chi=1024 complex: 4/4 27.2, 8/8 29.0, 16/8 29.2 TFLOP/s end to end
};

// x'[a + cL (s + S b)] = x[s + S (a + cL b)] (the layout stage of the matvec).
template<bool CPLX>
int permute_mps(const MatvecDims &d, const typename Scalar<CPLX>::T *x, typename Scalar<CPLX>::T *xp, cudaStream_t s);
// T2 = MPO mix of T1 (the MIX stage, FP64).
template<bool CPLX>
int mix_fp64(const MatvecDims &d, const typename Scalar<CPLX>::T *T1, typename Scalar<CPLX>::T *T2, const typename Scalar<CPLX>::T *W, cudaStream_t s);

// y = H_eff x with pre-permuted R'.  L and W in reference layout.  Launches 4 kernels on s.
// ev (optional): 5 events recorded before P and after P, G1, MIX, G2 (stage timing).
template<bool CPLX>
int matvec_fp64(const MatvecDims &d, const typename Scalar<CPLX>::T *x, typename Scalar<CPLX>::T *y, const typename Scalar<CPLX>::T *L,
                const typename Scalar<CPLX>::T *Rp, const typename Scalar<CPLX>::T *W, const MatvecScratch<CPLX> &ws, cudaStream_t s,
                cudaEvent_t *ev = nullptr);

// Deterministic dot product sum_i conj(x_i) y_i (conj only for complex) into a device scalar.
template<bool CPLX>
int dot_device(const typename Scalar<CPLX>::T *x, const typename Scalar<CPLX>::T *y, int64_t n, typename Scalar<CPLX>::T *out,
               double *partials /* >= 1024 * (CPLX ? 2 : 1) doubles */, cudaStream_t s);

// Stages 1-2 of the matvec (permute, GEMM 1 scaled by alpha, MPO mix into `out`): the L-side expansion term.
template<bool CPLX>
int matvec_left_stages(const MatvecDims &d, const typename Scalar<CPLX>::T *x, const typename Scalar<CPLX>::T *L, const typename Scalar<CPLX>::T *W,
                       typename Scalar<CPLX>::T *out, typename Scalar<CPLX>::T *xp, typename Scalar<CPLX>::T *T1, double alpha, cudaStream_t s);

// y = H_eff x with x, y in host memory: slabbed copies overlapped with GEMM 1 / mix and GEMM 2 (dx, dy device
// staging of the full vectors).  Synchronises hp.s before returning.
template<bool CPLX>
int matvec_fp64_host(const MatvecDims &d, const typename Scalar<CPLX>::T *xh, typename Scalar<CPLX>::T *yh, const typename Scalar<CPLX>::T *L,
                     const typename Scalar<CPLX>::T *Rp, const typename Scalar<CPLX>::T *W, const MatvecScratch<CPLX> &ws, typename Scalar<CPLX>::T *dx,
                     typename Scalar<CPLX>::T *dy, const HostPipe &hp);

}  // namespace heff
