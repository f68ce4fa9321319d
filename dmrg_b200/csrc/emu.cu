// H_eff matvec with both GEMMs emulated in FP64 accuracy on the INT8 tensor cores (gemm_i8.cuh).
//
// Same contraction order and stages as the FP64 path (matvec.cuh):
//   P   x' = layout of x                                                        (FP64)
//   G1  T1[(a',m),(s,b)]  = sum_a L[a,(a',m)] x'[a,(s,b)]     A = digit planes of L (per operator), B = of x'
//   MIX T2 = MPO mix of T1                                                      (FP64)
//   G2  y[(s',a'),b']     = sum_{(b,n)} T2[(s',a'),(b,n)] R'[(b,n),b']  A = digit planes of T2, B = of R' (per operator)
// The planes of L and R' are built on the first apply after a create or rebind; x' and T2 are sliced per
// matvec (a row-maximum pass, then the digit pass).  Complex operands use the real embedding of gemm_i8.cuh.
#include <algorithm>

#include "gemm_i8.cuh"
#include "matvec.cuh"
#include "op.cuh"
#include "runtime.cuh"

namespace heff {

// Buffer layout: err (256 B) | rmax[rmax_cap] | scales | planes A1 | B1 | A2 | B2.  The error flag and the
// row-maximum accumulators sit at fixed offsets (zeroed when the buffer is allocated and left zero by the
// kernels), so a rebind to other dimensions never finds stale bytes there.
struct EmuState {
    void   *buf = nullptr;
    size_t  cap = 0;
    int64_t rmax_cap = 0;  // rows of T2 the accumulators cover
    int    *err = nullptr;  // [0] sticky status; bad words of [1] x', [2] T2 (cleared per apply), [3] L, [4] R' (per slicing)
    ZPlanes A1, B1, A2, B2;
};

struct EmuDims {
    int64_t M1, N1, K1, kx1, M2, N2, K2, kx2;
    int     cf;
};

static EmuDims emu_dims(const heff_op *op) {
    const auto &d = op->d;
    EmuDims     e;
    e.cf  = op->cplx ? 2 : 1;
    e.M1  = d.cL * d.DL;
    e.N1  = d.S * d.cR;
    e.K1  = d.cL;
    e.kx1 = z_kx(e.K1, op->cplx);
    e.M2  = d.S * d.cL;
    e.N2  = d.cR;
    e.K2  = d.cR * d.DR;
    e.kx2 = z_kx(e.K2, op->cplx);
    return e;
}

bool emu_supported(const heff_op *op) {
    if(op->sequential) return false;
    const EmuDims e = emu_dims(op);
    return z_k_ok(e.kx1, op->emu_slices) && z_k_ok(e.kx2, op->emu_slices) && e.M1 <= 0x7fffffff && e.cf * e.N1 <= 0x7fffffff &&
           e.M2 <= 0x7fffffff && e.cf * e.N2 <= 0x7fffffff;
}

void emu_destroy(heff_op *op) {
    EmuState *e = reinterpret_cast<EmuState *>(op->emu);
    if(!e) return;
    if(e->buf) cudaFree(e->buf);
    delete e;
    op->emu       = nullptr;
    op->emu_stale = true;
}

static size_t up256(size_t b) { return (b + 255) / 256 * 256; }

struct EmuSizes {
    size_t A1, B1, A2, B2, S, R;
    size_t total() const { return 256 + R + S + A1 + B1 + A2 + B2; }
};
static EmuSizes emu_sizes(const EmuDims &e, int ns, int64_t rmax_rows) {
    EmuSizes z;
    z.A1 = up256((size_t)ns * e.M1 * e.kx1), z.B1 = up256((size_t)ns * e.cf * e.N1 * e.kx1);
    z.A2 = up256((size_t)ns * e.M2 * e.kx2), z.B2 = up256((size_t)ns * e.cf * e.N2 * e.kx2);
    z.S  = up256(sizeof(double) * 2 * (size_t)(e.M1 + e.N1 + e.M2 + e.N2));
    z.R  = up256(sizeof(unsigned long long) * (size_t)rmax_rows);
    return z;
}

// (Re)allocates the buffer for `need` bytes with row-maximum room for rmax_rows rows (zeroed).
static int emu_alloc(heff_op *op, EmuState *st, size_t need, int64_t rmax_rows) {
    if(st->buf) {
        HEFF_CUDA(cudaStreamSynchronize(op->stream));
        cudaFree(st->buf);
        st->buf = nullptr;
        st->cap = 0;
    }
    cudaError_t ce = cudaMalloc(&st->buf, need);
    if(ce != cudaSuccess) {
        set_last_cuda_error(ce, "emulated-FP64 digit planes", __FILE__, __LINE__);
        return HEFF_OOM;
    }
    st->cap      = need;
    st->rmax_cap = rmax_rows;
    HEFF_CUDA(cudaMemsetAsync(st->buf, 0, need, op->stream));
    op->emu_stale = true;
    return HEFF_OK;
}

// Carves the planes for the operator's current dimensions out of the state's buffer (grown when needed).
static int emu_layout(heff_op *op, EmuState *st) {
    const EmuDims e  = emu_dims(op);
    const int     ns = op->emu_slices;
    EmuSizes      z  = emu_sizes(e, ns, std::max<int64_t>(st->rmax_cap, e.M2));
    if(z.total() > st->cap || e.M2 > st->rmax_cap) HEFF_TRY(emu_alloc(op, st, z.total(), std::max<int64_t>(st->rmax_cap, e.M2)));
    unsigned char *p = reinterpret_cast<unsigned char *>(st->buf);
    st->err          = reinterpret_cast<int *>(p);
    p += 256;
    st->A2.rmax = reinterpret_cast<unsigned long long *>(p);
    p += z.R;
    double *sc = reinterpret_cast<double *>(p);
    st->A1.inv = sc, st->A1.fac = sc + e.M1, sc += 2 * e.M1;
    st->B1.inv = sc, st->B1.fac = sc + e.N1, sc += 2 * e.N1;
    st->A2.inv = sc, st->A2.fac = sc + e.M2, sc += 2 * e.M2;
    st->B2.inv = sc, st->B2.fac = sc + e.N2;
    p += z.S;
    auto planes = [&](ZPlanes &q, size_t bytes, int64_t rows, int64_t kx) {
        q.planes = reinterpret_cast<int8_t *>(p), q.rows = rows, q.kx = kx, q.nslice = ns;
        p += bytes;
    };
    planes(st->A1, z.A1, e.M1, e.kx1);
    planes(st->B1, z.B1, e.cf * e.N1, e.kx1);
    planes(st->A2, z.A2, e.M2, e.kx2);
    planes(st->B2, z.B2, e.cf * e.N2, e.kx2);
    return HEFF_OK;
}

int emu_reserve(heff_op *op, int64_t S, int64_t cmax, int64_t Dmax) {
    if(!op->emu) op->emu = new EmuState();
    EmuState *st = reinterpret_cast<EmuState *>(op->emu);
    EmuDims   e;
    e.cf = op->cplx ? 2 : 1;
    e.M1 = cmax * Dmax, e.N1 = S * cmax, e.K1 = cmax, e.kx1 = z_kx(e.K1, op->cplx);
    e.M2 = S * cmax, e.N2 = cmax, e.K2 = cmax * Dmax, e.kx2 = z_kx(e.K2, op->cplx);
    const EmuSizes z = emu_sizes(e, op->emu_slices, e.M2);
    if(z.total() <= st->cap && e.M2 <= st->rmax_cap) return HEFF_OK;
    return emu_alloc(op, st, z.total(), e.M2);
}

size_t emu_held_bytes(const heff_op *op) { return op->emu ? reinterpret_cast<const EmuState *>(op->emu)->cap : 0; }

size_t emu_bytes(int64_t S, int64_t cL, int64_t cR, int64_t DL, int64_t DR, bool cplx, int nslices) {
    EmuDims e;
    e.cf = cplx ? 2 : 1;
    e.M1 = cL * DL, e.N1 = S * cR, e.K1 = cL, e.kx1 = z_kx(e.K1, cplx);
    e.M2 = S * cL, e.N2 = cR, e.K2 = cR * DR, e.kx2 = z_kx(e.K2, cplx);
    return emu_sizes(e, nslices, e.M2).total();
}

template<bool CPLX>
static int emu_apply_impl(heff_op *op, const void *xv, void *yv) {
    using T = typename Scalar<CPLX>::T;
    if(!op->emu) op->emu = new EmuState();
    EmuState *st = reinterpret_cast<EmuState *>(op->emu);
    HEFF_TRY(emu_layout(op, st));
    const EmuDims e  = emu_dims(op);
    const auto   &d  = op->d;
    const int     ns = op->emu_slices;
    cudaStream_t  s  = op->stream;
    const double  a_extra = 1.0 / 4096.0;  // the 2^-12 of the two leading digits' units, carried by the A side
    int *err = st->err;
    if(op->emu_stale) {  // operator-side planes: L (A of G1) and R' (B of G2)
        const T *L = reinterpret_cast<const T *>(op->L), *Rp = reinterpret_cast<const T *>(op->Rp);
        HEFF_CUDA(cudaMemsetAsync(err + 3, 0, 2 * sizeof(int), s));
        HEFF_TRY(z_scale_kmajor<CPLX>(L, e.M1, e.K1, e.K1, a_extra, st->A1, err + 3, s));
        HEFF_TRY(z_slice_kmajor<CPLX>(L, e.M1, e.K1, e.K1, false, st->A1, err + 3, s));
        HEFF_TRY(z_scale_kmajor<CPLX>(Rp, e.N2, e.K2, e.K2, 1.0, st->B2, err + 4, s));
        HEFF_TRY(z_slice_kmajor<CPLX>(Rp, e.N2, e.K2, e.K2, CPLX, st->B2, err + 4, s));
        op->emu_stale = false;
    }
    HEFF_CUDA(cudaMemsetAsync(err + 1, 0, 2 * sizeof(int), s));  // this apply's operands start clean
    MatvecScratch<CPLX> ws;
    ws.carve(reinterpret_cast<T *>(op->scratch), d);
    const T *x = reinterpret_cast<const T *>(xv);
    T       *y = reinterpret_cast<T *>(yv);
    HEFF_TRY(permute_mps<CPLX>(d, x, ws.xp, s));
    HEFF_TRY(z_scale_kmajor<CPLX>(ws.xp, e.N1, e.K1, e.K1, 1.0, st->B1, err + 1, s));
    HEFF_TRY(z_slice_kmajor<CPLX>(ws.xp, e.N1, e.K1, e.K1, CPLX, st->B1, err + 1, s));
    ZGemmArgs g1{};
    g1.M = (int)e.M1, g1.N = (int)(e.cf * e.N1), g1.K = (int)e.kx1, g1.nslice = ns, g1.fa = st->A1.fac, g1.fb = st->B1.fac;
    g1.C = ws.T1, g1.ldc = e.M1, g1.cplx = CPLX, g1.err = err, g1.bad_a = err + 3, g1.bad_b = err + 1;
    HEFF_TRY(gemm_i8_ozaki(st->A1, st->B1, g1, s));
    HEFF_TRY(mix_fp64<CPLX>(d, ws.T1, ws.T2, reinterpret_cast<const T *>(op->W), s));
    HEFF_TRY(z_scale_mmajor<CPLX>(ws.T2, e.M2, e.K2, e.M2, a_extra, st->A2, err + 2, s));
    HEFF_TRY(z_slice_mmajor<CPLX>(ws.T2, e.M2, e.K2, e.M2, st->A2, err + 2, s));
    ZGemmArgs g2{};
    g2.M = (int)e.M2, g2.N = (int)(e.cf * e.N2), g2.K = (int)e.kx2, g2.nslice = ns, g2.fa = st->A2.fac, g2.fb = st->B2.fac;
    g2.C = y, g2.ldc = e.M2, g2.cplx = CPLX, g2.err = err, g2.bad_a = err + 2, g2.bad_b = err + 4;
    HEFF_TRY(gemm_i8_ozaki(st->A2, st->B2, g2, s));
    op->num_mv++;
    return HEFF_OK;
}

int emu_apply(heff_op *op, const void *x, void *y) {
    if(x == y) return HEFF_BAD_ARG;
    return op->cplx ? emu_apply_impl<true>(op, x, y) : emu_apply_impl<false>(op, x, y);
}

int emu_error_flag(heff_op *op, int *flag) {
    *flag         = 0;
    EmuState *st  = reinterpret_cast<EmuState *>(op->emu);
    if(!st || !st->err) return HEFF_OK;
    HEFF_CUDA(cudaMemcpyAsync(flag, st->err, sizeof(int), cudaMemcpyDeviceToHost, op->stream));
    HEFF_CUDA(cudaStreamSynchronize(op->stream));
    return HEFF_OK;
}

}  // namespace heff
