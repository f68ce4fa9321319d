// heff_op: the MatVecMPOS<T> / MatVecMPO<T> operator object behind the C ABI
// (source/math/eig/matvec/matvec_mpos.h:23-180, matvec_mpos.cpp:40-130, 963-984).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "matvec.cuh"
#include "eig.cuh"
#include "gemm_i8.cuh"
#include "op.cuh"
#include "runtime.cuh"

namespace heff {

// Merge site MPOs like matvec_mpos.cpp:104-119:
//   W2[mL, mR', s1 + dA*s2, t1 + dA*t2] = sum_c WA[mL, c, s1, t1] WB[c, mR', s2, t2]
template<class T>
static void merge_two(std::vector<T> &out, int64_t od[4], const std::vector<T> &A, const int64_t da[4], const std::vector<T> &B, const int64_t db[4]) {
    const int64_t mL = da[0], c = da[1], sA = da[2], tA = da[3], mR = db[1], sB = db[2], tB = db[3];
    const int64_t S = sA * sB, TT = tA * tB;
    out.assign((size_t)(mL * mR * S * TT), T{});
    for(int64_t t2 = 0; t2 < tB; t2++)
        for(int64_t t1 = 0; t1 < tA; t1++)
            for(int64_t s2 = 0; s2 < sB; s2++)
                for(int64_t s1 = 0; s1 < sA; s1++)
                    for(int64_t n = 0; n < mR; n++)
                        for(int64_t m = 0; m < mL; m++) {
                            T acc{};
                            for(int64_t k = 0; k < c; k++) {
                                const T &a = A[m + mL * (k + c * (s1 + sA * t1))];
                                const T &b = B[k + db[0] * (n + mR * (s2 + sB * t2))];
                                acc        = acc + a * b;
                            }
                            out[m + mL * (n + mR * ((s1 + sA * s2) + S * (t1 + tA * t2)))] = acc;
                        }
    od[0] = mL;
    od[1] = mR;
    od[2] = S;
    od[3] = TT;
}

struct HostC {
    double re = 0, im = 0;
    HostC() = default;
    HostC(double r, double i) : re(r), im(i) {}
    explicit HostC(double r) : re(r), im(0.0) {}
    HostC operator+(const HostC &o) const { return {re + o.re, im + o.im}; }
    HostC operator*(const HostC &o) const { return {re * o.re - im * o.im, re * o.im + im * o.re}; }
};

// Operator over more than 5 site MPOs: like the reference (matvec_mpos.cpp:104-123) the MPOs are not merged; the
// matvec applies them one at a time (matvec_multi).  FP64 only (the split-BF16 path needs the merged MPO).
template<bool CPLX>
static int create_sequential(heff_op **out, int nsites, const void *const *mpos, const int64_t *mdims, const void *envL, const int64_t ld[3],
                             const void *envR, const int64_t rd[3], heff_precision prec, cudaStream_t stream) {
    using T  = typename Scalar<CPLX>::T;
    using HT = typename std::conditional<CPLX, HostC, double>::type;
    if(prec != HEFF_PREC_FP64) {
        set_last_error_msg("operator over %d site MPOs: mixed precision needs the merged MPO (at most 5 sites)", nsites);
        return HEFF_BAD_ARG;
    }
    int64_t S = 1;
    for(int i = 0; i < nsites; i++) S *= mdims[4 * i + 2];
    const int64_t md[3] = {S, ld[0], rd[0]};
    MultiDims     mdm;
    HEFF_TRY(check_multi_dims(md, nsites, mdims, ld, rd, mdm));
    const int64_t D0 = mdims[0], DK = mdims[4 * (nsites - 1) + 1];
    heff_op      *op   = new heff_op();
    op->cplx           = CPLX;
    op->d              = MatvecDims{S, ld[0], rd[0], D0, DK};
    op->precision      = HEFF_PREC_FP64;
    op->stream         = stream;
    op->sequential     = true;
    op->multi          = mdm;
    op->mpo_dims[0] = D0, op->mpo_dims[1] = DK, op->mpo_dims[2] = S, op->mpo_dims[3] = S;
    const size_t es   = sizeof(T);
    auto         fail = [&](int rc) {
        heff_op_destroy(op);
        return rc;
    };
    // site MPOs to the device; the s == s' part of the merged MPO on the host:
    //   Wd[m0, mK, s] = sum_{m_1..m_{K-1}} prod_i W_i[m_{i-1}, m_i, s_i, s_i]
    std::vector<HT> Wd;
    int64_t         Dc = D0, Sc = 1;
    for(int i = 0; i < nsites; i++) {
        const int64_t *di = mdims + 4 * i;
        const size_t   n  = (size_t)(di[0] * di[1] * di[2] * di[3]);
        std::vector<HT> Wi(n);
        if(cudaMemcpy(Wi.data(), mpos[i], n * es, cudaMemcpyDefault) != cudaSuccess) return fail(HEFF_CUDA_ERROR);
        void *dW = nullptr;
        if(cudaMalloc(&dW, n * es) != cudaSuccess) return fail(HEFF_OOM);
        op->seq_W.push_back(dW);
        if(cudaMemcpy(dW, Wi.data(), n * es, cudaMemcpyHostToDevice) != cudaSuccess) return fail(HEFF_CUDA_ERROR);
        const int64_t   Dn = di[1], d = di[2];
        std::vector<HT> nxt((size_t)(D0 * Dn * Sc * d), HT{});
        for(int64_t t = 0; t < d; t++)
            for(int64_t sc = 0; sc < Sc; sc++)
                for(int64_t n2 = 0; n2 < Dn; n2++)
                    for(int64_t m0 = 0; m0 < D0; m0++) {
                        HT acc{};
                        for(int64_t k = 0; k < Dc; k++) {
                            const HT prev = i == 0 ? (k == m0 ? HT(1.0) : HT(0.0)) : Wd[m0 + D0 * (k + Dc * sc)];
                            acc           = acc + prev * Wi[k + di[0] * (n2 + Dn * (t + d * t))];
                        }
                        nxt[m0 + D0 * (n2 + Dn * (sc + Sc * t))] = acc;
                    }
        Wd = std::move(nxt);
        Dc = Dn;
        Sc *= d;
    }
    const int64_t nWfull = D0 * DK * S * S;
    if(nWfull <= (int64_t)1 << 24) {  // the diagonal-only merged MPO, laid out like a merged MPO for the diagonal kernel
        std::vector<HT> Wf((size_t)nWfull, HT{});
        for(int64_t s = 0; s < S; s++)
            for(int64_t n2 = 0; n2 < DK; n2++)
                for(int64_t m0 = 0; m0 < D0; m0++) Wf[m0 + D0 * (n2 + DK * (s + S * s))] = Wd[m0 + D0 * (n2 + DK * s)];
        if(cudaMalloc(&op->W, nWfull * es) != cudaSuccess) return fail(HEFF_OOM);
        if(cudaMemcpy(op->W, Wf.data(), nWfull * es, cudaMemcpyHostToDevice) != cudaSuccess) return fail(HEFF_CUDA_ERROR);
    }
    const MatvecDims &d  = op->d;
    const int64_t     nL = d.cL * d.cL * d.DL, nR = d.size_Rp();
    if(cudaMalloc(&op->L, nL * es) != cudaSuccess) return fail(HEFF_OOM);
    if(cudaMalloc(&op->Rp, nR * es) != cudaSuccess) return fail(HEFF_OOM);
    const int64_t nscr = multi_scratch_elems(mdm);
    if(cudaMalloc(&op->scratch, nscr * es) != cudaSuccess) return fail(HEFF_OOM);
    op->scratch_bytes = (size_t)nscr * es;
    void *Rtmp        = nullptr;
    if(cudaMalloc(&Rtmp, nR * es) != cudaSuccess) return fail(HEFF_OOM);
    cudaError_t e = cudaMemcpyAsync(op->L, envL, nL * es, cudaMemcpyDefault, stream);
    if(e == cudaSuccess) e = cudaMemcpyAsync(Rtmp, envR, nR * es, cudaMemcpyDefault, stream);
    int rc = e == cudaSuccess ? permute_R<CPLX>(reinterpret_cast<const T *>(Rtmp), reinterpret_cast<T *>(op->Rp), d, stream) : HEFF_CUDA_ERROR;
    const cudaError_t e2 = cudaStreamSynchronize(stream);
    cudaFree(Rtmp);
    if(e != cudaSuccess) {
        set_last_cuda_error(e, "heff_op_create copies", __FILE__, __LINE__);
        return fail(HEFF_CUDA_ERROR);
    }
    if(rc != HEFF_OK) return fail(rc);
    if(e2 != cudaSuccess) {
        set_last_cuda_error(e2, "heff_op_create sync", __FILE__, __LINE__);
        return fail(HEFF_CUDA_ERROR);
    }
    *out = op;
    return HEFF_OK;
}

template<bool CPLX>
static int create_impl(heff_op **out, int nsites, const void *const *mpos, const int64_t *mdims, const void *envL, const int64_t ld[3],
                       const void *envR, const int64_t rd[3], heff_mem where, heff_precision prec, cudaStream_t stream) {
    using T  = typename Scalar<CPLX>::T;
    using HT = typename std::conditional<CPLX, HostC, double>::type;
    static_assert(sizeof(HT) == sizeof(T), "host/device scalar size");
    if(!out || nsites < 1 || !mpos || !mdims || !envL || !envR || !ld || !rd) return HEFF_BAD_ARG;
    if(nsites > 5) return create_sequential<CPLX>(out, nsites, mpos, mdims, envL, ld, envR, rd, prec, stream);
    // --- gather the site MPOs on the host and merge them (setup only, tiny) ---
    std::vector<HT> W;
    int64_t         wd[4];
    for(int i = 0; i < nsites; i++) {
        const int64_t *di = mdims + 4 * i;
        if(di[0] <= 0 || di[1] <= 0 || di[2] <= 0 || di[3] <= 0 || di[2] != di[3]) return HEFF_BAD_SHAPE;
        size_t          n = (size_t)(di[0] * di[1] * di[2] * di[3]);
        std::vector<HT> Wi(n);
        // the MPO may live on the host even when the environments are on the device: let UVA decide
        HEFF_CUDA(cudaMemcpyAsync(Wi.data(), mpos[i], n * sizeof(HT), cudaMemcpyDefault, stream));
        HEFF_CUDA(cudaStreamSynchronize(stream));
        if(i == 0) {
            W = std::move(Wi);
            std::memcpy(wd, di, sizeof(wd));
        } else {
            if(wd[1] != di[0]) return HEFF_BAD_SHAPE;
            std::vector<HT> M2;
            int64_t         nd[4];
            merge_two(M2, nd, W, wd, Wi, di);
            W = std::move(M2);
            std::memcpy(wd, nd, sizeof(wd));
        }
    }
    const int64_t md[3] = {wd[2], ld[0], rd[0]};
    MatvecDims    d;
    HEFF_TRY(check_matvec_dims(md, wd, ld, rd, d));

    heff_op *op   = new heff_op();
    op->cplx      = CPLX;
    op->d         = d;
    op->precision   = prec;
    op->stream      = stream;
    op->mixed_apply = mixed_apply;  // split-BF16 tcgen05 path; its state is built on first use
    std::memcpy(op->mpo_dims, wd, sizeof(wd));
    const size_t es   = sizeof(T);
    auto         fail = [&](int rc) {
        heff_op_destroy(op);
        return rc;
    };
    // device buffers: L (reference layout), R' (permuted), W, scratch, staging for host MultAx
    const int64_t nL = d.cL * d.cL * d.DL, nR = d.size_Rp(), nW = wd[0] * wd[1] * wd[2] * wd[3];
    if(cudaMalloc(&op->L, nL * es) != cudaSuccess) return fail(HEFF_OOM);
    if(cudaMalloc(&op->Rp, nR * es) != cudaSuccess) return fail(HEFF_OOM);
    if(cudaMalloc(&op->W, nW * es) != cudaSuccess) return fail(HEFF_OOM);
    const int64_t nscr = MatvecScratch<CPLX>::elems(d);
    if(cudaMalloc(&op->scratch, nscr * es) != cudaSuccess) return fail(HEFF_OOM);
    op->scratch_bytes = (size_t)nscr * es;
    op->split_bytes   = matvec_split_bytes(op->scratch_bytes);
    if(cudaMalloc(&op->split_ws, op->split_bytes) != cudaSuccess) return fail(HEFF_OOM);
    void *Rtmp        = nullptr;
    if(cudaMalloc(&Rtmp, nR * es) != cudaSuccess) return fail(HEFF_OOM);
    (void)where;  // source location of each buffer is inferred from its address (unified addressing)
    const cudaMemcpyKind kind = cudaMemcpyDefault;
    cudaError_t          e    = cudaMemcpyAsync(op->L, envL, nL * es, kind, stream);
    if(e == cudaSuccess) e = cudaMemcpyAsync(Rtmp, envR, nR * es, kind, stream);
    if(e == cudaSuccess) e = cudaMemcpyAsync(op->W, W.data(), nW * es, cudaMemcpyHostToDevice, stream);
    if(e != cudaSuccess) {
        cudaFree(Rtmp);
        set_last_cuda_error(e, "heff_op_create copies", __FILE__, __LINE__);
        return fail(HEFF_CUDA_ERROR);
    }
    int rc = permute_R<CPLX>(reinterpret_cast<const T *>(Rtmp), reinterpret_cast<T *>(op->Rp), d, stream);
    e      = cudaStreamSynchronize(stream);  // W's host vector and Rtmp must outlive the copies
    cudaFree(Rtmp);
    if(rc != HEFF_OK) return fail(rc);
    if(e != cudaSuccess) {
        set_last_cuda_error(e, "heff_op_create sync", __FILE__, __LINE__);
        return fail(HEFF_CUDA_ERROR);
    }
    *out = op;
    return HEFF_OK;
}

// Operator with fixed-capacity buffers (spin S, bond <= cmax, MPO bond <= Dmax) for a sweep: every bond is
// bound with op_rebind, which reuses the buffers (no allocation, no device synchronisation per bond).
int op_create_capacity(heff_op **out, bool cplx, int64_t S, int64_t cmax, int64_t Dmax, heff_precision prec, cudaStream_t stream) {
    if(!out || S <= 0 || cmax <= 0 || Dmax <= 0) return HEFF_BAD_ARG;
    heff_op *op     = new heff_op();
    op->cplx        = cplx;
    op->precision   = prec;
    op->stream      = stream;
    op->mixed_apply = mixed_apply;
    const size_t es = cplx ? 16 : 8;
    auto         fail = [&](int rc) {
        heff_op_destroy(op);
        return rc;
    };
    const MatvecDims dmax{S, cmax, cmax, Dmax, Dmax};
    op->cap_env     = cmax * cmax * Dmax;
    op->cap_W       = Dmax * Dmax * S * S;
    op->cap_scratch = cplx ? MatvecScratch<true>::elems(dmax) : MatvecScratch<false>::elems(dmax);
    if(cudaMalloc(&op->L, op->cap_env * es) != cudaSuccess) return fail(HEFF_OOM);
    if(cudaMalloc(&op->Rp, op->cap_env * es) != cudaSuccess) return fail(HEFF_OOM);
    if(cudaMalloc(&op->Rtmp, op->cap_env * es) != cudaSuccess) return fail(HEFF_OOM);
    if(cudaMalloc(&op->W, op->cap_W * es) != cudaSuccess) return fail(HEFF_OOM);
    if(cudaMalloc(&op->scratch, op->cap_scratch * es) != cudaSuccess) return fail(HEFF_OOM);
    op->scratch_bytes = (size_t)op->cap_scratch * es;
    op->split_bytes   = matvec_split_bytes(op->scratch_bytes);
    if(cudaMalloc(&op->split_ws, op->split_bytes) != cudaSuccess) return fail(HEFF_OOM);
    op->diag_cap      = S * cmax * cmax;
    if(cudaMalloc(&op->diag, op->diag_cap * es) != cudaSuccess) return fail(HEFF_OOM);
    *out              = op;
    return HEFF_OK;
}

// Binds the operator to new site MPOs (host, merged like matvec_mpos.cpp:104-119) and environments
// (device, stream-ordered before the next apply).  Requires the capacities of op_create_capacity.
template<bool CPLX>
static int rebind_impl(heff_op *op, int nsites, const void *const *mpos_host, const int64_t *mdims, const void *envL, const int64_t ld[3],
                       const void *envR, const int64_t rd[3]) {
    using T  = typename Scalar<CPLX>::T;
    using HT = typename std::conditional<CPLX, HostC, double>::type;
    mixed_invalidate(op);                                      // split operands belong to the old environments (re-split in place)
    op->emu_stale  = true;                                     // so do the digit planes of L and R' (rebuilt in place)
    op->diag_ready = false;
    op->jcb_ready  = false;
    std::vector<HT> W;
    int64_t         wd[4];
    for(int i = 0; i < nsites; i++) {
        const int64_t  *di = mdims + 4 * i;
        const size_t    n  = (size_t)(di[0] * di[1] * di[2] * di[3]);
        std::vector<HT> Wi(reinterpret_cast<const HT *>(mpos_host[i]), reinterpret_cast<const HT *>(mpos_host[i]) + n);
        if(i == 0) {
            W = std::move(Wi);
            std::memcpy(wd, di, sizeof(wd));
        } else {
            if(wd[1] != di[0]) return HEFF_BAD_SHAPE;
            std::vector<HT> M2;
            int64_t         nd[4];
            merge_two(M2, nd, W, wd, Wi, di);
            W = std::move(M2);
            std::memcpy(wd, nd, sizeof(wd));
        }
    }
    const int64_t md[3] = {wd[2], ld[0], rd[0]};
    MatvecDims    d;
    HEFF_TRY(check_matvec_dims(md, wd, ld, rd, d));
    const int64_t nL = d.cL * d.cL * d.DL, nR = d.size_Rp(), nW = wd[0] * wd[1] * wd[2] * wd[3];
    if(nL > op->cap_env || nR > op->cap_env || nW > op->cap_W || MatvecScratch<CPLX>::elems(d) > op->cap_scratch) {
        set_last_error_msg("operator rebind: dimensions exceed the operator's capacity");
        return HEFF_BAD_SHAPE;
    }
    op->d = d;
    std::memcpy(op->mpo_dims, wd, sizeof(wd));
    op->w_host.resize(nW * sizeof(T));
    std::memcpy(op->w_host.data(), W.data(), nW * sizeof(T));  // stays alive until the next rebind
    const size_t es = sizeof(T);
    HEFF_CUDA(cudaMemcpyAsync(op->W, op->w_host.data(), nW * es, cudaMemcpyHostToDevice, op->stream));
    HEFF_CUDA(cudaMemcpyAsync(op->L, envL, nL * es, cudaMemcpyDefault, op->stream));
    HEFF_CUDA(cudaMemcpyAsync(op->Rtmp, envR, nR * es, cudaMemcpyDefault, op->stream));
    return permute_R<CPLX>(reinterpret_cast<const T *>(op->Rtmp), reinterpret_cast<T *>(op->Rp), d, op->stream);
}

int op_rebind(heff_op *op, int nsites, const void *const *mpos_host, const int64_t *mdims, const void *envL, const int64_t ld[3], const void *envR,
              const int64_t rd[3]) {
    if(!op || nsites < 1 || nsites > 5 || !mpos_host || !mdims || !envL || !envR) return HEFF_BAD_ARG;
    if(op->cap_env == 0) return HEFF_BAD_ARG;
    return op->cplx ? rebind_impl<true>(op, nsites, mpos_host, mdims, envL, ld, envR, rd)
                    : rebind_impl<false>(op, nsites, mpos_host, mdims, envL, ld, envR, rd);
}

ArenaBytes ArenaBytes::max_with(const ArenaBytes &o) const {
    ArenaBytes m;
    m.env     = std::max(env, o.env);
    m.W       = std::max(W, o.W);
    m.scratch = std::max(scratch, o.scratch);
    m.split   = std::max(split, o.split);
    m.diag    = std::max(diag, o.diag);
    m.mixed   = std::max(mixed, o.mixed);
    m.emu     = std::max(emu, o.emu);
    m.eig     = std::max(eig, o.eig);
    m.vec     = std::max(vec, o.vec);
    return m;
}

ArenaBytes arena_need(const heff_request &r, int max_basis) {
    const bool       cplx = r.dtype == HEFF_C128;
    const size_t     es   = cplx ? 16 : 8;
    const MatvecDims d{r.spin, r.chiL, r.chiR, r.mpoL, r.mpoR};
    ArenaBytes       a;
    a.env     = es * (size_t)std::max(d.cL * d.cL * d.DL, d.size_Rp());
    a.W       = es * (size_t)(d.DL * d.DR * d.S * d.S);
    a.scratch = es * (size_t)(cplx ? MatvecScratch<true>::elems(d) : MatvecScratch<false>::elems(d));
    a.split   = matvec_split_bytes(a.scratch);
    a.diag    = es * (size_t)d.size_mps();
    const bool mixed = r.precision == HEFF_PREC_MIXED;
    if(mixed) a.mixed = mixed_bytes(d.S, d.cL, d.cR, d.DL, d.DR, cplx);
    if(r.fp64_engine == HEFF_FP64_INT8) a.emu = emu_bytes(d.S, d.cL, d.cR, d.DL, d.DR, cplx, Z_DEFAULT_SLICES);
    a.eig = eig_workspace_bytes(d.size_mps(), max_basis, mixed, cplx);
    a.vec = 2 * es * (size_t)d.size_mps();
    return a;
}

ArenaBytes arena_held(const heff_op *op) {
    ArenaBytes a;
    a.env     = op->cap_env_b;
    a.W       = op->cap_W_b;
    a.scratch = op->cap_scratch_b;
    a.split   = op->cap_split_b;
    a.diag    = op->cap_diag_b;
    a.mixed   = mixed_held_bytes(op);
    a.emu     = emu_held_bytes(op);
    a.eig     = op->eig_ws_bytes;
    a.vec     = op->arena_vec_b;
    return a;
}

int op_create_arena(heff_op **out, cudaStream_t stream) {
    if(!out) return HEFF_BAD_ARG;
    heff_op *op     = new heff_op();
    op->arena       = true;
    op->stream      = stream;
    op->mixed_apply = mixed_apply;
    *out            = op;
    return HEFF_OK;
}

// Replaces *p by a buffer of `need` bytes when *cap is smaller (stream-synchronised free of the old buffer).
static int arena_grow(heff_op *op, void **p, size_t *cap, size_t need, const char *what) {
    if(*cap >= need) return HEFF_OK;
    if(*p) {
        HEFF_CUDA(cudaStreamSynchronize(op->stream));
        cudaFree(*p);
        *p   = nullptr;
        *cap = 0;
    }
    cudaError_t e = cudaMalloc(p, need);
    if(e != cudaSuccess) {
        *p = nullptr;
        set_last_cuda_error(e, what, __FILE__, __LINE__);
        return HEFF_OOM;
    }
    *cap = need;
    return HEFF_OK;
}

int op_arena_bind(heff_op *op, const heff_request &r, int max_basis, void **vec) {
    if(!op || !op->arena || !vec || !r.mpo || !r.envL || !r.envR) return HEFF_BAD_ARG;
    if(r.dtype != HEFF_F64 && r.dtype != HEFF_C128) return HEFF_BAD_ARG;
    const bool       cplx = r.dtype == HEFF_C128;
    const ArenaBytes need = arena_need(r, max_basis);
    size_t           env_cap = op->cap_env_b;
    // L, R' and the R staging share one capacity
    if(env_cap < need.env) {
        size_t c = env_cap;
        HEFF_TRY(arena_grow(op, &op->L, &c, need.env, "arena envL"));
        c = env_cap;
        HEFF_TRY(arena_grow(op, &op->Rp, &c, need.env, "arena envR"));
        c = env_cap;
        HEFF_TRY(arena_grow(op, &op->Rtmp, &c, need.env, "arena envR staging"));
        op->cap_env_b = need.env;
    }
    HEFF_TRY(arena_grow(op, &op->W, &op->cap_W_b, need.W, "arena MPO"));
    HEFF_TRY(arena_grow(op, &op->scratch, &op->cap_scratch_b, need.scratch, "arena matvec scratch"));
    HEFF_TRY(arena_grow(op, &op->split_ws, &op->cap_split_b, need.split, "arena tail-split partials"));
    op->split_bytes = need.split;  // this request's own share: the GEMMs' split plans (and rounding) do not depend on the arena's history
    HEFF_TRY(arena_grow(op, &op->diag, &op->cap_diag_b, need.diag, "arena preconditioner diagonal"));
    HEFF_TRY(arena_grow(op, &op->arena_vec, &op->arena_vec_b, need.vec, "arena start/result vectors"));
    if(cplx != op->cplx) op->emu_stale = true;
    op->cplx          = cplx;
    const size_t es   = cplx ? 16 : 8;
    op->cap_env       = (int64_t)(op->cap_env_b / es);
    op->cap_W         = (int64_t)(op->cap_W_b / es);
    op->cap_scratch   = (int64_t)(op->cap_scratch_b / es);
    op->scratch_bytes = op->cap_scratch_b;
    op->diag_cap      = (int64_t)(op->cap_diag_b / es);
    op->precision     = r.precision == HEFF_PREC_MIXED ? HEFF_PREC_MIXED : HEFF_PREC_FP64;
    if(need.mixed) HEFF_TRY(mixed_reserve(op, need.mixed));
    HEFF_TRY(heff_op_set_fp64_engine(op, r.fp64_engine == HEFF_FP64_INT8 ? HEFF_FP64_INT8 : HEFF_FP64_DMMA, 0));
    if(need.emu) HEFF_TRY(emu_reserve(op, r.spin, std::max(r.chiL, r.chiR), std::max(r.mpoL, r.mpoR)));
    const void   *mp[1] = {r.mpo};
    const int64_t md[4] = {r.mpoL, r.mpoR, r.spin, r.spin};
    const int64_t ld[3] = {r.chiL, r.chiL, r.mpoL};
    const int64_t rd[3] = {r.chiR, r.chiR, r.mpoR};
    HEFF_TRY(op_rebind(op, 1, mp, md, r.envL, ld, r.envR, rd));
    HEFF_TRY(eig_reserve(op, op->d.size_mps(), max_basis, r.precision == HEFF_PREC_MIXED));
    *vec = op->arena_vec;
    return HEFF_OK;
}

int op_prof_flush(heff_op *op) {
    if(op->prof_used == 0) return HEFF_OK;
    HEFF_CUDA(cudaStreamSynchronize(op->stream));
    for(int k = 0; k < op->prof_used; k++) {
        cudaEvent_t *e = op->prof_events.data() + 5 * k;
        for(int st = 0; st < 4; st++) {
            float ms = 0;
            HEFF_CUDA(cudaEventElapsedTime(&ms, e[st], e[st + 1]));
            op->prof_ms[st] += ms;
        }
        op->prof_count++;
    }
    op->prof_used = 0;
    return HEFF_OK;
}

cudaEvent_t *op_prof_slot(heff_op *op) {
    if(!op->profiling || op->prof_cap == 0) return nullptr;
    if(op->prof_used == op->prof_cap && op_prof_flush(op) != HEFF_OK) return nullptr;
    return op->prof_events.data() + 5 * (op->prof_used++);
}

// ---- CUDA graph of the FP64 matvec ----------------------------------------------------------------------------
// A small matvec is a handful of short kernels (permute, GEMM 1 [+ split reduction], MPO mix, GEMM 2 [+ split
// reduction]) whose launch costs are comparable to their run times; a sweep or an eigensolve applies the same
// operator shape tens to hundreds of times.  The first product of a shape runs as plain launches (which also perform
// every one-time set-up outside a capture) and is then recorded as a graph; later products patch the graph's two
// data-dependent parameters -- the permutation kernel's input and the output pointer in the GemmArgs of the last
// GEMM's kernels -- and launch it.  The graph is rebuilt when the shape or any operator buffer changes; a stream
// that cannot be captured (the legacy default stream) keeps the plain launches.
struct MatvecGraph {
    cudaGraph_t                       g  = nullptr;
    cudaGraphExec_t                   ex = nullptr;
    MatvecDims                        d{};
    bool                              cplx = false;
    const void                       *L = nullptr, *Rp = nullptr, *W = nullptr, *scr = nullptr, *split = nullptr;
    size_t                            split_bytes = 0;
    cudaGraphNode_t                   perm        = nullptr;
    cudaKernelNodeParams              perm_p{};
    std::vector<void *>               perm_args;
    std::vector<cudaGraphNode_t>      outs;
    std::vector<cudaKernelNodeParams> out_p;
    std::vector<GemmArgs>             out_a;
    int                               nkernels = 0;
    ~MatvecGraph() {
        if(ex) cudaGraphExecDestroy(ex);
        if(g) cudaGraphDestroy(g);
    }
    bool matches(const heff_op *op, bool c) const {
        return c == cplx && d.S == op->d.S && d.cL == op->d.cL && d.cR == op->d.cR && d.DL == op->d.DL && d.DR == op->d.DR && L == op->L &&
               Rp == op->Rp && W == op->W && scr == op->scratch && split == op->split_ws && split_bytes == op->split_bytes;
    }
};

// Step trace of the graph path on stderr (environment variable HEFF_GRAPHS_TRACE=1), for diagnosing a failure.
static bool graph_trace() {
    static const bool on = [] {
        const char *e = getenv("HEFF_GRAPHS_TRACE");
        return e && atoi(e) != 0;
    }();
    return on;
}
#define GTRACE(...)                                \
    do {                                           \
        if(graph_trace()) {                        \
            fprintf(stderr, "[heff graph] " __VA_ARGS__); \
            fputc('\n', stderr);                  \
            fflush(stderr);                        \
        }                                          \
    } while(0)

bool graphs_default() {
    static const bool on = [] {
        const char *e = getenv("HEFF_GRAPHS");
        return e && atoi(e) != 0;
    }();
    return on;
}

void op_graph_release(heff_op *op) {
    delete op->mg;
    op->mg = nullptr;
}

template<bool CPLX>
static int plain_apply(heff_op *op, const void *x, void *y) {
    using T = typename Scalar<CPLX>::T;
    MatvecScratch<CPLX> ws;
    ws.carve(reinterpret_cast<T *>(op->scratch), op->d);
    ws.split_ws    = op->split_ws;
    ws.split_bytes = op->split_bytes;
    return matvec_fp64<CPLX>(op->d, reinterpret_cast<const T *>(x), reinterpret_cast<T *>(y), reinterpret_cast<const T *>(op->L),
                             reinterpret_cast<const T *>(op->Rp), reinterpret_cast<const T *>(op->W), ws, op->stream, op_prof_slot(op));
}

// Records the matvec of the current shape (x, y as placeholders) and finds the nodes to retarget.  Any failure
// turns graphs off for this operator and leaves the plain launches in place.
template<bool CPLX>
static void graph_capture(heff_op *op, const void *x, void *y) {
    auto give_up = [&](MatvecGraph *G) {
        delete G;
        op->graphs = false;
        (void)cudaGetLastError();
    };
    MatvecGraph *G = new MatvecGraph();
    G->d = op->d, G->cplx = CPLX, G->L = op->L, G->Rp = op->Rp, G->W = op->W, G->scr = op->scratch, G->split = op->split_ws;
    G->split_bytes = op->split_bytes;
    GTRACE("capture begin (S=%lld cL=%lld cR=%lld DL=%lld DR=%lld cplx=%d)", (long long)op->d.S, (long long)op->d.cL, (long long)op->d.cR,
           (long long)op->d.DL, (long long)op->d.DR, (int)CPLX);
    if(cudaStreamBeginCapture(op->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return give_up(G);
    const int   rc = plain_apply<CPLX>(op, x, y);
    cudaGraph_t g  = nullptr;
    const cudaError_t e = cudaStreamEndCapture(op->stream, &g);
    GTRACE("capture end rc=%d err=%d graph=%p", rc, (int)e, (void *)g);
    G->g = g;
    if(rc != HEFF_OK || e != cudaSuccess || !g) return give_up(G);
    if(cudaGraphInstantiate(&G->ex, g, 0) != cudaSuccess) return give_up(G);
    size_t nn = 0;
    if(cudaGraphGetNodes(g, nullptr, &nn) != cudaSuccess) return give_up(G);
    GTRACE("instantiated, %zu nodes", nn);
    std::vector<cudaGraphNode_t> nodes(nn);
    if(cudaGraphGetNodes(g, nodes.data(), &nn) != cudaSuccess) return give_up(G);
    const void *pf = permute_kernel_fn(CPLX);
    for(cudaGraphNode_t nd : nodes) {
        cudaGraphNodeType t;
        if(cudaGraphNodeGetType(nd, &t) != cudaSuccess) return give_up(G);
        if(t != cudaGraphNodeTypeKernel) continue;
        G->nkernels++;
        cudaKernelNodeParams p{};
        if(cudaGraphKernelNodeGetParams(nd, &p) != cudaSuccess || !p.kernelParams) return give_up(G);
        GTRACE("kernel node func=%p permute=%d gemm=%d", p.func, (int)(p.func == pf), (int)gemm_fn_known(p.func));
        if(p.func == pf) {
            const void *x0 = nullptr;
            std::memcpy(&x0, p.kernelParams[0], sizeof(x0));  // the node's argument storage need not be aligned for the type
            if(G->perm || x0 != x) return give_up(G);
            G->perm   = nd;
            G->perm_p = p;
            G->perm_args.assign(p.kernelParams, p.kernelParams + 5);  // (x, xp, S, cL, n)
        } else if(gemm_fn_known(p.func)) {
            GemmArgs a;
            std::memcpy(&a, p.kernelParams[0], sizeof(a));  // byte copy: GemmArgs holds 16-byte-aligned members
            if(a.C == y) {
                G->outs.push_back(nd);
                G->out_p.push_back(p);
                G->out_a.push_back(a);
            }
        }
    }
    GTRACE("perm=%p outs=%zu", (void *)G->perm, G->outs.size());
    if(!G->perm || G->outs.empty()) return give_up(G);
    op->mg = G;
}

template<bool CPLX>
static int graph_replay(heff_op *op, const void *x, void *y) {
    MatvecGraph         *G  = op->mg;
    const void          *xv = x;
    std::vector<void *>  pa = G->perm_args;
    pa[0]                   = const_cast<void *>(reinterpret_cast<const void *>(&xv));
    cudaKernelNodeParams pp = G->perm_p;
    pp.kernelParams         = pa.data();
    pp.extra                = nullptr;
    GTRACE("replay: set input");
    HEFF_CUDA(cudaGraphExecKernelNodeSetParams(G->ex, G->perm, &pp));
    for(size_t i = 0; i < G->outs.size(); i++) {
        GemmArgs a             = G->out_a[i];
        a.C                    = y;
        void                *args[1] = {&a};
        cudaKernelNodeParams q = G->out_p[i];
        q.kernelParams         = args;
        q.extra                = nullptr;
        HEFF_CUDA(cudaGraphExecKernelNodeSetParams(G->ex, G->outs[i], &q));
    }
    GTRACE("replay: launch");
    HEFF_CUDA(cudaGraphLaunch(G->ex, op->stream));
    count_launches(G->nkernels);
    return HEFF_OK;
}

template<bool CPLX>
static int apply_impl(heff_op *op, const void *x, void *y) {
    using T = typename Scalar<CPLX>::T;
    if(x == y) {
        set_last_error_msg("MultAx: in and out must not alias");
        return HEFF_BAD_ARG;
    }
    if(op->sequential) {
        std::vector<const T *> W(op->seq_W.size());
        for(size_t i = 0; i < W.size(); i++) W[i] = reinterpret_cast<const T *>(op->seq_W[i]);
        HEFF_TRY(matvec_multi<CPLX>(op->multi, reinterpret_cast<const T *>(x), reinterpret_cast<T *>(y), reinterpret_cast<const T *>(op->L),
                                    reinterpret_cast<const T *>(op->Rp), W.data(), reinterpret_cast<T *>(op->scratch), op->stream));
        op->num_mv++;
        return HEFF_OK;
    }
    if(op->graphs && !op->profiling && op->stream) {
        if(op->mg && op->mg->matches(op, CPLX)) {
            HEFF_TRY(graph_replay<CPLX>(op, x, y));
        } else {
            op_graph_release(op);
            HEFF_TRY(plain_apply<CPLX>(op, x, y));  // this product, and every one-time set-up, outside a capture
            graph_capture<CPLX>(op, x, y);          // recorded for the next products of this shape
        }
    } else {
        HEFF_TRY(plain_apply<CPLX>(op, x, y));
    }
    op->num_mv++;
    return HEFF_OK;
}

int op_apply(heff_op *op, const void *x, void *y) {
    if(!op || !x || !y) return HEFF_BAD_ARG;
    if(op->precision == HEFF_PREC_MIXED && op->mixed_apply) return op->mixed_apply(op, x, y);
    if(op->fp64_engine == HEFF_FP64_INT8 && emu_supported(op)) return emu_apply(op, x, y);
    return op->cplx ? apply_impl<true>(op, x, y) : apply_impl<false>(op, x, y);
}

}  // namespace heff

using namespace heff;

extern "C" int heff_op_create(heff_op **op, heff_dtype dtype, int nsites, const void *const *mpos, const int64_t *mpo_dims, const void *envL,
                              const int64_t envL_dims[3], const void *envR, const int64_t envR_dims[3], heff_mem where, heff_precision precision,
                              void *stream) {
    if(dtype == HEFF_F64)
        return create_impl<false>(op, nsites, mpos, mpo_dims, envL, envL_dims, envR, envR_dims, where, precision, (cudaStream_t)stream);
    if(dtype == HEFF_C128)
        return create_impl<true>(op, nsites, mpos, mpo_dims, envL, envL_dims, envR, envR_dims, where, precision, (cudaStream_t)stream);
    return HEFF_BAD_ARG;
}

extern "C" int heff_op_destroy(heff_op *op) {
    if(!op) return HEFF_OK;
    op_graph_release(op);
    if(op->destroy_hook) op->destroy_hook(op);
    emu_destroy(op);
    for(cudaEvent_t e : op->prof_events) cudaEventDestroy(e);
    if(op->L) cudaFree(op->L);
    if(op->Rp) cudaFree(op->Rp);
    if(op->W) cudaFree(op->W);
    if(op->scratch) cudaFree(op->scratch);
    if(op->split_ws) cudaFree(op->split_ws);
    if(op->stage_x) cudaFree(op->stage_x);
    if(op->eig_ws) cudaFree(op->eig_ws);
    if(op->Rtmp) cudaFree(op->Rtmp);
    if(op->arena_vec) cudaFree(op->arena_vec);
    if(op->dense_ws) cudaFree(op->dense_ws);
    for(void *p : op->seq_W) cudaFree(p);
    if(op->pipe) {
        if(op->pipe->aux) cudaStreamDestroy(op->pipe->aux);
        if(op->pipe->copy) cudaStreamDestroy(op->pipe->copy);
        for(cudaEvent_t e : op->pipe->ev)
            if(e) cudaEventDestroy(e);
        delete op->pipe;
    }
    if(op->diag) cudaFree(op->diag);
    if(op->jcb) cudaFree(op->jcb);
    if(op->eig_host) cudaFreeHost(op->eig_host);
    if(op->eig_event) cudaEventDestroy(op->eig_event);
    delete op;
    return HEFF_OK;
}

extern "C" int64_t heff_op_rows(const heff_op *op) { return op ? op->d.size_mps() : -1; }

extern "C" int heff_op_shape(const heff_op *op, int64_t shape[3]) {
    if(!op || !shape) return HEFF_BAD_ARG;
    shape[0] = op->d.S;
    shape[1] = op->d.cL;
    shape[2] = op->d.cR;
    return HEFF_OK;
}

extern "C" int heff_op_multax(heff_op *op, const void *x, void *y) { return op_apply(op, x, y); }
extern "C" int heff_perform_op(heff_op *op, const void *x, void *y) { return op_apply(op, x, y); }

extern "C" int heff_op_multax_block(heff_op *op, const void *x, int64_t ldx, void *y, int64_t ldy, int block_size) {
    if(!op || !x || !y || block_size < 0) return HEFF_BAD_ARG;
    const int64_t n  = op->d.size_mps();
    const size_t  es = op->cplx ? 16 : 8;
    if(ldx < n || ldy < n) return HEFF_BAD_SHAPE;
    for(int i = 0; i < block_size; i++) {
        const char *xi = reinterpret_cast<const char *>(x) + (size_t)ldx * i * es;
        char       *yi = reinterpret_cast<char *>(y) + (size_t)ldy * i * es;
        HEFF_TRY(op_apply(op, xi, yi));
    }
    return HEFF_OK;
}

// Host-buffer matvec with the copies overlapped (matvec_fp64_host): FP64 operators of at least 8 MB per vector.
template<bool CPLX>
static int multax_host_pipelined(heff_op *op, const void *x_host, void *y_host, void *dx, void *dy) {
    using T = typename Scalar<CPLX>::T;
    if(!op->pipe) {
        HostPipe *hp = new HostPipe();
        op->pipe     = hp;
        HEFF_CUDA(cudaStreamCreateWithFlags(&hp->aux, cudaStreamNonBlocking));
        HEFF_CUDA(cudaStreamCreateWithFlags(&hp->copy, cudaStreamNonBlocking));
        for(cudaEvent_t &e : hp->ev) HEFF_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    op->pipe->s = op->stream;
    MatvecScratch<CPLX> ws;
    ws.carve(reinterpret_cast<T *>(op->scratch), op->d);
    HEFF_TRY(matvec_fp64_host<CPLX>(op->d, reinterpret_cast<const T *>(x_host), reinterpret_cast<T *>(y_host), reinterpret_cast<const T *>(op->L),
                                    reinterpret_cast<const T *>(op->Rp), reinterpret_cast<const T *>(op->W), ws, reinterpret_cast<T *>(dx),
                                    reinterpret_cast<T *>(dy), *op->pipe));
    op->num_mv++;
    return HEFF_OK;
}

extern "C" int heff_op_multax_host(heff_op *op, const void *x_host, void *y_host) {
    if(!op || !x_host || !y_host) return HEFF_BAD_ARG;
    const int64_t n     = op->d.size_mps();
    const size_t  bytes = (size_t)n * (op->cplx ? 16 : 8);
    if(op->stage_bytes < 2 * bytes + 256) {  // grown for a rebind to larger dimensions
        if(op->stage_x) {
            HEFF_CUDA(cudaStreamSynchronize(op->stream));
            cudaFree(op->stage_x);
            op->stage_x     = nullptr;
            op->stage_bytes = 0;
        }
        HEFF_CUDA(cudaMalloc(&op->stage_x, 2 * bytes + 256));
        op->stage_bytes = 2 * bytes + 256;
    }
    void *dx = op->stage_x;
    void *dy = reinterpret_cast<char *>(op->stage_x) + ((bytes + 255) / 256) * 256;
    if(op->precision == HEFF_PREC_FP64 && op->fp64_engine == HEFF_FP64_DMMA && !op->sequential && bytes >= ((size_t)8 << 20))
        return op->cplx ? multax_host_pipelined<true>(op, x_host, y_host, dx, dy) : multax_host_pipelined<false>(op, x_host, y_host, dx, dy);
    HEFF_CUDA(cudaMemcpyAsync(dx, x_host, bytes, cudaMemcpyHostToDevice, op->stream));
    HEFF_TRY(op_apply(op, dx, dy));
    HEFF_CUDA(cudaMemcpyAsync(y_host, dy, bytes, cudaMemcpyDeviceToHost, op->stream));
    HEFF_CUDA(cudaStreamSynchronize(op->stream));
    return HEFF_OK;
}

extern "C" int heff_op_set_stream(heff_op *op, void *stream) {
    if(!op) return HEFF_BAD_ARG;
    op->stream = (cudaStream_t)stream;
    return HEFF_OK;
}

extern "C" int heff_op_set_precision(heff_op *op, heff_precision precision) {
    if(!op) return HEFF_BAD_ARG;
    if(precision != HEFF_PREC_FP64 && precision != HEFF_PREC_MIXED) return HEFF_BAD_ARG;
    if(op->sequential && precision != HEFF_PREC_FP64) {
        set_last_error_msg("operator over more than 5 site MPOs: FP64 only");
        return HEFF_BAD_ARG;
    }
    op->precision = precision;
    return HEFF_OK;
}

extern "C" int heff_op_set_fp64_engine(heff_op *op, int engine, int nslices) {
    if(!op) return HEFF_BAD_ARG;
    if(engine != HEFF_FP64_DMMA && engine != HEFF_FP64_INT8) return HEFF_BAD_ARG;
    if(nslices == 0) nslices = Z_DEFAULT_SLICES;
    if(nslices < 3 || nslices > Z_MAX_SLICES) return HEFF_BAD_ARG;
    if(nslices != op->emu_slices) {
        if(op->emu) HEFF_CUDA(cudaStreamSynchronize(op->stream));
        emu_destroy(op);  // planes are laid out per slice count
        op->emu_slices = nslices;
    }
    op->fp64_engine = engine;
    return HEFF_OK;
}

extern "C" int heff_op_set_graphs(heff_op *op, int enable) {
    if(!op) return HEFF_BAD_ARG;
    op->graphs = enable != 0;
    if(!op->graphs) op_graph_release(op);
    return HEFF_OK;
}

extern "C" int64_t heff_op_num_mv(const heff_op *op) { return op ? op->num_mv : -1; }

extern "C" int heff_op_device_error(heff_op *op, int *code) {
    if(!op || !code) return HEFF_BAD_ARG;
    int m = 0, e = 0;
    HEFF_TRY(mixed_error_flag(op, &m));
    HEFF_TRY(emu_error_flag(op, &e));
    *code = m ? m : e;
    return HEFF_OK;
}

extern "C" int heff_op_set_profiling(heff_op *op, int enable) {
    if(!op) return HEFF_BAD_ARG;
    if(enable && op->prof_cap == 0) {
        op->prof_cap = 1024;
        op->prof_events.resize(5 * op->prof_cap);
        for(auto &e : op->prof_events) HEFF_CUDA(cudaEventCreate(&e));
    }
    if(!enable) HEFF_TRY(op_prof_flush(op));
    op->profiling = enable != 0;
    return HEFF_OK;
}

extern "C" int heff_op_stage_times(heff_op *op, double ms[4], int64_t *count, int reset) {
    if(!op || !ms) return HEFF_BAD_ARG;
    HEFF_TRY(op_prof_flush(op));
    for(int i = 0; i < 4; i++) ms[i] = op->prof_ms[i];
    if(count) *count = op->prof_count;
    if(reset) {
        for(int i = 0; i < 4; i++) op->prof_ms[i] = 0;
        op->prof_count = 0;
    }
    return HEFF_OK;
}
