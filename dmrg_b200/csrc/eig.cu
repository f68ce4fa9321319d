// Device eigensolver for H_eff, driving the operator through the same apply path the reference's
// PRIMME/ARPACK callback uses (MatVecMPOS::MultAx, solver_primme.cpp:122-128).
//
// Phase 1 -- thick-restart Davidson without preconditioner, i.e. a restarted Krylov (Lanczos) method:
//   * expansion with A v_last (for a Hermitian operator this spans the same Krylov space as expanding
//     with the Ritz residual, also after a thick restart); the projection coefficients of A v_last on
//     the basis are the new column of the Rayleigh-Ritz matrix, so one pass over the basis per iteration,
//   * FP64 Gram-Schmidt with DGKS selective re-orthogonalisation (a second pass only when the first
//     removed more than half of the vector's norm squared), decided and normalised on the device so the
//     next matvec is enqueued before the host reads the coefficients,
//   * Rayleigh-Ritz on the host in FP64; Ritz selection smallest / largest algebraic or closest to a target,
//   * residual norm |beta s_last| from the Krylov relation, checked explicitly (x = V s, r = AV s - theta x)
//     before convergence is declared.
// With an FP64 operator this phase runs to the tolerance: ||H x - theta x|| <= tol * ||H||_est
// (PRIMME eps, solver_primme.cpp:364; ||H||_est = largest |Ritz value| seen).
//
// Mixed precision (operator HEFF_PREC_MIXED): phase 1 runs on the split-BF16 matvec until its residual
// reaches mixed_tol * ||H||_est or stops improving (the inexact operator floors it), then
// Phase 2 -- Jacobi-Davidson refinement in FP64: an FP64 search space starting from the phase-1 Ritz
// vector, FP64 products of every basis vector, FP64 Rayleigh-Ritz (so the energy can only improve);
// each expansion vector is an approximate solution of the correction equation
//   (I - u u^H)(H - theta)(I - u u^H) t = -r
// by a few CG iterations on the mixed (cheap) matvec.  One FP64 matvec per refinement step.
#include <chrono>
#include <complex>
#include <cstring>
#include <numeric>
#include <type_traits>
#include <vector>

#include "blas1.cuh"
#include "eig.cuh"
#include "matvec.cuh"
#include "op.cuh"
#include "runtime.cuh"
#include "small_eig.hpp"

namespace heff {

__global__ void init_vec_kernel(double *x, int64_t nreal, uint64_t seed) {
    for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nreal; i += (int64_t)gridDim.x * blockDim.x) {
        uint64_t z = seed + 0x9E3779B97F4A7C15ull * (uint64_t)(i + 1);
        z          = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z          = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z ^= z >> 31;
        x[i] = 2.0 * ((double)(z >> 11) * (1.0 / 9007199254740992.0)) - 1.0;
    }
}

template<bool CPLX>
struct HostScalar;
template<>
struct HostScalar<false> {
    using T = double;
    static double conj(double v) { return v; }
    static double re(double v) { return v; }
};
template<>
struct HostScalar<true> {
    using T = std::complex<double>;
    static T      conj(T v) { return std::conj(v); }
    static double re(T v) { return v.real(); }
};

// Ritz decomposition of the k x k projected matrix (leading dimension ld): ascending w, vectors column-major.
template<bool CPLX>
static int ritz(int k, const std::vector<typename HostScalar<CPLX>::T> &Hk, int ld, std::vector<double> &w,
                std::vector<typename HostScalar<CPLX>::T> &vecs) {
    if constexpr(!CPLX) {
        std::vector<double> a((size_t)k * k);
        for(int j = 0; j < k; j++)
            for(int i = 0; i < k; i++) a[i + (size_t)k * j] = 0.5 * (Hk[i + (size_t)ld * j] + Hk[j + (size_t)ld * i]);
        if(sym_eig(k, a, w)) return HEFF_NOT_CONVERGED;
        vecs.swap(a);
    } else {
        std::vector<std::complex<double>> a((size_t)k * k);
        for(int j = 0; j < k; j++)
            for(int i = 0; i < k; i++) a[i + (size_t)k * j] = 0.5 * (Hk[i + (size_t)ld * j] + std::conj(Hk[j + (size_t)ld * i]));
        if(herm_eig(k, a, w, vecs)) return HEFF_NOT_CONVERGED;
    }
    return HEFF_OK;
}

static std::vector<int> ritz_order(const std::vector<double> &w, int rule, double target) {
    std::vector<int> o(w.size());
    std::iota(o.begin(), o.end(), 0);
    if(rule == HEFF_RITZ_LA) std::reverse(o.begin(), o.end());
    if(rule == HEFF_RITZ_TARGET) std::stable_sort(o.begin(), o.end(), [&](int a, int b) { return std::fabs(w[a] - target) < std::fabs(w[b] - target); });
    return o;
}

// Pinned host buffer and event through which the Krylov loop reads each iteration's coefficients while
// the next matvec runs (created once per operator).
int eig_host_ready(heff_op *op) {
    if(!op->eig_host) {
        cudaError_t e = cudaMallocHost(&op->eig_host, sizeof(double2) * (MD_MAXK + 2));
        if(e != cudaSuccess) {
            op->eig_host = nullptr;
            set_last_cuda_error(e, "eigensolver host buffer", __FILE__, __LINE__);
            return HEFF_OOM;
        }
    }
    if(!op->eig_event) HEFF_CUDA(cudaEventCreateWithFlags(&op->eig_event, cudaEventDisableTiming));
    return HEFF_OK;
}

template<bool CPLX>
struct Davidson {
    using T  = typename Scalar<CPLX>::T;
    using HT = typename HostScalar<CPLX>::T;
    heff_op               *op;
    const heff_eig_config &cfg;
    heff_eig_result       &res;
    cudaStream_t           s;
    int64_t                n;
    int                    maxb, minb;
    T *V = nullptr, *AV = nullptr, *V2 = nullptr, *AV2 = nullptr, *t = nullptr, *x = nullptr, *ax = nullptr, *r = nullptr;
    T *cg_p = nullptr, *cg_q = nullptr, *cg_z = nullptr, *cg_d = nullptr, *cg_r = nullptr;
    T *dh = nullptr, *dc = nullptr, *hres = nullptr;
    double             *partials = nullptr, *dscal = nullptr, *orth_st = nullptr, *cg_cs = nullptr;
    unsigned           *orth_counter = nullptr;
    std::vector<HT>     Hk, G2;
    std::vector<void *> allocs;
    double              anorm = 0.0;

    Davidson(heff_op *o, const heff_eig_config &c, heff_eig_result &r_) : op(o), cfg(c), res(r_), s(o->stream), n(o->d.size_mps()) {
        maxb = std::max(4, std::min(cfg.max_basis > 0 ? cfg.max_basis : 32, (int)MD_MAXK - 1));
        minb = std::max(1, std::min(cfg.min_basis > 0 ? cfg.min_basis : 8, maxb - 2));
        if((int64_t)maxb > n) maxb = (int)std::max<int64_t>(1, n);
        if(minb >= maxb) minb = std::max(1, maxb - 1);
    }
    // All device buffers are carved from the operator's eigensolver workspace, which persists across
    // solves on the same operator (no allocation per solve once it has grown to size).
    char  *carve_ptr = nullptr;
    size_t carve_left = 0;
    int    take(void **p, size_t bytes) {
        bytes = (bytes + 255) / 256 * 256;
        if(bytes > carve_left) return HEFF_OOM;
        *p = carve_ptr;
        carve_ptr += bytes;
        carve_left -= bytes;
        return HEFF_OK;
    }
    static size_t workspace_bytes(int64_t n, int maxb, bool mixed) {
        const size_t es  = sizeof(T);
        const size_t vec = (es * n + 255) / 256 * 256;
        return vec * (4 * (maxb + 1) + 4 + (mixed ? 5 : 0)) + es * MD_MAXK * 3 + es * MD_MAXK * MD_MAXK +
               sizeof(double) * MD_BLOCKS * MD_MAXK * 4 + 16 * sizeof(double) + es * (MD_MAXK + 2) +
               sizeof(double) * (8 + 4 * (MD_MAXK + 2)) + 21 * 256;
    }
    int setup(bool mixed) {
        const size_t es   = sizeof(T);
        const size_t need = workspace_bytes(n, maxb, mixed);
        if(op->eig_ws_bytes < need) {
            if(op->eig_ws) {
                HEFF_CUDA(cudaStreamSynchronize(s));
                cudaFree(op->eig_ws);
                op->eig_ws       = nullptr;
                op->eig_ws_bytes = 0;
            }
            cudaError_t e = cudaMalloc(&op->eig_ws, need);
            if(e != cudaSuccess) {
                set_last_cuda_error(e, "eigensolver workspace", __FILE__, __LINE__);
                return HEFF_OOM;
            }
            op->eig_ws_bytes = need;
        }
        carve_ptr  = reinterpret_cast<char *>(op->eig_ws);
        carve_left = op->eig_ws_bytes;
        HEFF_TRY(take((void **)&V, es * n * (maxb + 1)));  // column maxb holds the next Krylov vector
        HEFF_TRY(take((void **)&AV, es * n * (maxb + 1)));  // column maxb holds the product of the next Krylov vector
        HEFF_TRY(take((void **)&V2, es * n * (maxb + 1)));
        HEFF_TRY(take((void **)&AV2, es * n * (maxb + 1)));
        for(T **p : {&t, &x, &ax, &r}) HEFF_TRY(take((void **)p, es * n));
        if(mixed)
            for(T **p : {&cg_p, &cg_q, &cg_z, &cg_d, &cg_r}) HEFF_TRY(take((void **)p, es * n));
        HEFF_TRY(take((void **)&dh, es * MD_MAXK * 3));
        HEFF_TRY(take((void **)&dc, es * MD_MAXK * MD_MAXK));
        HEFF_TRY(take((void **)&partials, sizeof(double) * MD_BLOCKS * MD_MAXK * 4));
        HEFF_TRY(take((void **)&dscal, sizeof(double) * 16));
        HEFF_TRY(take((void **)&hres, es * (MD_MAXK + 2)));
        HEFF_TRY(take((void **)&orth_st, sizeof(double) * (8 + 4 * (MD_MAXK + 2))));
        HEFF_TRY(take((void **)&orth_counter, 256));
        HEFF_TRY(take((void **)&cg_cs, sizeof(double) * 16));
        HEFF_CUDA(cudaMemsetAsync(orth_counter, 0, sizeof(unsigned), s));
        HEFF_TRY(eig_host_ready(op));
        Hk.assign((size_t)maxb * maxb, HT(0));
        G2.assign((size_t)maxb * maxb, HT(0));
        return HEFF_OK;
    }
    int sync() {
        HEFF_CUDA(cudaStreamSynchronize(s));
        return HEFF_OK;
    }
    int dot(const T *a, const T *b, HT &out) {  // <a, b> -> host
        T d;
        HEFF_TRY(dot_device<CPLX>(a, b, n, reinterpret_cast<T *>(dscal), partials, s));
        HEFF_CUDA(cudaMemcpyAsync(&d, dscal, sizeof(T), cudaMemcpyDeviceToHost, s));
        HEFF_TRY(sync());
        std::memcpy((void *)&out, (void *)&d, sizeof(T));
        return HEFF_OK;
    }
    int norm2(const T *v, double &out) {
        HT d;
        HEFF_TRY(dot(v, v, d));
        out = HostScalar<CPLX>::re(d);
        return HEFF_OK;
    }
    // y += a * v (a real, host value)
    int axpy(double a, const T *v, T *y) {
        const T one = one_value();
        HEFF_CUDA(cudaMemcpyAsync(dh + 2 * MD_MAXK, &one, sizeof(T), cudaMemcpyHostToDevice, s));
        return multi_axpy<CPLX>(v, n, n, 1, dh + 2 * MD_MAXK, a, y, s);
    }
    int scale(T *v, double a) {
        HEFF_CUDA(cudaMemcpyAsync(dscal + 8, &a, sizeof(double), cudaMemcpyHostToDevice, s));
        HEFF_TRY(scale_dev<CPLX>(v, n, dscal + 8, false, s));
        return sync();  // the host scalar above must stay valid until the copy ran
    }
    static T one_value() {
        if constexpr(CPLX)
            return make_double2(1.0, 0.0);
        else
            return 1.0;
    }
    int apply(const T *in, T *out, bool fp64) {
        const heff_precision keep = op->precision;
        if(fp64) op->precision = HEFF_PREC_FP64;
        int rc        = op_apply(op, in, out);
        op->precision = keep;
        if(fp64 || keep == HEFF_PREC_FP64)
            res.num_mv_fp64++;
        else
            res.num_mv_mixed++;
        res.num_mv++;
        return rc;
    }
    // Orthonormalise t against V[:, :k] (Gram-Schmidt, DGKS second pass when needed).
    // nrm0: norm before, nrm: norm after (before normalisation).
    int orthonormalize(T *Vb, int k, double &nrm0, double &nrm) {
        double n2 = 0;
        HEFF_TRY(norm2(t, n2));
        nrm0 = std::sqrt(n2);
        nrm  = nrm0;
        for(int pass = 0; pass < 2 && k > 0; pass++) {
            HEFF_TRY(multi_dot<CPLX>(Vb, n, n, k, t, dh, partials, s));
            HEFF_TRY(multi_axpy<CPLX>(Vb, n, n, k, dh, -1.0, t, s));
            const double before = nrm;
            HEFF_TRY(norm2(t, n2));
            nrm = std::sqrt(n2);
            if(nrm > 0.7 * before) break;
        }
        if(!std::isfinite(nrm)) {
            set_last_error_msg("eigensolver: non-finite vector (NaN/Inf in the operator or start vector)");
            return HEFF_NAN_INPUT;
        }
        if(nrm > 0) HEFF_TRY(scale(t, 1.0 / nrm));
        return HEFF_OK;
    }
    int random_vector(T *v, uint64_t seed) {
        const int64_t nr = n * (CPLX ? 2 : 1);
        init_vec_kernel<<<(int)std::min<int64_t>((nr + 255) / 256, 4096), 256, 0, s>>>(reinterpret_cast<double *>(v), nr, seed);
        HEFF_LAUNCH_CHECK();
        return HEFF_OK;
    }
    // Append column k: V[:,k] = t (normalised), AV[:,k] = A t, projected-matrix column, AV-Gram column.
    int append(int k, bool fp64, bool track_g2) {
        HEFF_CUDA(cudaMemcpyAsync(V + (int64_t)k * n, t, sizeof(T) * n, cudaMemcpyDeviceToDevice, s));
        HEFF_TRY(apply(V + (int64_t)k * n, AV + (int64_t)k * n, fp64));
        HEFF_TRY(multi_dot<CPLX>(V, n, n, k + 1, AV + (int64_t)k * n, dh, partials, s));
        if(track_g2) HEFF_TRY(multi_dot<CPLX>(AV, n, n, k + 1, AV + (int64_t)k * n, dh + MD_MAXK, partials + 2 * MD_BLOCKS * MD_MAXK, s));
        std::vector<T> col(2 * (k + 1));
        HEFF_CUDA(cudaMemcpyAsync(col.data(), dh, sizeof(T) * (k + 1), cudaMemcpyDeviceToHost, s));
        if(track_g2) HEFF_CUDA(cudaMemcpyAsync(col.data() + (k + 1), dh + MD_MAXK, sizeof(T) * (k + 1), cudaMemcpyDeviceToHost, s));
        HEFF_TRY(sync());
        for(int i = 0; i <= k; i++) {
            HT v;
            std::memcpy((void *)&v, (void *)&col[i], sizeof(T));
            Hk[i + (size_t)maxb * k] = v;
            Hk[k + (size_t)maxb * i] = HostScalar<CPLX>::conj(v);
            if(track_g2) {
                std::memcpy((void *)&v, (void *)&col[k + 1 + i], sizeof(T));
                G2[i + (size_t)maxb * k] = v;
                G2[k + (size_t)maxb * i] = HostScalar<CPLX>::conj(v);
            }
        }
        return HEFF_OK;
    }
    // x = V s, ax = AV s, r = ax - theta x ; returns ||r||
    int explicit_residual(int k, const HT *svec, double theta, double &rn) {
        HEFF_CUDA(cudaMemcpyAsync(dc, (const void *)svec, sizeof(T) * k, cudaMemcpyHostToDevice, s));
        HEFF_TRY(combine<CPLX>(V, n, n, k, dc, x, s));
        HEFF_TRY(combine<CPLX>(AV, n, n, k, dc, ax, s));
        HEFF_TRY(residual<CPLX>(ax, x, theta, r, n, s));
        double r2 = 0;
        HEFF_TRY(norm2(r, r2));
        rn = std::sqrt(r2);
        return HEFF_OK;
    }
    // thick restart to the m best Ritz vectors
    int restart(int k, int m, const std::vector<double> &w, const std::vector<HT> &vecs, const std::vector<int> &ord, bool track_g2) {
        std::vector<HT> S((size_t)k * m);
        for(int q = 0; q < m; q++)
            for(int i = 0; i < k; i++) S[i + (size_t)k * q] = vecs[i + (size_t)k * ord[q]];
        HEFF_CUDA(cudaMemcpyAsync(dc, (const void *)S.data(), sizeof(T) * k * m, cudaMemcpyHostToDevice, s));
        GemmArgs g{};
        g.M = (int)n, g.N = m, g.K = k, g.batch = 1;
        g.A = V, g.lda = n, g.B = dc, g.ldb = k, g.C = V2, g.ldc = n;
        g.alpha = make_double2(1, 0), g.beta = make_double2(0, 0);
        HEFF_TRY(gemm_f64<CPLX>(false, false, false, g, s));
        g.A = AV, g.C = AV2;
        HEFF_TRY(gemm_f64<CPLX>(false, false, false, g, s));
        std::swap(V, V2);
        std::swap(AV, AV2);
        if(track_g2) {  // G2 <- S^H G2 S
            std::vector<HT> tmp((size_t)k * m, HT(0)), g2n((size_t)maxb * maxb, HT(0));
            for(int q = 0; q < m; q++)
                for(int i = 0; i < k; i++) {
                    HT acc(0);
                    for(int j = 0; j < k; j++) acc += G2[i + (size_t)maxb * j] * S[j + (size_t)k * q];
                    tmp[i + (size_t)k * q] = acc;
                }
            for(int q = 0; q < m; q++)
                for(int p = 0; p < m; p++) {
                    HT acc(0);
                    for(int i = 0; i < k; i++) acc += HostScalar<CPLX>::conj(S[i + (size_t)k * p]) * tmp[i + (size_t)k * q];
                    g2n[p + (size_t)maxb * q] = acc;
                }
            G2.swap(g2n);
        }
        std::fill(Hk.begin(), Hk.end(), HT(0));
        for(int q = 0; q < m; q++) Hk[q + (size_t)maxb * q] = HT(w[ord[q]]);
        res.restarts++;
        return sync();  // S must outlive its copy
    }

    // V[:, 0] = x0 / ||x0|| (a seeded random vector when x0 is NULL or zero)
    int init_start(const void *x0) {
        if(x0)
            HEFF_CUDA(cudaMemcpyAsync(V, x0, sizeof(T) * n, cudaMemcpyDeviceToDevice, s));
        else
            HEFF_TRY(random_vector(V, 0x5eedULL + (uint64_t)cfg.seed));
        double n2 = 0;
        HEFF_TRY(norm2(V, n2));
        if(!std::isfinite(n2)) {
            set_last_error_msg("eigensolver: non-finite start vector");
            return HEFF_NAN_INPUT;
        }
        if(!(n2 > 0)) {
            HEFF_TRY(random_vector(V, 0x5eedULL + (uint64_t)cfg.seed));
            HEFF_TRY(norm2(V, n2));
        }
        return scale(V, 1.0 / std::sqrt(n2));
    }

    // Phase 1 (thick-restart Krylov / Lanczos structure).  With w = A v_{k-1} projected out of V_k,
    //   A V_k = V_k H_k + beta v_k e_k^H,
    // so the projection coefficients ARE the last column of the Rayleigh-Ritz matrix H_k and the Ritz
    // residual norm is |beta * s_{k-1}|.  The projection (with its DGKS second pass) and the normalisation of
    // v_k run on the device (orth_cgs2), so the product A v_k is enqueued before the host reads the
    // coefficients: the host's Rayleigh-Ritz step overlaps the GPU's matvec.  A thick restart keeps
    // Y = V_k S_m (all residuals along v_k) and appends v_k with its product, preserving the relation.
    // Returns x = Ritz vector (normalised), theta, rnorm (explicit when converged).
    int run(const void *x0, bool use_mixed, double stop_tol, int64_t max_mv, double &theta, double &rnorm, bool &conv) {
        conv  = false;
        theta = 0;
        rnorm = INFINITY;
        HEFF_TRY(init_start(x0));
        std::fill(Hk.begin(), Hk.end(), HT(0));
        HEFF_TRY(apply(V, AV, !use_mixed));
        int                 k = 1;
        std::vector<double> w;
        std::vector<HT>     vecs;
        T                  *hh    = reinterpret_cast<T *>(op->eig_host);
        int                 stagn = 0;
        double              best = INFINITY, verify = 1.0;
        while(true) {
            T *vk = V + (int64_t)k * n;  // slot of the next basis vector
            HEFF_TRY(orth_cgs2<CPLX>(V, n, n, k, AV + (int64_t)(k - 1) * n, vk, partials, orth_counter, orth_st, hres, s));
            HEFF_CUDA(cudaMemcpyAsync(hh, hres, sizeof(T) * (k + 2), cudaMemcpyDeviceToHost, s));
            HEFF_CUDA(cudaEventRecord(op->eig_event, s));
            // the product of v_k, needed by the next iteration unless the solve stops here
            HEFF_TRY(apply(vk, AV + (int64_t)k * n, !use_mixed));
            HEFF_CUDA(cudaEventSynchronize(op->eig_event));
            std::vector<HT> h(k, HT(0));
            for(int i = 0; i < k; i++) std::memcpy((void *)&h[i], (void *)&hh[i], sizeof(T));
            HT bt, wf;
            std::memcpy((void *)&bt, (void *)&hh[k], sizeof(T));
            std::memcpy((void *)&wf, (void *)&hh[k + 1], sizeof(T));
            const double beta = HostScalar<CPLX>::re(bt), w2 = HostScalar<CPLX>::re(wf);
            if(!std::isfinite(w2) || !std::isfinite(beta)) {
                set_last_error_msg("eigensolver: non-finite vector (NaN/Inf in the operator or start vector)");
                return HEFF_NAN_INPUT;
            }
            for(int i = 0; i < k; i++) {
                Hk[i + (size_t)maxb * (k - 1)] = h[i];
                Hk[(k - 1) + (size_t)maxb * i] = HostScalar<CPLX>::conj(h[i]);
            }
            HEFF_TRY(ritz<CPLX>(k, Hk, maxb, w, vecs));
            for(double wi : w) anorm = std::max(anorm, std::fabs(wi));
            const std::vector<int> ord = ritz_order(w, cfg.ritz, cfg.target);
            theta                      = w[ord[0]];
            const HT *sv               = vecs.data() + (size_t)k * ord[0];
            const double est           = beta * std::abs(std::complex<double>(sv[k - 1]));
            rnorm                      = est;
            res.iters++;
            if(est <= verify * stop_tol * std::max(anorm, 1e-300) || res.num_mv >= max_mv) {
                HEFF_TRY(explicit_residual(k, sv, theta, rnorm));
                if(!std::isfinite(rnorm)) {
                    set_last_error_msg("eigensolver: non-finite residual");
                    return HEFF_NAN_INPUT;
                }
                if(rnorm <= stop_tol * std::max(anorm, 1e-300)) {
                    conv = true;
                    break;
                }
                verify *= 0.1;  // the estimate was optimistic: ask it for more before the next check
                if(res.num_mv >= max_mv) break;
            }
            if(use_mixed) {  // stop when the inexact operator floors the residual
                if(est < 0.5 * best) {
                    best  = est;
                    stagn = 0;
                } else if(++stagn >= 20) {
                    HEFF_TRY(explicit_residual(k, sv, theta, rnorm));
                    break;
                }
            }
            if(!(beta > 1e-13 * std::sqrt(std::max(w2, 1e-300)))) {
                // invariant subspace: the Ritz pair is exact for this operator
                HEFF_TRY(explicit_residual(k, sv, theta, rnorm));
                conv = rnorm <= stop_tol * std::max(anorm, 1e-300);
                break;
            }
            if(k == maxb) {
                // keep minb Ritz vectors, then append v_k and its product
                HEFF_TRY(restart(k, minb, w, vecs, ord, false));  // swaps V <-> V2, AV <-> AV2: v_k is now V2[:, k]
                HEFF_CUDA(cudaMemcpyAsync(V + (int64_t)minb * n, V2 + (int64_t)k * n, sizeof(T) * n, cudaMemcpyDeviceToDevice, s));
                HEFF_CUDA(cudaMemcpyAsync(AV + (int64_t)minb * n, AV2 + (int64_t)k * n, sizeof(T) * n, cudaMemcpyDeviceToDevice, s));
                k = minb + 1;
            } else {
                k++;
            }
        }
        return HEFF_OK;
    }

    // Jacobi-preconditioned Davidson (FP64): the expansion vector is t = (diag - theta)^-1 r for the current
    // Ritz pair (MultPc with the Ritz value as shift, matvec_mpos.cpp:1349-1364), orthonormalised against V
    // (DGKS), with its Rayleigh-Ritz column from a pass over the basis; thick restart to min_basis vectors.
    // Falls back to t = r when the preconditioned vector lies in the basis.
    int run_pc(const void *x0, double stop_tol, int64_t max_mv, double &theta, double &rnorm, bool &conv) {
        conv  = false;
        theta = 0;
        rnorm = INFINITY;
        HEFF_TRY(init_start(x0));
        HEFF_TRY(op_diagonal_ready(op));
        std::fill(Hk.begin(), Hk.end(), HT(0));
        HEFF_CUDA(cudaMemcpyAsync(t, V, sizeof(T) * n, cudaMemcpyDeviceToDevice, s));
        HEFF_TRY(append(0, true, false));
        int                 k = 1;
        std::vector<double> w;
        std::vector<HT>     vecs;
        while(true) {
            HEFF_TRY(ritz<CPLX>(k, Hk, maxb, w, vecs));
            for(double wi : w) anorm = std::max(anorm, std::fabs(wi));
            const std::vector<int> ord = ritz_order(w, cfg.ritz, cfg.target);
            theta                      = w[ord[0]];
            HEFF_TRY(explicit_residual(k, vecs.data() + (size_t)k * ord[0], theta, rnorm));
            res.iters++;
            if(!std::isfinite(rnorm)) {
                set_last_error_msg("eigensolver: non-finite residual");
                return HEFF_NAN_INPUT;
            }
            if(rnorm <= stop_tol * std::max(anorm, 1e-300)) {
                conv = true;
                break;
            }
            if(res.num_mv >= max_mv) break;
            HEFF_TRY(op_multpc(op, r, t, theta));
            if(k == maxb) {
                HEFF_TRY(restart(k, minb, w, vecs, ord, false));
                k = minb;
            }
            double n0 = 0, nrm = 0;
            HEFF_TRY(orthonormalize(V, k, n0, nrm));
            if(!(nrm > 1e-10 * n0)) {  // the preconditioned direction is already in the basis: use the residual
                HEFF_CUDA(cudaMemcpyAsync(t, r, sizeof(T) * n, cudaMemcpyDeviceToDevice, s));
                HEFF_TRY(orthonormalize(V, k, n0, nrm));
                if(!(nrm > 1e-10 * n0)) break;  // invariant subspace
            }
            HEFF_TRY(append(k, true, false));
            k++;
        }
        return HEFF_OK;
    }

    // CG on (I - u u^H)(H_mixed - theta)(I - u u^H) d = -r0 restricted to u^perp; d -> cg_d
    // The CG scalars stay on the device (cg_init / cg_step); the host only polls the stop flag every second
    // iteration, so at most one matvec runs past the stopping point.
    int correction(const T *u, const T *r0, double theta, double r0n) {
        HEFF_TRY(cg_init<CPLX>(cg_d, cg_r, cg_p, r0, n, cg_cs, r0n * r0n, theta, cfg.inner_tol * cfg.inner_tol, s));
        for(int it = 0; it < cfg.inner_iters; it++) {
            HEFF_TRY(apply(cg_p, cg_z, false));
            HEFF_TRY(cg_step<CPLX>(cg_z, cg_p, u, cg_q, cg_d, cg_r, n, cg_cs, partials, orth_counter, s));
            if((it & 1) == 1 && it + 1 < cfg.inner_iters) {
                HEFF_CUDA(cudaMemcpyAsync(&cg_done_, cg_cs + CG_DONE_SLOT, sizeof(double), cudaMemcpyDeviceToHost, s));
                HEFF_TRY(sync());
                if(cg_done_ != 0.0) break;
            }
        }
        return HEFF_OK;
    }
    double cg_done_ = 0.0;

    // Phase 2: Jacobi-Davidson in FP64 starting from x (normalised).
    int refine(double &theta, double &rnorm, bool &conv) {
        conv  = false;
        int k = 0;
        HEFF_CUDA(cudaMemcpyAsync(t, x, sizeof(T) * n, cudaMemcpyDeviceToDevice, s));
        std::fill(Hk.begin(), Hk.end(), HT(0));
        std::vector<double> w;
        std::vector<HT>     vecs;
        const int           kmax = std::min(maxb, 24);
        for(int outer = 0; outer < 60; outer++) {
            double n0 = 0, nrm = 0;
            HEFF_TRY(orthonormalize(V, k, n0, nrm));
            if(!(nrm > 1e-12 * n0) || !(nrm > 0)) break;  // correction lies in the space: nothing new
            HEFF_TRY(append(k, true, false));
            k++;
            HEFF_TRY(ritz<CPLX>(k, Hk, maxb, w, vecs));
            for(double wi : w) anorm = std::max(anorm, std::fabs(wi));
            const std::vector<int> ord = ritz_order(w, cfg.ritz, cfg.target);
            theta                      = w[ord[0]];
            HEFF_TRY(explicit_residual(k, vecs.data() + (size_t)k * ord[0], theta, rnorm));
            res.refine_steps++;
            if(rnorm <= cfg.tol * anorm) {
                conv = true;
                return HEFF_OK;
            }
            if(res.num_mv >= cfg.max_matvecs) return HEFF_OK;
            if(k == kmax) {
                HEFF_TRY(restart(k, 4, w, vecs, ord, false));
                k = 4;
            }
            HEFF_TRY(correction(x, r, theta, rnorm));
            HEFF_CUDA(cudaMemcpyAsync(t, cg_d, sizeof(T) * n, cudaMemcpyDeviceToDevice, s));
        }
        return HEFF_OK;
    }
};

template<class T>
__global__ void eig_pick_column_kernel(const T *__restrict__ evecs, int64_t n, int64_t col, T *__restrict__ x) {
    for(int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const T v = evecs[i + n * col];
        if constexpr(std::is_same<T, double2>::value)
            x[i] = make_double2(v.x, -v.y);  // get_matrix holds conj(H) for a Hermitian H: its eigenvectors are conjugated
        else
            x[i] = v;
    }
}

// Interior eigenpair (closest to cfg.target) of a small operator by the dense path: the reference switches to a
// dense eigensolver at problem sizes <= eig_max_size = 4096 (settings.h:249, AlgorithmFinite.cpp:318), and Krylov
// methods converge poorly to interior eigenvalues.  get_matrix + the device dense eigensolver, then the eigenvalue
// nearest the target and its eigenvector.
template<bool CPLX>
static int eigs_dense_target(heff_op *op, const heff_eig_config &cfg, void *x_out, heff_eig_result &res) {
    using T          = typename Scalar<CPLX>::T;
    auto          t0 = std::chrono::steady_clock::now();
    const int64_t n  = op->d.size_mps();
    const size_t  es = sizeof(T), nn = (size_t)n * n;
    const size_t  need = es * 2 * nn + sizeof(double) * n + 512;
    if(op->dense_bytes < need) {
        if(op->dense_ws) {
            HEFF_CUDA(cudaStreamSynchronize(op->stream));
            cudaFree(op->dense_ws);
            op->dense_ws    = nullptr;
            op->dense_bytes = 0;
        }
        cudaError_t e = cudaMalloc(&op->dense_ws, need);
        if(e != cudaSuccess) {
            set_last_cuda_error(e, "dense eigensolver buffers", __FILE__, __LINE__);
            return HEFF_OOM;
        }
        op->dense_bytes = need;
    }
    T      *M     = reinterpret_cast<T *>(op->dense_ws);
    T      *evecs = M + nn;
    double *evals = reinterpret_cast<double *>(evecs + nn);
    HEFF_TRY((int)heff_op_get_matrix(op, M));
    HEFF_TRY((int)heff_dense_eig(CPLX ? HEFF_C128 : HEFF_F64, n, M, n, evals, evecs, op->stream));
    std::vector<double> w(n);
    HEFF_CUDA(cudaMemcpyAsync(w.data(), evals, sizeof(double) * n, cudaMemcpyDeviceToHost, op->stream));
    HEFF_CUDA(cudaStreamSynchronize(op->stream));
    int64_t best = 0;
    for(int64_t i = 1; i < n; i++)
        if(std::fabs(w[i] - cfg.target) < std::fabs(w[best] - cfg.target)) best = i;
    if(x_out) {
        eig_pick_column_kernel<T><<<(int)std::min<int64_t>((n + 255) / 256, 1024), 256, 0, op->stream>>>(evecs, n, best, reinterpret_cast<T *>(x_out));
        HEFF_LAUNCH_CHECK();
    }
    HEFF_CUDA(cudaStreamSynchronize(op->stream));
    res.eigval    = w[best];
    res.resnorm   = 0.0;
    res.converged = 1;
    res.seconds   = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return HEFF_OK;
}

template<bool CPLX>
static int eigs_impl(heff_op *op, const heff_eig_config &cfg, const void *x0, void *x_out, heff_eig_result &res) {
    using T          = typename Scalar<CPLX>::T;
    if(cfg.ritz == HEFF_RITZ_TARGET && op->d.size_mps() <= 2048 && !op->sequential && op->W) return eigs_dense_target<CPLX>(op, cfg, x_out, res);
    auto       t0    = std::chrono::steady_clock::now();
    const bool mixed = cfg.mixed && op->precision == HEFF_PREC_MIXED && op->mixed_apply;
    Davidson<CPLX> D(op, cfg, res);
    HEFF_TRY(D.setup(mixed));
    double theta = 0, rnorm = INFINITY;
    bool   conv  = false;
    if(mixed) {
        const double mtol = cfg.mixed_tol > 0 ? cfg.mixed_tol : 1e-5;
        HEFF_TRY(D.run(x0, true, mtol, cfg.max_matvecs, theta, rnorm, conv));
        res.num_mv_phase1 = res.num_mv;
        if(std::fabs(theta) < 10.0 * mtol * std::max(D.anorm, 1e-300)) {
            // The eigenvalue sits within the split-BF16 operator's error (~4e-5 of its norm) of zero -- the folded
            // spectrum's (E_k - E_t)^2 near convergence: corrections solved on that operator cannot resolve it, so
            // the solve finishes in FP64 from the phase-1 vector (preconditioned when asked).
            if(cfg.precond == 1)
                HEFF_TRY(D.run_pc(D.x, cfg.tol, cfg.max_matvecs, theta, rnorm, conv));
            else
                HEFF_TRY(D.run(D.x, false, cfg.tol, cfg.max_matvecs, theta, rnorm, conv));
        } else {
            HEFF_TRY(D.refine(theta, rnorm, conv));
        }
    } else if(cfg.precond == 1) {
        HEFF_TRY(D.run_pc(x0, cfg.tol, cfg.max_matvecs, theta, rnorm, conv));
    } else {
        HEFF_TRY(D.run(x0, false, cfg.tol, cfg.max_matvecs, theta, rnorm, conv));
    }
    if(x_out) HEFF_CUDA(cudaMemcpyAsync(x_out, D.x, sizeof(T) * D.n, cudaMemcpyDeviceToDevice, D.s));
    HEFF_CUDA(cudaStreamSynchronize(D.s));
    res.eigval    = theta;
    res.resnorm   = rnorm;
    res.anorm     = D.anorm;
    res.converged = conv ? 1 : 0;
    res.seconds   = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return conv ? HEFF_OK : HEFF_NOT_CONVERGED;
}

size_t eig_workspace_bytes(int64_t n, int max_basis, bool mixed, bool cplx) {
    const int maxb = std::max(4, std::min(max_basis > 0 ? max_basis : 32, (int)MD_MAXK - 1));
    return cplx ? Davidson<true>::workspace_bytes(n, maxb, mixed) : Davidson<false>::workspace_bytes(n, maxb, mixed);
}

// Pre-sizes the operator's eigensolver workspace for problems up to n_max elements (so that solves on a
// rebound operator never allocate).
int eig_reserve(heff_op *op, int64_t n_max, int max_basis, bool mixed) {
    if(!op) return HEFF_BAD_ARG;
    HEFF_TRY(eig_host_ready(op));
    const int    maxb = std::max(4, std::min(max_basis > 0 ? max_basis : 32, (int)MD_MAXK - 1));
    const size_t need = op->cplx ? Davidson<true>::workspace_bytes(n_max, maxb, mixed) : Davidson<false>::workspace_bytes(n_max, maxb, mixed);
    if(op->eig_ws_bytes >= need) return HEFF_OK;
    if(op->eig_ws) {
        HEFF_CUDA(cudaStreamSynchronize(op->stream));
        cudaFree(op->eig_ws);
        op->eig_ws       = nullptr;
        op->eig_ws_bytes = 0;
    }
    cudaError_t e = cudaMalloc(&op->eig_ws, need);
    if(e != cudaSuccess) {
        set_last_cuda_error(e, "eigensolver workspace", __FILE__, __LINE__);
        return HEFF_OOM;
    }
    op->eig_ws_bytes = need;
    return HEFF_OK;
}

int eigs(heff_op *op, const heff_eig_config *cfg_in, const void *x0, void *x_out, heff_eig_result *res) {
    if(!op || !res) return HEFF_BAD_ARG;
    heff_eig_config cfg;
    heff_eig_config_default(&cfg);
    if(cfg_in) cfg = *cfg_in;
    std::memset(res, 0, sizeof(*res));
    return op->cplx ? eigs_impl<true>(op, cfg, x0, x_out, *res) : eigs_impl<false>(op, cfg, x0, x_out, *res);
}

}  // namespace heff

extern "C" void heff_eig_config_default(heff_eig_config *cfg) {
    if(!cfg) return;
    std::memset(cfg, 0, sizeof(*cfg));
    cfg->ritz        = HEFF_RITZ_SA;
    cfg->target      = 0.0;
    cfg->tol         = 1e-12;  // solver.cpp:378 default tolerance
    cfg->max_basis   = 24;
    cfg->min_basis   = 8;
    cfg->max_matvecs = 20000;
    cfg->mixed       = 1;
    cfg->mixed_tol   = 1e-5;
    cfg->inner_iters = 30;
    cfg->inner_tol   = 1e-3;
    cfg->seed        = 0;
}

extern "C" int heff_eigs(heff_op *op, const heff_eig_config *cfg, const void *x0, void *x_out, heff_eig_result *res) {
    return heff::eigs(op, cfg, x0, x_out, res);
}
