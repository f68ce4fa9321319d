// Device eigensolver for H_eff: thick-restart Davidson (no preconditioner, i.e. a restarted Krylov
// method) in FP64, driving the operator through the same apply path the reference's PRIMME/ARPACK
// callback uses (MatVecMPOS::MultAx, solver_primme.cpp:122-128).  Re-orthogonalisation is classical
// Gram-Schmidt applied twice (CGS2) in FP64; the Rayleigh-Ritz problem is solved on the host in FP64.
//
// Convergence (PRIMME-style, eps = tol, solver_primme.cpp:364): ||H x - theta x|| <= tol * ||H||_est,
// ||H||_est = largest |Ritz value| seen.  Ritz selection: smallest algebraic (ground state,
// optimize_energy.cpp:74-81), largest algebraic, or closest to a target (interior states).
//
// Mixed precision (op precision HEFF_PREC_MIXED, see mixed.cu): the Davidson phase runs on the
// split-BF16 matvec until ||r|| <= mixed_tol * ||H||_est; then FP64 refinement steps follow, each one
// FP64 matvec for the true residual r plus a correction (I - xx^H)(H - theta)(I - xx^H) d = -r solved
// with the mixed matvec by a few MINRES-like (CG on the projected operator) iterations, x <- x + d.
#include <chrono>
#include <complex>
#include <cstring>
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
    static double real(double v) { return v; }
};
template<>
struct HostScalar<true> {
    using T = std::complex<double>;
    static T      conj(T v) { return std::conj(v); }
    static double real(T v) { return v.real(); }
};

// Ritz decomposition of the k x k projected matrix; returns ascending eigenvalues and vectors (column-major).
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

// Order of Ritz values by the selection rule: indices into ascending w.
static std::vector<int> ritz_order(const std::vector<double> &w, int rule, double target) {
    std::vector<int> o(w.size());
    std::iota(o.begin(), o.end(), 0);
    if(rule == HEFF_RITZ_LA) std::reverse(o.begin(), o.end());
    if(rule == HEFF_RITZ_TARGET) std::stable_sort(o.begin(), o.end(), [&](int a, int b) { return std::fabs(w[a] - target) < std::fabs(w[b] - target); });
    return o;
}

template<bool CPLX>
struct Davidson {
    using T  = typename Scalar<CPLX>::T;
    using HT = typename HostScalar<CPLX>::T;
    heff_op                 *op;
    const heff_eig_config   &cfg;
    heff_eig_result         &res;
    cudaStream_t             s;
    int64_t                  n;
    int                      maxb, minb;
    T                       *V = nullptr, *AV = nullptr, *V2 = nullptr, *AV2 = nullptr, *t = nullptr, *x = nullptr, *ax = nullptr, *r = nullptr;
    T                       *dh = nullptr, *dc = nullptr;
    double                  *partials = nullptr, *dscal = nullptr;
    std::vector<HT>          Hk;
    std::vector<void *>      allocs;
    double                   anorm = 0.0;

    Davidson(heff_op *o, const heff_eig_config &c, heff_eig_result &r_) : op(o), cfg(c), res(r_), s(o->stream), n(o->d.size_mps()) {
        maxb = std::max(4, std::min(cfg.max_basis > 0 ? cfg.max_basis : 32, (int)MD_MAXK));
        minb = std::max(1, std::min(cfg.min_basis > 0 ? cfg.min_basis : 8, maxb - 2));
        if((int64_t)maxb > n) maxb = (int)std::max<int64_t>(1, n);
        if(minb >= maxb) minb = std::max(1, maxb - 1);
    }
    ~Davidson() {
        for(void *p : allocs) cudaFree(p);
    }
    int alloc(void **p, size_t bytes) {
        cudaError_t e = cudaMalloc(p, bytes);
        if(e != cudaSuccess) {
            set_last_cuda_error(e, "eigensolver workspace", __FILE__, __LINE__);
            return HEFF_OOM;
        }
        allocs.push_back(*p);
        return HEFF_OK;
    }
    int setup() {
        const size_t es = sizeof(T);
        HEFF_TRY(alloc((void **)&V, es * n * maxb));
        HEFF_TRY(alloc((void **)&AV, es * n * maxb));
        HEFF_TRY(alloc((void **)&V2, es * n * maxb));
        HEFF_TRY(alloc((void **)&AV2, es * n * maxb));
        HEFF_TRY(alloc((void **)&t, es * n));
        HEFF_TRY(alloc((void **)&x, es * n));
        HEFF_TRY(alloc((void **)&ax, es * n));
        HEFF_TRY(alloc((void **)&r, es * n));
        HEFF_TRY(alloc((void **)&dh, es * MD_MAXK * 2));
        HEFF_TRY(alloc((void **)&dc, es * MD_MAXK * MD_MAXK));
        HEFF_TRY(alloc((void **)&partials, sizeof(double) * MD_BLOCKS * MD_MAXK * 2));
        HEFF_TRY(alloc((void **)&dscal, sizeof(double) * 8));
        Hk.assign((size_t)maxb * maxb, HT(0));
        return HEFF_OK;
    }
    // ||v||^2 -> host (synchronises)
    int norm2(const T *v, double &out) {
        T d;
        HEFF_TRY(dot_device<CPLX>(v, v, n, reinterpret_cast<T *>(dscal), partials, s));
        HEFF_CUDA(cudaMemcpyAsync(&d, dscal, sizeof(T), cudaMemcpyDeviceToHost, s));
        HEFF_CUDA(cudaStreamSynchronize(s));
        if constexpr(CPLX)
            out = d.x;
        else
            out = d;
        return HEFF_OK;
    }
    int apply(const T *in, T *out, bool fp64) {
        const heff_precision keep = op->precision;
        if(fp64) op->precision = HEFF_PREC_FP64;
        int rc = op_apply(op, in, out);
        op->precision = keep;
        if(fp64 || keep == HEFF_PREC_FP64)
            res.num_mv_fp64++;
        else
            res.num_mv_mixed++;
        res.num_mv++;
        return rc;
    }
    // orthonormalise t against V[:, :k] (CGS2); returns the norm before normalisation (host)
    int orthonormalize(int k, double &nrm) {
        for(int pass = 0; pass < 2; pass++) {
            HEFF_TRY(multi_dot<CPLX>(V, n, n, k, t, dh, partials, s));
            HEFF_TRY(multi_axpy<CPLX>(V, n, n, k, dh, -1.0, t, s));
        }
        double n2 = 0;
        HEFF_TRY(norm2(t, n2));
        nrm = std::sqrt(n2);
        if(nrm > 0) {
            const double inv = 1.0 / nrm;
            HEFF_CUDA(cudaMemcpyAsync(dscal + 1, &inv, sizeof(double), cudaMemcpyHostToDevice, s));
            HEFF_TRY(scale_dev<CPLX>(t, n, dscal + 1, false, s));
            HEFF_CUDA(cudaStreamSynchronize(s));
        }
        return HEFF_OK;
    }
    int random_vector(T *v, uint64_t seed) {
        const int64_t nr = n * (CPLX ? 2 : 1);
        init_vec_kernel<<<(int)std::min<int64_t>((nr + 255) / 256, 4096), 256, 0, s>>>(reinterpret_cast<double *>(v), nr, seed);
        HEFF_LAUNCH_CHECK();
        return HEFF_OK;
    }

    // Davidson phase.  fp64_only forces FP64 matvecs.  stop_tol: relative residual target.
    int run(const void *x0, bool use_mixed, double stop_tol, int64_t max_mv, double &theta, double &rnorm, bool &conv) {
        int k = 0;
        if(x0)
            HEFF_CUDA(cudaMemcpyAsync(t, x0, sizeof(T) * n, cudaMemcpyDeviceToDevice, s));
        else
            HEFF_TRY(random_vector(t, 0x5eedULL + (uint64_t)cfg.seed));
        conv  = false;
        theta = 0;
        rnorm = INFINITY;
        std::vector<double> w;
        std::vector<HT>     vecs;
        int                 stagn = 0;
        double              best  = INFINITY;
        while(true) {
            double nrm = 0;
            HEFF_TRY(orthonormalize(k, nrm));
            if(!(nrm > 1e-14) || !std::isfinite(nrm)) {
                if(!std::isfinite(nrm)) {
                    set_last_error_msg("eigensolver: non-finite vector (NaN/Inf in the operator or start vector)");
                    return HEFF_NAN_INPUT;
                }
                // breakdown: the residual lies in the basis; continue with a fresh random direction
                HEFF_TRY(random_vector(t, 0xabcdefULL + (uint64_t)res.num_mv));
                HEFF_TRY(orthonormalize(k, nrm));
                if(!(nrm > 1e-14)) break;
            }
            HEFF_CUDA(cudaMemcpyAsync(V + (int64_t)k * n, t, sizeof(T) * n, cudaMemcpyDeviceToDevice, s));
            HEFF_TRY(apply(V + (int64_t)k * n, AV + (int64_t)k * n, !use_mixed));
            // new column of the projected matrix
            HEFF_TRY(multi_dot<CPLX>(V, n, n, k + 1, AV + (int64_t)k * n, dh, partials, s));
            std::vector<T> col(k + 1);
            HEFF_CUDA(cudaMemcpyAsync(col.data(), dh, sizeof(T) * (k + 1), cudaMemcpyDeviceToHost, s));
            HEFF_CUDA(cudaStreamSynchronize(s));
            for(int i = 0; i <= k; i++) {
                HT v;
                std::memcpy((void *)&v, (void *)&col[i], sizeof(T));
                Hk[i + (size_t)maxb * k] = v;
                Hk[k + (size_t)maxb * i] = HostScalar<CPLX>::conj(v);
            }
            k++;
            HEFF_TRY(ritz<CPLX>(k, Hk, maxb, w, vecs));
            for(double wi : w) anorm = std::max(anorm, std::fabs(wi));
            const std::vector<int> ord = ritz_order(w, cfg.ritz, cfg.target);
            const int              j0  = ord[0];
            theta                      = w[j0];
            // x = V s, ax = AV s, r = ax - theta x
            HEFF_CUDA(cudaMemcpyAsync(dc, (const void *)(vecs.data() + (size_t)k * j0), sizeof(T) * k, cudaMemcpyHostToDevice, s));
            HEFF_TRY(combine<CPLX>(V, n, n, k, dc, x, s));
            HEFF_TRY(combine<CPLX>(AV, n, n, k, dc, ax, s));
            HEFF_TRY(residual<CPLX>(ax, x, theta, r, n, s));
            double r2 = 0;
            HEFF_TRY(norm2(r, r2));
            rnorm = std::sqrt(r2);
            res.iters++;
            if(!std::isfinite(rnorm)) {
                set_last_error_msg("eigensolver: non-finite residual");
                return HEFF_NAN_INPUT;
            }
            if(rnorm <= stop_tol * std::max(anorm, 1e-300)) {
                conv = true;
                break;
            }
            // stagnation guard for the mixed phase (the inexact operator floors the residual)
            if(use_mixed) {
                if(rnorm < 0.9 * best) {
                    best  = rnorm;
                    stagn = 0;
                } else if(++stagn >= 12) {
                    break;
                }
            }
            if(res.num_mv >= max_mv) break;
            if(k == maxb) {
                // thick restart: keep the minb best Ritz vectors
                std::vector<HT> S((size_t)maxb * minb);
                for(int q = 0; q < minb; q++)
                    for(int i = 0; i < k; i++) S[i + (size_t)maxb * q] = vecs[i + (size_t)k * ord[q]];
                HEFF_CUDA(cudaMemcpyAsync(dc, (const void *)S.data(), sizeof(T) * maxb * minb, cudaMemcpyHostToDevice, s));
                GemmArgs g{};
                g.M = (int)n, g.N = minb, g.K = k, g.batch = 1;
                g.A = V, g.lda = n, g.B = dc, g.ldb = maxb, g.C = V2, g.ldc = n;
                g.alpha = make_double2(1, 0), g.beta = make_double2(0, 0);
                HEFF_TRY(gemm_f64<CPLX>(false, false, false, g, s));
                g.A = AV, g.C = AV2;
                HEFF_TRY(gemm_f64<CPLX>(false, false, false, g, s));
                std::swap(V, V2);
                std::swap(AV, AV2);
                std::fill(Hk.begin(), Hk.end(), HT(0));
                for(int q = 0; q < minb; q++) Hk[q + (size_t)maxb * q] = HT(w[ord[q]]);
                k = minb;
                res.restarts++;
                HEFF_CUDA(cudaStreamSynchronize(s));  // S must outlive the copy
            }
            HEFF_CUDA(cudaMemcpyAsync(t, r, sizeof(T) * n, cudaMemcpyDeviceToDevice, s));
        }
        return HEFF_OK;
    }

    // FP64 refinement of (x, theta): each step one FP64 matvec for the true residual and a correction
    // solved with the mixed operator by CG on (I - xx^H)(H - theta)(I - xx^H), restricted to x^perp.
    int refine(double &theta, double &rnorm, bool &conv) {
        T *p = V, *q = V + n, *z = V + 2 * n, *d = V + 3 * n, *rr = V + 4 * n;  // reuse the basis storage
        for(int outer = 0; outer < 12; outer++) {
            HEFF_TRY(apply(x, ax, true));
            // theta = <x, Hx> (x normalised), r = Hx - theta x
            T th;
            HEFF_TRY(dot_device<CPLX>(x, ax, n, reinterpret_cast<T *>(dscal), partials, s));
            HEFF_CUDA(cudaMemcpyAsync(&th, dscal, sizeof(T), cudaMemcpyDeviceToHost, s));
            HEFF_CUDA(cudaStreamSynchronize(s));
            if constexpr(CPLX)
                theta = th.x;
            else
                theta = th;
            HEFF_TRY(residual<CPLX>(ax, x, theta, r, n, s));
            double r2 = 0;
            HEFF_TRY(norm2(r, r2));
            rnorm = std::sqrt(r2);
            anorm = std::max(anorm, std::fabs(theta));
            res.refine_steps++;
            if(rnorm <= cfg.tol * anorm) {
                conv = true;
                return HEFF_OK;
            }
            if(res.num_mv >= cfg.max_matvecs) return HEFF_OK;
            // CG for A d = -r with A = P (H_mixed - theta) P, P = I - x x^H; d starts at 0
            HEFF_CUDA(cudaMemcpyAsync(rr, r, sizeof(T) * n, cudaMemcpyDeviceToDevice, s));
            const double  minus1 = -1.0;
            HEFF_CUDA(cudaMemcpyAsync(dscal + 2, &minus1, sizeof(double), cudaMemcpyHostToDevice, s));
            HEFF_TRY(scale_dev<CPLX>(rr, n, dscal + 2, false, s));  // rr = -r (residual of the linear system at d = 0)
            HEFF_CUDA(cudaMemsetAsync(d, 0, sizeof(T) * n, s));
            HEFF_CUDA(cudaMemcpyAsync(p, rr, sizeof(T) * n, cudaMemcpyDeviceToDevice, s));
            double rho = r2, rho0 = r2;
            for(int it = 0; it < cfg.inner_iters; it++) {
                // q = P (H - theta) P p   (p stays in x^perp)
                HEFF_TRY(apply(p, z, false));
                HEFF_TRY(residual<CPLX>(z, p, theta, q, n, s));
                HEFF_TRY(multi_dot<CPLX>(x, n, n, 1, q, dh, partials, s));
                HEFF_TRY(multi_axpy<CPLX>(x, n, n, 1, dh, -1.0, q, s));
                T pq;
                HEFF_TRY(dot_device<CPLX>(p, q, n, reinterpret_cast<T *>(dscal), partials, s));
                HEFF_CUDA(cudaMemcpyAsync(&pq, dscal, sizeof(T), cudaMemcpyDeviceToHost, s));
                HEFF_CUDA(cudaStreamSynchronize(s));
                double pqr;
                if constexpr(CPLX)
                    pqr = pq.x;
                else
                    pqr = pq;
                if(!(std::fabs(pqr) > 0)) break;
                const double alpha = rho / pqr;
                double       a2[2] = {alpha, -alpha};
                HEFF_CUDA(cudaMemcpyAsync(dscal + 3, a2, 2 * sizeof(double), cudaMemcpyHostToDevice, s));
                HEFF_TRY(axpy_dev(p, d, dscal + 3));   // d += alpha p
                HEFF_TRY(axpy_dev(q, rr, dscal + 4));  // rr -= alpha q
                double rho_new = 0;
                HEFF_TRY(norm2(rr, rho_new));
                if(rho_new <= cfg.inner_tol * cfg.inner_tol * rho0) break;
                const double beta = rho_new / rho;
                rho               = rho_new;
                // p = rr + beta p
                HEFF_CUDA(cudaMemcpyAsync(dscal + 5, &beta, sizeof(double), cudaMemcpyHostToDevice, s));
                HEFF_TRY(scale_dev<CPLX>(p, n, dscal + 5, false, s));
                const double one = 1.0;
                HEFF_CUDA(cudaMemcpyAsync(dscal + 6, &one, sizeof(double), cudaMemcpyHostToDevice, s));
                HEFF_TRY(axpy_dev(rr, p, dscal + 6));
                HEFF_CUDA(cudaStreamSynchronize(s));
            }
            // x <- (x + d) / ||x + d||
            const double one = 1.0;
            HEFF_CUDA(cudaMemcpyAsync(dscal + 6, &one, sizeof(double), cudaMemcpyHostToDevice, s));
            HEFF_TRY(axpy_dev(d, x, dscal + 6));
            double xn = 0;
            HEFF_TRY(norm2(x, xn));
            const double inv = 1.0 / std::sqrt(xn);
            HEFF_CUDA(cudaMemcpyAsync(dscal + 1, &inv, sizeof(double), cudaMemcpyHostToDevice, s));
            HEFF_TRY(scale_dev<CPLX>(x, n, dscal + 1, false, s));
            HEFF_CUDA(cudaStreamSynchronize(s));
        }
        return HEFF_OK;
    }
    // y += a * v  (a read on the device)
    int axpy_dev(const T *v, T *y, const double *a) {
        // multi_axpy with k = 1 and h = 1 scaled by alpha: y += alpha * v * h; use dh[0] = 1
        const T one_t = one_value();
        HEFF_CUDA(cudaMemcpyAsync(dh + MD_MAXK, &one_t, sizeof(T), cudaMemcpyHostToDevice, s));
        double ah = 0;
        HEFF_CUDA(cudaMemcpyAsync(&ah, a, sizeof(double), cudaMemcpyDeviceToHost, s));
        HEFF_CUDA(cudaStreamSynchronize(s));
        return multi_axpy<CPLX>(v, n, n, 1, dh + MD_MAXK, ah, y, s);
    }
    static T one_value() {
        if constexpr(CPLX)
            return make_double2(1.0, 0.0);
        else
            return 1.0;
    }
};

template<bool CPLX>
static int eigs_impl(heff_op *op, const heff_eig_config &cfg, const void *x0, void *x_out, heff_eig_result &res) {
    using T = typename Scalar<CPLX>::T;
    auto                t0 = std::chrono::steady_clock::now();
    Davidson<CPLX>      D(op, cfg, res);
    HEFF_TRY(D.setup());
    double theta = 0, rnorm = INFINITY;
    bool   conv  = false;
    const bool mixed = cfg.mixed && op->precision == HEFF_PREC_MIXED && op->mixed_apply;
    if(mixed) {
        HEFF_TRY(D.run(x0, true, cfg.mixed_tol > 0 ? cfg.mixed_tol : 1e-6, cfg.max_matvecs, theta, rnorm, conv));
        conv = false;
        res.num_mv_phase1 = res.num_mv;
        HEFF_TRY(D.refine(theta, rnorm, conv));
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
    cfg->max_basis   = 32;
    cfg->min_basis   = 8;
    cfg->max_matvecs = 20000;
    cfg->mixed       = 1;
    cfg->mixed_tol   = 1e-6;
    cfg->inner_iters = 40;
    cfg->inner_tol   = 1e-4;
    cfg->seed        = 0;
}

extern "C" int heff_eigs(heff_op *op, const heff_eig_config *cfg, const void *x0, void *x_out, heff_eig_result *res) {
    return heff::eigs(op, cfg, x0, x_out, res);
}
