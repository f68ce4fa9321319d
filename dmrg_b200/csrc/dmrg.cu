// Minimal two-site finite-DMRG sweep driver over the device hot path, for the random-field Ising chain
// H = -sum J sz_i sz_{i+1} - sum h_i sx_i (IsingRandomField, source/tensors/site/mpo/IsingRandomField.cpp:93-136),
// and the ensemble runner that overlaps many independent realisations on one GPU.
//
// The driver exists to run whole ground-state (fDMRG, fdmrg.cpp:282-360) calculations on the hot path
// and compare energies / entropies with exact answers; it is not a port of the reference's algorithm
// layer.  Per bond (i, i+1):
//   theta = M_i M_{i+1}                                    (merge, one DMMA GEMM + layout kernels)
//   (E, theta) = lowest eigenpair of H_eff                  (heff_op rebound to the bond + device Davidson)
//   theta -> U S V with the svd.cpp:257-280 rank rule        (device Jacobi SVD, schmidt_multisite)
//   right-moving: M_i = U, M_{i+1} = S V, L_{i+1} = build_block(L_i, M_i, W_i)
//   left-moving:  M_{i+1} = V, M_i = U S, R_i = build_block(R_{i+1}, M_{i+1}, W_{i+1})
// All device memory (MPS, environments, operator, eigensolver basis, SVD scratch) is allocated once per
// workspace and reused for every bond and every realisation, so a sweep step never allocates or
// synchronises the device -- realisations on different streams overlap.
#include <algorithm>
#include <array>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>

#include "dmrg.cuh"
#include "eig.cuh"
#include "env.cuh"
#include "matvec.cuh"
#include "op.cuh"
#include "runtime.cuh"
#include "svd.cuh"

namespace heff {

template<bool CPLX>
int expansion_term(int side, typename Scalar<CPLX>::T *P, const typename Scalar<CPLX>::T *B, const int64_t ed[3], const typename Scalar<CPLX>::T *M,
                   const int64_t md[3], const typename Scalar<CPLX>::T *W, const int64_t wd[4], double alpha, cudaStream_t s);  // expansion.cu

// The environment updates of a sweep run on the operator's stream between its matvecs, so they share the operator's
// tail-split scratch.
static int env_update_d(int side, double *out, const double *E, const int64_t ed[3], const double *M, const int64_t md[3], const double *W,
                        const int64_t wd[4], double *scratch, cudaStream_t s, void *split_ws, size_t split_bytes) {
    return env_update<false>(side, out, E, ed, M, md, W, wd, scratch, s, split_ws, split_bytes);
}

// splitmix64 -> uniform [0, 1): the generator shared with oracle/physics.py
static uint64_t splitmix(uint64_t &st) {
    st += 0x9E3779B97F4A7C15ull;
    uint64_t z = st;
    z          = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z          = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
static double uniform01(uint64_t &st) { return (double)(splitmix(st) >> 11) * (1.0 / 9007199254740992.0); }

// W[3,3,2,2] of IsingRandomField::get_mpo with edges (MpoSite.cpp:449-500) for site i of L
static void ising_site_mpo(std::vector<double> &W, int64_t wd[4], int i, int L, double J, double h, double eshift) {
    double full[36] = {0};
    auto   at       = [&](int m, int n, int s, int t) -> double & { return full[m + 3 * (n + 3 * (s + 2 * t))]; };
    const double id[2][2] = {{1, 0}, {0, 1}}, sx[2][2] = {{0, 1}, {1, 0}}, sz[2][2] = {{1, 0}, {0, -1}};
    for(int s = 0; s < 2; s++)
        for(int t = 0; t < 2; t++) {
            at(0, 0, s, t) = id[s][t];
            at(1, 0, s, t) = sz[s][t];
            at(2, 0, s, t) = -h * sx[s][t] - eshift * id[s][t];
            at(2, 1, s, t) = -J * sz[s][t];
            at(2, 2, s, t) = id[s][t];
        }
    const int m0 = (i == 0) ? 2 : 0, m1 = 3;       // left edge keeps row 2
    const int n0 = 0, n1 = (i == L - 1) ? 1 : 3;   // right edge keeps column 0
    wd[0] = m1 - m0;
    wd[1] = n1 - n0;
    wd[2] = wd[3] = 2;
    W.assign((size_t)(wd[0] * wd[1] * 4), 0.0);
    for(int t = 0; t < 2; t++)
        for(int s = 0; s < 2; s++)
            for(int n = n0; n < n1; n++)
                for(int m = m0; m < m1; m++) W[(m - m0) + wd[0] * ((n - n0) + wd[1] * (s + 2 * t))] = at(m, n, s, t);
}

// Uncompressed square of the energy-shifted site MPO (MpoSite.cpp:57-70, real):
//   W2[(m + 3 m~), (n + 3 n~), s, s''] = sum_s' W[m,n,s,s'] W[m~,n~,s',s'']
// with the MPO^2 edges (MpoSite.cpp:609-640): the left edge keeps row 8 = (2, 2), the right edge column 0.
static void ising_site_mpo2(std::vector<double> &W2, int64_t wd[4], int i, int L, double J, double h, double eshift) {
    std::vector<double> W;
    int64_t             w1[4];
    ising_site_mpo(W, w1, 1, 3, J, h, eshift);  // bulk site: full 3x3
    double full[81 * 4];
    for(int t = 0; t < 2; t++)
        for(int s = 0; s < 2; s++)
            for(int nt = 0; nt < 3; nt++)
                for(int n = 0; n < 3; n++)
                    for(int mt = 0; mt < 3; mt++)
                        for(int m = 0; m < 3; m++) {
                            double acc = 0;
                            for(int p = 0; p < 2; p++) acc += W[m + 3 * (n + 3 * (s + 2 * p))] * W[mt + 3 * (nt + 3 * (p + 2 * t))];
                            full[(m + 3 * mt) + 9 * ((n + 3 * nt) + 9 * (s + 2 * t))] = acc;
                        }
    const int m0 = (i == 0) ? 8 : 0, m1 = 9, n0 = 0, n1 = (i == L - 1) ? 1 : 9;
    wd[0] = m1 - m0;
    wd[1] = n1 - n0;
    wd[2] = wd[3] = 2;
    W2.assign((size_t)(wd[0] * wd[1] * 4), 0.0);
    for(int t = 0; t < 2; t++)
        for(int s = 0; s < 2; s++)
            for(int n = n0; n < n1; n++)
                for(int m = m0; m < m1; m++) W2[(m - m0) + wd[0] * ((n - n0) + wd[1] * (s + 2 * t))] = full[m + 9 * (n + 9 * (s + 2 * t))];
}

// C[(s1 + d a) + d ca (s2 + d b)] -> theta[(s1 + d s2) + d^2 (a + ca b)]
__global__ void merge_layout_kernel(const double *__restrict__ C, double *__restrict__ th, int64_t d, int64_t ca, int64_t cb) {
    const int64_t tot = d * d * ca * cb;
    for(int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < tot; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t s = e % (d * d), r = e / (d * d), a = r % ca, b = r / ca;
        const int64_t s1 = s % d, s2 = s / d;
        th[e]            = C[(s1 + d * a) + d * ca * (s2 + d * b)];
    }
}
// M2p[c + cc (s2 + d b)] = M2[s2 + d (c + cc b)]
__global__ void perm_sc_kernel(const double *__restrict__ M, double *__restrict__ P, int64_t d, int64_t cc, int64_t cb) {
    const int64_t tot = d * cc * cb;
    for(int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < tot; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t c = e % cc, r = e / cc, s2 = r % d, b = r / d;
        P[e]            = M[s2 + d * (c + cc * b)];
    }
}
// X[s, a, k] *= S[k] (which = 0) or X[s, k, b] *= S[k] (which = 1)
__global__ void scale_bond_kernel(double *__restrict__ X, const double *__restrict__ S, int64_t d, int64_t n1, int64_t n2, int which) {
    const int64_t tot = d * n1 * n2;
    for(int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < tot; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = e / d, i1 = r % n1, i2 = r / n1;
        X[e] *= S[which == 0 ? i2 : i1];
    }
}

// Warm-up schedule of both drivers: the first sweeps use the reduced bond limit and the loose eigensolver tolerance
static int warmup_sweeps(const heff_dmrg_config &cfg) {
    if(cfg.warmup_sweeps >= 0) return cfg.warmup_sweeps;
    return (cfg.algorithm == 1 || cfg.algorithm == 3) ? 2 : 0;
}
static int64_t sweep_bond_limit(const heff_dmrg_config &cfg, int sweep) {
    if(sweep >= warmup_sweeps(cfg)) return cfg.chi_max;
    return std::min<int64_t>(cfg.chi_max, cfg.bond_min > 0 ? cfg.bond_min : 8);
}
static double sweep_eig_tol(const heff_dmrg_config &cfg, int sweep) {
    const double tol = cfg.eig_tol > 0 ? cfg.eig_tol : 1e-12;
    return sweep >= warmup_sweeps(cfg) ? tol : std::max(1e-8, tol);
}

static int g1(int64_t n) {
    int64_t g = (n + 255) / 256, cap = (int64_t)device_sm_count() * 8;
    return (int)(g < 1 ? 1 : (g < cap ? g : cap));
}

// Device memory of one DMRG run, sized for chains up to Lcap sites and bonds up to chicap.
struct DmrgWorkspace {
    std::vector<void *>   ptrs;
    int                   Lcap   = 0;
    int64_t               chicap = 0, Dcap = 3;
    cudaStream_t          s      = nullptr;
    std::vector<double *> M, Lenv, Renv, W;
    double *theta = nullptr, *Cbuf = nullptr, *P2 = nullptr, *U = nullptr, *S = nullptr, *V = nullptr, *scr = nullptr, *red = nullptr;
    heff_op *op = nullptr;
    // one-site DMRG with subspace expansion (algorithms 2 and 3): expansion term, enlarged-bond matrix and its
    // transpose, SVD factors and GEMM temporaries, each d (1 + Dmax) chi^2 elements, and the SVD scratch
    double *eP = nullptr, *eX = nullptr, *eT = nullptr, *eU = nullptr, *eV = nullptr, *eY = nullptr, *eZ = nullptr, *escr = nullptr;
    bool    onesite = false;
    int init_onesite() {
        if(onesite) return HEFF_OK;
        const int64_t d = 2, chi = chicap;
        const size_t  big = (size_t)(d * (1 + Dcap) * chi * chi) + 64;
        for(double **p : {&eP, &eX, &eT, &eU, &eV, &eY, &eZ}) HEFF_TRY(get(p, big));
        const int64_t m = (1 + Dcap) * chi, n = d * chi;
        HEFF_TRY(get(&escr, (size_t)(svd_scratch_bytes(m, n, 8) / 8) + 64));
        onesite = true;
        return HEFF_OK;
    }
    ~DmrgWorkspace() {
        if(op) heff_op_destroy(op);
        for(void *p : ptrs) cudaFree(p);
    }
    int get(double **p, size_t n) {
        cudaError_t e = cudaMalloc((void **)p, n * sizeof(double) + 256);
        if(e != cudaSuccess) {
            set_last_cuda_error(e, "dmrg buffers", __FILE__, __LINE__);
            return HEFF_OOM;
        }
        ptrs.push_back(*p);
        return HEFF_OK;
    }
    int init(int L, int64_t chi, heff_precision prec, cudaStream_t stream, int64_t Dmax = 3, int engine = HEFF_FP64_DMMA) {
        const int64_t d = 2;
        Lcap = L;
        chicap = chi;
        Dcap   = Dmax;
        s = stream;
        M.resize(L);
        W.resize(L);
        Lenv.resize(L + 1);
        Renv.resize(L + 1);
        const size_t msz = (size_t)(d * chi * chi), tsz = (size_t)(d * d * chi * chi);
        for(int i = 0; i < L; i++) {
            HEFF_TRY(get(&M[i], msz));
            HEFF_TRY(get(&W[i], 9 * 9 * 4));
        }
        for(int i = 0; i <= L; i++) {
            HEFF_TRY(get(&Lenv[i], (size_t)(chi * chi * Dmax)));
            HEFF_TRY(get(&Renv[i], (size_t)(chi * chi * Dmax)));
        }
        HEFF_TRY(get(&red, 4096));
        HEFF_TRY(get(&theta, tsz));
        HEFF_TRY(get(&Cbuf, tsz));
        HEFF_TRY(get(&P2, msz));
        HEFF_TRY(get(&U, tsz));
        HEFF_TRY(get(&S, (size_t)(2 * chi + 64)));
        HEFF_TRY(get(&V, tsz));
        const int64_t md_max[3] = {d, chi, chi}, wd_max[4] = {Dmax, Dmax, 2, 2};
        const size_t  scr_elems = std::max<size_t>((size_t)env_scratch_elems(md_max, wd_max), (size_t)schmidt_scratch_bytes(d, d, chi, chi, chi) / 8 + 64);
        HEFF_TRY(get(&scr, scr_elems));
        HEFF_TRY(op_create_capacity(&op, false, d * d, chi, Dmax, prec, stream));
        if(engine == HEFF_FP64_INT8) {
            op->fp64_engine = HEFF_FP64_INT8;
            HEFF_TRY(emu_reserve(op, d * d, chi, Dmax));  // digit planes for the largest bond, once
        }
        if(prec == HEFF_PREC_MIXED) HEFF_TRY(mixed_reserve(op, mixed_bytes(d * d, chi, chi, Dmax, Dmax, false)));  // split operands, once
        heff_eig_config ec;
        heff_eig_config_default(&ec);
        return eig_reserve(op, d * d * chi * chi, ec.max_basis, prec == HEFF_PREC_MIXED);
    }
};

static int dmrg_run_ws(const heff_dmrg_config &cfg, heff_dmrg_result &res, DmrgWorkspace &ws) {
    auto      t0 = std::chrono::steady_clock::now();
    const int L  = cfg.L;
    if(L < 2 || L > ws.Lcap || !cfg.h || cfg.chi_max < 1 || cfg.chi_max > ws.chicap) return HEFF_BAD_ARG;
    const bool folded = cfg.algorithm == 1;
    if(folded && ws.Dcap < 9) return HEFF_BAD_ARG;
    const int64_t d = 2;
    cudaStream_t  s = ws.s;
    std::memset(&res, 0, sizeof(res));
    ws.op->precision = (heff_precision)cfg.precision;
    if(cfg.fp64_engine != HEFF_FP64_DMMA && cfg.fp64_engine != HEFF_FP64_INT8) return HEFF_BAD_ARG;
    ws.op->fp64_engine = cfg.fp64_engine;
    HEFF_TRY(heff_op_set_jacobi_blocksize(ws.op, cfg.jcb_blocksize > 0 ? cfg.jcb_blocksize : (folded ? 128 : 1)));
    // --- model (host copies stay alive until the stream has consumed them): H, or (H - E_t)^2 for xDMRG
    std::vector<std::vector<double>>    Wh(L);
    std::vector<std::array<int64_t, 4>> wd(L);
    for(int i = 0; i < L; i++) {
        int64_t dd[4];
        if(folded)
            ising_site_mpo2(Wh[i], dd, i, L, cfg.J, cfg.h[i], cfg.energy_shift_per_site);
        else
            ising_site_mpo(Wh[i], dd, i, L, cfg.J, cfg.h[i], cfg.energy_shift_per_site);
        for(int k = 0; k < 4; k++) wd[i][k] = dd[k];
        HEFF_CUDA(cudaMemcpyAsync(ws.W[i], Wh[i].data(), Wh[i].size() * sizeof(double), cudaMemcpyHostToDevice, s));
    }
    std::vector<int64_t> chi(L + 1, 1);
    // --- random product state (real, normalised per site), seed via splitmix64
    std::vector<double> init(2 * L);
    uint64_t            st = (uint64_t)cfg.seed * 0x2545F4914F6CDD1Dull + 17;
    for(int i = 0; i < L; i++) {
        double a = uniform01(st) - 0.5, b = uniform01(st) - 0.5, nn = std::sqrt(a * a + b * b);
        init[2 * i]     = a / nn;
        init[2 * i + 1] = b / nn;
        HEFF_CUDA(cudaMemcpyAsync(ws.M[i], init.data() + 2 * i, 2 * sizeof(double), cudaMemcpyHostToDevice, s));
    }
    const double one = 1.0;
    HEFF_CUDA(cudaMemcpyAsync(ws.Lenv[0], &one, sizeof(double), cudaMemcpyHostToDevice, s));
    HEFF_CUDA(cudaMemcpyAsync(ws.Renv[L - 1], &one, sizeof(double), cudaMemcpyHostToDevice, s));
    HEFF_CUDA(cudaStreamSynchronize(s));
    double t_env = 0.0, t_eig = 0.0, t_svd = 0.0;
    auto   now  = [] { return std::chrono::steady_clock::now(); };
    auto   secs = [](auto a, auto b) { return std::chrono::duration<double>(b - a).count(); };
    // R environments: Renv[i] = env of sites > i, dims [chi_{i+1}, chi_{i+1}, wd[i][1]]
    for(int i = L - 2; i >= 0; i--) {
        const int64_t ed[3] = {chi[i + 2], chi[i + 2], wd[i + 1][1]}, mdd[3] = {d, chi[i + 1], chi[i + 2]};
        HEFF_TRY(env_update_d(1, ws.Renv[i], ws.Renv[i + 1], ed, ws.M[i + 1], mdd, ws.W[i + 1], wd[i + 1].data(), ws.scr, s, ws.op->split_ws, ws.op->split_bytes));
    }
    heff_eig_config ecfg;
    heff_eig_config_default(&ecfg);
    ecfg.tol         = cfg.eig_tol > 0 ? cfg.eig_tol : 1e-12;
    ecfg.ritz        = cfg.ritz;
    ecfg.target      = cfg.target;
    ecfg.mixed       = cfg.precision == HEFF_PREC_MIXED;
    ecfg.precond     = cfg.precond >= 0 ? cfg.precond : (cfg.algorithm == 1 ? 1 : 0);  // H^2: Jacobi (optimize_folded_spectrum.cpp:303-304)
    ecfg.max_matvecs = cfg.eig_max_matvecs > 0 ? cfg.eig_max_matvecs : (folded ? 60000 : 4000);
    double energy    = 0;
    for(int sweep = 0; sweep < cfg.sweeps; sweep++) {
        const int64_t chi_lim = sweep_bond_limit(cfg, sweep);
        ecfg.tol              = sweep_eig_tol(cfg, sweep);
        for(int dir = 0; dir < 2; dir++) {
            for(int step = 0; step < L - 1; step++) {
                const int     i  = dir == 0 ? step : (L - 2 - step);
                const int64_t ca = chi[i], cc = chi[i + 1], cb = chi[i + 2];
                // theta = M_i M_{i+1}
                perm_sc_kernel<<<g1(d * cc * cb), 256, 0, s>>>(ws.M[i + 1], ws.P2, d, cc, cb);
                HEFF_LAUNCH_CHECK();
                GemmArgs g{};
                g.M = (int)(d * ca), g.N = (int)(d * cb), g.K = (int)cc, g.batch = 1;
                g.A = ws.M[i], g.lda = d * ca, g.B = ws.P2, g.ldb = cc, g.C = ws.Cbuf, g.ldc = d * ca;
                g.alpha = make_double2(1, 0), g.beta = make_double2(0, 0);
                HEFF_TRY(gemm_f64<false>(false, false, false, g, s));
                merge_layout_kernel<<<g1(d * d * ca * cb), 256, 0, s>>>(ws.Cbuf, ws.theta, d, ca, cb);
                HEFF_LAUNCH_CHECK();
                // eigensolve on the rebound operator
                auto          te0   = now();
                const void   *mp[2] = {Wh[i].data(), Wh[i + 1].data()};
                int64_t       mdims[8];
                for(int k = 0; k < 4; k++) {
                    mdims[k]     = wd[i][k];
                    mdims[4 + k] = wd[i + 1][k];
                }
                const int64_t ld[3] = {ca, ca, wd[i][0]}, rd[3] = {cb, cb, wd[i + 1][1]};
                HEFF_TRY(op_rebind(ws.op, 2, mp, mdims, ws.Lenv[i], ld, ws.Renv[i + 1], rd));
                heff_eig_result er;
                int             rc = eigs(ws.op, &ecfg, ws.theta, ws.theta, &er);
                if(rc != HEFF_OK && rc != HEFF_NOT_CONVERGED) return rc;
                res.num_mv += er.num_mv;
                res.num_mv_mixed += er.num_mv_mixed;
                if(!er.converged) res.unconverged_solves++;
                energy = er.eigval;
                t_eig += secs(te0, now());
                // split
                auto    ts0 = now();
                int64_t k   = 0;
                double  te  = 0;
                HEFF_TRY(schmidt_split(ws.theta, d, d, ca, cb, chi_lim, cfg.trunc_lim, ws.U, ws.S, ws.V, &k, &te, ws.scr, s));
                res.trunc_err_max = std::max(res.trunc_err_max, te);
                res.svd_sweeps_max = std::max(res.svd_sweeps_max, last_svd_sweeps());
                if(i + 1 == L / 2 && sweep == cfg.sweeps - 1) {
                    std::vector<double> hs(k);
                    HEFF_CUDA(cudaMemcpyAsync(hs.data(), ws.S, sizeof(double) * k, cudaMemcpyDeviceToHost, s));
                    HEFF_CUDA(cudaStreamSynchronize(s));
                    double ent = 0;
                    for(double v : hs)
                        if(v > 0) ent -= v * v * std::log(v * v);
                    res.entropy_mid = std::fabs(ent);
                    res.chi_mid     = k;
                }
                t_svd += secs(ts0, now());
                chi[i + 1] = k;
                auto tv0   = now();
                if(dir == 0) {
                    HEFF_CUDA(cudaMemcpyAsync(ws.M[i], ws.U, sizeof(double) * d * ca * k, cudaMemcpyDeviceToDevice, s));
                    scale_bond_kernel<<<g1(d * k * cb), 256, 0, s>>>(ws.V, ws.S, d, k, cb, 1);
                    HEFF_LAUNCH_CHECK();
                    HEFF_CUDA(cudaMemcpyAsync(ws.M[i + 1], ws.V, sizeof(double) * d * k * cb, cudaMemcpyDeviceToDevice, s));
                    const int64_t ed[3] = {ca, ca, wd[i][0]}, mdd[3] = {d, ca, k};
                    HEFF_TRY(env_update_d(0, ws.Lenv[i + 1], ws.Lenv[i], ed, ws.M[i], mdd, ws.W[i], wd[i].data(), ws.scr, s, ws.op->split_ws, ws.op->split_bytes));
                } else {
                    HEFF_CUDA(cudaMemcpyAsync(ws.M[i + 1], ws.V, sizeof(double) * d * k * cb, cudaMemcpyDeviceToDevice, s));
                    scale_bond_kernel<<<g1(d * ca * k), 256, 0, s>>>(ws.U, ws.S, d, ca, k, 0);
                    HEFF_LAUNCH_CHECK();
                    HEFF_CUDA(cudaMemcpyAsync(ws.M[i], ws.U, sizeof(double) * d * ca * k, cudaMemcpyDeviceToDevice, s));
                    const int64_t ed[3] = {cb, cb, wd[i + 1][1]}, mdd[3] = {d, k, cb};
                    HEFF_TRY(env_update_d(1, ws.Renv[i], ws.Renv[i + 1], ed, ws.M[i + 1], mdd, ws.W[i + 1], wd[i + 1].data(), ws.scr, s, ws.op->split_ws, ws.op->split_bytes));
                }
                t_env += secs(tv0, now());
            }
        }
        if(sweep < 64) res.energy_per_sweep[sweep] = energy;
        res.sweeps_done = sweep + 1;
    }
    if(folded) {
        // <H> at the final centre, bond (0, 1): right environments of the unshifted H (D = 3) built from the
        // converged MPS into the (now unused) left-environment storage, then one FP64 matvec and a dot.
        const double E_t = cfg.energy_shift_per_site * L;
        const double lam = energy;  // <(H - E_t)^2> of the last local eigensolve (normalised theta)
        std::vector<std::vector<double>>    W3h(L);
        std::vector<std::array<int64_t, 4>> w3(L);
        for(int i = 0; i < L; i++) {
            int64_t dd[4];
            ising_site_mpo(W3h[i], dd, i, L, cfg.J, cfg.h[i], 0.0);
            for(int k = 0; k < 4; k++) w3[i][k] = dd[k];
            HEFF_CUDA(cudaMemcpyAsync(ws.W[i], W3h[i].data(), W3h[i].size() * sizeof(double), cudaMemcpyHostToDevice, s));
        }
        HEFF_CUDA(cudaMemcpyAsync(ws.Lenv[L - 1], &one, sizeof(double), cudaMemcpyHostToDevice, s));
        for(int i = L - 2; i >= 1; i--) {
            const int64_t ed[3] = {chi[i + 2], chi[i + 2], w3[i + 1][1]}, mdd[3] = {d, chi[i + 1], chi[i + 2]};
            HEFF_TRY(env_update_d(1, ws.Lenv[i], ws.Lenv[i + 1], ed, ws.M[i + 1], mdd, ws.W[i + 1], w3[i + 1].data(), ws.scr, s, ws.op->split_ws, ws.op->split_bytes));
        }
        const int64_t ca = chi[0], cc = chi[1], cb = chi[2];
        perm_sc_kernel<<<g1(d * cc * cb), 256, 0, s>>>(ws.M[1], ws.P2, d, cc, cb);
        HEFF_LAUNCH_CHECK();
        GemmArgs g{};
        g.M = (int)(d * ca), g.N = (int)(d * cb), g.K = (int)cc, g.batch = 1;
        g.A = ws.M[0], g.lda = d * ca, g.B = ws.P2, g.ldb = cc, g.C = ws.Cbuf, g.ldc = d * ca;
        g.alpha = make_double2(1, 0), g.beta = make_double2(0, 0);
        HEFF_TRY(gemm_f64<false>(false, false, false, g, s));
        merge_layout_kernel<<<g1(d * d * ca * cb), 256, 0, s>>>(ws.Cbuf, ws.theta, d, ca, cb);
        HEFF_LAUNCH_CHECK();
        // Lenv[0] still holds the trivial left edge (1)
        const void   *mp[2] = {W3h[0].data(), W3h[1].data()};
        int64_t       mdims[8];
        for(int k = 0; k < 4; k++) {
            mdims[k]     = w3[0][k];
            mdims[4 + k] = w3[1][k];
        }
        const int64_t ld[3] = {ca, ca, w3[0][0]}, rd[3] = {cb, cb, w3[1][1]};
        HEFF_TRY(op_rebind(ws.op, 2, mp, mdims, ws.Lenv[0], ld, ws.Lenv[1], rd));
        ws.op->precision = HEFF_PREC_FP64;
        HEFF_TRY(op_apply(ws.op, ws.theta, ws.Cbuf));
        const int64_t n = d * d * ca * cb;
        double        hv[2];
        HEFF_TRY(dot_device<false>(ws.theta, ws.Cbuf, n, ws.red, ws.red + 8, s));
        HEFF_TRY(dot_device<false>(ws.theta, ws.theta, n, ws.red + 1, ws.red + 8, s));
        HEFF_CUDA(cudaMemcpyAsync(hv, ws.red, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
        HEFF_CUDA(cudaStreamSynchronize(s));
        const double Eh = hv[0] / hv[1];
        res.variance    = lam - (Eh - E_t) * (Eh - E_t);
        energy          = Eh;
    }
    HEFF_CUDA(cudaStreamSynchronize(s));
    res.energy  = energy;
    res.t_eig   = t_eig;
    res.t_svd   = t_svd;
    res.t_env   = t_env;
    res.seconds = secs(t0, now());
    return HEFF_OK;
}

// ---------------------------------------------------------------------------------------------------------------
// One-site DMRG with forward subspace expansion (algorithm 2: ground state of H; algorithm 3: lowest eigenpair of
// the energy-shifted (H - E_t)^2, the folded spectrum of xDMRG).  The reference's default single-site strategy
// (settings.h:225) with expand_environment_1site (tools/finite/env/env.cpp:1034-1262) before each local
// optimisation: moving right at site i, the next site B(i+1) is enriched with the expansion term of the
// operator being optimised, P = alpha * (env_R . B(i+1) . W(i+1)) (EnvBase::get_expansion_term), the rows
// [B(i+1); P] of the enlarged left bond are decomposed as U S V (rank <= min(d chi_i, d chi_{i+2}, chi_max),
// trunc_lim), B(i+1) <- V and the centre AC(i) <- [AC(i), 0] U S (merge_expansion_term_PR, case [AC, B]); the
// state is unchanged up to that truncation, but the optimisation of AC(i) now sees the enriched environment.
// Moving left mirrors it with [A(i-1), P_L] (merge_expansion_term_PL, case [A, AC]).  The R-side term is read
// by its index meaning [s', b', (a, m)]: heff_expansion_term_* reproduces the reference's bytes, whose final
// reshape to [spin, chiL*DL, chiR] reinterprets that order when chiR > 1.
// Mixing factor: the DMRG3S schedule (Hubig, McCulloch, Schollwoeck, Wolf, PRB 91, 155115 (2015)) in place of the
// reference's optimally mixed block (get_optimally_mixed_block_1site): alpha = expansion_alpha (default 1e-3)
// halved every sweep and switched off for the last two sweeps, so the final sweeps converge the fixed basis.
// ---------------------------------------------------------------------------------------------------------------

// X[a2 + c2 (s + d b)] (c2 = c (1 + DL)): rows a2 < c are B[s + d (a2 + c b)], rows c + (a + c m) the R-side
// expansion term P[s + d (b + cb (a + c m))]
__global__ void ex_rows_R_kernel(const double *__restrict__ B, const double *__restrict__ P, double *__restrict__ X, int64_t d, int64_t c, int64_t DL,
                                 int64_t cb) {
    const int64_t c2 = c * (1 + DL), tot = c2 * d * cb;
    for(int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < tot; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t a2 = e % c2, col = e / c2, s = col % d, b = col / d;
        X[e]             = a2 < c ? B[s + d * (a2 + c * b)] : P[s + d * (b + cb * (a2 - c))];
    }
}
// site tensor [s, a, b] -> its left-bond rows X[a + c (s + d b)]
__global__ void site_rows_kernel(const double *__restrict__ M, double *__restrict__ X, int64_t d, int64_t c, int64_t cb) {
    const int64_t tot = d * c * cb;
    for(int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < tot; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t a = e % c, col = e / c, s = col % d, b = col / d;
        X[e]            = M[s + d * (a + c * b)];
    }
}
// rows X[a + ldx (s + d b)] (a < c) -> site tensor M[s + d (a + c b)]
__global__ void rows_site_kernel(const double *__restrict__ X, int64_t ldx, double *__restrict__ M, int64_t d, int64_t c, int64_t cb) {
    const int64_t tot = d * c * cb;
    for(int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < tot; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t s = e % d, r = e / d, a = r % c, b = r / c;
        M[e]            = X[a + ldx * (s + d * b)];
    }
}
// which 0: X[r + ld k] *= S[k] (columns); which 1: X[k + ld j] *= S[k] (rows); rows x cols of X
__global__ void scale_mat_kernel(double *__restrict__ X, int64_t ld, int64_t rows, int64_t cols, const double *__restrict__ S, int which) {
    const int64_t tot = rows * cols;
    for(int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < tot; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = e % rows, c = e / rows;
        X[r + ld * c] *= S[which == 0 ? c : r];
    }
}
// Y[j + ldy i] = X[i + ldx j] for i < rows, j < cols
__global__ void transpose_kernel(const double *__restrict__ X, int64_t ldx, int64_t rows, int64_t cols, double *__restrict__ Y, int64_t ldy) {
    const int64_t tot = rows * cols;
    for(int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < tot; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = e % rows, j = e / rows;
        Y[j + ldy * i]  = X[i + ldx * j];
    }
}

// C (M x N, ldc) = A (M x K, lda) B (K x N, ldb), FP64 DMMA
static int gemm_nn(const double *A, int64_t lda, const double *B, int64_t ldb, double *C, int64_t ldc, int64_t M, int64_t N, int64_t K, cudaStream_t s) {
    GemmArgs g{};
    g.M = (int)M, g.N = (int)N, g.K = (int)K, g.batch = 1;
    g.A = A, g.lda = lda, g.B = B, g.ldb = ldb, g.C = C, g.ldc = ldc;
    g.alpha = make_double2(1, 0), g.beta = make_double2(0, 0);
    return gemm_f64<false>(false, false, false, g, s);
}

// A (m x n, lda) = U S VT with U m x k (ld m), VT k x n (ld k); the one-sided Jacobi always runs on the taller
// orientation (a wide matrix is transposed first and the factors swapped back).
static int svd_oriented(DmrgWorkspace &ws, const double *A, int64_t lda, int64_t m, int64_t n, int64_t rank_max, double trunc, double *U, double *S,
                        double *VT, int64_t *k, double *err, cudaStream_t s) {
    if(m >= n) return svd_truncated(A, lda, m, n, rank_max, trunc, U, S, VT, k, err, ws.escr, nullptr, s);
    transpose_kernel<<<g1(m * n), 256, 0, s>>>(A, lda, m, n, ws.eT, n);
    HEFF_LAUNCH_CHECK();
    HEFF_TRY(svd_truncated(ws.eT, n, n, m, rank_max, trunc, ws.eY, S, ws.eZ, k, err, ws.escr, nullptr, s));
    // A^T = U' S VT'  ->  A = VT'^T S U'^T
    transpose_kernel<<<g1(*k * m), 256, 0, s>>>(ws.eZ, *k, *k, m, U, m);
    HEFF_LAUNCH_CHECK();
    transpose_kernel<<<g1(n * *k), 256, 0, s>>>(ws.eY, n, n, *k, VT, *k);
    HEFF_LAUNCH_CHECK();
    return HEFF_OK;
}

// S <- S / ||S|| (the split keeps the state normalised, svd.h:172); returns ||S||^2 before and the values on the host
static int normalise_S(double *S, int64_t k, std::vector<double> &hs, cudaStream_t s) {
    hs.resize(k);
    HEFF_CUDA(cudaMemcpyAsync(hs.data(), S, sizeof(double) * k, cudaMemcpyDeviceToHost, s));
    HEFF_CUDA(cudaStreamSynchronize(s));
    double nrm = 0;
    for(double v : hs) nrm += v * v;
    nrm = std::sqrt(nrm);
    if(nrm > 0 && std::fabs(nrm - 1.0) > 0) {
        for(double &v : hs) v /= nrm;
        HEFF_CUDA(cudaMemcpyAsync(S, hs.data(), sizeof(double) * k, cudaMemcpyHostToDevice, s));
        HEFF_CUDA(cudaStreamSynchronize(s));  // hs is a host vector reused by the caller
    }
    return HEFF_OK;
}

static int dmrg1_run_ws(const heff_dmrg_config &cfg, heff_dmrg_result &res, DmrgWorkspace &ws) {
    auto      t0 = std::chrono::steady_clock::now();
    const int L  = cfg.L;
    if(L < 2 || L > ws.Lcap || !cfg.h || cfg.chi_max < 1 || cfg.chi_max > ws.chicap) return HEFF_BAD_ARG;
    const bool folded = cfg.algorithm == 3;
    if(folded && ws.Dcap < 9) return HEFF_BAD_ARG;
    HEFF_TRY(ws.init_onesite());
    const int64_t d = 2;
    cudaStream_t  s = ws.s;
    std::memset(&res, 0, sizeof(res));
    ws.op->precision = (heff_precision)cfg.precision;
    if(cfg.fp64_engine != HEFF_FP64_DMMA && cfg.fp64_engine != HEFF_FP64_INT8) return HEFF_BAD_ARG;
    ws.op->fp64_engine = cfg.fp64_engine;
    HEFF_TRY(heff_op_set_jacobi_blocksize(ws.op, cfg.jcb_blocksize > 0 ? cfg.jcb_blocksize : (folded ? 128 : 1)));
    std::vector<std::vector<double>>    Wh(L);
    std::vector<std::array<int64_t, 4>> wd(L);
    for(int i = 0; i < L; i++) {
        int64_t dd[4];
        if(folded)
            ising_site_mpo2(Wh[i], dd, i, L, cfg.J, cfg.h[i], cfg.energy_shift_per_site);
        else
            ising_site_mpo(Wh[i], dd, i, L, cfg.J, cfg.h[i], cfg.energy_shift_per_site);
        for(int k = 0; k < 4; k++) wd[i][k] = dd[k];
        HEFF_CUDA(cudaMemcpyAsync(ws.W[i], Wh[i].data(), Wh[i].size() * sizeof(double), cudaMemcpyHostToDevice, s));
    }
    std::vector<int64_t> chi(L + 1, 1);
    std::vector<double>  init(2 * L);
    uint64_t             st = (uint64_t)cfg.seed * 0x2545F4914F6CDD1Dull + 17;
    for(int i = 0; i < L; i++) {
        double a = uniform01(st) - 0.5, b = uniform01(st) - 0.5, nn = std::sqrt(a * a + b * b);
        init[2 * i]     = a / nn;
        init[2 * i + 1] = b / nn;
        HEFF_CUDA(cudaMemcpyAsync(ws.M[i], init.data() + 2 * i, 2 * sizeof(double), cudaMemcpyHostToDevice, s));
    }
    const double one = 1.0;
    HEFF_CUDA(cudaMemcpyAsync(ws.Lenv[0], &one, sizeof(double), cudaMemcpyHostToDevice, s));
    HEFF_CUDA(cudaMemcpyAsync(ws.Renv[L - 1], &one, sizeof(double), cudaMemcpyHostToDevice, s));
    HEFF_CUDA(cudaStreamSynchronize(s));
    void  *sw = ws.op->split_ws;
    size_t sb = ws.op->split_bytes;
    // Renv[i] = environment of the sites > i, dims [chi_{i+1}, chi_{i+1}, wd[i][1]]
    auto renv = [&](int i) {  // from Renv[i+1] and M[i+1]
        const int64_t ed[3] = {chi[i + 2], chi[i + 2], wd[i + 1][1]}, mdd[3] = {d, chi[i + 1], chi[i + 2]};
        return env_update_d(1, ws.Renv[i], ws.Renv[i + 1], ed, ws.M[i + 1], mdd, ws.W[i + 1], wd[i + 1].data(), ws.scr, s, sw, sb);
    };
    // Lenv[i] = environment of the sites < i, dims [chi_i, chi_i, wd[i][0]]
    auto lenv = [&](int i) {  // Lenv[i + 1] from Lenv[i] and M[i]
        const int64_t ed[3] = {chi[i], chi[i], wd[i][0]}, mdd[3] = {d, chi[i], chi[i + 1]};
        return env_update_d(0, ws.Lenv[i + 1], ws.Lenv[i], ed, ws.M[i], mdd, ws.W[i], wd[i].data(), ws.scr, s, sw, sb);
    };
    for(int i = L - 2; i >= 0; i--) HEFF_TRY(renv(i));
    heff_eig_config ecfg;
    heff_eig_config_default(&ecfg);
    ecfg.tol         = cfg.eig_tol > 0 ? cfg.eig_tol : 1e-12;
    ecfg.ritz        = cfg.ritz;
    ecfg.target      = cfg.target;
    ecfg.mixed       = cfg.precision == HEFF_PREC_MIXED;
    ecfg.precond     = cfg.precond >= 0 ? cfg.precond : (folded ? 1 : 0);
    ecfg.max_matvecs = cfg.eig_max_matvecs > 0 ? cfg.eig_max_matvecs : (folded ? 60000 : 4000);
    double              energy = 0, t_env = 0, t_eig = 0, t_svd = 0;
    auto                now  = [] { return std::chrono::steady_clock::now(); };
    auto                secs = [](auto a, auto b) { return std::chrono::duration<double>(b - a).count(); };
    std::vector<double> hs;
    const double        alpha0 = cfg.expansion_alpha > 0 ? cfg.expansion_alpha : 1e-3;
    auto optimise = [&](int i) -> int {
        auto          te0   = now();
        const void   *mp[1] = {Wh[i].data()};
        const int64_t ld[3] = {chi[i], chi[i], wd[i][0]}, rd[3] = {chi[i + 1], chi[i + 1], wd[i][1]};
        HEFF_TRY(op_rebind(ws.op, 1, mp, wd[i].data(), ws.Lenv[i], ld, ws.Renv[i], rd));
        heff_eig_result er;
        int             rc = eigs(ws.op, &ecfg, ws.M[i], ws.M[i], &er);
        if(rc != HEFF_OK && rc != HEFF_NOT_CONVERGED) return rc;
        res.num_mv += er.num_mv;
        res.num_mv_mixed += er.num_mv_mixed;
        if(!er.converged) res.unconverged_solves++;
        energy = er.eigval;
        t_eig += secs(te0, now());
        return HEFF_OK;
    };
    auto record_mid = [&](int bond, int sweep) {  // entanglement entropy at the middle bond, last sweep
        if(bond != L / 2 || sweep != cfg.sweeps - 1) return;
        double ent = 0;
        for(double v : hs)
            if(v > 0) ent -= v * v * std::log(v * v);
        res.entropy_mid = std::fabs(ent);
        res.chi_mid     = (int64_t)hs.size();
    };
    for(int sweep = 0; sweep < cfg.sweeps; sweep++) {
        const double  alpha   = (sweep + 2 < cfg.sweeps) ? alpha0 * std::ldexp(1.0, -sweep) : 0.0;
        const int64_t chi_lim = sweep_bond_limit(cfg, sweep);
        ecfg.tol              = sweep_eig_tol(cfg, sweep);
        // ---- left to right: sites 0 .. L-2, centre AC(i), B(i+1) enriched
        for(int i = 0; i + 1 < L; i++) {
            auto ts0 = now();
            if(alpha > 0) {
                const int64_t ca = chi[i], c = chi[i + 1], cb = chi[i + 2], DL = wd[i + 1][0];
                const int64_t ed[3] = {cb, cb, wd[i + 1][1]}, mdd[3] = {d, c, cb};
                HEFF_TRY(expansion_term<false>(1, ws.eP, ws.Renv[i + 1], ed, ws.M[i + 1], mdd, ws.W[i + 1], wd[i + 1].data(), alpha, s));
                const int64_t c2 = c * (1 + DL);
                ex_rows_R_kernel<<<g1(c2 * d * cb), 256, 0, s>>>(ws.M[i + 1], ws.eP, ws.eX, d, c, DL, cb);
                HEFF_LAUNCH_CHECK();
                const int64_t rmax = std::min(std::min(d * ca, d * cb), chi_lim);
                int64_t       k    = 0;
                double        te   = 0;
                HEFF_TRY(svd_oriented(ws, ws.eX, c2, c2, d * cb, rmax, cfg.trunc_lim, ws.eU, ws.S, ws.eV, &k, &te, s));
                // AC(i) <- AC(i) U[0:c, :] S ; B(i+1) <- V
                HEFF_TRY(gemm_nn(ws.M[i], d * ca, ws.eU, c2, ws.Cbuf, d * ca, d * ca, k, c, s));
                scale_mat_kernel<<<g1(d * ca * k), 256, 0, s>>>(ws.Cbuf, d * ca, d * ca, k, ws.S, 0);
                HEFF_LAUNCH_CHECK();
                HEFF_CUDA(cudaMemcpyAsync(ws.M[i], ws.Cbuf, sizeof(double) * d * ca * k, cudaMemcpyDeviceToDevice, s));
                rows_site_kernel<<<g1(d * k * cb), 256, 0, s>>>(ws.eV, k, ws.M[i + 1], d, k, cb);
                HEFF_LAUNCH_CHECK();
                chi[i + 1] = k;
                auto tv0   = now();
                HEFF_TRY(renv(i));
                t_env += secs(tv0, now());
            }
            t_svd += secs(ts0, now());
            HEFF_TRY(optimise(i));
            // split AC(i) = A(i) S V; AC(i+1) = S V B(i+1)
            auto          ts1 = now();
            const int64_t ca = chi[i], c = chi[i + 1], cb = chi[i + 2];
            int64_t       k  = 0;
            double        te = 0;
            HEFF_TRY(svd_oriented(ws, ws.M[i], d * ca, d * ca, c, chi_lim, cfg.trunc_lim, ws.eU, ws.S, ws.eV, &k, &te, s));
            HEFF_TRY(normalise_S(ws.S, k, hs, s));
            res.trunc_err_max = std::max(res.trunc_err_max, te);
            record_mid(i + 1, sweep);
            HEFF_CUDA(cudaMemcpyAsync(ws.M[i], ws.eU, sizeof(double) * d * ca * k, cudaMemcpyDeviceToDevice, s));
            scale_mat_kernel<<<g1(k * c), 256, 0, s>>>(ws.eV, k, k, c, ws.S, 1);
            HEFF_LAUNCH_CHECK();
            site_rows_kernel<<<g1(d * c * cb), 256, 0, s>>>(ws.M[i + 1], ws.eX, d, c, cb);
            HEFF_LAUNCH_CHECK();
            HEFF_TRY(gemm_nn(ws.eV, k, ws.eX, c, ws.eZ, k, k, d * cb, c, s));
            rows_site_kernel<<<g1(d * k * cb), 256, 0, s>>>(ws.eZ, k, ws.M[i + 1], d, k, cb);
            HEFF_LAUNCH_CHECK();
            chi[i + 1] = k;
            t_svd += secs(ts1, now());
            auto tv0 = now();
            HEFF_TRY(lenv(i));
            t_env += secs(tv0, now());
        }
        // ---- right to left: sites L-1 .. 1, centre AC(i), A(i-1) enriched
        for(int i = L - 1; i >= 1; i--) {
            auto ts0 = now();
            if(alpha > 0) {
                const int64_t ca = chi[i - 1], c = chi[i], cb = chi[i + 1], DR = wd[i - 1][1];
                const int64_t ed[3] = {ca, ca, wd[i - 1][0]}, mdd[3] = {d, ca, c};
                // [A(i-1), P_L] along the right bond: P_L's layout [s', a', (b, n)] continues A's columns
                HEFF_CUDA(cudaMemcpyAsync(ws.eX, ws.M[i - 1], sizeof(double) * d * ca * c, cudaMemcpyDeviceToDevice, s));
                HEFF_TRY(expansion_term<false>(0, ws.eX + d * ca * c, ws.Lenv[i - 1], ed, ws.M[i - 1], mdd, ws.W[i - 1], wd[i - 1].data(), alpha, s));
                const int64_t c2   = c * (1 + DR);
                const int64_t rmax = std::min(std::min(d * ca, d * cb), chi_lim);
                int64_t       k    = 0;
                double        te   = 0;
                HEFF_TRY(svd_oriented(ws, ws.eX, d * ca, d * ca, c2, rmax, cfg.trunc_lim, ws.eU, ws.S, ws.eV, &k, &te, s));
                // A(i-1) <- U ; AC(i) <- S V[:, 0:c] AC(i)
                HEFF_CUDA(cudaMemcpyAsync(ws.M[i - 1], ws.eU, sizeof(double) * d * ca * k, cudaMemcpyDeviceToDevice, s));
                scale_mat_kernel<<<g1(k * c), 256, 0, s>>>(ws.eV, k, k, c, ws.S, 1);
                HEFF_LAUNCH_CHECK();
                site_rows_kernel<<<g1(d * c * cb), 256, 0, s>>>(ws.M[i], ws.eP, d, c, cb);
                HEFF_LAUNCH_CHECK();
                HEFF_TRY(gemm_nn(ws.eV, k, ws.eP, c, ws.eZ, k, k, d * cb, c, s));
                rows_site_kernel<<<g1(d * k * cb), 256, 0, s>>>(ws.eZ, k, ws.M[i], d, k, cb);
                HEFF_LAUNCH_CHECK();
                chi[i] = k;
                auto tv0 = now();
                HEFF_TRY(lenv(i - 1));
                t_env += secs(tv0, now());
            }
            t_svd += secs(ts0, now());
            HEFF_TRY(optimise(i));
            // split AC(i) = U S B(i); AC(i-1) = A(i-1) U S
            auto          ts1 = now();
            const int64_t ca = chi[i - 1], c = chi[i], cb = chi[i + 1];
            site_rows_kernel<<<g1(d * c * cb), 256, 0, s>>>(ws.M[i], ws.eX, d, c, cb);
            HEFF_LAUNCH_CHECK();
            int64_t k  = 0;
            double  te = 0;
            HEFF_TRY(svd_oriented(ws, ws.eX, c, c, d * cb, chi_lim, cfg.trunc_lim, ws.eU, ws.S, ws.eV, &k, &te, s));
            HEFF_TRY(normalise_S(ws.S, k, hs, s));
            res.trunc_err_max = std::max(res.trunc_err_max, te);
            record_mid(i, sweep);
            rows_site_kernel<<<g1(d * k * cb), 256, 0, s>>>(ws.eV, k, ws.M[i], d, k, cb);
            HEFF_LAUNCH_CHECK();
            HEFF_TRY(gemm_nn(ws.M[i - 1], d * ca, ws.eU, c, ws.Cbuf, d * ca, d * ca, k, c, s));
            scale_mat_kernel<<<g1(d * ca * k), 256, 0, s>>>(ws.Cbuf, d * ca, d * ca, k, ws.S, 0);
            HEFF_LAUNCH_CHECK();
            HEFF_CUDA(cudaMemcpyAsync(ws.M[i - 1], ws.Cbuf, sizeof(double) * d * ca * k, cudaMemcpyDeviceToDevice, s));
            chi[i] = k;
            t_svd += secs(ts1, now());
            auto tv0 = now();
            HEFF_TRY(renv(i - 1));
            t_env += secs(tv0, now());
        }
        if(sweep < 64) res.energy_per_sweep[sweep] = energy;
        res.sweeps_done = sweep + 1;
    }
    if(res.chi_mid == 0) res.chi_mid = chi[L / 2];
    if(folded) {
        // <H> at the final centre AC(0): right environments of the unshifted H (D = 3) from the right-normalised
        // sites 1 .. L-1 into the (now unused) left-environment storage, Lenv[j + 1] = environment of the sites > j
        const double E_t = cfg.energy_shift_per_site * L;
        const double lam = energy;
        std::vector<std::vector<double>>    W3h(L);
        std::vector<std::array<int64_t, 4>> w3(L);
        for(int i = 0; i < L; i++) {
            int64_t dd[4];
            ising_site_mpo(W3h[i], dd, i, L, cfg.J, cfg.h[i], 0.0);
            for(int k = 0; k < 4; k++) w3[i][k] = dd[k];
            HEFF_CUDA(cudaMemcpyAsync(ws.W[i], W3h[i].data(), W3h[i].size() * sizeof(double), cudaMemcpyHostToDevice, s));
        }
        HEFF_CUDA(cudaMemcpyAsync(ws.Lenv[L], &one, sizeof(double), cudaMemcpyHostToDevice, s));
        for(int j = L - 2; j >= 0; j--) {
            const int64_t ed[3] = {chi[j + 2], chi[j + 2], w3[j + 1][1]}, mdd[3] = {d, chi[j + 1], chi[j + 2]};
            HEFF_TRY(env_update_d(1, ws.Lenv[j + 1], ws.Lenv[j + 2], ed, ws.M[j + 1], mdd, ws.W[j + 1], w3[j + 1].data(), ws.scr, s, sw, sb));
        }
        const void   *mp[1] = {W3h[0].data()};
        const int64_t ld[3] = {chi[0], chi[0], w3[0][0]}, rd[3] = {chi[1], chi[1], w3[0][1]};
        HEFF_TRY(op_rebind(ws.op, 1, mp, w3[0].data(), ws.Lenv[0], ld, ws.Lenv[1], rd));
        ws.op->precision = HEFF_PREC_FP64;
        HEFF_TRY(op_apply(ws.op, ws.M[0], ws.Cbuf));
        const int64_t n = d * chi[0] * chi[1];
        double        hv[2];
        HEFF_TRY(dot_device<false>(ws.M[0], ws.Cbuf, n, ws.red, ws.red + 8, s));
        HEFF_TRY(dot_device<false>(ws.M[0], ws.M[0], n, ws.red + 1, ws.red + 8, s));
        HEFF_CUDA(cudaMemcpyAsync(hv, ws.red, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
        HEFF_CUDA(cudaStreamSynchronize(s));
        const double Eh = hv[0] / hv[1];
        res.variance    = lam - (Eh - E_t) * (Eh - E_t);
        energy          = Eh;
    }
    HEFF_CUDA(cudaStreamSynchronize(s));
    res.energy  = energy;
    res.t_eig   = t_eig;
    res.t_svd   = t_svd;
    res.t_env   = t_env;
    res.seconds = secs(t0, now());
    return HEFF_OK;
}

static int dmrg_any_ws(const heff_dmrg_config &cfg, heff_dmrg_result &res, DmrgWorkspace &ws) {
    if(cfg.algorithm == 2 || cfg.algorithm == 3) return dmrg1_run_ws(cfg, res, ws);
    if(cfg.algorithm != 0 && cfg.algorithm != 1) return HEFF_BAD_ARG;
    return dmrg_run_ws(cfg, res, ws);
}

int dmrg_run(const heff_dmrg_config &cfg, heff_dmrg_result &res, cudaStream_t s) {
    if(cfg.L < 2 || cfg.L > 4096 || !cfg.h || cfg.chi_max < 1) return HEFF_BAD_ARG;
    DmrgWorkspace ws;
    const bool    folded = cfg.algorithm == 1 || cfg.algorithm == 3;
    HEFF_TRY(ws.init(cfg.L, cfg.chi_max, (heff_precision)cfg.precision, s, folded ? 9 : 3, cfg.fp64_engine));
    return dmrg_any_ws(cfg, res, ws);
}

// Estimated device time of one realisation, in units of one chi=32 two-site split (~0.75 ms): per bond and sweep, a
// local eigensolve (~30 launch-bound matvecs at small chi, about 1.8 units; folded spectra need about ten times the
// iterations) plus the Jacobi SVD of the (2 chi_b) x (2 chi_b) split, whose time grows as chi_b^2.2 over 32..256
// (64^2: 0.75 ms, 512^2: 23-72 ms).  The bond dimension at bond b of an L-site spin-1/2 chain is
// min(2^min(b, L-b), chi_max).  Only the ordering of realisations by this estimate matters.
static double realisation_cost(const heff_dmrg_config &c) {
    const bool   folded = c.algorithm == 1 || c.algorithm == 3;
    const double eig    = folded ? 18.0 : 1.8;
    double       t      = 0;
    for(int b = 1; b < c.L; b++) {
        const int    e   = std::min(b, c.L - b);
        const double chb = e >= 62 ? (double)c.chi_max : std::min<double>((double)(int64_t(1) << e), (double)std::max<int64_t>(c.chi_max, 1));
        t += eig + std::pow(chb / 32.0, 2.2);
    }
    return t * std::max(c.sweeps, 1);
}

// Many independent realisations: nthreads workers, each with its own stream and workspace (sized for the
// largest chain and bond dimension), take realisations from a shared counter, longest first by
// realisation_cost (a list schedule: the longest chains do not start last while the other workers idle; input
// order with HEFF_ENSEMBLE_ORDER=input, for measurements).  Results stay at their input index, and each
// realisation's result does not depend on the worker or the order.  Different streams overlap on the device;
// nthreads = 1 runs them one at a time.
int ensemble_run(const heff_dmrg_config *cfgs, int n, int nthreads, heff_dmrg_result *results, int *status, double *seconds) {
    int     Lmax   = 2;
    int64_t chimax = 1;
    for(int i = 0; i < n; i++) {
        Lmax   = std::max(Lmax, cfgs[i].L);
        chimax = std::max(chimax, cfgs[i].chi_max);
    }
    int dev = 0;
    HEFF_CUDA(cudaGetDevice(&dev));
    std::vector<int> order(n);
    for(int i = 0; i < n; i++) order[i] = i;
    static const bool input_order = [] {
        const char *e = getenv("HEFF_ENSEMBLE_ORDER");
        return e && std::strcmp(e, "input") == 0;
    }();
    if(!input_order) {
        std::vector<double> cost(n);
        for(int i = 0; i < n; i++) cost[i] = realisation_cost(cfgs[i]);
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cost[a] > cost[b]; });
    }
    std::atomic<int>         next{0};
    std::vector<int>         rcs(nthreads, HEFF_OK);
    std::vector<std::thread> pool;
    HEFF_CUDA(cudaDeviceSynchronize());
    // workspaces are built before the clock starts (one-time allocation)
    std::vector<cudaStream_t>                   streams(nthreads);
    std::vector<std::unique_ptr<DmrgWorkspace>> wss(nthreads);
    for(int t = 0; t < nthreads; t++) {
        HEFF_CUDA(cudaStreamCreateWithFlags(&streams[t], cudaStreamNonBlocking));
        wss[t] = std::make_unique<DmrgWorkspace>();
        int64_t Dmax   = 3;
        int     engine = HEFF_FP64_DMMA;
        for(int i = 0; i < n; i++) {
            if(cfgs[i].algorithm == 1 || cfgs[i].algorithm == 3) Dmax = 9;
            if(cfgs[i].fp64_engine == HEFF_FP64_INT8) engine = HEFF_FP64_INT8;
        }
        int rc = wss[t]->init(Lmax, chimax, (heff_precision)cfgs[0].precision, streams[t], Dmax, engine);
        if(rc != HEFF_OK) return rc;
    }
    auto t0 = std::chrono::steady_clock::now();
    for(int t = 0; t < nthreads; t++) {
        pool.emplace_back([&, t] {
            cudaSetDevice(dev);
            while(true) {
                const int k = next.fetch_add(1);
                if(k >= n) break;
                const int i = order[k];
                status[i]   = dmrg_any_ws(cfgs[i], results[i], *wss[t]);
            }
        });
    }
    for(auto &th : pool) th.join();
    if(seconds) *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    wss.clear();
    for(auto st : streams) cudaStreamDestroy(st);
    return HEFF_OK;
}

}  // namespace heff

extern "C" void heff_dmrg_config_default(heff_dmrg_config *cfg) {
    if(!cfg) return;
    std::memset(cfg, 0, sizeof(*cfg));
    cfg->L         = 16;
    cfg->J         = 1.0;
    cfg->chi_max   = 64;
    cfg->sweeps    = 10;
    cfg->trunc_lim = 1e-12;
    cfg->precond   = -1;
    cfg->eig_tol   = 1e-12;
    cfg->ritz      = HEFF_RITZ_SA;
    cfg->precision = HEFF_PREC_FP64;
    cfg->warmup_sweeps = -1;
}

extern "C" int heff_dmrg_run(const heff_dmrg_config *cfg, heff_dmrg_result *res, void *stream) {
    if(!cfg || !res) return HEFF_BAD_ARG;
    return heff::dmrg_run(*cfg, *res, (cudaStream_t)stream);
}

extern "C" int heff_ensemble_run(const heff_dmrg_config *cfgs, int n, int nthreads, heff_dmrg_result *results, int *status, double *seconds) {
    if(!cfgs || n <= 0 || nthreads < 1 || nthreads > 64 || !results || !status) return HEFF_BAD_ARG;
    return heff::ensemble_run(cfgs, n, nthreads, results, status, seconds);
}
