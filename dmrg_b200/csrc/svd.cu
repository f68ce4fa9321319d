// Truncated SVD on the device: svd::solver::do_svd_ptr (source/math/svd/svd.cpp:113-206) with the rank
// rule get_rank_from_truncation_error (svd.cpp:257-280) and the two-site Schmidt split
// schmidt_multisite (source/math/svd.h:189-220).
//
// Algorithm: one-sided (Hestenes) block Jacobi in FP64.  The columns of the work matrix G (= A, m x n,
// column-major, n padded to a multiple of 32 with zero columns) are grouped into blocks of 16.  A sweep
// pairs every block with every other block once (round-robin tournament, B-1 rounds of B/2 disjoint
// pairs).  For one pair, a CTA
//   1. forms the 32 x 32 Gram matrix P^T P of the pair's 32 columns (streamed through shared memory),
//   2. diagonalises it with a cyclic two-sided Jacobi eigensolver in shared memory (16 disjoint
//      rotations per step), accumulating the orthogonal Q,
//   3. applies P <- P Q and V[:, pair] <- V[:, pair] Q.
// A pair whose Gram is already diagonal to |g_ij| <= tol*sqrt(g_ii g_jj) is skipped; the sweep loop
// stops when every pair was skipped.  The relative criterion, evaluated on freshly computed Gram
// entries, is what lets one-sided Jacobi resolve small singular values to high relative accuracy
// (Demmel & Veselic 1992), which the truncation rule at 1e-12 needs.  Then sigma_j = ||G_j||,
// U_j = G_j / sigma_j, sorted descending.
#include <algorithm>
#include <cmath>
#include <numeric>
#include <vector>

#include "matvec.cuh"
#include "runtime.cuh"
#include "svd.cuh"

namespace heff {

constexpr int JB     = 16;       // columns per block
constexpr int JP     = 2 * JB;   // columns per pair
constexpr int JROWS  = 64;       // rows per streamed tile
constexpr int JTHR   = 256;

// Pair k of round r in the circle-method tournament over B (even) players.
__host__ __device__ inline void rr_pair(int B, int r, int k, int &p, int &q) {
    if(k == 0) {
        p = B - 1;
        q = r;
    } else {
        p = (r + k) % (B - 1);
        q = (r - k + (B - 1)) % (B - 1);
    }
}

__device__ inline void atomic_max_pos(double *addr, double v) {
    // non-negative doubles order like their bit patterns
    atomicMax(reinterpret_cast<unsigned long long *>(addr), (unsigned long long)__double_as_longlong(v));
}

// One round of the block Jacobi sweep: blockIdx.x = pair index.
__global__ void __launch_bounds__(JTHR) jacobi_round_kernel(double *__restrict__ G, int64_t ldg, int m, double *__restrict__ V, int64_t ldv, int nv,
                                                           int B, int round, double tol, double *__restrict__ offmax, int *__restrict__ rotated) {
    __shared__ double sG[JP][JP + 1];
    __shared__ double sQ[JP][JP + 1];
    __shared__ double sT[JROWS][JP + 1];
    __shared__ double cs_c[JP / 2], cs_s[JP / 2];
    __shared__ int    s_idx[JP];
    __shared__ double s_red[JTHR];
    __shared__ int    s_rot[2];

    int p, q;
    rr_pair(B, round, blockIdx.x, p, q);
    const int tid = threadIdx.x;
    if(tid < JP) s_idx[tid] = (tid < JB) ? p * JB + tid : q * JB + (tid - JB);
    __syncthreads();

    // ---- 1. Gram matrix of the 32 columns: thread owns entries (i, j) = (tid / 8, 4*(tid % 8) + 0..3)
    const int gi = tid / 8, gj0 = 4 * (tid % 8);
    double    acc[4] = {0, 0, 0, 0};
    for(int r0 = 0; r0 < m; r0 += JROWS) {
        for(int e = tid; e < JROWS * JP; e += JTHR) {
            const int rr = e % JROWS, cc = e / JROWS, row = r0 + rr;
            sT[rr][cc]   = row < m ? G[row + ldg * (int64_t)s_idx[cc]] : 0.0;
        }
        __syncthreads();
        for(int rr = 0; rr < JROWS; rr++) {
            const double a = sT[rr][gi];
#pragma unroll
            for(int u = 0; u < 4; u++) acc[u] = fma(a, sT[rr][gj0 + u], acc[u]);
        }
        __syncthreads();
    }
#pragma unroll
    for(int u = 0; u < 4; u++) sG[gi][gj0 + u] = acc[u];
    __syncthreads();

    // ---- off-diagonal measure of the fresh Gram (relative to the diagonal)
    auto off_measure = [&]() -> double {
        double mx = 0;
        for(int e = tid; e < JP * JP; e += JTHR) {
            const int i = e / JP, j = e % JP;
            if(i < j) {
                const double d = sqrt(fabs(sG[i][i]) * fabs(sG[j][j]));
                const double o = fabs(sG[i][j]);
                if(o > 0) mx = fmax(mx, d > 0 ? o / d : 1.0);
            }
        }
        s_red[tid] = mx;
        __syncthreads();
        for(int w = JTHR / 2; w > 0; w >>= 1) {
            if(tid < w) s_red[tid] = fmax(s_red[tid], s_red[tid + w]);
            __syncthreads();
        }
        const double r = s_red[0];
        __syncthreads();
        return r;
    };
    const double off0 = off_measure();
    if(tid == 0) atomic_max_pos(offmax, off0);
    if(off0 <= tol) return;  // uniform across the CTA
    if(tid == 0) atomicAdd(rotated, 1);

    // ---- 2. cyclic Jacobi on sG, accumulating sQ.  Rotations are applied in Rutishauser's form
    //      x' = x - s (y + tau x), y' = y + s (x - tau y), tau = s / (1 + c), which keeps the rounding of c
    //      (c -> 1 for tiny angles) from inflating column norms; only numerically significant
    //      off-diagonals (|g_ab| > tol sqrt(g_aa g_bb)) are rotated, at most 8 sweeps (the outer sweep
    //      re-checks every pair on a freshly computed Gram matrix).
    for(int e = tid; e < JP * JP; e += JTHR) sQ[e / JP][e % JP] = (e / JP == e % JP) ? 1.0 : 0.0;
    if(tid < 2) s_rot[tid] = 0;
    __syncthreads();
    for(int sweep = 0; sweep < 8; sweep++) {
        const int par = sweep & 1;
        for(int step = 0; step < JP - 1; step++) {
            if(tid < JP / 2) {
                int a, b;
                rr_pair(JP, step, tid, a, b);
                const double app = sG[a][a], aqq = sG[b][b], apq = sG[a][b];
                double       sn = 0.0, tau = 0.0;
                if(fabs(apq) > 1e-300 && fabs(apq) > tol * sqrt(fabs(app) * fabs(aqq))) {
                    const double th = (aqq - app) / (2.0 * apq);
                    const double t  = (th >= 0 ? 1.0 : -1.0) / (fabs(th) + sqrt(1.0 + th * th));
                    const double c  = 1.0 / sqrt(1.0 + t * t);
                    sn              = t * c;
                    tau             = sn / (1.0 + c);
                    s_rot[par]      = 1;
                }
                cs_c[tid] = tau;
                cs_s[tid] = sn;
            }
            __syncthreads();
            // columns of G and Q: col_a' = c col_a - s col_b ; col_b' = s col_a + c col_b
            for(int e = tid; e < (JP / 2) * JP; e += JTHR) {
                const int k = e / JP, row = e % JP;
                int       a, b;
                rr_pair(JP, step, k, a, b);
                const double tau = cs_c[k], sn = cs_s[k];
                if(sn != 0.0) {
                    const double ga = sG[row][a], gb = sG[row][b];
                    sG[row][a]      = ga - sn * (gb + tau * ga);
                    sG[row][b]      = gb + sn * (ga - tau * gb);
                    const double qa = sQ[row][a], qb = sQ[row][b];
                    sQ[row][a]      = qa - sn * (qb + tau * qa);
                    sQ[row][b]      = qb + sn * (qa - tau * qb);
                }
            }
            __syncthreads();
            // rows of G
            for(int e = tid; e < (JP / 2) * JP; e += JTHR) {
                const int k = e / JP, col = e % JP;
                int       a, b;
                rr_pair(JP, step, k, a, b);
                const double tau = cs_c[k], sn = cs_s[k];
                if(sn != 0.0) {
                    const double ga = sG[a][col], gb = sG[b][col];
                    sG[a][col]      = ga - sn * (gb + tau * ga);
                    sG[b][col]      = gb + sn * (ga - tau * gb);
                }
            }
            __syncthreads();
        }
        const int rotated_this_sweep = s_rot[par];
        __syncthreads();
        if(tid == 0) s_rot[par] = 0;  // reused two sweeps later; read above before this reset
        if(!rotated_this_sweep) break;
    }

    // ---- 3. apply Q to the pair's columns of G (m rows) and V (nv rows)
    for(int pass = 0; pass < 2; pass++) {
        double       *X    = pass == 0 ? G : V;
        const int64_t ldx  = pass == 0 ? ldg : ldv;
        const int     rows = pass == 0 ? m : nv;
        for(int r0 = 0; r0 < rows; r0 += JROWS) {
            for(int e = tid; e < JROWS * JP; e += JTHR) {
                const int rr = e % JROWS, cc = e / JROWS, row = r0 + rr;
                sT[rr][cc]   = row < rows ? X[row + ldx * (int64_t)s_idx[cc]] : 0.0;
            }
            __syncthreads();
            for(int e = tid; e < JROWS * JP; e += JTHR) {
                const int rr = e % JROWS, cc = e / JROWS, row = r0 + rr;
                if(row < rows) {
                    double v = 0;
#pragma unroll 8
                    for(int k = 0; k < JP; k++) v = fma(sT[rr][k], sQ[k][cc], v);
                    X[row + ldx * (int64_t)s_idx[cc]] = v;
                }
            }
            __syncthreads();
        }
    }
}

// sigma_j = ||G_j||_2 (column norms), one warp per column.
__global__ void col_norms_kernel(const double *__restrict__ G, int64_t ldg, int m, int n, double *__restrict__ sig) {
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) / 32, lane = threadIdx.x & 31;
    if(w >= n) return;
    double acc = 0;
    for(int i = lane; i < m; i += 32) {
        const double v = G[i + ldg * (int64_t)w];
        acc            = fma(v, v, acc);
    }
    for(int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if(lane == 0) sig[w] = sqrt(acc);
}

// U[:, i] = G[:, perm[i]] / sigma[perm[i]],  VT[i, :] = V[:, perm[i]]^T  (i < k)
__global__ void svd_gather_kernel(const double *__restrict__ G, int64_t ldg, int m, const double *__restrict__ V, int64_t ldv, int n,
                                  const int *__restrict__ perm, const double *__restrict__ sig, int k, double *__restrict__ U, double *__restrict__ VT) {
    const int64_t tot_u = (int64_t)m * k, tot_v = (int64_t)n * k;
    for(int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < tot_u + tot_v; e += (int64_t)gridDim.x * blockDim.x) {
        if(e < tot_u) {
            const int64_t i = e / m, r = e % m;
            const int     j = perm[i];
            const double  s = sig[j];
            U[r + (int64_t)m * i] = s > 0 ? G[r + ldg * (int64_t)j] / s : 0.0;
        } else {
            const int64_t f = e - tot_u, c = f / k, i = f % k;  // VT is k x n column-major
            VT[i + (int64_t)k * c] = V[c + ldv * (int64_t)perm[i]];
        }
    }
}

__global__ void copy_pad_kernel(const double *__restrict__ A, int64_t lda, int m, int n, double *__restrict__ G, int64_t ldg, int npad) {
    const int64_t tot = (int64_t)ldg * npad;
    for(int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < tot; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = e % ldg, c = e / ldg;
        G[e]            = (r < m && c < n) ? A[r + lda * c] : 0.0;
    }
}

__global__ void eye_kernel(double *__restrict__ V, int64_t ldv, int npad) {
    const int64_t tot = (int64_t)ldv * npad;
    for(int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < tot; e += (int64_t)gridDim.x * blockDim.x)
        V[e] = (e % ldv == e / ldv) ? 1.0 : 0.0;
}

static int g1(int64_t n) {
    int64_t g = (n + 255) / 256, cap = (int64_t)device_sm_count() * 8;
    return (int)(g < 1 ? 1 : (g < cap ? g : cap));
}

int64_t svd_scratch_bytes(int64_t m, int64_t n) {
    const int64_t npad = (n + JP - 1) / JP * JP;
    const int64_t ldg  = (m + 1) / 2 * 2;
    return 8 * (ldg * npad + npad * npad + npad + 64) + 4 * npad + 256;
}

// Rank rule of svd.cpp:257-280 on descending sigma (only exactly-nonzero values count, like
// svd_lapacke.cpp:453 S.nonZeros()).  Returns rank (>0) or -1 (the reference throws there).
int64_t truncation_rank(const double *S, int64_t n, int64_t rank_max, int64_t rank_min, double lim, double *trunc_err) {
    int64_t nz = 0;
    for(int64_t i = 0; i < n; i++) nz += S[i] != 0.0;
    std::vector<double> err(nz + 1, 0.0);
    double              acc = 0;
    for(int64_t s = nz; s >= 0; s--) {
        if(s < nz) acc += S[s] * S[s];
        err[s] = std::sqrt(acc);
    }
    int64_t rank = 0;
    for(int64_t s = 0; s <= nz; s++) rank += err[s] >= lim;
    int64_t rank_lim = nz;
    if(rank_max > 0) rank_lim = std::min(nz, rank_max);
    rank = std::min(rank, rank_lim);
    if(rank_min > 0) rank = std::max(rank, std::min(nz, rank_min));
    if(rank <= 0) return -1;
    if(trunc_err) *trunc_err = err[rank];
    return rank;
}

// Full SVD driver.  A: m x n (lda), not modified.  Outputs (device): U (m x kmax), S (kmax), VT (kmax x n)
// with kmax = min(m, n, rank_max>0 ? rank_max : inf); *rank and *trunc_err on the host.
int svd_truncated(const double *A, int64_t lda, int64_t m, int64_t n, int64_t rank_max, double trunc_lim, double *U, double *S, double *VT,
                  int64_t *rank, double *trunc_err, void *scratch, int *sweeps_out, cudaStream_t s) {
    if(m <= 0 || n <= 0 || m > (1 << 24) || n > 16384) return HEFF_BAD_SHAPE;
    const int     npad = (int)((n + JP - 1) / JP * JP);
    const int64_t ldg  = (m + 1) / 2 * 2;
    double       *G    = reinterpret_cast<double *>(scratch);
    double       *V    = G + ldg * npad;
    double       *sig  = V + (int64_t)npad * npad;
    double       *dmax = sig + npad;                     // [0] offmax, [1..] spare
    int          *drot = reinterpret_cast<int *>(dmax + 8);
    int          *perm = reinterpret_cast<int *>(dmax + 64);
    copy_pad_kernel<<<g1(ldg * npad), 256, 0, s>>>(A, lda, (int)m, (int)n, G, ldg, npad);
    HEFF_LAUNCH_CHECK();
    eye_kernel<<<g1((int64_t)npad * npad), 256, 0, s>>>(V, npad, npad);
    HEFF_LAUNCH_CHECK();
    const int    B   = npad / JB;  // even
    // off-diagonal tolerance just above the rounding noise of a length-m dot product
    const double tol = std::max(1e-14, 8.0 * 2.2e-16 * std::sqrt((double)m));
    int          sweep = 0;
    for(; sweep < 40; sweep++) {
        HEFF_CUDA(cudaMemsetAsync(dmax, 0, 8 * 8 + sizeof(int), s));
        for(int r = 0; r < B - 1; r++) {
            jacobi_round_kernel<<<B / 2, JTHR, 0, s>>>(G, ldg, (int)m, V, npad, npad, B, r, tol, dmax, drot);
            HEFF_LAUNCH_CHECK();
        }
        int rot = 0;
        HEFF_CUDA(cudaMemcpyAsync(&rot, drot, sizeof(int), cudaMemcpyDeviceToHost, s));
        HEFF_CUDA(cudaStreamSynchronize(s));
        if(rot == 0) break;
    }
    if(sweeps_out) *sweeps_out = sweep + 1;
    col_norms_kernel<<<(npad * 32 + 255) / 256, 256, 0, s>>>(G, ldg, (int)m, npad, sig);
    HEFF_LAUNCH_CHECK();
    std::vector<double> hs(npad);
    HEFF_CUDA(cudaMemcpyAsync(hs.data(), sig, sizeof(double) * npad, cudaMemcpyDeviceToHost, s));
    HEFF_CUDA(cudaStreamSynchronize(s));
    std::vector<int> order(npad);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return hs[a] > hs[b]; });
    const int64_t       kfull = std::min(m, n);
    std::vector<double> sorted(kfull);
    for(int64_t i = 0; i < kfull; i++) sorted[i] = hs[order[i]];
    const int64_t r = truncation_rank(sorted.data(), kfull, rank_max, 0, trunc_lim, trunc_err);
    if(r <= 0) {
        set_last_error_msg("svd: rank <= 0 (all singular values zero or below the truncation limit)");
        return HEFF_BAD_ARG;
    }
    *rank = r;
    HEFF_CUDA(cudaMemcpyAsync(perm, order.data(), sizeof(int) * r, cudaMemcpyHostToDevice, s));
    HEFF_CUDA(cudaMemcpyAsync(S, sorted.data(), sizeof(double) * r, cudaMemcpyHostToDevice, s));
    svd_gather_kernel<<<g1((m + n) * r), 256, 0, s>>>(G, ldg, (int)m, V, npad, (int)n, perm, sig, (int)r, U, VT);
    HEFF_LAUNCH_CHECK();
    HEFF_CUDA(cudaStreamSynchronize(s));  // host vectors above must outlive the copies
    return HEFF_OK;
}

// theta [dL*dR, chiL, chiR] -> A[(s1 + dL a), (s2 + dR b)] = theta[s1 + dL s2, a, b]   (svd.h:217 reshape+shuffle)
__global__ void schmidt_pack_kernel(const double *__restrict__ th, double *__restrict__ A, int64_t dL, int64_t dR, int64_t cL, int64_t cR) {
    const int64_t m = dL * cL, tot = m * dR * cR;
    for(int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < tot; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t row = e % m, col = e / m;
        const int64_t s1 = row % dL, a = row / dL, s2 = col % dR, b = col / dR;
        A[e]             = th[(s1 + dL * s2) + dL * dR * (a + cL * b)];
    }
}
// VT [k, dR*chiR] -> V [dR, k, chiR] (svd.h:173 shuffle {1,0,2});  S <- S / ||S||
__global__ void schmidt_unpack_kernel(const double *__restrict__ VT, double *__restrict__ Vout, double *__restrict__ S, double inv_norm, int64_t k,
                                      int64_t dR, int64_t cR) {
    const int64_t tot = k * dR * cR;
    for(int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < tot; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t s2 = e % dR, r = e / dR, i = r % k, b = r / k;
        Vout[e]          = VT[i + k * (s2 + dR * b)];
        if(e < k) S[e] *= inv_norm;
    }
}

int schmidt_split(const double *theta, int64_t dL, int64_t dR, int64_t cL, int64_t cR, int64_t rank_max, double trunc_lim, double *U, double *S,
                  double *V, int64_t *rank, double *trunc_err, void *scratch, cudaStream_t s) {
    const int64_t m = dL * cL, n = dR * cR;
    double       *A      = reinterpret_cast<double *>(scratch);
    double       *VT     = A + (m * n + 31) / 32 * 32;
    const int64_t kmax   = std::min(std::min(m, n), rank_max > 0 ? rank_max : INT64_MAX);
    void         *jscr   = VT + (kmax * n + 31) / 32 * 32;
    schmidt_pack_kernel<<<g1(m * n), 256, 0, s>>>(theta, A, dL, dR, cL, cR);
    HEFF_LAUNCH_CHECK();
    HEFF_TRY(svd_truncated(A, m, m, n, rank_max, trunc_lim, U, S, VT, rank, trunc_err, jscr, nullptr, s));
    std::vector<double> hs(*rank);
    HEFF_CUDA(cudaMemcpyAsync(hs.data(), S, sizeof(double) * (*rank), cudaMemcpyDeviceToHost, s));
    HEFF_CUDA(cudaStreamSynchronize(s));
    double nrm = 0;
    for(double v : hs) nrm += v * v;
    nrm = std::sqrt(nrm);
    schmidt_unpack_kernel<<<g1((*rank) * n), 256, 0, s>>>(VT, V, S, nrm > 0 ? 1.0 / nrm : 1.0, *rank, dR, cR);
    HEFF_LAUNCH_CHECK();
    return HEFF_OK;
}

int64_t schmidt_scratch_bytes(int64_t dL, int64_t dR, int64_t cL, int64_t cR, int64_t rank_max) {
    const int64_t m = dL * cL, n = dR * cR;
    const int64_t kmax = std::min(std::min(m, n), rank_max > 0 ? rank_max : INT64_MAX);
    return 8 * ((m * n + 31) / 32 * 32 + (kmax * n + 31) / 32 * 32) + svd_scratch_bytes(m, n) + 512;
}

}  // namespace heff

using namespace heff;

extern "C" int heff_svd_d(const double *A, int64_t rows, int64_t cols, int64_t rank_max, double trunc_lim, double *U, double *S, double *VT,
                          int64_t *rank, double *trunc_err, void *stream) {
    if(!A || !U || !S || !VT || !rank || rows <= 0 || cols <= 0) return HEFF_BAD_ARG;
    cudaStream_t s    = (cudaStream_t)stream;
    void        *base = nullptr;
    HEFF_TRY(stream_workspace(s, (size_t)svd_scratch_bytes(rows, cols), &base));
    double te = 0;
    HEFF_TRY(svd_truncated(A, rows, rows, cols, rank_max, trunc_lim, U, S, VT, rank, &te, base, nullptr, s));
    if(trunc_err) *trunc_err = te;
    return HEFF_OK;
}

extern "C" int heff_schmidt_d(const double *theta, int64_t dL, int64_t dR, int64_t chiL, int64_t chiR, int64_t rank_max, double trunc_lim, double *U,
                              double *S, double *V, int64_t *rank, double *trunc_err, void *stream) {
    if(!theta || !U || !S || !V || !rank || dL <= 0 || dR <= 0 || chiL <= 0 || chiR <= 0) return HEFF_BAD_ARG;
    cudaStream_t s    = (cudaStream_t)stream;
    void        *base = nullptr;
    HEFF_TRY(stream_workspace(s, (size_t)schmidt_scratch_bytes(dL, dR, chiL, chiR, rank_max), &base));
    double te = 0;
    HEFF_TRY(schmidt_split(theta, dL, dR, chiL, chiR, rank_max, trunc_lim, U, S, V, rank, &te, base, s));
    if(trunc_err) *trunc_err = te;
    return HEFF_OK;
}
