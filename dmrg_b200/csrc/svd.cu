// Truncated SVD on the device: svd::solver::do_svd_ptr (source/math/svd/svd.cpp:113-206) with the rank
// rule get_rank_from_truncation_error (svd.cpp:257-280) and the two-site Schmidt split
// schmidt_multisite (source/math/svd.h:189-220), for real (double) and complex (double2) matrices.
//
// Algorithm: one-sided (Hestenes) block Jacobi in FP64.  The columns of the work matrix G (= A, m x n,
// column-major, n padded to a multiple of 32 with zero columns) are ordered by norm before every sweep and
// grouped into blocks of 16 neighbours.  A sweep pairs every block with every other block once
// (round-robin tournament, B-1 rounds of B/2 disjoint pairs).  For one pair, a cluster of 1-4 CTAs
//   1. forms the 32 x 32 Gram matrix P^H P of the pair's 32 columns (rows streamed through shared memory,
//      DMMA products, row shares summed across the cluster),
//   2. runs one sweep of a cyclic two-sided Jacobi eigensolver on it in shared memory (16 disjoint
//      rotations per step), accumulating the unitary Q,
//   3. applies P <- P Q and V[:, pair] <- V[:, pair] Q (DMMA, row shares).
// A pair whose Gram is already diagonal to |g_ij| <= max(tol*sqrt(g_ii g_jj), floor) is skipped; the
// sweep loop stops when every pair was skipped.  The relative criterion, evaluated on freshly computed
// Gram entries, is what lets one-sided Jacobi resolve small singular values to high relative accuracy
// (Demmel & Veselic 1992), which the truncation rule at 1e-12 needs.  The absolute floor
// m eps^2 max_j ||G_j||^2 (from the previous sweep) stops the sweeps on columns that are rounding
// noise (singular values below ~eps sigma_max, which no rotation can make relatively orthogonal); an
// off-diagonal below it moves a singular value sigma by at most ~floor / sigma, the eps ||A|| level
// of LAPACK's gesdd.  Then sigma_j = ||G_j||, U_j = G_j / sigma_j, sorted descending, VT = V^H.
//
// Complex rotation: for the Hermitian 2x2 block [[a, h], [conj(h), b]] with h = |h| e (|e| = 1) the
// unitary J = diag(1, conj(e)) R diag(1, e), R the real Jacobi rotation of [[a, |h|], [|h|, b]], acts as
//   col_p' = c col_p - s conj(e) col_q,   col_q' = s e col_p + c col_q
// (rows of the Gram with the conjugate coefficients); it reduces to the real rotation for e = +-1.
#include <algorithm>
#include <cmath>
#include <cooperative_groups.h>
#include <numeric>
#include <type_traits>
#include <vector>

#include "matvec.cuh"
#include "runtime.cuh"
#include "svd.cuh"

namespace heff {

constexpr int JB   = 16;      // columns per block
constexpr int JP   = 2 * JB;  // columns per pair
constexpr int JTHR = 256;
constexpr int JINNER = 1;   // two-sided Jacobi sweeps on a pair's 32 x 32 Gram per visit
constexpr int JOUTER = 60;  // outer sweeps at most

// Scalar operations of the Jacobi kernels for real and complex FP64.
template<class T>
struct JS;
template<>
struct JS<double> {
    static constexpr int ROWS = 64;  // rows per streamed tile (shared memory fits 48 KB)
    __device__ static double zero() { return 0.0; }
    __device__ static double one() { return 1.0; }
    __device__ static double fma_cj(double a, double b, double acc) { return fma(a, b, acc); }  // acc + conj(a) b
    __device__ static double fma_(double a, double b, double acc) { return fma(a, b, acc); }    // acc + a b
    __device__ static double abs2(double a) { return a * a; }
    __device__ static double absv(double a) { return fabs(a); }
    __device__ static double re(double a) { return a; }
    __device__ static double unit(double a) { return a >= 0 ? 1.0 : -1.0; }
    __device__ static double unit_r(double a, double) { return a >= 0 ? 1.0 : -1.0; }  // a / |a| given 1 / |a|
    __device__ static double conj(double a) { return a; }
    __device__ static double mul(double a, double b) { return a * b; }
    __device__ static double axpy(double a, double x, double y) { return fma(a, x, y); }  // y + a x, a real
    __device__ static double scale(double x, double a) { return x * a; }
};
template<>
struct JS<double2> {
    static constexpr int ROWS = 16;
    __device__ static double2 zero() { return make_double2(0.0, 0.0); }
    __device__ static double2 one() { return make_double2(1.0, 0.0); }
    __device__ static double2 fma_cj(double2 a, double2 b, double2 acc) {
        return make_double2(fma(a.x, b.x, fma(a.y, b.y, acc.x)), fma(a.x, b.y, fma(-a.y, b.x, acc.y)));
    }
    __device__ static double2 fma_(double2 a, double2 b, double2 acc) {
        return make_double2(fma(a.x, b.x, fma(-a.y, b.y, acc.x)), fma(a.x, b.y, fma(a.y, b.x, acc.y)));
    }
    __device__ static double  abs2(double2 a) { return a.x * a.x + a.y * a.y; }
    __device__ static double  absv(double2 a) { return hypot(a.x, a.y); }
    __device__ static double  re(double2 a) { return a.x; }
    __device__ static double2 unit(double2 a) {
        const double r = hypot(a.x, a.y);
        return r > 0 ? make_double2(a.x / r, a.y / r) : make_double2(1.0, 0.0);
    }
    __device__ static double2 unit_r(double2 a, double rinv) { return make_double2(a.x * rinv, a.y * rinv); }
    __device__ static double2 conj(double2 a) { return make_double2(a.x, -a.y); }
    __device__ static double2 mul(double2 a, double2 b) { return cmul(a, b); }
    __device__ static double2 axpy(double a, double2 x, double2 y) { return make_double2(fma(a, x.x, y.x), fma(a, x.y, y.y)); }
    __device__ static double2 scale(double2 x, double a) { return make_double2(x.x * a, x.y * a); }
};

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

// C += A B on the FP64 tensor pipe: mma.sync m16n8k4 (A fragment rows g, g+8 at column t; B at row t,
// column g; C entries (g + 8 (r >> 1), 2 t + (r & 1)), g = lane / 4, t = lane % 4).
__device__ __forceinline__ void dmma_f64(double (&c)[4], double a0, double a1, double b0) {
    asm volatile("mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};\n"
                 : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
                 : "d"(a0), "d"(a1), "d"(b0));
}

// x' = x - s (e y + tau x)  (one half of a Rutishauser-form rotation; e unit-modulus)
template<class T>
__device__ __forceinline__ T rot_lo(T x, T y, T e, double sn, double tau) {
    using S = JS<T>;
    return S::axpy(-sn, S::fma_(e, y, S::scale(x, tau)), x);
}

// One round of the block Jacobi sweep.  A pair is handled by a cluster of CL CTAs (blockIdx.x = pair * CL + rank):
// each forms the Gram of its share of the rows, the partials are summed through distributed shared memory in
// rank order (so every CTA holds the same full Gram), every CTA runs the small Jacobi on it (the same Q
// everywhere, no broadcast) and updates its share of the rows of G and V.  CL = 1: a plain launch, one CTA
// per pair.  The two cluster barriers are reached by every CTA; the early exit comes after them.
template<class T>
__global__ void __launch_bounds__(JTHR) jacobi_round_kernel(T *__restrict__ G, int64_t ldg, int m, T *__restrict__ V, int64_t ldv, int nv, int B,
                                                           int round, double tol, double floor_abs, const int *__restrict__ colmap,
                                                           double *__restrict__ offmax, int *__restrict__ rotated, int CL) {
    using S                = JS<T>;
    constexpr int JROWS    = S::ROWS;
    __shared__ T      sG[JP][JP + 1];
    __shared__ T      sQ[JP][JP + 1];
    __shared__ T      sT[JROWS][JP + 1];
    __shared__ double cs_t[JP / 2], cs_s[JP / 2];
    __shared__ T      cs_e[JP / 2];
    __shared__ int    s_idx[JP];
    __shared__ double s_red[JTHR];
    __shared__ int    s_rot[2];

    int       p, q;
    const int rank = (int)(blockIdx.x % CL);
    rr_pair(B, round, (int)(blockIdx.x / CL), p, q);
    const int tid = threadIdx.x;
    if(tid < JP) s_idx[tid] = colmap[(tid < JB) ? p * JB + tid : q * JB + (tid - JB)];
    __syncthreads();

    // ---- 1. Gram matrix of the 32 columns over this CTA's rows [ga, gb)
    const int ga = (int)((int64_t)m * rank / CL), gb = (int)((int64_t)m * (rank + 1) / CL);
    // warp w forms the 16 x 8 tile (w / 4, w % 4) of the Gram on the FP64 tensor pipe (m16n8k4 DMMA,
    // A = P^H, B = P from the staged rows); complex: Re = Pr^T Pr + Pi^T Pi, Im = Pr^T Pi - Pi^T Pr
    const int lane = tid & 31, wg = lane >> 2, wt = lane & 3, wmt = (tid >> 5) >> 2, wnt = (tid >> 5) & 3;
    double    accr[4] = {0, 0, 0, 0}, acci[4] = {0, 0, 0, 0};
    for(int r0 = ga; r0 < gb; r0 += JROWS) {
        for(int e = tid; e < JROWS * JP; e += JTHR) {
            const int rr = e % JROWS, cc = e / JROWS, row = r0 + rr;
            sT[rr][cc]   = row < gb ? G[row + ldg * (int64_t)s_idx[cc]] : S::zero();
        }
        __syncthreads();
#pragma unroll 4
        for(int k4 = 0; k4 < JROWS; k4 += 4) {
            const T a0 = sT[k4 + wt][wmt * 16 + wg], a1 = sT[k4 + wt][wmt * 16 + wg + 8], b = sT[k4 + wt][wnt * 8 + wg];
            if constexpr(std::is_same<T, double>::value) {
                dmma_f64(accr, a0, a1, b);
            } else {
                dmma_f64(accr, a0.x, a1.x, b.x);
                dmma_f64(accr, a0.y, a1.y, b.y);
                dmma_f64(acci, a0.x, a1.x, b.y);
                dmma_f64(acci, -a0.y, -a1.y, b.x);
            }
        }
        __syncthreads();
    }
    T acc[4];
#pragma unroll
    for(int u = 0; u < 4; u++) {
        if constexpr(std::is_same<T, double>::value)
            acc[u] = accr[u];
        else
            acc[u] = make_double2(accr[u], acci[u]);
    }
    // the Gram entry acc[u] holds: the fragment entry u of the warp's DMMA tile
    auto g_row = [&](int u) { return wmt * 16 + wg + 8 * (u >> 1); };
    auto g_col = [&](int u) { return wnt * 8 + 2 * wt + (u & 1); };
    if(CL == 1) {
#pragma unroll
        for(int u = 0; u < 4; u++) sG[g_row(u)][g_col(u)] = acc[u];
        __syncthreads();
    } else {
        // partials in sQ (free until the Jacobi below), summed over the cluster in rank order
        namespace cg = cooperative_groups;
        cg::cluster_group cluster = cg::this_cluster();
#pragma unroll
        for(int u = 0; u < 4; u++) sQ[g_row(u)][g_col(u)] = acc[u];
        cluster.sync();
        T tot[4] = {S::zero(), S::zero(), S::zero(), S::zero()};
        for(int r = 0; r < CL; r++) {
            const T *rq = cluster.map_shared_rank(&sQ[0][0], r);
#pragma unroll
            for(int u = 0; u < 4; u++) tot[u] = JS<T>::axpy(1.0, rq[g_row(u) * (JP + 1) + g_col(u)], tot[u]);
        }
#pragma unroll
        for(int u = 0; u < 4; u++) sG[g_row(u)][g_col(u)] = tot[u];
        cluster.sync();  // every CTA has read the partials before any overwrites its sQ
    }

    // ---- off-diagonal measure of the fresh Gram (relative to the diagonal; entries under the floor ignored)
    //      and the largest squared column norm of the pair (offmax[1], the next sweep's floor)
    double mx = 0, gmx = 0;
    for(int e = tid; e < JP * JP; e += JTHR) {
        const int i = e / JP, j = e % JP;
        if(i < j) {
            const double d = sqrt(fabs(S::re(sG[i][i])) * fabs(S::re(sG[j][j])));
            const double o = S::absv(sG[i][j]);
            if(o > floor_abs) mx = fmax(mx, d > 0 ? o / d : 1.0);
        } else if(i == j) {
            gmx = fmax(gmx, fabs(S::re(sG[i][i])));
        }
    }
    s_red[tid] = mx;
    __syncthreads();
    for(int w = JTHR / 2; w > 0; w >>= 1) {
        if(tid < w) s_red[tid] = fmax(s_red[tid], s_red[tid + w]);
        __syncthreads();
    }
    const double off0 = s_red[0];
    __syncthreads();
    s_red[tid] = gmx;
    __syncthreads();
    for(int w = JTHR / 2; w > 0; w >>= 1) {
        if(tid < w) s_red[tid] = fmax(s_red[tid], s_red[tid + w]);
        __syncthreads();
    }
    if(tid == 0 && rank == 0) {
        atomic_max_pos(offmax, off0);
        atomic_max_pos(offmax + 1, s_red[0]);
    }
    if(off0 <= tol) return;  // uniform across the CTA and the cluster (the same Gram everywhere)
    if(tid == 0 && rank == 0) atomicAdd(rotated, 1);

    // ---- 2. cyclic Jacobi on sG, accumulating sQ.  Rotations are applied in Rutishauser's form
    //      x' = x - s (conj(e) y + tau x), y' = y + s (e x - tau y), tau = s / (1 + c), which keeps the
    //      rounding of c (c -> 1 for tiny angles) from inflating column norms; only numerically
    //      significant off-diagonals (|g_ab| > tol sqrt(g_aa g_bb)) are rotated, one sweep per visit of the
    //      pair (the outer sweep re-checks every pair on a freshly computed Gram matrix; measured on 1024^2 and
    //      2048^2: one inner sweep costs at most a few more outer sweeps and halves the time against eight).
    for(int e = tid; e < JP * JP; e += JTHR) sQ[e / JP][e % JP] = (e / JP == e % JP) ? S::one() : S::zero();
    if(tid < 2) s_rot[tid] = 0;
    __syncthreads();
    for(int sweep = 0; sweep < JINNER; sweep++) {
        const int par = sweep & 1;
        for(int step = 0; step < JP - 1; step++) {
            if(tid < JP / 2) {
                int a, b;
                rr_pair(JP, step, tid, a, b);
                const double app = S::re(sG[a][a]), aqq = S::re(sG[b][b]);
                const T      apq = sG[a][b];
                const double h   = S::absv(apq);
                double       sn = 0.0, tau = 0.0;
                if(h > 1e-300 && h > floor_abs && h > tol * sqrt(fabs(app) * fabs(aqq))) {
                    const double th = (aqq - app) / (2.0 * h);
                    const double t  = (th >= 0 ? 1.0 : -1.0) / (fabs(th) + sqrt(1.0 + th * th));
                    const double c  = 1.0 / sqrt(1.0 + t * t);
                    sn              = t * c;
                    tau             = sn / (1.0 + c);
                    s_rot[par]      = 1;
                }
                cs_t[tid] = tau;
                cs_s[tid] = sn;
                cs_e[tid] = S::unit(apq);
            }
            __syncthreads();
            // columns of G and Q: col_a' = col_a - s (conj(e) col_b + tau col_a), col_b' = col_b + s (e col_a - tau col_b)
            for(int e = tid; e < (JP / 2) * JP; e += JTHR) {
                const int k = e / JP, row = e % JP;
                int       a, b;
                rr_pair(JP, step, k, a, b);
                const double tau = cs_t[k], sn = cs_s[k];
                if(sn != 0.0) {
                    const T ph = cs_e[k], phc = S::conj(ph);
                    const T ga = sG[row][a], gb = sG[row][b];
                    sG[row][a] = rot_lo(ga, gb, phc, sn, tau);
                    sG[row][b] = rot_lo(gb, ga, ph, -sn, -tau);
                    const T qa = sQ[row][a], qb = sQ[row][b];
                    sQ[row][a] = rot_lo(qa, qb, phc, sn, tau);
                    sQ[row][b] = rot_lo(qb, qa, ph, -sn, -tau);
                }
            }
            __syncthreads();
            // rows of G (left multiplication by J^H): row_a' = row_a - s (e row_b + tau row_a), row_b' = row_b + s (conj(e) row_a - tau row_b)
            for(int e = tid; e < (JP / 2) * JP; e += JTHR) {
                const int k = e / JP, col = e % JP;
                int       a, b;
                rr_pair(JP, step, k, a, b);
                const double tau = cs_t[k], sn = cs_s[k];
                if(sn != 0.0) {
                    const T ph = cs_e[k], phc = S::conj(ph);
                    const T ga = sG[a][col], gb = sG[b][col];
                    sG[a][col] = rot_lo(ga, gb, ph, sn, tau);
                    sG[b][col] = rot_lo(gb, ga, phc, -sn, -tau);
                }
            }
            __syncthreads();
        }
        const int rotated_this_sweep = s_rot[par];
        __syncthreads();
        if(tid == 0) s_rot[par] = 0;  // reused two sweeps later; read above before this reset
        if(!rotated_this_sweep) break;
    }

    // ---- 3. apply Q to this CTA's share of the pair's columns of G (m rows) and V (nv rows)
    for(int pass = 0; pass < 2; pass++) {
        T            *X    = pass == 0 ? G : V;
        const int64_t ldx  = pass == 0 ? ldg : ldv;
        const int     all  = pass == 0 ? m : nv;
        const int     ra = (int)((int64_t)all * rank / CL), rows = (int)((int64_t)all * (rank + 1) / CL);
        for(int r0 = ra; r0 < rows; r0 += JROWS) {
            for(int e = tid; e < JROWS * JP; e += JTHR) {
                const int rr = e % JROWS, cc = e / JROWS, row = r0 + rr;
                sT[rr][cc]   = row < rows ? X[row + ldx * (int64_t)s_idx[cc]] : S::zero();
            }
            __syncthreads();
            if constexpr(std::is_same<T, double>::value) {
                // (64 rows x 32) Q on the tensor pipe: warp w owns row tile w / 2 and column tiles 2 (w % 2) + 0, 1;
                // the products go back through the staged tile so the stores below stay coalesced
                const int mt = (tid >> 5) >> 1, nt0 = 2 * ((tid >> 5) & 1);
                double    c[2][4] = {{0, 0, 0, 0}, {0, 0, 0, 0}};
#pragma unroll
                for(int k4 = 0; k4 < JP; k4 += 4) {
                    const double a0 = sT[mt * 16 + wg][k4 + wt], a1 = sT[mt * 16 + wg + 8][k4 + wt];
#pragma unroll
                    for(int j = 0; j < 2; j++) dmma_f64(c[j], a0, a1, sQ[k4 + wt][(nt0 + j) * 8 + wg]);
                }
                __syncthreads();
#pragma unroll
                for(int j = 0; j < 2; j++)
#pragma unroll
                    for(int u = 0; u < 4; u++) sT[mt * 16 + wg + 8 * (u >> 1)][(nt0 + j) * 8 + 2 * wt + (u & 1)] = c[j][u];
                __syncthreads();
                for(int e = tid; e < JROWS * JP; e += JTHR) {
                    const int rr = e % JROWS, cc = e / JROWS, row = r0 + rr;
                    if(row < rows) X[row + ldx * (int64_t)s_idx[cc]] = sT[rr][cc];
                }
            } else {
                // (16 rows x 32) Q, complex: warp w owns column tile w % 4 and the real (w < 4) or imaginary part
                const int nt = (tid >> 5) & 3, im = (tid >> 5) >> 2;
                double    c[4] = {0, 0, 0, 0};
#pragma unroll
                for(int k4 = 0; k4 < JP; k4 += 4) {
                    const T a0 = sT[wg][k4 + wt], a1 = sT[wg + 8][k4 + wt], qv = sQ[k4 + wt][nt * 8 + wg];
                    if(im == 0) {  // Re = Tr Qr - Ti Qi
                        dmma_f64(c, a0.x, a1.x, qv.x);
                        dmma_f64(c, -a0.y, -a1.y, qv.y);
                    } else {       // Im = Tr Qi + Ti Qr
                        dmma_f64(c, a0.x, a1.x, qv.y);
                        dmma_f64(c, a0.y, a1.y, qv.x);
                    }
                }
                __syncthreads();
#pragma unroll
                for(int u = 0; u < 4; u++) {
                    T &dst = sT[wg + 8 * (u >> 1)][nt * 8 + 2 * wt + (u & 1)];
                    if(im == 0)
                        dst.x = c[u];
                    else
                        dst.y = c[u];
                }
                __syncthreads();
                for(int e = tid; e < JROWS * JP; e += JTHR) {
                    const int rr = e % JROWS, cc = e / JROWS, row = r0 + rr;
                    if(row < rows) X[row + ldx * (int64_t)s_idx[cc]] = sT[rr][cc];
                }
            }
            __syncthreads();
        }
    }
}

// sigma_j = ||G_j||_2 (column norms), one warp per column.
template<class T>
__global__ void col_norms_kernel(const T *__restrict__ G, int64_t ldg, int m, int n, double *__restrict__ sig) {
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) / 32, lane = threadIdx.x & 31;
    if(w >= n) return;
    double acc = 0;
    for(int i = lane; i < m; i += 32) acc += JS<T>::abs2(G[i + ldg * (int64_t)w]);
    for(int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if(lane == 0) sig[w] = sqrt(acc);
}

// U[:, i] = G[:, perm[i]] / sigma[perm[i]],  VT[i, :] = V[:, perm[i]]^H  (i < k)
template<class T>
__global__ void svd_gather_kernel(const T *__restrict__ G, int64_t ldg, int m, const T *__restrict__ V, int64_t ldv, int n, const int *__restrict__ perm,
                                  const double *__restrict__ sig, int k, T *__restrict__ U, T *__restrict__ VT) {
    const int64_t tot_u = (int64_t)m * k, tot_v = (int64_t)n * k;
    for(int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < tot_u + tot_v; e += (int64_t)gridDim.x * blockDim.x) {
        if(e < tot_u) {
            const int64_t i = e / m, r = e % m;
            const int     j = perm[i];
            const double  s = sig[j];
            U[r + (int64_t)m * i] = s > 0 ? JS<T>::scale(G[r + ldg * (int64_t)j], 1.0 / s) : JS<T>::zero();
        } else {
            const int64_t f = e - tot_u, c = f / k, i = f % k;  // VT is k x n column-major
            VT[i + (int64_t)k * c] = JS<T>::conj(V[c + ldv * (int64_t)perm[i]]);
        }
    }
}

template<class T>
__global__ void copy_pad_kernel(const T *__restrict__ A, int64_t lda, int m, int n, T *__restrict__ G, int64_t ldg, int npad) {
    const int64_t tot = (int64_t)ldg * npad;
    for(int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < tot; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = e % ldg, c = e / ldg;
        G[e]            = (r < m && c < n) ? A[r + lda * c] : JS<T>::zero();
    }
}

template<class T>
__global__ void eye_kernel(T *__restrict__ V, int64_t ldv, int npad) {
    const int64_t tot = (int64_t)ldv * npad;
    for(int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < tot; e += (int64_t)gridDim.x * blockDim.x)
        V[e] = (e % ldv == e / ldv) ? JS<T>::one() : JS<T>::zero();
}

// Small matrices (at most 64 padded columns, G and V together in shared memory): one CTA runs the whole cyclic
// one-sided Jacobi -- every sweep of nc - 1 steps over the nc / 2 disjoint column pairs of the round-robin
// tournament on the first nc (even) columns, one warp per pair -- with the block path's rotation (Rutishauser form),
// relative criterion and absolute floor, and no host round trip between sweeps.  On the block path each sweep costs a norm ordering on the host, two
// synchronisations and B - 1 launches, most of the time of a 64 x 64 split.  G (m x npad, column stride ldg) and V
// (npad x npad, the identity on entry) are read from and written back to global memory; sweeps_out receives the
// number of sweeps run (max_sweeps when the last one still rotated).
constexpr int    JSMALL_THR  = 1024;
constexpr size_t JSMALL_SMEM = 200 * 1024;
template<class T>
static size_t jacobi_small_bytes(int64_t m, int64_t npad) {
    return (size_t)(m * npad + npad * npad) * sizeof(T);
}
template<class T>
__device__ __forceinline__ T warp_sum(T v);
template<>
__device__ __forceinline__ double warp_sum(double v) {
    for(int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
template<>
__device__ __forceinline__ double2 warp_sum(double2 v) {
    for(int o = 16; o > 0; o >>= 1) {
        v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
        v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
    }
    return v;
}
template<class T>
__global__ void __launch_bounds__(JSMALL_THR, 1) jacobi_small_kernel(T *__restrict__ G, int64_t ldg, int m, T *__restrict__ V, int npad, int nc,
                                                                    double tol, int max_sweeps, int *__restrict__ sweeps_out) {
    using S = JS<T>;
    extern __shared__ __align__(16) unsigned char js_smem[];
    T *sG = reinterpret_cast<T *>(js_smem);  // m x npad, column-major, column stride m
    T *sV = sG + (int64_t)m * npad;           // npad x npad, column-major
    __shared__ double s_norm[64];
    __shared__ double s_gmax;
    __shared__ int    s_rot;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for(int64_t e = tid; e < (int64_t)m * npad; e += JSMALL_THR) sG[e] = G[(e % m) + ldg * (e / m)];
    for(int e = tid; e < npad * npad; e += JSMALL_THR) sV[e] = V[e];
    const double eps       = 2.220446049250313e-16;
    double       floor_abs = 0.0;  // first sweep: relative criterion only
    int          done      = max_sweeps;
    for(int sweep = 0; sweep < max_sweeps; sweep++) {
        __syncthreads();  // the previous sweep's flag has been read by every thread
        if(tid == 0) s_rot = 0;
        __syncthreads();
        for(int step = 0; step < nc - 1; step++) {
            if(warp < nc / 2) {
                int p, q;
                rr_pair(nc, step, warp, p, q);
                T     *gp = sG + (int64_t)m * p, *gq = sG + (int64_t)m * q;
                double app = 0.0, aqq = 0.0;
                T      apq = S::zero();
                for(int i = lane; i < m; i += 32) {
                    const T x = gp[i], y = gq[i];
                    app += S::abs2(x);
                    aqq += S::abs2(y);
                    apq = S::fma_cj(x, y, apq);  // += conj(x) y
                }
                app = warp_sum(app);
                aqq = warp_sum(aqq);
                apq = warp_sum(apq);
                // the block path's criterion |apq| > max(tol sqrt(app aqq), floor, 1e-300), in the same form (squaring |apq|
                // would underflow for entries below ~1e-81), and the rotation with one reciprocal of |apq| shared by the
                // angle and the phase: every step waits on this chain of reciprocals and square roots
                const double h = S::absv(apq);
                if(h > 1e-300 && h > floor_abs && h > tol * sqrt(app * aqq)) {  // the same value in every lane
                    const double rh  = 1.0 / h;
                    const double th  = 0.5 * (aqq - app) * rh;
                    const double t   = (th >= 0 ? 1.0 : -1.0) / (fabs(th) + sqrt(fma(th, th, 1.0)));
                    const double c   = rsqrt(fma(t, t, 1.0));
                    const double sn  = t * c;
                    const double tau = sn / (1.0 + c);
                    const T      ph = S::unit_r(apq, rh), phc = S::conj(ph);
                    // col_p' = col_p - s (conj(e) col_q + tau col_p), col_q' = col_q + s (e col_p - tau col_q), on G and V
                    for(int i = lane; i < m; i += 32) {
                        const T x = gp[i], y = gq[i];
                        gp[i]     = rot_lo(x, y, phc, sn, tau);
                        gq[i]     = rot_lo(y, x, ph, -sn, -tau);
                    }
                    T *vp = sV + (int64_t)npad * p, *vq = sV + (int64_t)npad * q;
                    for(int i = lane; i < npad; i += 32) {
                        const T x = vp[i], y = vq[i];
                        vp[i]     = rot_lo(x, y, phc, sn, tau);
                        vq[i]     = rot_lo(y, x, ph, -sn, -tau);
                    }
                    if(lane == 0) s_rot = 1;
                }
            }
            __syncthreads();
        }
        // squared column norms: their maximum sets the next sweep's absolute floor m eps^2 max ||G_j||^2
        for(int c = warp; c < nc; c += JSMALL_THR / 32) {
            double v = 0.0;
            for(int i = lane; i < m; i += 32) v += S::abs2(sG[(int64_t)m * c + i]);
            v = warp_sum(v);
            if(lane == 0) s_norm[c] = v;
        }
        __syncthreads();
        if(tid == 0) {
            double g = 0.0;
            for(int c = 0; c < nc; c++) g = fmax(g, s_norm[c]);
            s_gmax = g;
        }
        __syncthreads();
        if(s_rot == 0) {  // uniform: read after the barrier by every thread
            done = sweep + 1;
            break;
        }
        floor_abs = (double)m * eps * eps * s_gmax;
    }
    __syncthreads();
    for(int64_t e = tid; e < (int64_t)m * npad; e += JSMALL_THR) G[(e % m) + ldg * (e / m)] = sG[e];
    for(int e = tid; e < npad * npad; e += JSMALL_THR) V[e] = sV[e];
    if(tid == 0) *sweeps_out = done;
}

int &last_svd_sweeps() {
    static thread_local int n = 0;
    return n;
}

static int g1(int64_t n) {
    int64_t g = (n + 255) / 256, cap = (int64_t)device_sm_count() * 8;
    return (int)(g < 1 ? 1 : (g < cap ? g : cap));
}

int64_t svd_scratch_bytes(int64_t m, int64_t n, int64_t esize) {
    const int64_t npad = (n + JP - 1) / JP * JP;
    const int64_t ldg  = (m + 1) / 2 * 2;
    return esize * (ldg * npad + npad * npad) + 8 * (npad + 64) + 8 * npad + 256;
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
template<class T>
static int svd_truncated_t(const T *A, int64_t lda, int64_t m, int64_t n, int64_t rank_max, double trunc_lim, T *U, double *S, T *VT, int64_t *rank,
                           double *trunc_err, void *scratch, int *sweeps_out, cudaStream_t s) {
    if(m <= 0 || n <= 0 || m > (1 << 24) || n > 16384) return HEFF_BAD_SHAPE;
    const int     npad = (int)((n + JP - 1) / JP * JP);
    const int64_t ldg  = (m + 1) / 2 * 2;
    T            *G    = reinterpret_cast<T *>(scratch);
    T            *V    = G + ldg * npad;
    double       *sig  = reinterpret_cast<double *>(V + (int64_t)npad * npad);
    double       *dmax = sig + npad;  // [0] largest relative off-diagonal, [1] largest squared column norm
    int          *drot = reinterpret_cast<int *>(dmax + 8);
    int          *perm = reinterpret_cast<int *>(dmax + 64);
    int          *cmap = perm + npad;  // column order of the current sweep (block b = columns cmap[16 b .. 16 b + 15])
    copy_pad_kernel<T><<<g1(ldg * npad), 256, 0, s>>>(A, lda, (int)m, (int)n, G, ldg, npad);
    HEFF_LAUNCH_CHECK();
    eye_kernel<T><<<g1((int64_t)npad * npad), 256, 0, s>>>(V, npad, npad);
    HEFF_LAUNCH_CHECK();
    const int B = npad / JB;  // even
    // off-diagonal tolerance just above the rounding noise of a length-m dot product
    const double tol   = std::max(1e-14, 8.0 * 2.2e-16 * std::sqrt((double)m));
    const double eps   = 2.220446049250313e-16;
    double       floor_abs = 0.0;  // first sweep: relative criterion only
    int          sweep     = 0;
    // Norm-ordered blocks (the block form of de Rijk's pivoting in LAPACK's ?gesvj): before every sweep the
    // columns are ordered by norm and blocks are formed from neighbours, so clusters of close singular values
    // meet inside one pair block.  On a 1024 x 1024 matrix with a dense spectrum (3 % gaps, 1 .. 1e-13) the
    // fixed column order had not converged after 40 sweeps; with the ordering it converges in 35-40.
    std::vector<double> hn(npad);
    std::vector<int>    hmap(npad);
    // CTAs per pair: enough to fill the SMs with one wave (the pairs of a round are only B / 2), when the rows
    // are long enough to share out
    int CL = 1;
    while(CL < 4 && (int64_t)(B / 2) * CL * 2 <= device_sm_count() && m >= 128 * CL * 2) CL *= 2;
    const size_t small     = jacobi_small_bytes<T>(m, npad);
    const bool   use_small = npad <= 64 && small <= JSMALL_SMEM;
    if(use_small) {
        static int attr_done[64] = {0};
        int        dev           = 0;
        HEFF_CUDA(cudaGetDevice(&dev));
        if(dev < 0 || dev >= 64 || !attr_done[dev]) {
            HEFF_CUDA(cudaFuncSetAttribute(jacobi_small_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)JSMALL_SMEM));
            if(dev >= 0 && dev < 64) attr_done[dev] = 1;
        }
        // the tournament runs over the n columns rounded up to even, not over the padding to 32: padded columns are
        // zero and never rotate
        const int nc = (int)std::min<int64_t>(npad, (n + 1) / 2 * 2);
        jacobi_small_kernel<T><<<1, JSMALL_THR, small, s>>>(G, ldg, (int)m, V, npad, nc, tol, JOUTER, drot);
        HEFF_LAUNCH_CHECK();
        int ran = 0;
        HEFF_CUDA(cudaMemcpyAsync(&ran, drot, sizeof(int), cudaMemcpyDeviceToHost, s));
        HEFF_CUDA(cudaStreamSynchronize(s));
        sweep = ran - 1;
    }
    for(; !use_small && sweep < JOUTER; sweep++) {
        col_norms_kernel<T><<<(npad * 32 + 255) / 256, 256, 0, s>>>(G, ldg, (int)m, npad, sig);
        HEFF_LAUNCH_CHECK();
        HEFF_CUDA(cudaMemcpyAsync(hn.data(), sig, sizeof(double) * npad, cudaMemcpyDeviceToHost, s));
        HEFF_CUDA(cudaStreamSynchronize(s));
        std::iota(hmap.begin(), hmap.end(), 0);
        std::stable_sort(hmap.begin(), hmap.end(), [&](int a, int b) { return hn[a] > hn[b]; });
        HEFF_CUDA(cudaMemcpyAsync(cmap, hmap.data(), sizeof(int) * npad, cudaMemcpyHostToDevice, s));
        HEFF_CUDA(cudaMemsetAsync(dmax, 0, 8 * 8 + sizeof(int), s));
        for(int r = 0; r < B - 1; r++) {
            if(CL == 1) {
                jacobi_round_kernel<T><<<B / 2, JTHR, 0, s>>>(G, ldg, (int)m, V, npad, npad, B, r, tol, floor_abs, cmap, dmax, drot, 1);
                HEFF_LAUNCH_CHECK();
            } else {
                cudaLaunchConfig_t  lc = {};
                cudaLaunchAttribute at[1];
                at[0].id               = cudaLaunchAttributeClusterDimension;
                at[0].val.clusterDim.x = (unsigned)CL;
                at[0].val.clusterDim.y = 1;
                at[0].val.clusterDim.z = 1;
                lc.gridDim             = dim3((unsigned)(B / 2 * CL));
                lc.blockDim            = dim3(JTHR);
                lc.dynamicSmemBytes    = 0;
                lc.stream              = s;
                lc.attrs               = at;
                lc.numAttrs            = 1;
                HEFF_CUDA(cudaLaunchKernelEx(&lc, jacobi_round_kernel<T>, G, ldg, (int)m, V, (int64_t)npad, (int)npad, B, r, tol, floor_abs,
                                             (const int *)cmap, dmax, drot, CL));
            }
        }
        struct {
            double gmax;
            int    rot;
        } st{};
        HEFF_CUDA(cudaMemcpyAsync(&st.rot, drot, sizeof(int), cudaMemcpyDeviceToHost, s));
        HEFF_CUDA(cudaMemcpyAsync(&st.gmax, dmax + 1, sizeof(double), cudaMemcpyDeviceToHost, s));
        HEFF_CUDA(cudaStreamSynchronize(s));
        if(st.rot == 0) break;
        floor_abs = (double)m * eps * eps * st.gmax;
    }
    last_svd_sweeps() = sweep + 1;
    if(sweeps_out) *sweeps_out = sweep + 1;
    col_norms_kernel<T><<<(npad * 32 + 255) / 256, 256, 0, s>>>(G, ldg, (int)m, npad, sig);
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
    svd_gather_kernel<T><<<g1((m + n) * r), 256, 0, s>>>(G, ldg, (int)m, V, npad, (int)n, perm, sig, (int)r, U, VT);
    HEFF_LAUNCH_CHECK();
    HEFF_CUDA(cudaStreamSynchronize(s));  // host vectors above must outlive the copies
    return HEFF_OK;
}

int svd_truncated(const double *A, int64_t lda, int64_t m, int64_t n, int64_t rank_max, double trunc_lim, double *U, double *S, double *VT,
                  int64_t *rank, double *trunc_err, void *scratch, int *sweeps_out, cudaStream_t s) {
    return svd_truncated_t<double>(A, lda, m, n, rank_max, trunc_lim, U, S, VT, rank, trunc_err, scratch, sweeps_out, s);
}
int svd_truncated(const double2 *A, int64_t lda, int64_t m, int64_t n, int64_t rank_max, double trunc_lim, double2 *U, double *S, double2 *VT,
                  int64_t *rank, double *trunc_err, void *scratch, int *sweeps_out, cudaStream_t s) {
    return svd_truncated_t<double2>(A, lda, m, n, rank_max, trunc_lim, U, S, VT, rank, trunc_err, scratch, sweeps_out, s);
}

// theta [dL*dR, chiL, chiR] -> A[(s1 + dL a), (s2 + dR b)] = theta[s1 + dL s2, a, b]   (svd.h:217 reshape+shuffle)
template<class T>
__global__ void schmidt_pack_kernel(const T *__restrict__ th, T *__restrict__ A, int64_t dL, int64_t dR, int64_t cL, int64_t cR) {
    const int64_t m = dL * cL, tot = m * dR * cR;
    for(int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < tot; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t row = e % m, col = e / m;
        const int64_t s1 = row % dL, a = row / dL, s2 = col % dR, b = col / dR;
        A[e]             = th[(s1 + dL * s2) + dL * dR * (a + cL * b)];
    }
}
// VT [k, dR*chiR] -> V [dR, k, chiR] (svd.h:173 shuffle {1,0,2});  S <- S / ||S||
template<class T>
__global__ void schmidt_unpack_kernel(const T *__restrict__ VT, T *__restrict__ Vout, double *__restrict__ S, double inv_norm, int64_t k, int64_t dR,
                                      int64_t cR) {
    const int64_t tot = k * dR * cR;
    for(int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < tot; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t s2 = e % dR, r = e / dR, i = r % k, b = r / k;
        Vout[e]          = VT[i + k * (s2 + dR * b)];
        if(e < k) S[e] *= inv_norm;
    }
}

int64_t schmidt_scratch_bytes(int64_t dL, int64_t dR, int64_t cL, int64_t cR, int64_t rank_max, int64_t esize) {
    const int64_t m = dL * cL, n = dR * cR;
    const int64_t kmax = std::min(std::min(m, n), rank_max > 0 ? rank_max : INT64_MAX);
    return esize * ((m * n + 31) / 32 * 32 + (kmax * n + 31) / 32 * 32) + svd_scratch_bytes(m, n, esize) + 512;
}

template<class T>
static int schmidt_split_t(const T *theta, int64_t dL, int64_t dR, int64_t cL, int64_t cR, int64_t rank_max, double trunc_lim, T *U, double *S, T *V,
                           int64_t *rank, double *trunc_err, void *scratch, cudaStream_t s) {
    const int64_t m = dL * cL, n = dR * cR;
    T            *A    = reinterpret_cast<T *>(scratch);
    T            *VT   = A + (m * n + 31) / 32 * 32;
    const int64_t kmax = std::min(std::min(m, n), rank_max > 0 ? rank_max : INT64_MAX);
    void         *jscr = VT + (kmax * n + 31) / 32 * 32;
    schmidt_pack_kernel<T><<<g1(m * n), 256, 0, s>>>(theta, A, dL, dR, cL, cR);
    HEFF_LAUNCH_CHECK();
    HEFF_TRY(svd_truncated_t<T>(A, m, m, n, rank_max, trunc_lim, U, S, VT, rank, trunc_err, jscr, nullptr, s));
    std::vector<double> hs(*rank);
    HEFF_CUDA(cudaMemcpyAsync(hs.data(), S, sizeof(double) * (*rank), cudaMemcpyDeviceToHost, s));
    HEFF_CUDA(cudaStreamSynchronize(s));
    double nrm = 0;
    for(double v : hs) nrm += v * v;
    nrm = std::sqrt(nrm);
    schmidt_unpack_kernel<T><<<g1((*rank) * n), 256, 0, s>>>(VT, V, S, nrm > 0 ? 1.0 / nrm : 1.0, *rank, dR, cR);
    HEFF_LAUNCH_CHECK();
    return HEFF_OK;
}

int schmidt_split(const double *theta, int64_t dL, int64_t dR, int64_t cL, int64_t cR, int64_t rank_max, double trunc_lim, double *U, double *S,
                  double *V, int64_t *rank, double *trunc_err, void *scratch, cudaStream_t s) {
    return schmidt_split_t<double>(theta, dL, dR, cL, cR, rank_max, trunc_lim, U, S, V, rank, trunc_err, scratch, s);
}
int schmidt_split(const double2 *theta, int64_t dL, int64_t dR, int64_t cL, int64_t cR, int64_t rank_max, double trunc_lim, double2 *U, double *S,
                  double2 *V, int64_t *rank, double *trunc_err, void *scratch, cudaStream_t s) {
    return schmidt_split_t<double2>(theta, dL, dR, cL, cR, rank_max, trunc_lim, U, S, V, rank, trunc_err, scratch, s);
}

}  // namespace heff

using namespace heff;

template<class T>
static int svd_entry(const T *A, int64_t rows, int64_t cols, int64_t rank_max, double trunc_lim, T *U, double *S, T *VT, int64_t *rank,
                     double *trunc_err, void *stream) {
    if(!A || !U || !S || !VT || !rank || rows <= 0 || cols <= 0) return HEFF_BAD_ARG;
    cudaStream_t s    = (cudaStream_t)stream;
    void        *base = nullptr;
    HEFF_TRY(stream_workspace(s, (size_t)svd_scratch_bytes(rows, cols, sizeof(T)), &base));
    double te = 0;
    HEFF_TRY(svd_truncated(A, rows, rows, cols, rank_max, trunc_lim, U, S, VT, rank, &te, base, nullptr, s));
    if(trunc_err) *trunc_err = te;
    return HEFF_OK;
}

template<class T>
static int schmidt_entry(const T *theta, int64_t dL, int64_t dR, int64_t chiL, int64_t chiR, int64_t rank_max, double trunc_lim, T *U, double *S, T *V,
                         int64_t *rank, double *trunc_err, void *stream) {
    if(!theta || !U || !S || !V || !rank || dL <= 0 || dR <= 0 || chiL <= 0 || chiR <= 0) return HEFF_BAD_ARG;
    cudaStream_t s    = (cudaStream_t)stream;
    void        *base = nullptr;
    HEFF_TRY(stream_workspace(s, (size_t)schmidt_scratch_bytes(dL, dR, chiL, chiR, rank_max, sizeof(T)), &base));
    double te = 0;
    HEFF_TRY(schmidt_split(theta, dL, dR, chiL, chiR, rank_max, trunc_lim, U, S, V, rank, &te, base, s));
    if(trunc_err) *trunc_err = te;
    return HEFF_OK;
}

extern "C" int heff_svd_d(const double *A, int64_t rows, int64_t cols, int64_t rank_max, double trunc_lim, double *U, double *S, double *VT,
                          int64_t *rank, double *trunc_err, void *stream) {
    return svd_entry<double>(A, rows, cols, rank_max, trunc_lim, U, S, VT, rank, trunc_err, stream);
}

extern "C" int heff_svd_z(const heff_z *A, int64_t rows, int64_t cols, int64_t rank_max, double trunc_lim, heff_z *U, double *S, heff_z *VT,
                          int64_t *rank, double *trunc_err, void *stream) {
    return svd_entry<double2>(reinterpret_cast<const double2 *>(A), rows, cols, rank_max, trunc_lim, reinterpret_cast<double2 *>(U), S,
                              reinterpret_cast<double2 *>(VT), rank, trunc_err, stream);
}

extern "C" int heff_schmidt_d(const double *theta, int64_t dL, int64_t dR, int64_t chiL, int64_t chiR, int64_t rank_max, double trunc_lim, double *U,
                              double *S, double *V, int64_t *rank, double *trunc_err, void *stream) {
    return schmidt_entry<double>(theta, dL, dR, chiL, chiR, rank_max, trunc_lim, U, S, V, rank, trunc_err, stream);
}

extern "C" int heff_schmidt_z(const heff_z *theta, int64_t dL, int64_t dR, int64_t chiL, int64_t chiR, int64_t rank_max, double trunc_lim, heff_z *U,
                              double *S, heff_z *V, int64_t *rank, double *trunc_err, void *stream) {
    return schmidt_entry<double2>(reinterpret_cast<const double2 *>(theta), dL, dR, chiL, chiR, rank_max, trunc_lim, reinterpret_cast<double2 *>(U), S,
                                  reinterpret_cast<double2 *>(V), rank, trunc_err, stream);
}
