/*
 * heff_oracle.c -- CPU restatement of DMRG++'s H_eff hot path (see heff_oracle.h).
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA library, never part of it.
 * Parity with the reference's own outputs is unpinned (the reference cannot be
 * built here and ships no golden vectors for this path); the restatement is
 * pinned against independent answers in tests/.
 */
#include "heff_oracle.h"
#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define T double
#define CONJ(x) (x)
#define SFX d
#include "oracle_body.inc"
#undef T
#undef CONJ
#undef SFX

#define T double _Complex
#define CONJ(x) conj(x)
#define SFX z
#include "oracle_body.inc"
#undef T
#undef CONJ
#undef SFX

int oracle_matvec_d(double *res, const double *mps, const int64_t md[3], const double *mpo, const int64_t wd[4], const double *L,
                    const int64_t ld[3], const double *R, const int64_t rd[3], int branch) {
    return matvec_impl_d(res, mps, md, mpo, wd, L, ld, R, rd, branch);
}
int oracle_matvec_z(double *res, const double *mps, const int64_t md[3], const double *mpo, const int64_t wd[4], const double *L,
                    const int64_t ld[3], const double *R, const int64_t rd[3], int branch) {
    return matvec_impl_z((double _Complex *)res, (const double _Complex *)mps, md, (const double _Complex *)mpo, wd,
                         (const double _Complex *)L, ld, (const double _Complex *)R, rd, branch);
}
int oracle_expval_d(double *result, const double *mps, const int64_t md[3], const double *mpo, const int64_t wd[4], const double *L,
                    const int64_t ld[3], const double *R, const int64_t rd[3]) {
    double v = 0;
    int    rc = expval_impl_d(&v, mps, md, mpo, wd, L, ld, R, rd);
    result[0] = v;
    result[1] = 0;
    return rc;
}
int oracle_expval_z(double *result, const double *mps, const int64_t md[3], const double *mpo, const int64_t wd[4], const double *L,
                    const int64_t ld[3], const double *R, const int64_t rd[3]) {
    double _Complex v  = 0;
    int             rc = expval_impl_z(&v, (const double _Complex *)mps, md, (const double _Complex *)mpo, wd, (const double _Complex *)L, ld,
                                       (const double _Complex *)R, rd);
    result[0]          = creal(v);
    result[1]          = cimag(v);
    return rc;
}
int oracle_env_update_d(int side, double *out, const double *env, const int64_t ed[3], const double *mps, const int64_t md[3], const double *mpo,
                        const int64_t wd[4]) {
    return env_impl_d(side, out, env, ed, mps, md, mpo, wd);
}
int oracle_env_update_z(int side, double *out, const double *env, const int64_t ed[3], const double *mps, const int64_t md[3], const double *mpo,
                        const int64_t wd[4]) {
    return env_impl_z(side, (double _Complex *)out, (const double _Complex *)env, ed, (const double _Complex *)mps, md,
                      (const double _Complex *)mpo, wd);
}

/* The matrix of the matvec, H[(s',a',b'),(s,a,b)] = sum_{m,n} L[a,a',m] W[m,n,s,s'] R[b,b',n], so that y = H x
 * reproduces oracle_matvec_d for x = theta (contraction_tblis.cpp:277-290).  The reference's get_matrix
 * (oracle_get_matrix_*) is its transpose. */
int oracle_dense_heff_d(double *H, const int64_t md[3], const double *W, const int64_t wd[4], const double *L, const int64_t ld[3], const double *R,
                        const int64_t rd[3]) {
    const int64_t S = md[0], cL = md[1], cR = md[2], DL = wd[0], DR = wd[1];
    if(cL != ld[0] || cR != rd[0] || S != wd[2] || ld[2] != DL || rd[2] != DR) return 1;
    const int64_t N = S * cL * cR;
    for(int64_t b = 0; b < cR; b++)
        for(int64_t a = 0; a < cL; a++)
            for(int64_t s = 0; s < S; s++) {
                int64_t col = s + S * (a + cL * b);
                for(int64_t bp = 0; bp < cR; bp++)
                    for(int64_t ap = 0; ap < cL; ap++)
                        for(int64_t sp = 0; sp < S; sp++) {
                            double acc = 0;
                            for(int64_t n = 0; n < DR; n++)
                                for(int64_t m = 0; m < DL; m++)
                                    acc += L[a + cL * (ap + cL * m)] * W[m + DL * (n + DR * (s + S * sp))] * R[b + cR * (bp + cR * n)];
                            H[(sp + S * (ap + cL * bp)) + N * col] = acc;
                        }
            }
    return 0;
}

int oracle_get_matrix_d(double *M, const int64_t md[3], const double *W, const int64_t wd[4], const double *L, const int64_t ld[3], const double *R,
                        const int64_t rd[3]) {
    return get_matrix_impl_d(M, md, W, wd, L, ld, R, rd);
}
int oracle_get_matrix_z(double *M, const int64_t md[3], const double *W, const int64_t wd[4], const double *L, const int64_t ld[3], const double *R,
                        const int64_t rd[3]) {
    return get_matrix_impl_z((double _Complex *)M, md, (const double _Complex *)W, wd, (const double _Complex *)L, ld, (const double _Complex *)R,
                             rd);
}

/* IsingRandomField::get_mpo, IsingRandomField.cpp:122-129, Pauli matrices qm/spin/half.cpp:9-17.
 *   W[0,0]=I, W[1,0]=sz, W[2,0]=-h*sx - e_shift*I, W[2,1]=-J*sz, W[2,2]=I  (slices are [s, s'] matrices). */
void oracle_mpo_ising(double *W, double J, double h, double eshift) {
    memset(W, 0, sizeof(double) * 36);
#define WI(m, n, s, t) W[(m) + 3 * ((n) + 3 * ((s) + 2 * (t)))]
    const double id[2][2] = {{1, 0}, {0, 1}}, sx[2][2] = {{0, 1}, {1, 0}}, sz[2][2] = {{1, 0}, {0, -1}};
    for(int s = 0; s < 2; s++)
        for(int t = 0; t < 2; t++) {
            WI(0, 0, s, t) = id[s][t];
            WI(1, 0, s, t) = sz[s][t];
            WI(2, 0, s, t) = -h * sx[s][t] - eshift * id[s][t];
            WI(2, 1, s, t) = -J * sz[s][t];
            WI(2, 2, s, t) = id[s][t];
        }
#undef WI
}

/* MpoSite.cpp:449-500 (parity_shift_sign == 0 branch) and apply_edge_left: keep row mL-1 -> dims [1, mR, d, d]. */
void oracle_mpo_edge_left(double *Wout, const double *W, int64_t mL, int64_t mR, int64_t d) {
    for(int64_t t = 0; t < d; t++)
        for(int64_t s = 0; s < d; s++)
            for(int64_t n = 0; n < mR; n++) Wout[n + mR * (s + d * t)] = W[(mL - 1) + mL * (n + mR * (s + d * t))];
}
/* get_MPO_edge_right / apply_edge_right: keep column 0 -> dims [mL, 1, d, d]. */
void oracle_mpo_edge_right(double *Wout, const double *W, int64_t mL, int64_t mR, int64_t d) {
    for(int64_t t = 0; t < d; t++)
        for(int64_t s = 0; s < d; s++)
            for(int64_t m = 0; m < mL; m++) Wout[m + mL * (s + d * t)] = W[m + mL * (0 + mR * (s + d * t))];
}
void oracle_mpo_merge_d(double *W2, const double *WA, const int64_t dA[4], const double *WB, const int64_t dB[4]) {
    merge_impl_d(W2, WA, dA, WB, dB);
}
void oracle_mpo_merge_z(double *W2, const double *WA, const int64_t dA[4], const double *WB, const int64_t dB[4]) {
    merge_impl_z((double _Complex *)W2, (const double _Complex *)WA, dA, (const double _Complex *)WB, dB);
}
void oracle_mpo_square_d(double *Wsq, const double *W, const int64_t dims[4]) { square_impl_d(Wsq, W, dims); }
void oracle_mpo_square_z(double *Wsq, const double *W, const int64_t dims[4]) {
    square_impl_z((double _Complex *)Wsq, (const double _Complex *)W, dims);
}

/* svd.cpp:257-280: truncation_errors[s] = ||S[s:]||; rank = #(errors >= lim), clipped to rank_max, raised to rank_min. */
int64_t oracle_truncation_rank(const double *S, int64_t n, int64_t rank_max, int64_t rank_min, double lim, double *trunc_err) {
    double *err = (double *)malloc(sizeof(double) * (size_t)(n + 1));
    for(int64_t s = 0; s <= n; s++) {
        double acc = 0;
        for(int64_t i = s; i < n; i++) acc += S[i] * S[i];
        err[s] = sqrt(acc);
    }
    int64_t rank = 0;
    for(int64_t s = 0; s <= n; s++) rank += (err[s] >= lim) ? 1 : 0;
    int64_t rank_lim = n;
    if(rank_max > 0) rank_lim = rank_max < n ? rank_max : n;
    if(rank > rank_lim) rank = rank_lim;
    if(rank_min > 0) {
        int64_t rmin = rank_min < n ? rank_min : n;
        if(rank < rmin) rank = rmin;
    }
    if(rank <= 0) {
        free(err);
        return -1;
    }
    if(trunc_err) *trunc_err = err[rank];
    free(err);
    return rank;
}

/* measure.cpp:134-138: S_vN = |-sum_i L_i^2 log(L_i^2)| */
double oracle_entropy(const double *S, int64_t n) {
    double acc = 0;
    for(int64_t i = 0; i < n; i++) {
        double p = S[i] * S[i];
        if(p > 0) acc += p * log(p);
    }
    return fabs(-acc);
}
