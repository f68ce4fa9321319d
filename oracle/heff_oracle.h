/*
 * heff_oracle.h -- CPU restatement of DMRG++'s effective-Hamiltonian hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker that the CUDA path is
 * compared against; it is never linked into, called by, or used as a fallback
 * for the product library (dmrg_b200/libheff_b200.so).  Only tests/, the smoke
 * check in __graft_entry__.py and the cpu_baseline leg of bench.py load it.
 *
 * Parity status: the reference (DavidAce/DMRG v3.5.0) cannot be built here
 * (Eigen 3.4.0, PRIMME, arpack-ng, LAPACKE, h5pp are absent and there is no
 * network) and its own tests hold no golden vectors for this path, so parity
 * with the reference's *outputs* is UNPINNED.  The restatement follows the
 * reference's contraction sequences index-for-index (file:line cited at each
 * function) and is pinned instead against independent answers: an independent
 * numpy einsum restatement, the dense H_eff matrix, exact diagonalisation of
 * the full chain and the free-fermion solution of the transverse-field Ising
 * chain (tests/golden/make_golden.py).
 *
 * Layout (identical to Eigen's default column-major Tensor storage):
 *   mps   [spin, chiL, chiR]      element (s,a,b)   at s + spin*(a + chiL*b)
 *   mpo   [mL, mR, s_in, s_out]   element (m,n,s,t) at m + mL*(n + mR*(s + spin*t))
 *   env   [chi, chi, m]           element (a,a',m)  at a + chi*(a' + chi*m)
 * Complex data is interleaved (re, im) = std::complex<double> = C99 double _Complex.
 */
#ifndef HEFF_ORACLE_H
#define HEFF_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

/* y = H_eff * theta, both branches of contraction_tblis.cpp:277-290.
 * branch: -1 = choose like the reference (chiL >= chiR -> L first), 0 = L first, 1 = R first. */
int oracle_matvec_d(double *res, const double *mps, const int64_t mps_dims[3], const double *mpo, const int64_t mpo_dims[4],
                    const double *envL, const int64_t envL_dims[3], const double *envR, const int64_t envR_dims[3], int branch);
int oracle_matvec_z(double *res, const double *mps, const int64_t mps_dims[3], const double *mpo, const int64_t mpo_dims[4],
                    const double *envL, const int64_t envL_dims[3], const double *envR, const int64_t envR_dims[3], int branch);

/* <theta| W |theta> with envs, contraction_tblis.cpp:64-69 (result[0]=re, result[1]=im). */
int oracle_expval_d(double *result, const double *mps, const int64_t mps_dims[3], const double *mpo, const int64_t mpo_dims[4],
                    const double *envL, const int64_t envL_dims[3], const double *envR, const int64_t envR_dims[3]);
int oracle_expval_z(double *result, const double *mps, const int64_t mps_dims[3], const double *mpo, const int64_t mpo_dims[4],
                    const double *envL, const int64_t envL_dims[3], const double *envR, const int64_t envR_dims[3]);

/* EnvBase::build_block, EnvBase.cpp:109-112 (side 'L') and :146-149 (side 'R'). */
int oracle_env_update_d(int side, double *out, const double *env, const int64_t env_dims[3], const double *mps, const int64_t mps_dims[3],
                        const double *mpo, const int64_t mpo_dims[4]);
int oracle_env_update_z(int side, double *out, const double *env, const int64_t env_dims[3], const double *mps, const int64_t mps_dims[3],
                        const double *mpo, const int64_t mpo_dims[4]);

/* Dense matrix of the matvec: H[(s',a',b'), (s,a,b)] column-major (y = H theta), rows = spin*chiL*chiR. */
int oracle_dense_heff_d(double *H, const int64_t mps_dims[3], const double *mpo, const int64_t mpo_dims[4], const double *envL,
                        const int64_t envL_dims[3], const double *envR, const int64_t envR_dims[3]);
/* MatVecMPO::get_tensor/get_matrix (matvec_mpo.cpp:313-332): M[(s,a,b), (s',a',b')] column-major, the
 * transpose of the dense matvec matrix above.  _z: interleaved complex buffers. */
int oracle_get_matrix_d(double *M, const int64_t mps_dims[3], const double *mpo, const int64_t mpo_dims[4], const double *envL,
                        const int64_t envL_dims[3], const double *envR, const int64_t envR_dims[3]);
int oracle_get_matrix_z(double *M, const int64_t mps_dims[3], const double *mpo, const int64_t mpo_dims[4], const double *envL,
                        const int64_t envL_dims[3], const double *envR, const int64_t envR_dims[3]);

/* IsingRandomField::get_mpo (IsingRandomField.cpp:122-129): W[3,3,2,2] real. */
void oracle_mpo_ising(double *W, double J, double h_field, double energy_shift);
/* Edge-applied boundary MPOs (MpoSite.cpp:449-500, no parity shift): left keeps row D-1, right keeps column 0. */
void oracle_mpo_edge_left(double *Wout, const double *W, int64_t mL, int64_t mR, int64_t d);
void oracle_mpo_edge_right(double *Wout, const double *W, int64_t mL, int64_t mR, int64_t d);
/* Two-site merge, matvec_mpos.cpp:104-119: W2[mL, mR', s1+d1*s2, t1+d1*t2] = sum_c WA[mL,c,s1,t1] WB[c,mR',s2,t2]. */
void oracle_mpo_merge_d(double *W2, const double *WA, const int64_t dA[4], const double *WB, const int64_t dB[4]);
void oracle_mpo_merge_z(double *W2, const double *WA, const int64_t dA[4], const double *WB, const int64_t dB[4]);
/* Uncompressed MPO squared, MpoSite.cpp:57-70: Wsq[(m + D*m~), (n + D*n~), s, s''] = sum_s' W[m,n,s,s'] conj(W)[m~,n~,s',s'']. */
void oracle_mpo_square_d(double *Wsq, const double *W, const int64_t dims[4]);
void oracle_mpo_square_z(double *Wsq, const double *W, const int64_t dims[4]);

/* svd::solver::get_rank_from_truncation_error (svd.cpp:257-280). S sorted descending, normalised.
 * Returns rank (>0) or -1 when the rule yields rank <= 0 (the reference throws there). */
int64_t oracle_truncation_rank(const double *S, int64_t n, int64_t rank_max, int64_t rank_min, double trunc_lim, double *trunc_err);
/* Von Neumann entropy -sum S^2 log S^2 (natural log), measure.cpp:134-138. */
double oracle_entropy(const double *S, int64_t n);

#ifdef __cplusplus
}
#endif
#endif
