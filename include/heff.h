/*
 * heff.h -- C ABI of heff_b200, a B200-native (sm_100a) implementation of the
 * effective-Hamiltonian hot path of DMRG++ (DavidAce/DMRG v3.5.0).
 *
 * Every entry point is extern "C", takes plain pointers and sizes, returns an
 * int status (heff_status) and never throws.  Tensors keep the reference's
 * layout (Eigen column-major):
 *   mps   [spin, chiL, chiR]       (s,a,b)   at s + spin*(a + chiL*b)
 *   mpo   [mL, mR, s_in, s_out]    (m,n,s,t) at m + mL*(n + mR*(s + spin*t))
 *   env   [chi, chi, m]            (a,a',m)  at a + chi*(a' + chi*m)
 * Complex scalars are interleaved (re, im) pairs (heff_z), layout-compatible
 * with std::complex<double> (the reference's cx64) and C99 double _Complex.
 * Unless a name says _host, pointers are device pointers; `stream` is a
 * cudaStream_t (NULL = legacy default stream).  Calls are stream-ordered and
 * do not synchronise the host.
 */
#ifndef HEFF_B200_H
#define HEFF_B200_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    double re, im;
} heff_z;

typedef enum {
    HEFF_OK            = 0,
    HEFF_BAD_SHAPE     = 1, /* dimension mismatch (reference: except::runtime_error, contraction_tblis.cpp:230-234) */
    HEFF_NAN_INPUT     = 2,
    HEFF_OOM           = 3,
    HEFF_TIMEOUT       = 4,
    HEFF_NOT_CONVERGED = 5,
    HEFF_CUDA_ERROR    = 6,
    HEFF_BAD_ARG       = 7,
    HEFF_NO_DEVICE     = 8
} heff_status;

typedef enum { HEFF_F64 = 0, HEFF_C128 = 1 } heff_dtype;
typedef enum { HEFF_MEM_DEVICE = 0, HEFF_MEM_HOST = 1 } heff_mem;
typedef enum { HEFF_PREC_FP64 = 0, HEFF_PREC_MIXED = 1 } heff_precision;
typedef enum { HEFF_FP64_DMMA = 0, HEFF_FP64_INT8 = 1 } heff_fp64_engine;

/* Human-readable description of the last error raised on the calling thread. */
const char *heff_last_error(void);
/* Library version string. */
const char *heff_version(void);

/* ---------------------------------------------------------------------------
 * Contraction kernels
 * ------------------------------------------------------------------------- */

/* res = H_eff * mps.  Replaces tools::common::contraction::matrix_vector_product
 * (source/tools/common/contraction.h:31-36, contraction_tblis.cpp:213-292), real
 * (fp64) and complex (cx64) instantiations.  res must not alias mps.  Scratch is
 * taken from a per-device workspace that grows on demand (a growth allocates,
 * so a first call at a new size should come before any stream capture). */
int heff_matvec_d(double *res, const double *mps, const int64_t mps_dims[3], const double *mpo, const int64_t mpo_dims[4], const double *envL,
                  const int64_t envL_dims[3], const double *envR, const int64_t envR_dims[3], void *stream);
int heff_matvec_z(heff_z *res, const heff_z *mps, const int64_t mps_dims[3], const heff_z *mpo, const int64_t mpo_dims[4], const heff_z *envL,
                  const int64_t envL_dims[3], const heff_z *envR, const int64_t envR_dims[3], void *stream);

/* res = H_eff * mps with a chain of nmpo site MPOs (mpos[i] device pointers, unshuffled
 * [D_{i-1}, D_i, d_i, d_i], dims 4 per MPO in mpo_dims), replacing the multi-MPO
 * matrix_vector_product (contraction_tblis.cpp:307-420, used for more than 5 sites,
 * matvec_mpos.cpp:104-123): the MPOs are applied one at a time, never merged;
 * mps [prod d_i, chiL, chiR] with site 1's index fastest.  The reference also
 * accepts MPOs pre-shuffled {2,3,0,1}; this entry point takes them unshuffled. */
int heff_matvec_multi_d(double *res, const double *mps, const int64_t mps_dims[3], int nmpo, const double *const *mpos, const int64_t *mpo_dims,
                        const double *envL, const int64_t envL_dims[3], const double *envR, const int64_t envR_dims[3], void *stream);
int heff_matvec_multi_z(heff_z *res, const heff_z *mps, const int64_t mps_dims[3], int nmpo, const heff_z *const *mpos, const int64_t *mpo_dims,
                        const heff_z *envL, const int64_t envL_dims[3], const heff_z *envR, const int64_t envR_dims[3], void *stream);

/* Same product and arguments as heff_matvec_d, but allocating no device memory.
 * No counterpart in the reference: it exists for callers that cannot let a
 * library call cudaMalloc (a process that has already split all device memory
 * among its own pools, or that cannot afford the device-wide synchronisation a
 * cudaMalloc/cudaFree implies).  Scratch comes from one fixed 32 MiB array
 * inside the library (held on every GPU that loads the library until exit);
 * calls needing more return HEFF_BAD_SHAPE (real two-site D=3 fits up to
 * chi=367).  All calls on a device share that array: calls that may overlap on
 * the GPU race, so serialise them.  The first call on a device looks up the
 * array's device address and keeps it for the life of the process; make it
 * before any stream capture.  A cudaDeviceReset of that device makes the kept
 * address (and heff_matvec_d's kept workspaces) stale: do not call the library
 * on a device again after resetting it in the same process. */
int heff_matvec_d_noalloc(double *res, const double *mps, const int64_t mps_dims[3], const double *mpo, const int64_t mpo_dims[4],
                          const double *envL, const int64_t envL_dims[3], const double *envR, const int64_t envR_dims[3], void *stream);

/* <mps| mpo |mps> with environments.  Replaces
 * tools::common::contraction::expectation_value (contraction.h:18-22,
 * contraction_tblis.cpp:30-87).  result is a HOST pointer: result[0]=re,
 * result[1]=im; the call synchronises `stream`. */
int heff_expval_d(double *result, const double *mps, const int64_t mps_dims[3], const double *mpo, const int64_t mpo_dims[4], const double *envL,
                  const int64_t envL_dims[3], const double *envR, const int64_t envR_dims[3], void *stream);
int heff_expval_z(double *result, const heff_z *mps, const int64_t mps_dims[3], const heff_z *mpo, const int64_t mpo_dims[4], const heff_z *envL,
                  const int64_t envL_dims[3], const heff_z *envR, const int64_t envR_dims[3], void *stream);

/* ---------------------------------------------------------------------------
 * Environment update
 * ------------------------------------------------------------------------- */

/* out = EnvBase::build_block(env, mps, mpo) (source/tensors/site/env/EnvBase.cpp:67-151):
 *   side 0 ('L', :109-112): out[b,b',n] = sum env[a,a',m] mps[s,a,b] conj(mps)[s',a',b'] mpo[m,n,s,s']
 *   side 1 ('R', :146-149): out[a,a',m] = sum env[b,b',n] mps[s,a,b] conj(mps)[s',a',b'] mpo[m,n,s,s']
 * env [chi,chi,D] (chi = mps dim 1 for L, dim 2 for R), mps [d,chiL,chiR], mpo [DL,DR,d,d];
 * out is [chiR,chiR,DR] (L) or [chiL,chiL,DL] (R).  The reference keeps environments complex
 * (EnvBase.h:26); the _d form is for environments whose imaginary part is identically zero.
 * Dimension checks follow EnvBase.cpp:93-101 / :130-138 (HEFF_BAD_SHAPE). */
int heff_env_update_d(int side, double *out, const double *env, const int64_t env_dims[3], const double *mps, const int64_t mps_dims[3],
                      const double *mpo, const int64_t mpo_dims[4], void *stream);
int heff_env_update_z(int side, heff_z *out, const heff_z *env, const int64_t env_dims[3], const heff_z *mps, const int64_t mps_dims[3],
                      const heff_z *mpo, const int64_t mpo_dims[4], void *stream);

/* Subspace-expansion term of one-site DMRG, replacing EnvBase::get_expansion_term(mps,
 * mpo, alpha) (source/tensors/site/env/EnvBase.cpp:303-364), no conjugation:
 *   side 0 ('L'): P[s',a',b + chiR*n] = alpha sum env[a,a',m] mps[s,a,b] mpo[m,n,s,s'],
 *                 P [spin, chiL, chiR*DR], env [chiL,chiL,DL]
 *   side 1 ('R'): P_flat[s' + spin*(b' + chiR*(a + chiL*m))] = alpha sum env[b,b',n] mps[s,a,b] mpo[m,n,s,s'],
 *                 P [spin, chiL*DL, chiR] in the reference's memory order (its shuffle
 *                 {3,0,1,2} of [b',a,m,s'] then a reshape), env [chiR,chiR,DR]
 * alpha == 0 writes zeros; a NaN alpha returns HEFF_NAN_INPUT (the reference throws).
 * Device pointers, stream-ordered. */
int heff_expansion_term_d(int side, double *P, const double *env, const int64_t env_dims[3], const double *mps, const int64_t mps_dims[3],
                          const double *mpo, const int64_t mpo_dims[4], double alpha, void *stream);
int heff_expansion_term_z(int side, heff_z *P, const heff_z *env, const int64_t env_dims[3], const heff_z *mps, const int64_t mps_dims[3],
                          const heff_z *mpo, const int64_t mpo_dims[4], double alpha, void *stream);

/* ---------------------------------------------------------------------------
 * SVD truncation
 * ------------------------------------------------------------------------- */

/* Truncated SVD A = U S VT of a rows x cols column-major matrix, replacing
 * svd::solver::do_svd_ptr (source/math/svd/svd.cpp:113-206; geauto resolves to
 * LAPACK ?gesdd for the two-site split).  FP64 one-sided block Jacobi on the
 * device.  The rank follows get_rank_from_truncation_error (svd.cpp:257-280):
 * keep singular values while the norm of the discarded tail stays >= trunc_lim,
 * at most rank_max (<= 0: no limit).  U [rows x k], S [k] (not normalised, like
 * svd_lapacke.cpp:457), VT [k x cols] are device buffers sized for
 * k = min(rows, cols, rank_max); *rank and *trunc_err are host outputs.
 * Synchronises the stream. */
int heff_svd_d(const double *A, int64_t rows, int64_t cols, int64_t rank_max, double trunc_lim, double *U, double *S, double *VT, int64_t *rank,
               double *trunc_err, void *stream);
/* Two-site Schmidt split, replacing svd::solver::schmidt_multisite
 * (source/math/svd.h:189-220): theta [dL*dR, chiL, chiR] is reshaped to
 * [dL, dR, chiL, chiR], shuffled {0,2,1,3} and decomposed as a (dL chiL) x
 * (dR chiR) matrix.  Outputs U [dL, chiL, k], S [k] normalised to unit norm
 * (svd.h:172), V [dR, k, chiR] (svd.h:173).  Synchronises the stream. */
int heff_schmidt_d(const double *theta, int64_t dL, int64_t dR, int64_t chiL, int64_t chiR, int64_t rank_max, double trunc_lim, double *U,
                   double *S, double *V, int64_t *rank, double *trunc_err, void *stream);
/* Complex128 forms of the two above (the reference instantiates svd::solver for
 * cx64 = std::complex<double>, svd.cpp:208-217): A = U S VT with VT = V^H, the
 * LAPACK zgesdd convention; same rank rule, layouts and synchronisation. */
int heff_svd_z(const heff_z *A, int64_t rows, int64_t cols, int64_t rank_max, double trunc_lim, heff_z *U, double *S, heff_z *VT, int64_t *rank,
               double *trunc_err, void *stream);
int heff_schmidt_z(const heff_z *theta, int64_t dL, int64_t dR, int64_t chiL, int64_t chiR, int64_t rank_max, double trunc_lim, heff_z *U,
                   double *S, heff_z *V, int64_t *rank, double *trunc_err, void *stream);

/* ---------------------------------------------------------------------------
 * Operator object: MatVecMPOS<T> / MatVecMPO<T>
 * (source/math/eig/matvec/matvec_mpos.h:23-180, matvec_mpo.h:18-103)
 * ------------------------------------------------------------------------- */
typedef struct heff_op heff_op;

/* Constructor: MatVecMPOS<T>(mpos, env_pair) (matvec_mpos.cpp:40-130).  The
 * nsites site MPOs (each [mL, mR, d, d]) are merged into one
 * [mL0, mR_last, prod d, prod d] MPO as in matvec_mpos.cpp:104-119 (nsites <= 5);
 * with more sites they are kept apart and applied one at a time (as
 * matvec_mpos.cpp:120-123 / contraction_tblis.cpp:307-420; FP64 only, no
 * heff_op_get_matrix).
 * envL [chiL, chiL, mL0], envR [chiR, chiR, mR_last].  Buffers live in `where`
 * (host or device); the operator keeps its own device copies, laid out for the
 * kernels.  precision selects the FP64 tensor-core path or the mixed split
 * path (HEFF_PREC_MIXED: bulk matvec in split-BF16 with FP32 accumulation). */
int heff_op_create(heff_op **op, heff_dtype dtype, int nsites, const void *const *mpos, const int64_t *mpo_dims /* nsites x 4 */,
                   const void *envL, const int64_t envL_dims[3], const void *envR, const int64_t envR_dims[3], heff_mem where,
                   heff_precision precision, void *stream);
int heff_op_destroy(heff_op *op);
/* rows() = spin * chiL * chiR (matvec_mpos.h: rows()). */
int64_t heff_op_rows(const heff_op *op);
/* shape of the mps this operator acts on: {spin, chiL, chiR}. */
int heff_op_shape(const heff_op *op, int64_t shape[3]);
/* MatVecMPOS::MultAx(T* in, T* out) (matvec_mpos.cpp:963-974), device buffers. */
int heff_op_multax(heff_op *op, const void *x, void *y);
/* ARPACK-style alias of heff_op_multax (the eigensolver's perform_op(x, y)). */
int heff_perform_op(heff_op *op, const void *x, void *y);
/* PRIMME form MultAx(x, ldx, y, ldy, blockSize, primme, err) (matvec_mpos.cpp:976-984):
 * block_size columns of length rows(), leading dims ldx / ldy (elements). */
int heff_op_multax_block(heff_op *op, const void *x, int64_t ldx, void *y, int64_t ldy, int block_size);
/* MultAx with HOST buffers: copies x in, applies H_eff, copies y out, synchronises. */
int heff_op_multax_host(heff_op *op, const void *x_host, void *y_host);
int heff_op_set_stream(heff_op *op, void *stream);
int heff_op_set_precision(heff_op *op, heff_precision precision);
/* Engine of the operator's FP64-accurate matvecs (HEFF_PREC_FP64 applies and the
 * FP64 refinement steps of mixed eigensolves): HEFF_FP64_DMMA, the FP64 tensor
 * cores (default); or HEFF_FP64_INT8, both GEMMs emulated on the INT8 tensor
 * cores with `nslices` digit slices (0 = 7; 3..8) as in heff_gemm_i8_emu --
 * normwise error a few 2^-48 relative at 7 slices.  Operators over more than 5
 * site MPOs, and shapes whose GEMMs exceed the exact-INT32 range, keep DMMA.
 * No counterpart in the reference (its matvec is Eigen FP64). */
int heff_op_set_fp64_engine(heff_op *op, int engine, int nslices);
/* Number of matvecs applied so far (MatVecMPOS::num_mv). */
int64_t heff_op_num_mv(const heff_op *op);
/* Stage timing (the reference's tid:: timers around MultAx, matvec_mpo.h:70-102):
 * when enabled, every FP64 matvec records CUDA events around its four kernels
 * (layout, GEMM 1, MPO mix, GEMM 2).  heff_op_stage_times synchronises the op's
 * stream and returns the summed milliseconds per stage and the matvec count. */
int heff_op_set_profiling(heff_op *op, int enable);
/* CUDA graphs for the FP64 matvec (off by default, or on for every operator when the
 * environment variable HEFF_GRAPHS=1; no counterpart in the reference):
 * on an operator created with a non-default stream, the first product of a shape
 * runs as plain kernel launches and is recorded as a graph; later products of that
 * shape replay it with the input and output retargeted (one launch instead of
 * four to six).  Results are bitwise identical either way.  0 turns it off. */
int heff_op_set_graphs(heff_op *op, int enable);
int heff_op_stage_times(heff_op *op, double ms[4], int64_t *count, int reset);
/* Device-side status of the operator's tensor-core pipeline: *code = 0 when every
 * bounded wait in the tensor-core kernels completed, nonzero when one timed out
 * (the kernel then skipped its work and returned); 5 when the INT8 engine met a
 * non-finite input (or one of magnitude >= 2^1022).  Synchronises the stream. */
int heff_op_device_error(heff_op *op, int *code);
/* Diagonal of H_eff, replacing MatVecMPOS::get_diagonal_new(0, ...)
 * (source/math/eig/matvec/matvec_mpos.cpp:300-407): diag[s + S(a + chiL b)] =
 * sum_{m,n} envL[a,a,m] W[m,n,s,s] envR[b,b,n] into a device buffer of rows()
 * elements of the operator's dtype (stream-ordered).  Computed once per operator
 * (and per rebind) like CalcPc's readyCalcPc flag. */
int heff_op_diagonal(heff_op *op, void *diag_out);
/* Dense effective Hamiltonian, replacing MatVecMPO(S)::get_matrix (source/math/eig/
 * matvec/matvec_mpo.cpp:313-332, matvec_mpos.cpp:1570-1588): M[(s,a,b), (s',a',b')] =
 * sum_{m,n} envL[a,a',m] W[m,n,s,s'] envR[b,b',n], rows() x rows() column-major in
 * the operator's dtype.  As in the reference the row index is the matvec's input
 * index, so M is the transpose of the matrix applied by MultAx (its complex
 * conjugate when H_eff is Hermitian).  Device buffer, stream-ordered. */
int heff_op_get_matrix(heff_op *op, void *M_out);
/* All eigenpairs of a Hermitian n x n device matrix (lda >= n), replacing the dense
 * eig::solver path (LAPACK ?syevr / ?heevd on get_matrix, used by the reference for
 * problem sizes <= eig_max_size = 4096, AlgorithmFinite.cpp:318): evals (device, n
 * doubles) ascending, evecs (device, n x n, leading dimension n) the matching
 * orthonormal eigenvectors.  FP64 one-sided Jacobi on the Gershgorin-shifted
 * positive-definite matrix; n <= 16384.  Synchronises the stream. */
int heff_dense_eig(heff_dtype dtype, int64_t n, const void *A, int64_t lda, double *evals, void *evecs, void *stream);
/* Jacobi preconditioner, replacing MatVecMPOS::MultPc(T*, T*, T shift)
 * (matvec_mpos.cpp:1349-1416).  Block size 1 (the default): y = x / (diag - shift),
 * the denominator kept >= 1e-10 max(|shift|, 1) in magnitude.  Block size bs > 1
 * (jcbMaxBlockSize, CalcPc matvec_mpos.cpp:1087-1240): the rows are cut into
 * consecutive blocks of bs (the last one shorter), each block B = H[blk,blk] - shift I
 * is formed and inverted on the device at the shift of the first call after a create
 * or rebind (later shifts reuse it, like readyCalcPc), and y_blk = B^-1 x_blk.
 * Device buffers, stream-ordered. */
int heff_op_multpc(heff_op *op, const void *x, void *y, double shift);
/* Block size of the Jacobi preconditioner, replacing MatVecMPOS::set_jcbMaxBlockSize
 * (matvec_mpos.h:147): 1 = diagonal; 2 .. HEFF_JCB_MAX_BLOCK = block Jacobi (the
 * inverted blocks take rows() * bs elements of device memory).  A change takes effect
 * at the next MultPc. */
#define HEFF_JCB_MAX_BLOCK 1024
int heff_op_set_jacobi_blocksize(heff_op *op, int64_t block_size);
/* Number of block-Jacobi pivots that were below 1e-14 of their block's largest entry
 * and floored there (0 for a well-conditioned preconditioner).  Synchronises the stream. */
int heff_op_jacobi_singular(heff_op *op, int *count);

/* ---------------------------------------------------------------------------
 * BF16 tensor-core GEMM used by the mixed-precision path (tcgen05 + TMA)
 * ------------------------------------------------------------------------- */
/* C[m + M*n] (float, column-major) = sum_k A[m*K + k] * B[n*K + k]; A (M x K) and
 * B (N x K) bf16 row-major (K contiguous), K a multiple of 8, 16-byte aligned
 * buffers.  No counterpart in the reference (its matvec is FP64/cx64 only); exposed
 * so the split-precision building block can be validated on its own.
 * Synchronises the stream; HEFF_TIMEOUT if a pipeline wait timed out. */
int heff_gemm_bf16_f32(const void *A, const void *B, float *C, int64_t M, int64_t N, int64_t K, void *stream);

/* FP64-accurate GEMM on the INT8 tensor cores (tcgen05 kind::i8, exact INT32
 * accumulation): C[m + M*n] = sum_k A[m*K + k] * B[n*K + k] (no conjugation),
 * dtype HEFF_F64 or HEFF_C128, device buffers, A (M x K) and B (N x K) with K
 * contiguous, C column-major.  Each row is scaled by a power of two and split
 * into `nslices` signed 7-bit digit planes (0 = default 7, at most 8); digit
 * products of equal weight are summed exactly and the weights combined in FP64,
 * so the normwise error is a few 2^-(7*nslices-1) of |A||B| (2^-48 at 7).  No
 * counterpart in the reference (its products are Eigen FP64); exposed so the
 * emulated-FP64 building block can be validated on its own.  Synchronises the
 * stream; HEFF_NAN_INPUT for a non-finite entry (or one of magnitude >= 2^1022;
 * C is then NaN, as an FP64 product would be),
 * HEFF_BAD_SHAPE when K is too long for exact INT32 sums (K' * nslices >= 2^19,
 * K' = round16(K), doubled for complex), HEFF_TIMEOUT if a pipeline wait timed out. */
int heff_gemm_i8_emu(int dtype, const void *A, const void *B, void *C, int64_t M, int64_t N, int64_t K, int nslices, void *stream);
/* Tile width of the INT8 emulated-FP64 GEMMs: 128, 192 or 256 columns; 0 for the
 * cost model (fewest waves weighted by measured per-width costs); 1 (the default)
 * for the autotuner: the first GEMM of each shape runs once with every width,
 * timed with CUDA events on its stream (which it synchronises then), and the
 * fastest width is cached for that shape.  The initial value comes from the
 * environment variable HEFF_I8_BN.  Results do not depend on it (every width sums
 * the same exact level products in the same order).  Returns the previous
 * setting, or -1 for an invalid value.  Process-wide tuning knob; no counterpart
 * in the reference. */
int heff_i8_set_tile_width(int bn);
/* Kernels launched so far by the FP64 matvec path (its permutation and MPO mix) and by every DMMA
 * GEMM (with its tail-split reduction), graph replays included, process-wide; read it around a
 * timed region of matvecs to count their launches.  No counterpart in the reference. */
int64_t heff_matvec_launches(void);
/* Number of GEMM shapes the INT8 tile-width autotuner has timed so far. */
int heff_i8_tuned_shapes(void);

/* Tail split of the FP64 (DMMA) GEMMs of the matvec: when a GEMM's tiles leave
 * the last wave of the device partly empty, the tiles of that wave are split
 * along K into pieces whose partial tiles a second kernel sums in piece order.
 * mode 0 = off, 1 = automatic (a cost model of waves, partial traffic and the
 * extra launch; default), 2..16 = that many pieces whenever a wave is partial.
 * The initial value comes from the environment variable HEFF_GEMM_SPLIT.  Results
 * are deterministic for a given mode and device but differ from the unsplit
 * product at the rounding level.  Returns the previous mode, or -1 for an invalid
 * one.  Process-wide tuning knob; no counterpart in the reference. */
int heff_gemm_set_tail_split(int mode);

/* ---------------------------------------------------------------------------
 * Eigensolver (the caller side of MultAx: eig::solver, source/math/eig/solver.h:15-88)
 * ------------------------------------------------------------------------- */
typedef enum { HEFF_RITZ_SA = 0, HEFF_RITZ_LA = 1, HEFF_RITZ_TARGET = 2 } heff_ritz;

typedef struct {
    int     ritz;        /* heff_ritz: smallest / largest algebraic, or closest to `target` (interior:
                            at rows() <= 2048 solved densely, get_matrix + heff_dense_eig, as the
                            reference's dense path for small problems, AlgorithmFinite.cpp:318) */
    double  target;      /* target eigenvalue for HEFF_RITZ_TARGET */
    double  tol;         /* ||H x - theta x|| <= tol * ||H||_est (PRIMME eps, solver_primme.cpp:364); default 1e-12 */
    int     max_basis;   /* Davidson basis size (<= 128), default 24 */
    int     min_basis;   /* vectors kept at a thick restart, default 8 */
    int64_t max_matvecs; /* default 20000 */
    int     mixed;       /* 1: when the operator is HEFF_PREC_MIXED, split-BF16 phase then FP64 refinement */
    double  mixed_tol;   /* relative residual at which the mixed phase hands over, default 1e-5 */
    int     inner_iters; /* CG iterations of one refinement correction (mixed operator), default 30 */
    double  inner_tol;   /* relative CG residual that ends a correction, default 1e-3 */
    int64_t seed;        /* start vector seed when x0 is NULL */
    int     precond;     /* 0 (default): Krylov expansion A v_last;  1: Jacobi-preconditioned
                            Davidson, expansion (diag - theta)^-1 r (PRIMME with MultPc,
                            optimize_folded_spectrum.cpp:303-304); FP64 operators */
} heff_eig_config;

typedef struct {
    double  eigval, resnorm, anorm, seconds;
    int64_t num_mv, num_mv_fp64, num_mv_mixed, num_mv_phase1;
    int     iters, restarts, refine_steps, converged;
} heff_eig_result;

void heff_eig_config_default(heff_eig_config *cfg);
/* One extremal/interior eigenpair of the operator (Davidson, thick restart, FP64 CGS2
 * re-orthogonalisation and Rayleigh-Ritz).  x0: device start vector or NULL; x_out:
 * device output (normalised), may be NULL.  Returns HEFF_NOT_CONVERGED (result still
 * filled) when max_matvecs is reached first.  Synchronises the operator's stream. */
int heff_eigs(heff_op *op, const heff_eig_config *cfg, const void *x0, void *x_out, heff_eig_result *res);

/* ---------------------------------------------------------------------------
 * Minimal two-site DMRG sweep driver over the hot path (random-field Ising chain
 * H = -sum J sz_i sz_{i+1} - sum h_i sx_i, IsingRandomField.cpp:93-136, open chain,
 * real FP64).  Stands in for the caller layer (fdmrg::update_state, fdmrg.cpp:282-360)
 * so whole calculations can run and be checked; not a port of the algorithm layer.
 * ------------------------------------------------------------------------- */
typedef struct {
    int           L;
    double        J;
    const double *h;                     /* host array of L fields */
    int64_t       chi_max;               /* bond dimension limit (svd rank_max) */
    int           sweeps;                /* full left-right-left sweeps */
    double        trunc_lim;             /* svd truncation limit (svd.cpp:257-280), default 1e-12 */
    double        eig_tol;               /* eigensolver tolerance, default 1e-12 */
    int           ritz;                  /* heff_ritz */
    double        target;                /* target for HEFF_RITZ_TARGET */
    int           precision;             /* heff_precision of the matvecs */
    int64_t       seed;                  /* random product-state initialisation */
    double        energy_shift_per_site; /* MPO energy shift (IsingRandomField.cpp:127) */
    int           algorithm;             /* 0: two-site ground state (fDMRG, H);  1: two-site excited state
                                            (xDMRG): lowest eigenpair of (H - E_t)^2 with E_t = L *
                                            energy_shift_per_site, MPO^2 uncompressed (MpoSite.cpp:57-70,
                                            D = 9), as in optimize_folded_spectrum.cpp:236-370;  2 and 3: the
                                            same two problems with one-site DMRG and forward subspace
                                            expansion before each local optimisation (the reference's
                                            single-site strategy, expand_environment_1site,
                                            tools/finite/env/env.cpp:1034-1262) */
    int           precond;               /* eigensolver expansion (heff_eig_config.precond); default -1:
                                            Jacobi for xDMRG (as the reference's PRIMME set-up for H^2,
                                            optimize_folded_spectrum.cpp:303-304), Krylov for fDMRG */
    int           fp64_engine;           /* heff_fp64_engine of the FP64-accurate matvecs (heff_op_set_fp64_engine);
                                            default HEFF_FP64_DMMA.  With HEFF_FP64_INT8 the digit planes are
                                            reserved once for chi_max, so sweeps still allocate nothing */
    double        expansion_alpha;       /* algorithms 2 and 3: mixing factor of the expansion term in the first
                                            sweep (0: 1e-3), halved every sweep, off for the last two sweeps */
    int           warmup_sweeps;         /* first sweeps run at bond limit bond_min and eigensolver tolerance
                                            max(1e-8, eig_tol) (the reference's warm-up iterations with bond_min and
                                            eigs_tol_max, AlgorithmFinite.cpp:530-545, 812-822); -1 (default): 2 for
                                            the folded-spectrum algorithms (1, 3), 0 for the ground state */
    int64_t       bond_min;              /* bond limit of the warm-up sweeps (0: 8, the xDMRG bond_min of
                                            settings.h:432) */
    int64_t       jcb_blocksize;         /* Jacobi block size of the preconditioned local solves
                                            (heff_op_set_jacobi_blocksize); 0: 128 for the folded spectrum (the
                                            reference's eigs_jcb_min_blocksize, settings.h:261), 1 (diagonal)
                                            otherwise */
    int64_t       eig_max_matvecs;       /* matvec limit of one local solve; 0: 4000 for the ground state,
                                            60000 for the folded spectrum (the reference allows eigs_iter_max =
                                            100000, settings.h:251) */
} heff_dmrg_config;

typedef struct {
    double  energy, entropy_mid, trunc_err_max, seconds, t_eig, t_svd, t_env;
    int64_t chi_mid, num_mv, num_mv_mixed, unconverged_solves;
    int     sweeps_done;
    double  energy_per_sweep[64]; /* last eigenvalue of each sweep (energy, or <(H-E_t)^2> for xDMRG) */
    double  variance;             /* xDMRG: <(H-E_t)^2> - (<H> - E_t)^2 (measure.cpp:575-640); energy = <H> */
    int     svd_sweeps_max;       /* most Jacobi sweeps one two-site split needed */
} heff_dmrg_result;

void heff_dmrg_config_default(heff_dmrg_config *cfg);
int  heff_dmrg_run(const heff_dmrg_config *cfg, heff_dmrg_result *res, void *stream);
/* Ensemble of independent realisations (disorder average): n configurations run by nthreads
 * workers, each with its own stream and a workspace allocated once for the largest chain and
 * bond dimension, so sweeps never allocate and realisations overlap on the device; nthreads = 1
 * runs them one at a time.  status[i] is realisation i's return code; *seconds the wall time of
 * the runs (workspace set-up excluded).  The reference runs one realisation per OS process
 * (slurm/submit_jobarray.py:49-95). */
int  heff_ensemble_run(const heff_dmrg_config *cfgs, int n, int nthreads, heff_dmrg_result *results, int *status, double *seconds);

/* ---------------------------------------------------------------------------
 * Eigensolve server: continuous batching of site-optimisation eigensolves.
 * No counterpart in the reference (it solves one site problem at a time on the
 * calling thread, solver_primme.cpp:298-517).  max_inflight worker slots, each
 * with its own stream, admit queued requests first-fit while the device memory
 * the in-flight requests hold stays within hbm_budget_bytes; environments stay
 * on the device for the whole solve; work of concurrent requests overlaps.
 * Results do not depend on the mix (every reduction has a fixed order).
 * ------------------------------------------------------------------------- */
typedef struct heff_server heff_server;

typedef struct {
    size_t hbm_budget_bytes; /* admission limit on the device memory held by in-flight requests */
    int    max_inflight;     /* concurrent slots */
    int    device;           /* CUDA device of the worker threads */
    int    max_basis;        /* eigensolver basis size per request, default 24 */
} heff_server_config;

typedef struct {
    int           dtype;                       /* HEFF_F64 / HEFF_C128 */
    int64_t       spin, chiL, chiR, mpoL, mpoR; /* mps [spin, chiL, chiR], mpo [mpoL, mpoR, spin, spin] */
    const void   *mpo;                         /* HOST mpo (merged) */
    const void   *envL, *envR;                 /* [chiL,chiL,mpoL], [chiR,chiR,mpoR] in env_where */
    int           env_where;                   /* heff_mem */
    const void   *theta0;                      /* start vector (host or device) or NULL */
    int           ritz;                        /* heff_ritz */
    double        target;                      /* for HEFF_RITZ_TARGET */
    double        tol;                         /* eigensolver tolerance, default 1e-10 */
    int           precision;                   /* heff_precision */
    void         *theta_out;                   /* HOST output eigenvector (rows elements) or NULL */
    int           fp64_engine;                 /* heff_fp64_engine of the FP64-accurate matvecs, default 0 (DMMA) */
} heff_request; /* buffers must stay valid until the request is answered; device buffers must be
                   complete (their producing work finished) when the request is submitted */

typedef struct {
    int64_t id;
    int     status; /* HEFF_OK, HEFF_NOT_CONVERGED, HEFF_OOM (larger than the whole budget), ... */
    int     converged;
    double  eigval, resnorm;
    int64_t num_mv, num_mv_mixed;
    double  t_submit, t_start, t_done; /* seconds on the server clock */
} heff_response;

typedef struct {
    int64_t completed, failed, queued;
    int     inflight, peak_inflight;
    size_t  peak_bytes;
    double  p50_latency_s, p99_latency_s, max_latency_s, solves_per_s;
    /* slot arenas: device bytes they hold now, and how many requests had to grow one (a growth frees and
     * reallocates buffers, which synchronises the device; a stream of sizes seen before grows none) */
    size_t  arena_bytes;
    int64_t arena_grows;
} heff_server_stats;

void   heff_server_config_default(heff_server_config *cfg);
int    heff_server_create(const heff_server_config *cfg, heff_server **srv);
/* Device bytes a request holds while it runs (the admission estimate). */
size_t heff_request_bytes(const heff_request *req, int max_basis);
int    heff_server_submit(heff_server *srv, const heff_request *req, int64_t *id);
/* Blocks until request `id` is answered (or timeout_s passes: HEFF_TIMEOUT). */
int    heff_server_wait(heff_server *srv, int64_t id, double timeout_s, heff_response *resp);
int    heff_server_get_stats(heff_server *srv, heff_server_stats *stats);
/* Finishes queued requests, joins the workers, frees the server. */
int    heff_server_destroy(heff_server *srv);

/* ---------------------------------------------------------------------------
 * Seeded synthetic inputs on the device (workload generators, not on the hot path)
 * ------------------------------------------------------------------------- */
/* env[a,a',mu] = (g(a,a',mu) + conj(g(a',a,pair(mu))))/2, g counter-based Gaussian:
 * pair = identity (swap_base <= 1: every slice Hermitian) or, for D = swap_base^2,
 * the swap (m + b*m~) <-> (m~ + b*m) matching the uncompressed MPO squared. */
int heff_make_env(int dtype, int64_t chi, int64_t D, int64_t swap_base, uint64_t seed, void *out, void *stream);
/* n Gaussian entries (complex: N(0,1) + i N(0,1)). */
int heff_make_vector(int dtype, int64_t n, uint64_t seed, void *out, void *stream);

#ifdef __cplusplus
}
#endif
#endif
