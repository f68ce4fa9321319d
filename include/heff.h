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

/* Same product and arguments as heff_matvec_d, but allocating no device memory.
 * No counterpart in the reference: it exists for callers that cannot let a
 * library call cudaMalloc (a process that has already split all device memory
 * among its own pools, or that cannot afford the device-wide synchronisation a
 * cudaMalloc/cudaFree implies).  Scratch comes from one fixed 32 MiB array
 * inside the library (held on every GPU that loads the library until exit);
 * calls needing more return HEFF_BAD_SHAPE (real two-site D=3 fits up to about
 * chi=360).  All calls on a device share that array: calls that may overlap on
 * the GPU race, so serialise them.  The first call on a device looks up the
 * array's device address; make it before any stream capture. */
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
 * Operator object: MatVecMPOS<T> / MatVecMPO<T>
 * (source/math/eig/matvec/matvec_mpos.h:23-180, matvec_mpo.h:18-103)
 * ------------------------------------------------------------------------- */
typedef struct heff_op heff_op;

/* Constructor: MatVecMPOS<T>(mpos, env_pair) (matvec_mpos.cpp:40-130).  The
 * nsites site MPOs (each [mL, mR, d, d]) are merged into one
 * [mL0, mR_last, prod d, prod d] MPO as in matvec_mpos.cpp:104-119 (nsites <= 5).
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
/* Number of matvecs applied so far (MatVecMPOS::num_mv). */
int64_t heff_op_num_mv(const heff_op *op);
/* Stage timing (the reference's tid:: timers around MultAx, matvec_mpo.h:70-102):
 * when enabled, every FP64 matvec records CUDA events around its four kernels
 * (layout, GEMM 1, MPO mix, GEMM 2).  heff_op_stage_times synchronises the op's
 * stream and returns the summed milliseconds per stage and the matvec count. */
int heff_op_set_profiling(heff_op *op, int enable);
int heff_op_stage_times(heff_op *op, double ms[4], int64_t *count, int reset);

#ifdef __cplusplus
}
#endif
#endif
