// Internal definition of the heff_op operator object (opaque in include/heff.h).
#pragma once
#include <vector>

#include "matvec.cuh"
#include "multi.cuh"

namespace heff {
struct MatvecGraph;     // op.cu
bool graphs_default();  // op.cu: environment variable HEFF_GRAPHS (1 on, default off)
}

struct heff_op {
    bool               cplx = false;
    heff::MatvecDims   d{};
    int64_t            mpo_dims[4] = {0, 0, 0, 0};
    heff_precision     precision   = HEFF_PREC_FP64;
    cudaStream_t       stream      = nullptr;
    void              *L = nullptr, *Rp = nullptr, *W = nullptr;  // device: envL (reference layout), R', merged W
    // more than 5 site MPOs (matvec_mpos.cpp:104-123): applied one at a time (multi.cu); W then holds only the
    // s == s' entries of the merged MPO (for the preconditioner diagonal)
    bool               sequential = false;
    heff::MultiDims    multi{};
    std::vector<void *> seq_W;
    void              *scratch       = nullptr;                    // x' | T1 | T2
    size_t             scratch_bytes = 0;
    void              *split_ws      = nullptr;  // tail-split partial tiles of the matvec GEMMs (matvec_split_bytes)
    size_t             split_bytes   = 0;
    void              *stage_x       = nullptr;  // device staging for MultAx with host buffers
    size_t             stage_bytes   = 0;
    heff::HostPipe    *pipe          = nullptr;  // streams/events of the overlapped host-buffer matvec (created on first use)
    int64_t            num_mv        = 0;
    // fixed-capacity operators (op_create_capacity / op_rebind): element capacities, R staging, host MPO copy
    int64_t            cap_env = 0, cap_W = 0, cap_scratch = 0;
    void              *Rtmp    = nullptr;
    std::vector<unsigned char> w_host;
    // arena operators (server slots, op_create_arena): byte capacities of the buffers above and of the
    // start/result vector pair; cap_env/cap_W/cap_scratch/diag_cap follow from them for the bound dtype
    bool               arena = false;
    size_t             cap_env_b = 0, cap_W_b = 0, cap_scratch_b = 0, cap_diag_b = 0, cap_split_b = 0;
    void              *arena_vec   = nullptr;
    size_t             arena_vec_b = 0;
    // eigensolver workspace, kept across heff_eigs calls on this operator (grown on demand)
    void              *eig_ws       = nullptr;
    size_t             eig_ws_bytes = 0;
    void              *eig_host     = nullptr;  // pinned: per-iteration coefficients (Krylov loop)
    cudaEvent_t        eig_event    = nullptr;
    // diagonal of H_eff for the Jacobi preconditioner (computed on first use after create / rebind)
    void              *diag         = nullptr;
    int64_t            diag_cap     = 0;
    bool               diag_ready   = false;
    // block-Jacobi preconditioner (heff_op_set_jacobi_blocksize > 1): [0, 256) singular-pivot count, then the
    // inverted blocks; formed at the shift of the first MultPc after a (re)bind
    int64_t            jcb_block    = 1;
    void              *jcb          = nullptr;
    size_t             jcb_bytes    = 0;
    bool               jcb_ready    = false;
    double             jcb_shift    = 0.0;
    // stage profiling (heff_op_set_profiling): ring of 5-event sets, summed on query
    bool               profiling     = false;
    std::vector<cudaEvent_t> prof_events;  // 5 * prof_cap
    int                prof_cap      = 0, prof_used = 0;
    double             prof_ms[4]    = {0, 0, 0, 0};
    int64_t            prof_count    = 0;
    // engine of the FP64-accurate matvecs: HEFF_FP64_DMMA, or HEFF_FP64_INT8 (emulated on the INT8 tensor cores,
    // emu.cu; its digit planes of L and R' are rebuilt after a rebind)
    int                fp64_engine   = HEFF_FP64_DMMA;
    int                emu_slices    = 7;
    void              *emu           = nullptr;
    bool               emu_stale     = true;
    // dense interior solve (heff_eigs with HEFF_RITZ_TARGET at rows() <= 4096): matrix, eigenvalues, eigenvectors
    void              *dense_ws      = nullptr;
    size_t             dense_bytes   = 0;
    // CUDA graph of the FP64 DMMA matvec (heff_op_set_graphs; default from HEFF_GRAPHS): recorded after the first product of a
    // shape on a non-default stream and replayed with the input and output retargeted
    bool               graphs        = heff::graphs_default();
    heff::MatvecGraph *mg            = nullptr;
    // mixed-precision state (owned by the mixed path; null until first use)
    void              *mixed         = nullptr;
    int (*mixed_apply)(heff_op *, const void *, void *) = nullptr;
    void (*destroy_hook)(heff_op *)                     = nullptr;
};

namespace heff {
int op_apply(heff_op *op, const void *x, void *y);
int mixed_apply(heff_op *op, const void *x, void *y);     // mixed.cu
int mixed_error_flag(heff_op *op, int *flag);              // mixed.cu
void mixed_invalidate(heff_op *op);                        // mixed.cu: split operands are rebuilt on the next mixed matvec
int mixed_reserve(heff_op *op, size_t bytes);              // mixed.cu: pooled split-operand buffer of at least `bytes`
size_t mixed_bytes(int64_t S, int64_t cL, int64_t cR, int64_t DL, int64_t DR, bool cplx);  // mixed.cu: pool bytes of one shape
size_t mixed_held_bytes(const heff_op *op);                // mixed.cu
size_t eig_workspace_bytes(int64_t n, int max_basis, bool mixed, bool cplx);  // eig.cu: Davidson workspace of one solve
bool emu_supported(const heff_op *op);                     // emu.cu: both GEMMs within the exact-INT32 range
int emu_apply(heff_op *op, const void *x, void *y);        // emu.cu
int emu_error_flag(heff_op *op, int *flag);                // emu.cu
void emu_destroy(heff_op *op);                             // emu.cu
int emu_reserve(heff_op *op, int64_t S, int64_t cmax, int64_t Dmax);  // emu.cu: digit-plane buffer for the largest bond
size_t emu_bytes(int64_t S, int64_t cL, int64_t cR, int64_t DL, int64_t DR, bool cplx, int nslices);  // emu.cu
int op_create_capacity(heff_op **out, bool cplx, int64_t S, int64_t cmax, int64_t Dmax, heff_precision prec, cudaStream_t stream);
size_t emu_held_bytes(const heff_op *op);  // emu.cu: bytes of the digit-plane buffer

// Arena operators (one per eigensolve-server slot): every device buffer is kept across requests and grown only when
// a request needs more, so a request costs no cudaMalloc/cudaFree (which synchronise the whole device) once the
// arena has grown to the stream's sizes.  Byte capacities, so one arena serves real and complex requests.
struct ArenaBytes {
    size_t env = 0, W = 0, scratch = 0, split = 0, diag = 0, mixed = 0, emu = 0, eig = 0, vec = 0;
    size_t total() const { return 3 * env + W + scratch + split + diag + mixed + emu + eig + vec; }
    ArenaBytes max_with(const ArenaBytes &o) const;
};
ArenaBytes arena_need(const heff_request &r, int max_basis);  // bytes each buffer needs for this request
ArenaBytes arena_held(const heff_op *op);                      // bytes each buffer holds now
int op_create_arena(heff_op **out, cudaStream_t stream);
// Grows the arena to cover `r`, binds its MPO and environments (copied onto the device, stream-ordered) and sets its
// dtype, precision and FP64 engine.  *vec receives a device buffer of 2 * rows elements (start vector and result).
int op_arena_bind(heff_op *op, const heff_request &r, int max_basis, void **vec);
int op_rebind(heff_op *op, int nsites, const void *const *mpos_host, const int64_t *mdims, const void *envL, const int64_t ld[3], const void *envR,
              const int64_t rd[3]);
int eig_host_ready(heff_op *op);     // eig.cu: pinned coefficient buffer + event of the Krylov loop
int op_diagonal_ready(heff_op *op);  // precond.cu: op->diag holds the diagonal of H_eff (stream-ordered)
int op_multpc(heff_op *op, const void *x, void *y, double shift);  // precond.cu: y = x / (diag - shift)
int op_prof_flush(heff_op *op);  // synchronises the op's stream and folds recorded events into prof_ms
cudaEvent_t *op_prof_slot(heff_op *op);  // next free 5-event set or nullptr (profiling off)
}
