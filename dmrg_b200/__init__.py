"""heff_b200: B200-native (sm_100a) effective-Hamiltonian hot path of DMRG++.

Python mirror of the reference's operator surface over the C ABI in
``include/heff.h`` (ctypes).  Device buffers are torch CUDA tensors (plumbing
only); every computation runs in ``libheff_b200.so``.  There is no CPU
fallback: if the library is missing, :func:`lib` raises.

Tensors use the reference's Eigen column-major layout.  A column-major tensor
of shape ``(s, chiL, chiR)`` is passed as a flat (1-D) device tensor plus its
dims; :func:`to_device` / :func:`to_host` convert Fortran-ordered numpy arrays.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libheff_b200.so")
_lib = None

HEFF_OK = 0
STATUS = {
    0: "HEFF_OK",
    1: "HEFF_BAD_SHAPE",
    2: "HEFF_NAN_INPUT",
    3: "HEFF_OOM",
    4: "HEFF_TIMEOUT",
    5: "HEFF_NOT_CONVERGED",
    6: "HEFF_CUDA_ERROR",
    7: "HEFF_BAD_ARG",
    8: "HEFF_NO_DEVICE",
}
F64, C128 = 0, 1
MEM_DEVICE, MEM_HOST = 0, 1
PREC_FP64, PREC_MIXED = 0, 1
FP64_DMMA, FP64_INT8 = 0, 1  # engines of the FP64-accurate matvecs (heff_op_set_fp64_engine)


class HeffError(RuntimeError):
    def __init__(self, code, where):
        self.code = code
        msg = lib().heff_last_error().decode(errors="replace") if _lib is not None else ""
        super().__init__(f"{where}: {STATUS.get(code, code)} {msg}")


_P = ctypes.c_void_p
_I64 = ctypes.c_int64
_I64P = ctypes.POINTER(ctypes.c_int64)


def _sig(L, name, res, args):
    f = getattr(L, name)
    f.restype = res
    f.argtypes = args
    return f


def lib():
    """Load libheff_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: run `python -m dmrg_b200.build` (nvcc, sm_100a)")
        L = ctypes.CDLL(LIB_PATH)
        _sig(L, "heff_last_error", ctypes.c_char_p, [])
        _sig(L, "heff_version", ctypes.c_char_p, [])
        for n in ("heff_matvec_d", "heff_matvec_z"):
            _sig(L, n, ctypes.c_int, [_P, _P, _I64P, _P, _I64P, _P, _I64P, _P, _I64P, _P])
        for n in ("heff_expval_d", "heff_expval_z"):
            _sig(L, n, ctypes.c_int, [ctypes.POINTER(ctypes.c_double), _P, _I64P, _P, _I64P, _P, _I64P, _P, _I64P, _P])
        _sig(L, "heff_op_create", ctypes.c_int,
             [ctypes.POINTER(_P), ctypes.c_int, ctypes.c_int, ctypes.POINTER(_P), _I64P, _P, _I64P, _P, _I64P, ctypes.c_int, ctypes.c_int, _P])
        _sig(L, "heff_op_destroy", ctypes.c_int, [_P])
        _sig(L, "heff_op_rows", _I64, [_P])
        _sig(L, "heff_op_shape", ctypes.c_int, [_P, _I64P])
        _sig(L, "heff_op_multax", ctypes.c_int, [_P, _P, _P])
        _sig(L, "heff_perform_op", ctypes.c_int, [_P, _P, _P])
        _sig(L, "heff_op_multax_block", ctypes.c_int, [_P, _P, _I64, _P, _I64, ctypes.c_int])
        _sig(L, "heff_op_multax_host", ctypes.c_int, [_P, _P, _P])
        _sig(L, "heff_op_set_stream", ctypes.c_int, [_P, _P])
        _sig(L, "heff_op_set_precision", ctypes.c_int, [_P, ctypes.c_int])
        _sig(L, "heff_op_num_mv", _I64, [_P])
        _sig(L, "heff_op_set_profiling", ctypes.c_int, [_P, ctypes.c_int])
        _sig(L, "heff_op_stage_times", ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_double), _I64P, ctypes.c_int])
        _lib = L
        _extend_signatures(L)
    return _lib


def _extend_signatures(L):
    """Signatures of the entry points added beyond the matvec (env, svd, eigensolver, ...)."""
    from . import _sigs

    _sigs.declare(L, _sig)


def check(rc, where):
    if rc != HEFF_OK:
        raise HeffError(rc, where)


def dims(shape):
    return (ctypes.c_int64 * len(shape))(*[int(x) for x in shape])


# ---------------------------------------------------------------- torch plumbing
def _torch():
    import torch

    return torch


def to_device(a, device="cuda"):
    """Fortran-ordered numpy array -> flat torch CUDA tensor holding the same column-major bytes."""
    torch = _torch()
    a = np.asarray(a)
    flat = np.ascontiguousarray(a.ravel(order="F"))
    return torch.from_numpy(flat).to(device)


def to_host(t, shape):
    """Flat torch tensor -> Fortran-ordered numpy array of the given column-major shape."""
    return np.asarray(t.detach().cpu().numpy()).reshape(shape, order="F")


def ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _stream_handle(stream):
    if stream is None:
        torch = _torch()
        return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    if isinstance(stream, int):
        return ctypes.c_void_p(stream)
    return ctypes.c_void_p(stream.cuda_stream)


# ---------------------------------------------------------------- contraction API
def matrix_vector_product(res, mps, mps_dims, mpo, mpo_dims, envL, envL_dims, envR, envR_dims, stream=None):
    """tools::common::contraction::matrix_vector_product (contraction.h:31-36) on device tensors."""
    cplx = mps.is_complex()
    fn = lib().heff_matvec_z if cplx else lib().heff_matvec_d
    rc = fn(ptr(res), ptr(mps), dims(mps_dims), ptr(mpo), dims(mpo_dims), ptr(envL), dims(envL_dims), ptr(envR), dims(envR_dims),
            _stream_handle(stream))
    check(rc, "heff_matvec")
    return res


def expectation_value(mps, mps_dims, mpo, mpo_dims, envL, envL_dims, envR, envR_dims, stream=None):
    """tools::common::contraction::expectation_value (contraction.h:18-22)."""
    cplx = mps.is_complex()
    out = (ctypes.c_double * 2)()
    fn = lib().heff_expval_z if cplx else lib().heff_expval_d
    rc = fn(out, ptr(mps), dims(mps_dims), ptr(mpo), dims(mpo_dims), ptr(envL), dims(envL_dims), ptr(envR), dims(envR_dims),
            _stream_handle(stream))
    check(rc, "heff_expval")
    return complex(out[0], out[1]) if cplx else float(out[0])


def env_update(side, out, env, env_dims, mps, mps_dims, mpo, mpo_dims, stream=None):
    """EnvBase::build_block (EnvBase.cpp:67-151) on device tensors; side 'L' or 'R'."""
    cplx = mps.is_complex()
    fn = lib().heff_env_update_z if cplx else lib().heff_env_update_d
    sd = 0 if side in ("L", 0) else 1
    rc = fn(sd, ptr(out), ptr(env), dims(env_dims), ptr(mps), dims(mps_dims), ptr(mpo), dims(mpo_dims), _stream_handle(stream))
    check(rc, "heff_env_update")
    return out


def matrix_vector_product_multi(res, mps, mps_dims, mpos, mpo_dims, envL, envL_dims, envR, envR_dims, stream=None):
    """Multi-MPO matrix_vector_product (contraction_tblis.cpp:307-420): a list of device site MPOs [D, D', d, d]
    applied one at a time; mps [prod d, chiL, chiR] (site 1 fastest)."""
    cplx = mps.is_complex()
    fn = lib().heff_matvec_multi_z if cplx else lib().heff_matvec_multi_d
    arr = (_P * len(mpos))(*[ctypes.c_void_p(m.data_ptr()) for m in mpos])
    md = (ctypes.c_int64 * (4 * len(mpos)))(*[int(x) for d4 in mpo_dims for x in d4])
    rc = fn(ptr(res), ptr(mps), dims(mps_dims), len(mpos), arr, md, ptr(envL), dims(envL_dims), ptr(envR), dims(envR_dims), _stream_handle(stream))
    check(rc, "heff_matvec_multi")
    return res


def get_expansion_term(side, P, env, env_dims, mps, mps_dims, mpo, mpo_dims, alpha, stream=None):
    """EnvBase::get_expansion_term (EnvBase.cpp:303-364) on device tensors; side 'L' or 'R'.  P holds
    spin*chiL*chiR*D elements ([spin, chiL, chiR*DR] for L, the reference's [spin, chiL*DL, chiR] order for R)."""
    cplx = mps.is_complex()
    fn = lib().heff_expansion_term_z if cplx else lib().heff_expansion_term_d
    sd = 0 if side in ("L", 0) else 1
    rc = fn(sd, ptr(P), ptr(env), dims(env_dims), ptr(mps), dims(mps_dims), ptr(mpo), dims(mpo_dims), float(alpha), _stream_handle(stream))
    check(rc, "heff_expansion_term")
    return P


def dense_eig(A, n, stream=None):
    """All eigenpairs of a Hermitian n x n device matrix (flat, column-major): heff_dense_eig.  Returns
    (evals ascending [n] float64, evecs flat column-major [n x n]) as device tensors."""
    torch = _torch()
    cplx = A.dtype == torch.complex128
    ev = torch.empty(n, dtype=torch.float64, device=A.device)
    V = torch.empty(n * n, dtype=A.dtype, device=A.device)
    check(lib().heff_dense_eig(C128 if cplx else F64, n, ptr(A), n, ptr(ev), ptr(V), _stream_handle(stream)), "heff_dense_eig")
    return ev, V


def svd(A, rows, cols, rank_max=0, trunc_lim=1e-12, stream=None):
    """svd::solver::do_svd_ptr + truncation (svd.cpp:113-206, 257-280) on a device matrix (float64 or complex128).

    Returns (U [rows x k], S [k], VT [k x cols]) as flat device tensors plus (k, truncation_error); VT = V^H."""
    torch = _torch()
    cplx = A.dtype == torch.complex128
    dt = torch.complex128 if cplx else torch.float64
    kmax = min(rows, cols, rank_max if rank_max > 0 else rows * cols)
    U = torch.empty(rows * kmax, dtype=dt, device=A.device)
    S = torch.empty(kmax, dtype=torch.float64, device=A.device)
    VT = torch.empty(kmax * cols, dtype=dt, device=A.device)
    k = ctypes.c_int64(0)
    err = ctypes.c_double(0)
    name = "heff_svd_z" if cplx else "heff_svd_d"
    check(getattr(lib(), name)(ptr(A), rows, cols, rank_max, trunc_lim, ptr(U), ptr(S), ptr(VT), ctypes.byref(k), ctypes.byref(err),
                               _stream_handle(stream)), name)
    k = int(k.value)
    return U[: rows * k], S[:k], VT[: k * cols], k, float(err.value)


def schmidt_multisite(theta, dL, dR, chiL, chiR, rank_max=0, trunc_lim=1e-12, stream=None):
    """svd::solver::schmidt_multisite (svd.h:189-220): returns U [dL,chiL,k], S [k] (unit norm), V [dR,k,chiR]
    as flat device tensors, and (k, truncation_error).  theta float64 or complex128."""
    torch = _torch()
    cplx = theta.dtype == torch.complex128
    dt = torch.complex128 if cplx else torch.float64
    m, n = dL * chiL, dR * chiR
    kmax = min(m, n, rank_max if rank_max > 0 else m * n)
    U = torch.empty(m * kmax, dtype=dt, device=theta.device)
    S = torch.empty(kmax, dtype=torch.float64, device=theta.device)
    V = torch.empty(kmax * n, dtype=dt, device=theta.device)
    k = ctypes.c_int64(0)
    err = ctypes.c_double(0)
    name = "heff_schmidt_z" if cplx else "heff_schmidt_d"
    check(getattr(lib(), name)(ptr(theta), dL, dR, chiL, chiR, rank_max, trunc_lim, ptr(U), ptr(S), ptr(V), ctypes.byref(k), ctypes.byref(err),
                               _stream_handle(stream)), name)
    k = int(k.value)
    return U[: m * k], S[:k], V[: k * n], k, float(err.value)


def xdmrg(h, energy_target, one_site=False, **kw):
    """Excited-state DMRG (folded spectrum): the eigenstate closest to energy_target (heff_dmrg_run, algorithm 1, or 3:
    one-site with subspace expansion)."""
    return fdmrg(h, energy_shift_per_site=energy_target / len(h), algorithm=3 if one_site else 1, **kw)


def fdmrg(h, J=1.0, chi_max=64, sweeps=10, trunc_lim=1e-12, eig_tol=1e-12, precision=PREC_FP64, seed=0, ritz="SA", target=0.0,
          energy_shift_per_site=0.0, algorithm=0, precond=-1, fp64_engine=FP64_DMMA, expansion_alpha=0.0, warmup_sweeps=-1, bond_min=0,
          jcb_blocksize=0, eig_max_matvecs=0, stream=None):
    """DMRG of the random-field Ising chain on the device (heff_dmrg_run); returns the result dict.  algorithm 0: two-site
    ground state, 1: two-site folded spectrum, 2 / 3: the same with one-site DMRG and forward subspace expansion."""
    from ._sigs import DmrgConfig, DmrgResult

    hs = np.ascontiguousarray(np.asarray(h, dtype=np.float64))
    cfg = DmrgConfig()
    lib().heff_dmrg_config_default(ctypes.byref(cfg))
    cfg.L = len(hs)
    cfg.J = J
    cfg.h = hs.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    cfg.chi_max = chi_max
    cfg.sweeps = sweeps
    cfg.trunc_lim = trunc_lim
    cfg.eig_tol = eig_tol
    cfg.precision = precision
    cfg.seed = seed
    cfg.ritz = {"SA": 0, "LA": 1, "TARGET": 2}[ritz]
    cfg.target = target
    cfg.energy_shift_per_site = energy_shift_per_site
    cfg.algorithm = int(algorithm)
    cfg.precond = int(precond)
    cfg.fp64_engine = int(fp64_engine)
    cfg.expansion_alpha = float(expansion_alpha)
    cfg.warmup_sweeps = int(warmup_sweeps)
    cfg.bond_min = int(bond_min)
    cfg.jcb_blocksize = int(jcb_blocksize)
    cfg.eig_max_matvecs = int(eig_max_matvecs)
    res = DmrgResult()
    check(lib().heff_dmrg_run(ctypes.byref(cfg), ctypes.byref(res), _stream_handle(stream)), "heff_dmrg_run")
    return res.as_dict()


def ensemble(realisations, nthreads=16, chi_max=64, sweeps=10, trunc_lim=1e-12, eig_tol=1e-12, J=1.0, precision=PREC_FP64,
             fp64_engine=FP64_DMMA):
    """Independent fDMRG realisations (heff_ensemble_run).  realisations: list of (h_fields, chi_max or None, seed).
    Returns (list of result dicts, list of status codes, wall seconds)."""
    from ._sigs import DmrgConfig, DmrgResult

    n = len(realisations)
    cfgs = (DmrgConfig * n)()
    keep = []
    for i, (h, chi, seed) in enumerate(realisations):
        hs = np.ascontiguousarray(np.asarray(h, dtype=np.float64))
        keep.append(hs)
        c = cfgs[i]
        lib().heff_dmrg_config_default(ctypes.byref(c))
        c.L = len(hs)
        c.J = J
        c.h = hs.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        c.chi_max = int(chi or chi_max)
        c.sweeps = sweeps
        c.trunc_lim = trunc_lim
        c.eig_tol = eig_tol
        c.precision = precision
        c.fp64_engine = int(fp64_engine)
        c.seed = int(seed)
    res = (DmrgResult * n)()
    st = (ctypes.c_int * n)()
    secs = ctypes.c_double(0)
    check(lib().heff_ensemble_run(cfgs, n, int(nthreads), res, st, ctypes.byref(secs)), "heff_ensemble_run")
    return [res[i].as_dict() for i in range(n)], list(st), float(secs.value)


def make_env(chi, D, cplx, seed, swap_base=0, stream=None):
    """Seeded [chi, chi, D] environment on the device (heff_make_env): every slice Hermitian, or for
    D = swap_base^2 the MPO-squared swap symmetry.  Returns a flat device tensor."""
    torch = _torch()
    out = torch.empty(chi * chi * D, dtype=torch.complex128 if cplx else torch.float64, device="cuda")
    check(lib().heff_make_env(C128 if cplx else F64, chi, D, swap_base, seed & (2**64 - 1), ptr(out), _stream_handle(stream)), "heff_make_env")
    return out


def make_vector(n, cplx, seed, stream=None):
    torch = _torch()
    out = torch.empty(n, dtype=torch.complex128 if cplx else torch.float64, device="cuda")
    check(lib().heff_make_vector(C128 if cplx else F64, n, seed & (2**64 - 1), ptr(out), _stream_handle(stream)), "heff_make_vector")
    return out


class EigServer:
    """Continuous-batching eigensolve server (heff_server_*): submit requests, wait for answers, read stats."""

    def __init__(self, hbm_budget_bytes=64 << 30, max_inflight=4, device=0, max_basis=24):
        from ._sigs import ServerConfig

        cfg = ServerConfig()
        lib().heff_server_config_default(ctypes.byref(cfg))
        cfg.hbm_budget_bytes = int(hbm_budget_bytes)
        cfg.max_inflight = int(max_inflight)
        cfg.device = int(device)
        cfg.max_basis = int(max_basis)
        h = ctypes.c_void_p()
        check(lib().heff_server_create(ctypes.byref(cfg), ctypes.byref(h)), "heff_server_create")
        self.handle = h
        self._keep = {}

    @staticmethod
    def request(mpo, envL, envR, spin, chiL, chiR, cplx, theta0=None, ritz="SA", target=0.0, tol=1e-10, precision=PREC_FP64, theta_out=None,
                fp64_engine=FP64_DMMA):
        """Builds an heff_request; mpo: host numpy [mL,mR,spin,spin]; envs/theta0: device tensors; theta_out: host numpy or None."""
        from ._sigs import Request

        dt = np.complex128 if cplx else np.float64
        W = np.asfortranarray(np.asarray(mpo, dtype=dt))
        r = Request()
        r.dtype = C128 if cplx else F64
        r.spin, r.chiL, r.chiR, r.mpoL, r.mpoR = spin, chiL, chiR, W.shape[0], W.shape[1]
        r.mpo = W.ctypes.data
        r.envL = envL.data_ptr()
        r.envR = envR.data_ptr()
        r.env_where = MEM_DEVICE
        r.theta0 = theta0.data_ptr() if theta0 is not None else None
        r.ritz = {"SA": 0, "LA": 1, "TARGET": 2}[ritz]
        r.target = float(target)
        r.tol = float(tol)
        r.precision = int(precision)
        r.theta_out = theta_out.ctypes.data if theta_out is not None else None
        r.fp64_engine = int(fp64_engine)
        return r, (W, envL, envR, theta0, theta_out)

    @staticmethod
    def request_bytes(req, max_basis=24):
        """Admission estimate: device bytes the request holds while it runs."""
        return int(lib().heff_request_bytes(ctypes.byref(req), max_basis))

    def submit(self, req_and_keep):
        req, keep = req_and_keep
        rid = ctypes.c_int64(0)
        check(lib().heff_server_submit(self.handle, ctypes.byref(req), ctypes.byref(rid)), "heff_server_submit")
        self._keep[rid.value] = (req, keep)
        return rid.value

    def wait(self, rid, timeout=0.0):
        from ._sigs import Response

        resp = Response()
        check(lib().heff_server_wait(self.handle, rid, float(timeout), ctypes.byref(resp)), "heff_server_wait")
        self._keep.pop(rid, None)
        return resp.as_dict()

    def stats(self):
        from ._sigs import ServerStats

        st = ServerStats()
        check(lib().heff_server_get_stats(self.handle, ctypes.byref(st)), "heff_server_get_stats")
        return st.as_dict()

    def close(self):
        if getattr(self, "handle", None):
            lib().heff_server_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def two_site_ising_mpo(D, cplx, h1=0.8, h2=1.2, J=1.0):
    """Merged two-site random-field Ising MPO (D=3; IsingRandomField.cpp:122-129, merged as matvec_mpos.cpp:104-119)
    or the merged uncompressed MPO squared (D=9; MpoSite.cpp:57-70), Fortran-ordered [D, D, 4, 4] numpy."""
    def site(h):
        W = np.zeros((3, 3, 2, 2))
        sx = np.array([[0.0, 1.0], [1.0, 0.0]])
        sz = np.array([[1.0, 0.0], [0.0, -1.0]])
        W[0, 0] = np.eye(2)
        W[1, 0] = sz
        W[2, 0] = -h * sx
        W[2, 1] = -J * sz
        W[2, 2] = np.eye(2)
        return W

    def square(W):
        return np.einsum("mnsp,MNpt->mMnNst", W, W).reshape(9, 9, 2, 2, order="F")

    if D not in (3, 9):
        raise ValueError("D must be 3 (H) or 9 (H squared)")
    WA, WB = site(h1), site(h2)
    if D == 9:
        WA, WB = square(WA), square(WB)
    X = np.einsum("mcst,cnuv->mnsutv", WA, WB)
    W = X.reshape(WA.shape[0], WB.shape[1], 4, 4, order="F")
    return np.asfortranarray(W.astype(np.complex128 if cplx else np.float64))


def serve_specs(specs, hbm_budget_bytes=None, max_inflight=8, max_basis=24, wait_timeout=3600.0, max_pending_bytes=16 << 30):
    """Runs a stream of synthetic eigensolve requests through one EigServer on this process's GPU.

    specs: list of dicts with chi, D (3: H, lowest eigenpair; 9: H squared, lowest eigenpair of the folded
    operator), cplx, seed and optionally precision (PREC_FP64), tol (1e-10), arrival (seconds after the stream
    starts; requests are submitted in list order, each not before its arrival time).  A request's environments
    (Hermitian slices, seeded) and start vector are generated on the device when it arrives and released once it is
    answered; while the generated inputs of unanswered requests exceed `max_pending_bytes`, the next arrival waits
    for the oldest answer (its latency from arrival then includes that wait).  Returns (list of response dicts,
    list of status codes, wall seconds of the stream, server stats plus the latency percentiles measured from each
    request's arrival time)."""
    import collections
    import time

    torch = _torch()
    n = len(specs)
    torch.cuda.synchronize()
    if hbm_budget_bytes is None:
        torch.cuda.empty_cache()
        free, _ = torch.cuda.mem_get_info()
        hbm_budget_bytes = max(int(0.85 * free) - int(max_pending_bytes), 1 << 30)
    srv = EigServer(hbm_budget_bytes=hbm_budget_bytes, max_inflight=max_inflight, max_basis=max_basis)
    resp = [None] * n
    pending = collections.deque()
    pend_bytes = 0

    def settle_oldest():
        nonlocal pend_bytes
        j, rid, keep, nb = pending.popleft()
        resp[j] = srv.wait(rid, timeout=wait_timeout)
        pend_bytes -= nb
        del keep

    try:
        t0 = time.perf_counter()
        for i, sp in enumerate(specs):
            chi, D, cplx, seed = int(sp["chi"]), int(sp["D"]), bool(sp["cplx"]), int(sp["seed"])
            nb = (2 * chi * chi * D + 4 * chi * chi) * (16 if cplx else 8)
            while pending and pend_bytes + nb > max_pending_bytes:
                settle_oldest()
            dt = float(sp.get("arrival", 0.0)) - (time.perf_counter() - t0)
            if dt > 0:
                time.sleep(dt)
            envL = make_env(chi, D, cplx, seed=2 * seed, swap_base=3 if D == 9 else 0)
            envR = make_env(chi, D, cplx, seed=2 * seed + 1, swap_base=3 if D == 9 else 0)
            th0 = make_vector(4 * chi * chi, cplx, seed=7 * seed + 3)
            req = EigServer.request(two_site_ising_mpo(D, cplx), envL, envR, 4, chi, chi, cplx, theta0=th0,
                                    tol=float(sp.get("tol", 1e-10)), precision=int(sp.get("precision", PREC_FP64)))
            torch.cuda.current_stream().synchronize()  # the inputs are complete before the server reads them
            pending.append((i, srv.submit(req), req, nb))
            pend_bytes += nb
        while pending:
            settle_oldest()
        secs = time.perf_counter() - t0
        st = srv.stats()
    finally:
        srv.close()
    start = min(r["t_submit"] for r in resp) if resp else 0.0
    lat = sorted(r["t_done"] - (start + float(sp.get("arrival", 0.0))) for r, sp in zip(resp, specs))
    if lat:
        st["p50_latency_from_arrival_s"] = lat[min(len(lat) - 1, int(0.50 * (len(lat) - 1) + 0.5))]
        st["p99_latency_from_arrival_s"] = lat[min(len(lat) - 1, int(0.99 * (len(lat) - 1) + 0.5))]
    return resp, [r["status"] for r in resp], secs, st


class MatVecMPOS:
    """MatVecMPOS<T> (matvec_mpos.h:23-180): operator object handed to an eigensolver.

    ``mpos``: list of Fortran-ordered numpy site MPOs [mL, mR, d, d] (merged like
    matvec_mpos.cpp:104-119); ``envL``/``envR``: numpy [chi, chi, m].  The operator
    keeps device copies; ``MultAx`` takes device tensors, ``MultAx_host`` numpy.
    """

    def __init__(self, mpos, envL, envR, cplx=None, precision=PREC_FP64, stream=None):
        if cplx is None:
            cplx = any(np.iscomplexobj(x) for x in list(mpos) + [envL, envR])
        self.cplx = bool(cplx)
        dt = np.complex128 if self.cplx else np.float64
        self._keep = [np.asfortranarray(np.asarray(w, dtype=dt)) for w in mpos]
        self._envL = np.asfortranarray(np.asarray(envL, dtype=dt))
        self._envR = np.asfortranarray(np.asarray(envR, dtype=dt))
        n = len(self._keep)
        ptrs = (ctypes.c_void_p * n)(*[w.ctypes.data for w in self._keep])
        md = (ctypes.c_int64 * (4 * n))(*[int(x) for w in self._keep for x in w.shape])
        h = ctypes.c_void_p()
        self._stream = _stream_handle(stream)
        rc = lib().heff_op_create(ctypes.byref(h), C128 if self.cplx else F64, n, ptrs, md, self._envL.ctypes.data_as(_P), dims(self._envL.shape),
                                  self._envR.ctypes.data_as(_P), dims(self._envR.shape), MEM_HOST, int(precision), self._stream)
        check(rc, "heff_op_create")
        self.handle = h
        sh = (ctypes.c_int64 * 3)()
        check(lib().heff_op_shape(h, sh), "heff_op_shape")
        self.shape_mps = (sh[0], sh[1], sh[2])

    def rows(self):
        return int(lib().heff_op_rows(self.handle))

    def MultAx(self, x, y):
        check(lib().heff_op_multax(self.handle, ptr(x), ptr(y)), "MultAx")
        return y

    def MultAx_block(self, x, ldx, y, ldy, block_size):
        check(lib().heff_op_multax_block(self.handle, ptr(x), int(ldx), ptr(y), int(ldy), int(block_size)), "MultAx_block")
        return y

    def MultAx_host(self, x):
        dt = np.complex128 if self.cplx else np.float64
        xin = np.ascontiguousarray(np.asarray(x, dtype=dt).ravel(order="F"))
        out = np.empty_like(xin)
        check(lib().heff_op_multax_host(self.handle, xin.ctypes.data_as(_P), out.ctypes.data_as(_P)), "MultAx_host")
        return out.reshape(self.shape_mps, order="F")

    def set_precision(self, precision):
        check(lib().heff_op_set_precision(self.handle, int(precision)), "set_precision")

    def set_fp64_engine(self, engine, nslices=0):
        """FP64-accurate matvecs on the FP64 tensor cores (FP64_DMMA) or emulated on the INT8 tensor cores (FP64_INT8)."""
        check(lib().heff_op_set_fp64_engine(self.handle, int(engine), int(nslices)), "set_fp64_engine")

    def set_graphs(self, enable=True):
        """CUDA-graph replay of the FP64 matvec (heff_op_set_graphs; on by default, needs a non-default stream)."""
        check(lib().heff_op_set_graphs(self.handle, int(bool(enable))), "heff_op_set_graphs")

    def set_profiling(self, enable=True):
        check(lib().heff_op_set_profiling(self.handle, int(bool(enable))), "set_profiling")

    def stage_times(self, reset=False):
        """Summed milliseconds of (layout, GEMM1, mix, GEMM2) over profiled matvecs, and their count."""
        ms = (ctypes.c_double * 4)()
        cnt = ctypes.c_int64(0)
        check(lib().heff_op_stage_times(self.handle, ms, ctypes.byref(cnt), int(bool(reset))), "stage_times")
        return list(ms), int(cnt.value)

    def eigs(self, x0=None, x_out=None, ritz="SA", target=0.0, tol=1e-12, mixed=True, **kw):
        """Eigenpair through the device Davidson solver (heff_eigs).  x0/x_out: device tensors or None.
        Returns (eigval, result dict); raises on errors other than non-convergence."""
        from ._sigs import EigConfig, EigResult

        cfg = EigConfig()
        lib().heff_eig_config_default(ctypes.byref(cfg))
        cfg.ritz = {"SA": 0, "LA": 1, "TARGET": 2}[ritz]
        cfg.target = float(target)
        cfg.tol = float(tol)
        cfg.mixed = int(bool(mixed))
        for k, v in kw.items():
            setattr(cfg, k, v)
        res = EigResult()
        rc = lib().heff_eigs(self.handle, ctypes.byref(cfg), ptr(x0) if x0 is not None else None, ptr(x_out) if x_out is not None else None,
                             ctypes.byref(res))
        if rc not in (HEFF_OK, 5):
            check(rc, "heff_eigs")
        return res.eigval, res.as_dict()

    def get_matrix(self):
        """Dense H_eff as the reference's get_matrix (matvec_mpo.cpp:313-332): device [rows x rows] column-major
        tensor (a flat tensor viewed as its transpose in torch's row-major view), M[(s,a,b),(s',a',b')]."""
        torch = _torch()
        n = self.rows()
        M = torch.empty(n * n, dtype=torch.complex128 if self.cplx else torch.float64, device="cuda")
        check(lib().heff_op_get_matrix(self.handle, ptr(M)), "heff_op_get_matrix")
        return M

    def diagonal(self):
        """Diagonal of H_eff (get_diagonal_new, matvec_mpos.cpp:300-407) as a device tensor of rows() elements."""
        torch = _torch()
        out = torch.empty(self.rows(), dtype=torch.complex128 if self.cplx else torch.float64, device="cuda")
        check(lib().heff_op_diagonal(self.handle, ptr(out)), "heff_op_diagonal")
        return out

    def set_jacobi_blocksize(self, block_size):
        """Block size of the Jacobi preconditioner (set_jcbMaxBlockSize, matvec_mpos.h:147): 1 = diagonal."""
        check(lib().heff_op_set_jacobi_blocksize(self.handle, int(block_size)), "heff_op_set_jacobi_blocksize")

    def jacobi_singular(self):
        """Pivots of the block-Jacobi inversion that were floored (0 for a well-conditioned preconditioner)."""
        c = ctypes.c_int(0)
        check(lib().heff_op_jacobi_singular(self.handle, ctypes.byref(c)), "heff_op_jacobi_singular")
        return int(c.value)

    def MultPc(self, x, y, shift):
        """Jacobi preconditioner (MultPc, matvec_mpos.cpp:1349-1416); device tensors.  Block size 1: y = x / (diag - shift);
        block size > 1: y_blk = (H[blk, blk] - shift0 I)^-1 x_blk with shift0 the shift of the first call."""
        check(lib().heff_op_multpc(self.handle, ptr(x), ptr(y), float(shift)), "heff_op_multpc")

    def device_error(self):
        """Device-side status of the tensor-core pipeline (heff_op_device_error): 0 when every bounded wait completed,
        5 after a non-finite input on the INT8 engine, other nonzero codes after a timed-out wait."""
        code = ctypes.c_int(0)
        check(lib().heff_op_device_error(self.handle, ctypes.byref(code)), "heff_op_device_error")
        return int(code.value)

    @property
    def num_mv(self):
        return int(lib().heff_op_num_mv(self.handle))

    def close(self):
        if getattr(self, "handle", None):
            lib().heff_op_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
