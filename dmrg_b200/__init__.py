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

    def set_profiling(self, enable=True):
        check(lib().heff_op_set_profiling(self.handle, int(bool(enable))), "set_profiling")

    def stage_times(self, reset=False):
        """Summed milliseconds of (layout, GEMM1, mix, GEMM2) over profiled matvecs, and their count."""
        ms = (ctypes.c_double * 4)()
        cnt = ctypes.c_int64(0)
        check(lib().heff_op_stage_times(self.handle, ms, ctypes.byref(cnt), int(bool(reset))), "stage_times")
        return list(ms), int(cnt.value)

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
