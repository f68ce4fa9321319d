"""ctypes binding of the C oracle (heff_oracle.c).  TEST INFRASTRUCTURE ONLY.

All tensors are numpy arrays in Fortran (column-major) order, which is the
layout of Eigen's Tensor, e.g. ``mps.shape == (spin, chiL, chiR)``.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "liboracle_heff.so")
_lib = None

_I64x = ctypes.POINTER(ctypes.c_int64)
_DP = ctypes.POINTER(ctypes.c_double)


def build():
    """Compile the oracle with its Makefile (gcc, a few seconds)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_SO):
            build()
        L = ctypes.CDLL(_SO)
        for name in ("oracle_matvec_d", "oracle_matvec_z"):
            f = getattr(L, name)
            f.argtypes = [_DP, _DP, _I64x, _DP, _I64x, _DP, _I64x, _DP, _I64x, ctypes.c_int]
            f.restype = ctypes.c_int
        for name in ("oracle_expval_d", "oracle_expval_z"):
            f = getattr(L, name)
            f.argtypes = [_DP, _DP, _I64x, _DP, _I64x, _DP, _I64x, _DP, _I64x]
            f.restype = ctypes.c_int
        for name in ("oracle_env_update_d", "oracle_env_update_z"):
            f = getattr(L, name)
            f.argtypes = [ctypes.c_int, _DP, _DP, _I64x, _DP, _I64x, _DP, _I64x]
            f.restype = ctypes.c_int
        L.oracle_dense_heff_d.argtypes = [_DP, _I64x, _DP, _I64x, _DP, _I64x, _DP, _I64x]
        L.oracle_dense_heff_d.restype = ctypes.c_int
        for nm in ("oracle_get_matrix_d", "oracle_get_matrix_z"):
            f = getattr(L, nm)
            f.argtypes = [_DP, _I64x, _DP, _I64x, _DP, _I64x, _DP, _I64x]
            f.restype = ctypes.c_int
        L.oracle_mpo_ising.argtypes = [_DP, ctypes.c_double, ctypes.c_double, ctypes.c_double]
        L.oracle_mpo_ising.restype = None
        for name in ("oracle_mpo_edge_left", "oracle_mpo_edge_right"):
            f = getattr(L, name)
            f.argtypes = [_DP, _DP, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64]
            f.restype = None
        for name in ("oracle_mpo_merge_d", "oracle_mpo_merge_z"):
            f = getattr(L, name)
            f.argtypes = [_DP, _DP, _I64x, _DP, _I64x]
            f.restype = None
        for name in ("oracle_mpo_square_d", "oracle_mpo_square_z"):
            f = getattr(L, name)
            f.argtypes = [_DP, _DP, _I64x]
            f.restype = None
        L.oracle_truncation_rank.argtypes = [_DP, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64, ctypes.c_double, _DP]
        L.oracle_truncation_rank.restype = ctypes.c_int64
        L.oracle_entropy.argtypes = [_DP, ctypes.c_int64]
        L.oracle_entropy.restype = ctypes.c_double
        _lib = L
    return _lib


def _f(a, cplx):
    a = np.asarray(a)
    a = np.asfortranarray(a.astype(np.complex128 if cplx else np.float64))
    return a


def _p(a):
    return a.ctypes.data_as(_DP)


def _dims(a):
    d = (ctypes.c_int64 * a.ndim)(*a.shape)
    return d


def _is_cplx(*arrs):
    return any(np.iscomplexobj(a) for a in arrs)


def matvec(mps, mpo, envL, envR, branch=-1):
    """y = H_eff theta (contraction_tblis.cpp:277-290).  branch -1: like the reference."""
    c = _is_cplx(mps, mpo, envL, envR)
    mps, mpo, envL, envR = (_f(x, c) for x in (mps, mpo, envL, envR))
    res = np.zeros(mps.shape, dtype=mps.dtype, order="F")
    fn = lib().oracle_matvec_z if c else lib().oracle_matvec_d
    rc = fn(_p(res), _p(mps), _dims(mps), _p(mpo), _dims(mpo), _p(envL), _dims(envL), _p(envR), _dims(envR), branch)
    if rc != 0:
        raise ValueError("oracle_matvec: dimension mismatch")
    return res


def expval(mps, mpo, envL, envR):
    """<theta|W|theta> with environments (contraction_tblis.cpp:64-69)."""
    c = _is_cplx(mps, mpo, envL, envR)
    mps, mpo, envL, envR = (_f(x, c) for x in (mps, mpo, envL, envR))
    out = np.zeros(2)
    fn = lib().oracle_expval_z if c else lib().oracle_expval_d
    rc = fn(_p(out), _p(mps), _dims(mps), _p(mpo), _dims(mpo), _p(envL), _dims(envL), _p(envR), _dims(envR))
    if rc != 0:
        raise ValueError("oracle_expval: dimension mismatch")
    return complex(out[0], out[1]) if c else float(out[0])


def env_update(side, env, mps, mpo):
    """EnvBase::build_block (EnvBase.cpp:109-112 for 'L', :146-149 for 'R')."""
    c = _is_cplx(env, mps, mpo)
    env, mps, mpo = (_f(x, c) for x in (env, mps, mpo))
    if side == "L":
        shape = (mps.shape[2], mps.shape[2], mpo.shape[1])
    else:
        shape = (mps.shape[1], mps.shape[1], mpo.shape[0])
    out = np.zeros(shape, dtype=mps.dtype, order="F")
    fn = lib().oracle_env_update_z if c else lib().oracle_env_update_d
    rc = fn(0 if side == "L" else 1, _p(out), _p(env), _dims(env), _p(mps), _dims(mps), _p(mpo), _dims(mpo))
    if rc != 0:
        raise ValueError("oracle_env_update: dimension mismatch")
    return out


def dense_heff(mps_shape, mpo, envL, envR):
    """Dense H_eff matrix (real), rows/cols ordered like a column-major mps."""
    mpo, envL, envR = (_f(x, False) for x in (mpo, envL, envR))
    n = int(np.prod(mps_shape))
    H = np.zeros((n, n), order="F")
    md = (ctypes.c_int64 * 3)(*mps_shape)
    rc = lib().oracle_dense_heff_d(_p(H), md, _p(mpo), _dims(mpo), _p(envL), _dims(envL), _p(envR), _dims(envR))
    if rc != 0:
        raise ValueError("oracle_dense_heff: dimension mismatch")
    return H


def get_matrix(mps_shape, mpo, envL, envR):
    """MatVecMPO::get_matrix (matvec_mpo.cpp:313-332): M[(s,a,b),(s',a',b')], the transpose of dense_heff."""
    c = _is_cplx(mpo, envL, envR)
    mpo, envL, envR = (_f(x, c) for x in (mpo, envL, envR))
    n = int(np.prod(mps_shape))
    M = np.zeros((n, n), dtype=np.complex128 if c else np.float64, order="F")
    md = (ctypes.c_int64 * 3)(*mps_shape)
    fn = lib().oracle_get_matrix_z if c else lib().oracle_get_matrix_d
    if fn(_p(M), md, _p(mpo), _dims(mpo), _p(envL), _dims(envL), _p(envR), _dims(envR)) != 0:
        raise ValueError("oracle_get_matrix: dimension mismatch")
    return M


def mpo_ising(J, h, eshift=0.0):
    """IsingRandomField::get_mpo -> W[3,3,2,2] (IsingRandomField.cpp:122-129)."""
    W = np.zeros((3, 3, 2, 2), order="F")
    lib().oracle_mpo_ising(_p(W), float(J), float(h), float(eshift))
    return W


def mpo_edge_left(W):
    W = _f(W, False)
    out = np.zeros((1,) + W.shape[1:], order="F")
    lib().oracle_mpo_edge_left(_p(out), _p(W), W.shape[0], W.shape[1], W.shape[2])
    return out


def mpo_edge_right(W):
    W = _f(W, False)
    out = np.zeros((W.shape[0], 1) + W.shape[2:], order="F")
    lib().oracle_mpo_edge_right(_p(out), _p(W), W.shape[0], W.shape[1], W.shape[2])
    return out


def mpo_merge(WA, WB):
    """Two-site merged MPO (matvec_mpos.cpp:104-119)."""
    c = _is_cplx(WA, WB)
    WA, WB = _f(WA, c), _f(WB, c)
    out = np.zeros((WA.shape[0], WB.shape[1], WA.shape[2] * WB.shape[2], WA.shape[3] * WB.shape[3]), dtype=WA.dtype, order="F")
    fn = lib().oracle_mpo_merge_z if c else lib().oracle_mpo_merge_d
    fn(_p(out), _p(WA), _dims(WA), _p(WB), _dims(WB))
    return out


def mpo_square(W):
    """Uncompressed MPO^2 (MpoSite.cpp:57-70)."""
    c = _is_cplx(W)
    W = _f(W, c)
    D0, D1, d, _ = W.shape
    out = np.zeros((D0 * D0, D1 * D1, d, d), dtype=W.dtype, order="F")
    fn = lib().oracle_mpo_square_z if c else lib().oracle_mpo_square_d
    fn(_p(out), _p(W), _dims(W))
    return out


def truncation_rank(S, rank_max, trunc_lim, rank_min=0):
    """svd::solver::get_rank_from_truncation_error (svd.cpp:257-280) -> (rank, truncation_error)."""
    S = np.ascontiguousarray(S, dtype=np.float64)
    err = ctypes.c_double(0)
    r = lib().oracle_truncation_rank(_p(S), S.size, int(rank_max), int(rank_min), float(trunc_lim), ctypes.byref(err))
    if r <= 0:
        raise ValueError("rank <= 0")
    return int(r), float(err.value)


def entropy(S):
    """Von Neumann entropy (measure.cpp:134-138)."""
    S = np.ascontiguousarray(S, dtype=np.float64)
    return float(lib().oracle_entropy(_p(S), S.size))
