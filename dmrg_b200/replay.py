"""Replay of the reference's HDF5 dumps of hot-path operands on the device.

The reference can dump the operands of its hot path to HDF5 through h5pp:

* contraction_tblis.cpp:72-84 (built with ``DMRG_SAVE_CONTRACTION``) appends a group ``contraction_<n>`` holding
  ``mps`` [spin, chiL, chiR], ``mpo`` [D, D, spin, spin], ``envL`` [chiL, chiL, D] and ``envR`` [chiR, chiR, D] to
  ``dmrg-contractions.h5`` for every ``expectation_value`` call;
* math/svd/svd_save.cpp:32-66 and 112-181 write the SVDs of a run to ``svd-save-<seed>.h5``: groups ``svd_<n>`` (or
  ``svd-last`` / ``svd-fail``) holding ``A`` (``A_real`` / ``A_cplx``), the factors ``U``, ``S``, ``VT`` and
  attributes such as ``rank_max``, ``truncation_lim`` and LAPACK's ``info``;
* the reference's SVD tests and bench read the same layouts: one root dataset ``svdmatrix`` per file
  (tests/svd/main.cpp:69-87, truncation limit 1e-8) and groups ``svd_<...>`` with ``A``, ``U``, ``S``, ``V`` and
  attributes ``rank_max`` and ``threshold`` (bench/svd/main.cpp:89-108);
* the reference's eigensolver bench reads ``eigs.h5`` (bench/eig/main.cpp:45-62, 151-160): groups ``eigs-<...>``
  holding the folded-spectrum local problem of an xDMRG step, ``mps`` (complex; its real part is the initial guess),
  ``mpo2`` [D, D, spin, spin], ``envL2``, ``envR2`` (float64), with the solve's recorded attributes ``eval`` (the
  lowest eigenvalue of H^2 found), ``rnorm``, ``iter``, ``mv``, ``op``, ``time``, ``dims`` and ``size``.

``contraction_dumps`` / ``svd_dumps`` / ``eig_dumps`` read those files with :mod:`dmrg_b200.h5read` (no HDF5 library
needed) and return host arrays in the reference's column-major layout; ``replay_contractions`` / ``replay_svds`` /
``replay_eigs`` run every dumped problem through the device (``heff_expval`` + ``heff_matvec``, ``heff_svd``, an
operator + ``heff_eigs``) and return the results next to the dumped reference outputs where the dump holds them.
"""
import re

import numpy as np

from .h5read import H5Dataset, H5File, H5Group

__all__ = ["contraction_dumps", "svd_dumps", "eig_dumps", "replay_contractions", "replay_svds", "replay_eigs"]


def _numbered(names, prefix):
    """Group names with the prefix, in the order the reference wrote them (numeric suffix, then the rest)."""
    picked = [n for n in names if n.startswith(prefix)]

    def key(n):
        m = re.search(r"(\d+)$", n)
        return (0, int(m.group(1)), n) if m else (1, 0, n)

    return sorted(picked, key=key)


def _contraction_dims_ok(mps, mpo, envL, envR):
    """The asserts of contraction_tblis.cpp:56-60 (expectation_value), plus the square environments and square MPO
    site block that the matrix_vector_product contraction (contraction_tblis.cpp:277-290) needs."""
    return (mps.ndim == 3 and mpo.ndim == 4 and envL.ndim == 3 and envR.ndim == 3 and mps.shape[1] == envL.shape[0]
            and mps.shape[2] == envR.shape[0] and mps.shape[0] == mpo.shape[2] and envL.shape[2] == mpo.shape[0]
            and envR.shape[2] == mpo.shape[1] and envL.shape[0] == envL.shape[1] and envR.shape[0] == envR.shape[1]
            and mpo.shape[2] == mpo.shape[3])


def contraction_dumps(path):
    """Every ``contraction_<n>`` group of a ``dmrg-contractions.h5`` file as a dict with ``name`` and the four
    operands as Fortran-ordered arrays with the reference's dimensions.

    h5pp stores Eigen's column-major tensors converted to row-major with unchanged dimensions; a file whose datasets
    carry the reversed dimensions instead (raw column-major buffers) is recognised by the contraction's dimension
    rules and read accordingly.  A group whose operands fit neither raises ``ValueError``."""
    out = []
    with H5File(path) as f:
        for name in _numbered(f.root.keys(), "contraction_"):
            g = f.root[name]
            if not isinstance(g, H5Group):
                continue
            raw = {k: g[k].read() for k in ("mps", "mpo", "envL", "envR")}
            ops = {k: np.asfortranarray(v) for k, v in raw.items()}
            if not _contraction_dims_ok(ops["mps"], ops["mpo"], ops["envL"], ops["envR"]):
                rev = {k: np.asfortranarray(v.transpose()) for k, v in raw.items()}
                if not _contraction_dims_ok(rev["mps"], rev["mpo"], rev["envL"], rev["envR"]):
                    shapes = {k: v.shape for k, v in raw.items()}
                    raise ValueError(f"{path}:{name}: operand dimensions {shapes} do not form a contraction")
                ops = rev
            cplx = any(np.iscomplexobj(v) for v in ops.values())
            dt = np.complex128 if cplx else np.float64
            out.append({"name": name, **{k: np.asfortranarray(v.astype(dt, copy=False)) for k, v in ops.items()}})
    return out


def _first(g, names):
    for n in names:
        if n in g.keys() and isinstance(g[n], H5Dataset):
            return g[n].read()
    return None


def svd_dumps(path, truncation_lim=None):
    """Every SVD problem in an HDF5 file written by the reference, as dicts with ``name``, ``A`` (Fortran-ordered),
    ``rank_max`` (0: none), ``truncation_lim``, and, where the dump holds them, the reference's ``U``, ``S``, ``VT``
    and LAPACK ``info``.

    Recognised layouts: a root dataset ``svdmatrix`` (the reference's SVD test matrices; truncation limit 1e-8 as in
    tests/svd/main.cpp:71 unless ``truncation_lim`` is given) and groups named ``svd...`` holding ``A``/``A_real``/
    ``A_cplx`` with attributes ``rank_max`` and ``truncation_lim`` (svd_save.cpp:67-71) or ``threshold``
    (bench/svd/main.cpp:41-42).  ``truncation_lim``, when given, overrides the dumped limit."""
    out = []
    with H5File(path) as f:
        root = f.root
        if "svdmatrix" in root.keys() and isinstance(root["svdmatrix"], H5Dataset):
            out.append({"name": "svdmatrix", "A": np.asfortranarray(root["svdmatrix"].read()), "rank_max": 0,
                        "truncation_lim": 1e-8 if truncation_lim is None else float(truncation_lim)})
        for name in _numbered(root.keys(), "svd"):
            g = root[name]
            if not isinstance(g, H5Group):
                continue
            A = _first(g, ("A", "A_cplx", "A_real"))
            if A is None or A.ndim != 2 or A.size == 0:
                continue
            at = g.attrs
            lim = truncation_lim
            if lim is None:
                lim = at.get("truncation_lim", at.get("truncation_limit", at.get("threshold", 1e-8)))
            e = {"name": name, "A": np.asfortranarray(A), "rank_max": int(at.get("rank_max", 0)), "truncation_lim": float(lim)}
            U = _first(g, ("U", "U_cplx", "U_real"))
            S = _first(g, ("S",))
            VT = _first(g, ("VT", "VT_cplx", "VT_real", "V"))
            if "info" in at:
                e["info"] = int(at["info"])
            if S is not None and S.size:
                e["S"] = np.real(np.asarray(S)).ravel()
            if U is not None and U.size:
                e["U"] = np.asfortranarray(U)
            if VT is not None and VT.size:
                e["VT"] = np.asfortranarray(VT)
            out.append(e)
    return out


def replay_contractions(path, stream=None, matvec=True):
    """Runs every dumped contraction on the device: ``energy`` = heff_expval (the call the dump came from) and,
    with ``matvec``, ``Hpsi`` = heff_matvec of the same operands (host Fortran-ordered array).  Returns a list of
    dicts with ``name``, ``dims`` and those results."""
    from . import expectation_value, matrix_vector_product, to_device, to_host

    res = []
    for d in contraction_dumps(path):
        mps, mpo, envL, envR = d["mps"], d["mpo"], d["envL"], d["envR"]
        t = {k: to_device(v) for k, v in (("mps", mps), ("mpo", mpo), ("envL", envL), ("envR", envR))}
        e = expectation_value(t["mps"], mps.shape, t["mpo"], mpo.shape, t["envL"], envL.shape, t["envR"], envR.shape, stream)
        r = {"name": d["name"], "dims": {k: d[k].shape for k in ("mps", "mpo", "envL", "envR")}, "energy": e}
        if matvec:
            out = t["mps"].new_empty(t["mps"].shape)
            matrix_vector_product(out, t["mps"], mps.shape, t["mpo"], mpo.shape, t["envL"], envL.shape, t["envR"], envR.shape, stream)
            r["Hpsi"] = to_host(out, mps.shape)
        res.append(r)
    return res


def replay_svds(path, truncation_lim=None, rank_max=None, stream=None):
    """Runs every dumped SVD problem through the device SVD (heff_svd_d / heff_svd_z) with the dump's rank limit
    and truncation limit (or the overrides).  Returns dicts with ``name``, ``shape``, ``rank``, ``S``,
    ``truncation_error``, host ``U`` / ``VT``, and ``reference_S`` where the dump holds singular values from a
    LAPACK call that succeeded (``info`` absent or 0)."""
    from . import svd, to_device, to_host

    res = []
    for d in svd_dumps(path, truncation_lim):
        A = d["A"]
        A = A.astype(np.complex128 if np.iscomplexobj(A) else np.float64, copy=False)
        m, n = A.shape
        rmax = d["rank_max"] if rank_max is None else int(rank_max)
        U, S, VT, k, err = svd(to_device(A), m, n, rmax, d["truncation_lim"], stream)
        r = {"name": d["name"], "shape": (m, n), "rank": k, "S": S.cpu().numpy(), "truncation_error": err,
             "U": to_host(U, (m, k)), "VT": to_host(VT, (k, n)), "rank_max": rmax, "truncation_lim": d["truncation_lim"]}
        if "S" in d and d.get("info", 0) == 0:
            r["reference_S"] = d["S"]
        res.append(r)
    return res


def _attr_value(v):
    if isinstance(v, np.ndarray):
        return v.tolist()
    if isinstance(v, np.generic):
        return v.item()
    return v


def eig_dumps(path):
    """Every ``eigs-<...>`` group of an eigensolver bench file: dicts with ``name``, ``mps`` (the dumped state, complex
    as stored), ``mpo2``, ``envL2``, ``envR2`` (Fortran-ordered float64; the bench reads them as real,
    bench/eig/main.cpp:59-62) and ``attrs`` (the recorded solve: eval, rnorm, iter, mv, op, time, dims, size).  The
    operands must form a contraction (contraction_tblis.cpp:56-60), in h5pp's layout or the reversed one."""
    out = []
    with H5File(path) as f:
        for name in _numbered(f.root.keys(), "eigs-"):
            g = f.root[name]
            if not isinstance(g, H5Group):
                continue
            raw = {"mps": g["mps"].read(), "mpo": g["mpo2"].read(), "envL": g["envL2"].read(), "envR": g["envR2"].read()}
            ops = {k: np.asfortranarray(v) for k, v in raw.items()}
            if not _contraction_dims_ok(ops["mps"], ops["mpo"], ops["envL"], ops["envR"]):
                ops = {k: np.asfortranarray(v.transpose()) for k, v in raw.items()}
                if not _contraction_dims_ok(ops["mps"], ops["mpo"], ops["envL"], ops["envR"]):
                    raise ValueError(f"{path}:{name}: operand dimensions do not form a contraction")
            out.append({"name": name, "mps": ops["mps"], "mpo2": np.asfortranarray(np.real(ops["mpo"]).astype(np.float64)),
                        "envL2": np.asfortranarray(np.real(ops["envL"]).astype(np.float64)),
                        "envR2": np.asfortranarray(np.real(ops["envR"]).astype(np.float64)),
                        "attrs": {k: _attr_value(v) for k, v in g.attrs.items()}})
    return out


def replay_eigs(path, tol=1e-12, precision=None, max_size=None, **eig_kw):
    """Solves every dumped problem as the reference's eigensolver bench does (bench/eig/main.cpp:64-71, 125-135): the
    lowest eigenpair (Ritz SA) of the single-MPO operator MatVecMPO(envL2, envR2, mpo2) at tolerance ``tol``, started
    from the real part of the dumped state, here with the device Davidson solver (heff_eigs).  ``max_size`` skips
    problems with more rows (the bench skips size > 1024).  Returns dicts with ``name``, ``rows``, ``eigval``,
    ``reference_eval`` (the dump's ``eval``, when recorded), ``resnorm``, ``num_mv``, ``seconds``, ``converged``."""
    from . import PREC_FP64, MatVecMPOS, to_device

    res = []
    for d in eig_dumps(path):
        rows = int(np.prod(d["mps"].shape))
        if max_size is not None and rows > max_size:
            continue
        op = MatVecMPOS([d["mpo2"]], d["envL2"], d["envR2"], cplx=False, precision=PREC_FP64 if precision is None else precision)
        try:
            x0 = to_device(np.asfortranarray(np.real(d["mps"]).astype(np.float64)))
            ev, r = op.eigs(x0=x0, ritz="SA", tol=tol, **eig_kw)
        finally:
            op.close()
        out = {"name": d["name"], "rows": rows, "eigval": ev, "resnorm": r["resnorm"], "num_mv": r["num_mv"], "seconds": r["seconds"],
               "converged": bool(r["converged"])}
        if "eval" in d["attrs"]:
            out["reference_eval"] = float(d["attrs"]["eval"])
        res.append(out)
    return res
