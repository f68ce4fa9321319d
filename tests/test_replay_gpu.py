"""Replay of HDF5 dumps on the device.

* The reference's own SVD test matrices and SVD bench matrices (HDF5 files written by the reference through h5pp,
  committed under tests/golden/reference_h5) go through the device SVD with the reference's settings (truncation
  limit 1e-8, tests/svd/main.cpp:71; rank_max and threshold attributes, bench/svd/main.cpp:41-42).  The rank must
  equal the oracle's (LAPACK gesdd + the rank rule of svd.cpp:257-280); singular values agree to 1e-13 of the largest
  and the truncated products to 1e-12 of the matrix norm.  The bench file's matrices are the ones on which the
  reference's MKL gesdd returned info = 1 and -13.
* The golden contraction cases, written into a ``dmrg-contractions.h5`` in the layout of contraction_tblis.cpp:72-84,
  replay through heff_expval and heff_matvec to the golden expectation values and products.
* The reference's dense eigenproblem fixtures (tests/testmatrices/lapacke_matrix-*.h5: a real symmetric 8 x 8 or
  64 x 64 matrix with the eigenvalues and eigenvectors its LAPACK computed, a state theta and the overlaps
  |<v_i|theta>|) go through the device dense eigensolver (heff_dense_eig, the ?syevr of the small-problem path):
  eigenvalues to 1e-13 of the largest, overlaps with theta to 1e-10 (eigenvalue gaps >= 0.12).
"""
import glob
import os

import numpy as np
import pytest

import dmrg_b200 as hb
from dmrg_b200 import replay
from dmrg_b200.h5read import H5File
from oracle import physics as ph
from oracle import ref_numpy as rn

import h5writer

pytestmark = pytest.mark.gpu

FIXTURES = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_h5")


def check_against_oracle(r, A):
    U, S, VT, k, err = rn.svd_truncated(A, r["rank_max"], r["truncation_lim"])
    assert r["rank"] == k, (r["name"], r["rank"], k)
    smax = S[0]
    assert np.max(np.abs(r["S"] - S)) <= 1e-13 * smax
    assert abs(r["truncation_error"] - err) <= 1e-13 * smax
    Ud, VTd = r["U"], r["VT"]
    m, n = A.shape
    assert np.linalg.norm(Ud.conj().T @ Ud - np.eye(k)) < 1e-13 * max(m, n)
    assert np.linalg.norm(VTd @ VTd.conj().T - np.eye(k)) < 1e-13 * max(m, n)
    assert np.linalg.norm((Ud * r["S"]) @ VTd - (U * S) @ VT) <= 1e-12 * np.linalg.norm(A)


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(FIXTURES, "svdmatrix_*.h5"))), ids=os.path.basename)
def test_reference_svd_test_matrices(cuda, path):
    (r,) = replay.replay_svds(path)
    (d,) = replay.svd_dumps(path)
    assert r["truncation_lim"] == 1e-8 and r["shape"] == d["A"].shape
    check_against_oracle(r, d["A"])


def test_reference_svd_bench_matrices(cuda):
    path = os.path.join(FIXTURES, "svd-failed.h5")
    dumps = {d["name"]: d for d in replay.svd_dumps(path)}
    res = replay.replay_svds(path)
    assert [r["name"] for r in res] == [f"svd_lapacke_{i}" for i in range(4)]
    for r in res:
        assert "reference_S" not in r  # the dumped factors come from failed LAPACK calls
        check_against_oracle(r, dumps[r["name"]]["A"])
    assert [r["rank"] for r in res] == [58, 20, 20, 20]


def test_replay_golden_contractions(cuda, golden, tmp_path):
    root = {}
    for i in range(10):
        g = lambda k: golden[f"mv{i}_{k}"]
        # h5pp stores the column-major tensors row-major with the same dimensions: a C-ordered copy of each
        root[f"contraction_{i}"] = {k: np.ascontiguousarray(g(k)) for k in ("mps", "mpo", "envL", "envR")}
    path = str(tmp_path / "dmrg-contractions.h5")
    h5writer.write(path, root)
    res = replay.replay_contractions(path)
    assert [r["name"] for r in res] == [f"contraction_{i}" for i in range(10)]
    for i, r in enumerate(res):
        g = lambda k: golden[f"mv{i}_{k}"]
        scale = np.linalg.norm(g("mps")) * np.linalg.norm(g("res"))
        assert abs(r["energy"] - complex(g("expval")[0])) <= 1e-13 * scale
        assert np.linalg.norm(r["Hpsi"] - g("res")) <= 1e-12 * np.linalg.norm(g("res"))
        assert r["dims"]["mps"] == g("mps").shape


@pytest.mark.parametrize("name", ["lapacke_matrix-1A.h5", "lapacke_matrix-1B.h5", "lapacke_matrix-2A.h5", "lapacke_matrix-2B.h5"])
def test_reference_dense_eigenproblems(cuda, name):
    with H5File(os.path.join(FIXTURES, name)) as f:
        A, w, V = f["matrix"].read(), f["eigvals"].read().ravel(), f["eigvecs"].read()
        th, ov = f["theta"].read().ravel(), f["overlaps"].read().ravel()
    n = A.shape[0]
    ev, Vd = hb.dense_eig(hb.to_device(np.asfortranarray(A)), n)
    ev, Vd = ev.cpu().numpy(), hb.to_host(Vd, (n, n))
    order = np.argsort(w)
    scale = np.abs(w).max()
    assert np.max(np.abs(ev - w[order])) <= 1e-13 * scale
    assert np.max(np.abs(np.abs(Vd.T @ th) - ov[order])) < 1e-10
    assert np.linalg.norm(A @ Vd - Vd * ev) <= 1e-12 * scale * n


def folded_env(rng, chi, base=3):
    """Real environment of an MPO squared: slice (m, m~) is the transpose of slice (m~, m), the symmetry the
    environments of H^2 have, which makes H_eff symmetric for the uncompressed square of a Hermitian MPO."""
    E = np.zeros((chi, chi, base * base))
    for m in range(base):
        for mt in range(m, base):
            X = rng.standard_normal((chi, chi))
            if m == mt:
                X = 0.5 * (X + X.T)
            E[:, :, m + base * mt] = X
            E[:, :, mt + base * m] = X.T
    return np.asfortranarray(E)


def test_replay_eigensolver_bench_dump(cuda, tmp_path):
    """An eigs.h5 in the layout the reference's eigensolver bench reads (bench/eig/main.cpp:45-62): folded local
    problems (the two-site Ising MPO squared, D=9) at chi 6 x 7 and 10 x 10, each with the lowest eigenvalue of its
    dense operator recorded as ``eval``.  replay_eigs solves them like the bench (Ritz SA, tol 1e-12, started from the
    real part of the stored state) on the device and must reach those eigenvalues."""
    from oracle import clib

    root = {}
    for i, (cl, cr) in enumerate([(6, 7), (10, 10)]):
        rng = np.random.default_rng(40 + i)
        W = ph.ising_two_site_mpo(0.7, 1.3, squared=True)
        L, R = folded_env(rng, cl), folded_env(rng, cr)
        mps = rng.standard_normal((4, cl, cr)) + 1j * rng.standard_normal((4, cl, cr))
        H = clib.dense_heff(mps.shape, W, L, R)
        assert np.abs(H - H.T).max() < 1e-12 * np.abs(H).max()
        w = np.linalg.eigvalsh(H)
        root[f"eigs-{i}"] = {"mps": np.ascontiguousarray(mps), "mpo2": np.ascontiguousarray(W), "envL2": np.ascontiguousarray(L),
                             "envR2": np.ascontiguousarray(R),
                             "__attrs__": {"eval": float(w[0]), "size": np.int64(mps.size), "dims": np.array(mps.shape, dtype=np.int64)}}
    path = str(tmp_path / "eigs.h5")
    h5writer.write(path, root)
    res = replay.replay_eigs(path)
    assert [r["name"] for r in res] == ["eigs-0", "eigs-1"]
    for r in res:
        assert r["converged"] and r["num_mv"] > 0
        assert abs(r["eigval"] - r["reference_eval"]) <= 1e-10 * max(1.0, abs(r["reference_eval"]))
    small = replay.replay_eigs(path, max_size=300)
    assert [r["name"] for r in small] == ["eigs-0"]
