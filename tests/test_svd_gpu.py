"""SVD truncation parity: device one-sided Jacobi SVD vs LAPACK gesdd (the routine the reference's
svd::solver resolves to for the two-site split) + the reference's rank rule (svd.cpp:257-280)."""
import numpy as np
import pytest
import torch

import dmrg_b200 as hb
import oracle
from oracle import ref_numpy as rn

pytestmark = pytest.mark.gpu


def dev(a):
    return hb.to_device(np.asfortranarray(a))


def run_svd(A, rank_max=0, lim=1e-12):
    m, n = A.shape
    U, S, VT, k, err = hb.svd(dev(A), m, n, rank_max, lim)
    torch.cuda.synchronize()
    return hb.to_host(U, (m, k)), S.cpu().numpy(), hb.to_host(VT, (k, n)), k, err


def graded(m, n, sig, seed):
    rng = np.random.default_rng(seed)
    Q1, _ = np.linalg.qr(rng.standard_normal((m, m)))
    Q2, _ = np.linalg.qr(rng.standard_normal((n, n)))
    k = len(sig)
    return (Q1[:, :k] * sig) @ Q2[:, :k].T


def check_against_gesdd(A, rank_max=0, lim=1e-12, sv_tol=1e-13):
    U, S, VT, k, err = run_svd(A, rank_max, lim)
    Ur, Sr, VTr, kr, errr = rn.svd_truncated(A, rank_max, lim)
    assert k == kr
    smax = Sr[0]
    assert np.max(np.abs(S - Sr)) <= sv_tol * smax
    assert abs(err - errr) <= 1e-13 * smax
    # orthonormal factors (Frobenius norm over k x k entries: bound scales with the size)
    m, n = A.shape
    assert np.linalg.norm(U.T @ U - np.eye(k)) < 1e-13 * max(m, n)
    assert np.linalg.norm(VT @ VT.T - np.eye(k)) < 1e-13 * max(m, n)
    # the truncated product matches gesdd's truncated product
    assert np.linalg.norm(U * S @ VT - (Ur * Sr) @ VTr) <= 1e-12 * np.linalg.norm(A)
    return S, k


@pytest.mark.parametrize("m,n", [(8, 8), (32, 32), (33, 47), (47, 33), (128, 128), (200, 64), (256, 256)])
def test_svd_random_vs_gesdd(cuda, m, n):
    A = np.random.default_rng(m * 1000 + n).standard_normal((m, n))
    check_against_gesdd(A)


def test_svd_rank_deficient_rank_rule(cuda):
    """Exact rank 4 in 128x128 plus 1e-16 noise: the rule with lim=1e-12 must give rank 4 like gesdd."""
    sig = np.array([0.8, 0.5, 0.3, 0.1])
    A = graded(128, 128, sig, 1) + 1e-17 * np.random.default_rng(2).standard_normal((128, 128))
    S, k = check_against_gesdd(A)
    assert k == 4


def test_svd_graded_spectrum(cuda):
    """Singular values spanning 1 .. 1e-13.  gesdd is accurate to ~eps*sigma_max in absolute terms, so the
    comparison is absolute; the rank decision at the 1e-14 truncation limit must agree."""
    sig = np.logspace(0, -13, 40)
    A = graded(96, 96, sig, 3)
    U, S, VT, k, err = run_svd(A, 0, 1e-14)
    Ur, Sr, VTr, kr, errr = rn.svd_truncated(A, 0, 1e-14)
    assert k == kr
    assert np.max(np.abs(S - Sr)) < 1e-14
    assert np.max(np.abs(S[:30] - sig[:30])) < 1e-15  # the constructed spectrum, to the rounding of building A


def test_svd_rank_max(cuda):
    A = np.random.default_rng(5).standard_normal((160, 160))
    S, k = check_against_gesdd(A, rank_max=64)
    assert k == 64


def test_svd_repeated_values(cuda):
    sig = np.array([1.0, 1.0, 1.0, 0.5, 0.5, 0.25])
    A = graded(64, 64, sig, 7)
    S, k = check_against_gesdd(A)
    assert k == 6


@pytest.mark.parametrize("chiL,chiR,rank_max", [(16, 16, 0), (32, 24, 20), (64, 64, 64), (100, 80, 64)])
def test_schmidt_two_site_split(cuda, chiL, chiR, rank_max):
    rng = np.random.default_rng(chiL + chiR)
    theta = np.asfortranarray(rng.standard_normal((4, chiL, chiR)))
    theta /= np.linalg.norm(theta)
    U, S, V, k, err = hb.schmidt_multisite(hb.to_device(theta), 2, 2, chiL, chiR, rank_max, 1e-12)
    torch.cuda.synchronize()
    Ur, Sr, Vr, kr, errr = rn.schmidt_multisite(theta, 2, 2, rank_max, 1e-12)
    assert k == kr
    Sg = S.cpu().numpy()
    assert np.max(np.abs(Sg - Sr)) < 1e-13
    assert abs(np.linalg.norm(Sg) - 1.0) < 1e-14
    assert oracle.entropy(Sg) == pytest.approx(oracle.entropy(Sr), abs=1e-12)
    Ug = hb.to_host(U, (2, chiL, k))
    Vg = hb.to_host(V, (2, k, chiR))
    # U S V reproduces the oracle's truncated theta (gauge-invariant check)
    th_g = np.einsum("sak,k,tkb->stab", Ug, Sg, Vg).reshape(4, chiL, chiR, order="F")
    th_r = np.einsum("sak,k,tkb->stab", Ur, Sr, Vr).reshape(4, chiL, chiR, order="F")
    assert np.linalg.norm(th_g - th_r) < 1e-12


def test_svd_full_size_properties(cuda):
    """2048 x 2048 (two-site split at chi=1024): orthonormality and reconstruction (size-independent)."""
    n = 1024 * 2
    rng = np.random.default_rng(11)
    A = rng.standard_normal((n, n)) / np.sqrt(n)
    U, S, VT, k, err = run_svd(A, 1024, 1e-12)
    assert k == 1024
    Sr = np.linalg.svd(A, compute_uv=False)
    assert np.max(np.abs(S - Sr[:1024])) < 1e-12 * Sr[0]
    assert np.linalg.norm(U.T @ U - np.eye(k)) < 1e-13 * n
    assert err == pytest.approx(np.linalg.norm(Sr[1024:]), rel=1e-10)


@pytest.mark.parametrize("n,cplx", [(512, False), (1024, False), (512, True)])
def test_svd_clustered_rounds_graded(cuda, n, cplx):
    """Sizes whose Jacobi rounds run each pair on a cluster of CTAs (row shares, Gram summed across the cluster):
    a dense graded spectrum (3 % gaps, 1 .. 1e-13) against LAPACK in absolute terms, orthonormal kept factors."""
    rng = np.random.default_rng(n + cplx)
    sig = np.exp(-np.arange(n) * (30.0 / n))
    A = (cgraded if cplx else graded)(n, n, sig, n + 1)
    U, S, VT, k, err = (run_svd_z if cplx else run_svd)(A, n // 2, 1e-12)
    Sr = np.linalg.svd(A, compute_uv=False)
    assert k == n // 2
    assert np.max(np.abs(S - Sr[:k])) < 1e-13
    assert np.linalg.norm(U.conj().T @ U - np.eye(k)) < 1e-13 * n
    assert np.linalg.norm(VT @ VT.conj().T - np.eye(k)) < 1e-13 * n


# ---- complex128 (svd::solver instantiated for cx64, svd.cpp:208-217; zgesdd convention VT = V^H)

def cgauss(rng, *shape):
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


def cgraded(m, n, sig, seed):
    rng = np.random.default_rng(seed)
    Q1, _ = np.linalg.qr(cgauss(rng, m, m))
    Q2, _ = np.linalg.qr(cgauss(rng, n, n))
    k = len(sig)
    return (Q1[:, :k] * sig) @ Q2[:, :k].conj().T


def run_svd_z(A, rank_max=0, lim=1e-12):
    m, n = A.shape
    U, S, VT, k, err = hb.svd(hb.to_device(np.asfortranarray(A.astype(np.complex128))), m, n, rank_max, lim)
    torch.cuda.synchronize()
    assert U.dtype == torch.complex128 and S.dtype == torch.float64
    return hb.to_host(U, (m, k)), S.cpu().numpy(), hb.to_host(VT, (k, n)), k, err


def check_z_against_gesdd(A, rank_max=0, lim=1e-12):
    U, S, VT, k, err = run_svd_z(A, rank_max, lim)
    Ur, Sr, VTr, kr, errr = rn.svd_truncated(A, rank_max, lim)
    assert k == kr
    smax = Sr[0]
    assert np.max(np.abs(S - Sr)) <= 1e-13 * smax
    assert abs(err - errr) <= 1e-13 * smax
    m, n = A.shape
    assert np.linalg.norm(U.conj().T @ U - np.eye(k)) < 1e-13 * max(m, n)
    assert np.linalg.norm(VT @ VT.conj().T - np.eye(k)) < 1e-13 * max(m, n)
    assert np.linalg.norm(U * S @ VT - (Ur * Sr) @ VTr) <= 1e-12 * np.linalg.norm(A)
    return S, k


@pytest.mark.parametrize("m,n", [(8, 8), (33, 47), (47, 33), (128, 128), (200, 64)])
def test_svd_complex_random_vs_zgesdd(cuda, m, n):
    A = cgauss(np.random.default_rng(7 * m + n), m, n)
    check_z_against_gesdd(A)


def test_svd_complex_real_input_matches_real_path(cuda):
    """A real matrix given as complex128 has the real path's singular values."""
    A = np.random.default_rng(21).standard_normal((96, 80))
    Sz = run_svd_z(A.astype(np.complex128))[1]
    Sd = run_svd(A)[1]
    assert np.max(np.abs(Sz - Sd)) < 1e-13 * Sd[0]


def test_svd_complex_rank_deficient_and_graded(cuda):
    S, k = check_z_against_gesdd(cgraded(128, 128, np.array([0.9, 0.4, 0.2, 0.05]), 3) + 1e-17 * cgauss(np.random.default_rng(4), 128, 128))
    assert k == 4
    sig = np.logspace(0, -13, 40)
    A = cgraded(96, 96, sig, 5)
    U, S, VT, k, err = run_svd_z(A, 0, 1e-14)
    Ur, Sr, VTr, kr, errr = rn.svd_truncated(A, 0, 1e-14)
    assert k == kr
    assert np.max(np.abs(S - Sr)) < 1e-14
    # a complex rotation is ~4 real multiply-adds per entry update: a few ulps of sigma_max (real path: 1e-15)
    assert np.max(np.abs(S[:30] - sig[:30])) < 2e-15


def test_svd_complex_rank_max(cuda):
    S, k = check_z_against_gesdd(cgauss(np.random.default_rng(6), 160, 160), rank_max=48)
    assert k == 48


@pytest.mark.parametrize("chiL,chiR,rank_max", [(16, 16, 0), (32, 24, 20), (100, 80, 64)])
def test_schmidt_two_site_split_complex(cuda, chiL, chiR, rank_max):
    rng = np.random.default_rng(3 * chiL + chiR)
    theta = np.asfortranarray(cgauss(rng, 4, chiL, chiR))
    theta /= np.linalg.norm(theta)
    U, S, V, k, err = hb.schmidt_multisite(hb.to_device(theta), 2, 2, chiL, chiR, rank_max, 1e-12)
    torch.cuda.synchronize()
    Ur, Sr, Vr, kr, errr = rn.schmidt_multisite(theta, 2, 2, rank_max, 1e-12)
    assert k == kr
    Sg = S.cpu().numpy()
    assert np.max(np.abs(Sg - Sr)) < 1e-13
    assert abs(err - errr) < 1e-13
    assert oracle.entropy(Sg) == pytest.approx(oracle.entropy(Sr), abs=1e-12)
    Ug = hb.to_host(U, (2, chiL, k))
    Vg = hb.to_host(V, (2, k, chiR))
    th_g = np.einsum("sak,k,tkb->stab", Ug, Sg, Vg).reshape(4, chiL, chiR, order="F")
    th_r = np.einsum("sak,k,tkb->stab", Ur, Sr, Vr).reshape(4, chiL, chiR, order="F")
    assert np.linalg.norm(th_g - th_r) < 1e-12
    # left-canonical U: sum_{s,a} conj(U[s,a,k]) U[s,a,l] = delta_kl
    Um = Ug.reshape(2 * chiL, k, order="F")
    assert np.linalg.norm(Um.conj().T @ Um - np.eye(k)) < 1e-13 * k


def test_svd_complex_large_properties(cuda):
    """1024 x 1024 complex (two-site split at chi=512): singular values, unitarity, tail norm."""
    n = 1024
    A = cgauss(np.random.default_rng(12), n, n) / np.sqrt(2 * n)
    U, S, VT, k, err = run_svd_z(A, 512, 1e-12)
    assert k == 512
    Sr = np.linalg.svd(A, compute_uv=False)
    assert np.max(np.abs(S - Sr[:512])) < 1e-12 * Sr[0]
    assert np.linalg.norm(U.conj().T @ U - np.eye(k)) < 1e-13 * n
    assert err == pytest.approx(np.linalg.norm(Sr[512:]), rel=1e-10)
