"""The CPU oracle against the golden fixtures (CPU only).

The golden vectors come from computations that share no code with the C oracle
(numpy einsum restatements, exact diagonalisation, the free-fermion solution,
hand-worked truncation cases); see tests/golden/make_golden.py.
"""
import numpy as np
import pytest

import oracle
from oracle import physics as ph
from oracle import ref_numpy as rn

from conftest import relerr

N_MV = 10
N_ENV = 5


@pytest.mark.parametrize("i", range(N_MV))
@pytest.mark.parametrize("branch", [-1, 0, 1])
def test_matvec_oracle_golden(golden, i, branch):
    g = lambda k: golden[f"mv{i}_{k}"]
    y = oracle.matvec(g("mps"), g("mpo"), g("envL"), g("envR"), branch=branch)
    assert relerr(y, g("res")) < 1e-13


@pytest.mark.parametrize("i", range(N_MV))
def test_matvec_blas_baseline_golden(golden, i):
    g = lambda k: golden[f"mv{i}_{k}"]
    y = rn.matvec_blas(g("mps"), g("mpo"), g("envL"), g("envR"))
    assert relerr(y, g("res")) < 1e-13


@pytest.mark.parametrize("i", range(N_MV))
def test_expval_oracle_golden(golden, i):
    g = lambda k: golden[f"mv{i}_{k}"]
    e = oracle.expval(g("mps"), g("mpo"), g("envL"), g("envR"))
    ref = complex(g("expval")[0])
    scale = np.linalg.norm(g("mps")) * np.linalg.norm(g("res"))
    assert abs(e - ref) <= 1e-13 * scale


def test_dense_heff_golden(golden):
    n = 0
    for i in range(N_MV):
        k = f"mv{i}_dense"
        if k not in golden:
            continue
        g = lambda s: golden[f"mv{i}_{s}"]
        H = oracle.dense_heff(g("mps").shape, g("mpo"), g("envL"), g("envR"))
        assert relerr(H, golden[k]) < 1e-14
        y = H @ g("mps").ravel(order="F")
        assert relerr(y, g("res").ravel(order="F")) < 1e-13
        n += 1
    assert n >= 4


@pytest.mark.parametrize("i", range(N_ENV))
@pytest.mark.parametrize("side", ["L", "R"])
def test_env_update_oracle_golden(golden, i, side):
    g = lambda k: golden[f"env{i}_{k}"]
    env = g("L") if side == "L" else g("R")
    out = oracle.env_update(side, env, g("M"), g("W"))
    assert relerr(out, g("out" + side)) < 1e-13


def test_mpo_builders_golden(golden):
    W = oracle.mpo_ising(1.0, 0.83)
    assert np.array_equal(W, golden["mpo_ising_h083"])
    WB = oracle.mpo_ising(1.0, 1.21)
    assert relerr(oracle.mpo_merge(W, WB), golden["mpo_merge"]) == 0.0
    assert relerr(oracle.mpo_square(W), golden["mpo_square"]) == 0.0
    # edges (MpoSite.cpp:449-500): left keeps the last row, right the first column
    assert np.array_equal(oracle.mpo_edge_left(W)[0], W[2])
    assert np.array_equal(oracle.mpo_edge_right(W)[:, 0], W[:, 0])


def test_truncation_rule_golden(physics):
    for case in physics["truncation"]:
        r, err = oracle.truncation_rank(np.array(case["S"]), case["rank_max"], case["lim"])
        assert r == case["rank"], case
        assert err == pytest.approx(np.linalg.norm(np.array(case["S"])[r:]), abs=1e-15)


def test_entropy_formula():
    S = np.array([0.8, 0.6])
    assert oracle.entropy(S) == pytest.approx(-(0.64 * np.log(0.64) + 0.36 * np.log(0.36)), rel=1e-15)
    assert oracle.entropy(np.array([1.0])) == 0.0


def test_splitmix_fields_golden(physics):
    for f in physics["fields"]:
        assert np.array_equal(ph.random_fields(f["seed"], len(f["h"])), np.array(f["h"]))


def test_free_fermion_matches_ed(physics):
    for case in physics["ed"]:
        assert ph.free_fermion_ground(case["h"]) == pytest.approx(case["E0"], abs=1e-10)


def test_mpo_chain_reproduces_ed(physics):
    """Contracting the edge-applied MPO chain into a dense H gives the ED spectrum (L=8)."""
    case = physics["ed"][0]
    mpos = ph.ising_mpos(case["h"])
    # contract W1 ... WL into H[(s1..sL),(t1..tL)] with a boundary-dimension-1 chain
    T = mpos[0][0]  # [mR, d, d]
    H = T  # [m, S_in, S_out] where S indices accumulate site 0 fastest
    for W in mpos[1:]:
        # H[m, P, Q] W[m, n, s, t] -> H'[n, (P, s), (Q, t)]
        m, P, Q = H.shape
        X = np.einsum("mpq,mnst->npsqt", H, W)
        H = X.reshape(W.shape[1], P * W.shape[2], Q * W.shape[3], order="F")
    Hd = H[0]
    w = np.linalg.eigvalsh(Hd)
    assert w[0] == pytest.approx(case["E0"], abs=1e-10)


@pytest.mark.parametrize("i", range(N_ENV))
@pytest.mark.parametrize("side", ["L", "R"])
def test_env_update_blas_baseline_golden(golden, i, side):
    g = lambda k: golden[f"env{i}_{k}"]
    env = g("L") if side == "L" else g("R")
    assert relerr(rn.env_update_blas(side, env, g("M"), g("W")), g("out" + side)) < 1e-13


@pytest.mark.parametrize("c", [False, True])
def test_diagonal_restatement_matches_dense_heff(c):
    """The preconditioner diagonal (get_matrix_element at I == J) equals the diagonal of the dense H_eff."""
    th, W, L, R = ph.heff_inputs(5, D=3, cplx=c, seed=31, chiR=4)
    H = np.einsum("axm,mnst,byn->txysab", L, W, R).reshape(th.size, th.size, order="F")
    d = rn.diagonal_einsum(th.shape, W, L, R)
    assert np.linalg.norm(d - np.diag(H)) < 1e-13 * np.linalg.norm(d)
    if not c:
        Hc = oracle.dense_heff(th.shape, W, L, R)
        assert np.linalg.norm(d - np.diag(Hc)) < 1e-13 * np.linalg.norm(d)


def _expansion_literal(side, B, M, W, alpha):
    """The Eigen expression of EnvBase.cpp:326-330 / :351-355 written with tensordot (same result-dim order
    as Eigen's contract: free dims of the left operand, then of the right) and transpose for shuffle."""
    S, cL, cR = M.shape
    if side == "L":
        X = np.tensordot(B, M, axes=([0], [1]))
        Y = np.tensordot(X, W, axes=([1, 2], [0, 2]))
        shape = (S, cL, cR * W.shape[1])
    else:
        X = np.tensordot(B, M, axes=([0], [2]))
        Y = np.tensordot(X, W, axes=([1, 2], [1, 2]))
        shape = (S, cL * W.shape[0], cR)
    return alpha * Y.transpose(3, 0, 1, 2).reshape(shape, order="F")


@pytest.mark.parametrize("side", ["L", "R"])
@pytest.mark.parametrize("c", [False, True])
def test_expansion_term_restatement(side, c):
    rng = np.random.default_rng(5 if side == "L" else 6)
    S, cL, cR, D = 2, 5, 4, 3
    g = (lambda *s: rng.standard_normal(s) + 1j * rng.standard_normal(s)) if c else (lambda *s: rng.standard_normal(s))
    M = np.asfortranarray(g(S, cL, cR))
    W = np.asfortranarray(g(D, D, S, S))
    B = np.asfortranarray(g(cL, cL, D) if side == "L" else g(cR, cR, D))
    P = rn.expansion_term_einsum(side, B, M, W, 0.7)
    assert np.linalg.norm(P - _expansion_literal(side, B, M, W, 0.7)) < 1e-13 * np.linalg.norm(P)
    assert not np.any(rn.expansion_term_einsum(side, B, M, W, 0.0))


@pytest.mark.parametrize("c", [False, True])
def test_get_matrix_restatement_is_transpose_of_matvec_matrix(c):
    """get_tensor's shuffle {2,0,4,3,1,5} puts the input index first: get_matrix = (matrix of the matvec)^T."""
    th, W, L, R = ph.heff_inputs(4, D=3, cplx=c, seed=41, chiR=3)
    M = oracle.get_matrix(th.shape, W, L, R)
    H = np.einsum("axm,mnst,byn->txysab", L, W, R).reshape(th.size, th.size, order="F")
    assert np.linalg.norm(M - H.T) < 1e-13 * np.linalg.norm(H)
    # the literal Eigen expression (contract, contract, shuffle, column-major cast)
    G = np.tensordot(np.tensordot(L, W, axes=([2], [0])), R, axes=([2], [2])).transpose(2, 0, 4, 3, 1, 5)
    assert np.linalg.norm(M - G.reshape(th.size, th.size, order="F")) < 1e-13 * np.linalg.norm(H)


@pytest.mark.parametrize("nsites,c", [(1, False), (2, True), (3, False), (6, True)])
def test_multi_mpo_literal_equals_merged(nsites, c):
    """The reference's sequential multi-MPO contraction equals the matvec with the merged MPO
    (matvec_mpos.cpp:104-119 order: site 1's physical index fastest)."""
    rng = np.random.default_rng(nsites)
    g = (lambda *s: rng.standard_normal(s) + 1j * rng.standard_normal(s)) if c else (lambda *s: rng.standard_normal(s))
    Ds = [3, 2, 4, 3, 2, 3, 2][: nsites + 1]
    mpos = [np.asfortranarray(g(Ds[i], Ds[i + 1], 2, 2)) for i in range(nsites)]
    W = mpos[0]
    for Wi in mpos[1:]:
        W = oracle.mpo_merge(W, Wi)
    chiL, chiR = 5, 4
    th = np.asfortranarray(g(2 ** nsites, chiL, chiR))
    L = np.asfortranarray(g(chiL, chiL, Ds[0]))
    R = np.asfortranarray(g(chiR, chiR, Ds[nsites]))
    y = rn.matvec_multi_literal(th, mpos, L, R)
    ref = rn.matvec_einsum(th, W, L, R)
    assert np.linalg.norm(y - ref) < 1e-12 * np.linalg.norm(ref)
