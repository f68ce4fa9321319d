"""Subspace-expansion term (EnvBase::get_expansion_term, EnvBase.cpp:303-364) on the device vs the oracle's
restatement: both sides, real and complex, ragged bond dimensions, D = 3 and 9, alpha = 0 / NaN edge cases."""
import numpy as np
import pytest
import torch

import dmrg_b200 as hb
from oracle import clib
from oracle import ref_numpy as rn

pytestmark = pytest.mark.gpu


def inputs(side, S, cL, cR, D, c, seed):
    rng = np.random.default_rng(seed)
    g = (lambda *s: rng.standard_normal(s) + 1j * rng.standard_normal(s)) if c else (lambda *s: rng.standard_normal(s))
    M = np.asfortranarray(g(S, cL, cR))
    if D == 3:
        W = clib.mpo_ising(1.0, 0.8)
    elif D == 9:
        W = clib.mpo_square(clib.mpo_ising(1.0, 0.8))
    else:
        W = np.asfortranarray(g(D, D, S, S))
    if S == 4 and D in (3, 9):
        W = clib.mpo_merge(W, W)
    W = np.asfortranarray(W.astype(np.complex128) if c else W)
    B = np.asfortranarray(g(cL, cL, W.shape[0]) if side == "L" else g(cR, cR, W.shape[1]))
    return B, M, W


def run(side, B, M, W, alpha):
    S, cL, cR = M.shape
    D = W.shape[1] if side == "L" else W.shape[0]
    P = torch.empty(S * cL * cR * D, dtype=torch.complex128 if np.iscomplexobj(M) else torch.float64, device="cuda")
    hb.get_expansion_term(side, P, hb.to_device(B), B.shape, hb.to_device(M), M.shape, hb.to_device(W), W.shape, alpha)
    torch.cuda.synchronize()
    shape = (S, cL, cR * D) if side == "L" else (S, cL * D, cR)
    return hb.to_host(P, shape)


@pytest.mark.parametrize("side", ["L", "R"])
@pytest.mark.parametrize("S,cL,cR,D,c", [(2, 7, 5, 3, False), (2, 5, 9, 3, True), (2, 33, 17, 9, False), (4, 20, 24, 3, True),
                                          (2, 64, 64, 3, False), (2, 128, 96, 9, True), (3, 6, 6, 4, False)])
def test_expansion_term_vs_oracle(cuda, side, S, cL, cR, D, c):
    B, M, W = inputs(side, S, cL, cR, D, c, seed=S * 100 + cL + cR + D)
    P = run(side, B, M, W, 0.35)
    ref = rn.expansion_term_einsum(side, B, M, W, 0.35)
    assert np.linalg.norm(P - ref) <= 1e-12 * np.linalg.norm(ref)


def test_expansion_term_alpha_zero_and_nan(cuda):
    B, M, W = inputs("L", 2, 8, 8, 3, False, seed=1)
    assert not np.any(run("L", B, M, W, 0.0))
    assert not np.any(run("R", *inputs("R", 2, 8, 8, 3, False, seed=2), 0.0))
    with pytest.raises(hb.HeffError):
        run("L", B, M, W, float("nan"))


def test_expansion_term_bad_shape(cuda):
    B, M, W = inputs("L", 2, 8, 6, 3, False, seed=3)
    with pytest.raises(hb.HeffError):
        run("R", B, M, W, 1.0)  # an L-sized environment on the R side
