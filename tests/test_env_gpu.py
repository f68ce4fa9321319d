"""Environment update (EnvBase::build_block) parity: CUDA path vs the CPU oracle, tolerance 1e-12 relative."""
import numpy as np
import pytest
import torch

import dmrg_b200 as hb
import oracle
from oracle import physics as ph
from oracle import ref_numpy as rn

from conftest import relerr

pytestmark = pytest.mark.gpu
TOL = 1e-12


def gpu_env(side, E, M, W):
    dE, dM, dW = (hb.to_device(a) for a in (E, M, W))
    if side == "L":
        shape = (M.shape[2], M.shape[2], W.shape[1])
    else:
        shape = (M.shape[1], M.shape[1], W.shape[0])
    out = torch.empty(int(np.prod(shape)), dtype=dE.dtype, device="cuda")
    hb.env_update(side, out, dE, E.shape, dM, M.shape, dW, W.shape)
    torch.cuda.synchronize()
    return hb.to_host(out, shape)


@pytest.mark.parametrize("i", range(5))
@pytest.mark.parametrize("side", ["L", "R"])
def test_env_golden(cuda, golden, i, side):
    g = lambda k: golden[f"env{i}_{k}"]
    E = g("L") if side == "L" else g("R")
    assert relerr(gpu_env(side, E, g("M"), g("W")), g("out" + side)) < TOL


CASES = [
    # chiL, chiR, D, complex
    (1, 1, 3, False), (1, 3, 1, True), (7, 5, 3, False), (5, 7, 9, True), (31, 17, 3, True), (17, 31, 9, False), (64, 64, 3, True),
    (100, 37, 9, True), (130, 129, 3, False),
]


@pytest.mark.parametrize("cL,cR,D,c", CASES)
@pytest.mark.parametrize("side", ["L", "R"])
def test_env_vs_c_oracle(cuda, cL, cR, D, c, side):
    rng = np.random.default_rng(cL * 7 + cR)
    M = rng.standard_normal((2, cL, cR)) + (1j * rng.standard_normal((2, cL, cR)) if c else 0)
    M = np.asfortranarray(M)
    if D == 1:
        W = np.asfortranarray(rng.standard_normal((1, 1, 2, 2)))
    elif D == 3:
        W = oracle.mpo_ising(1.0, 0.9)
    else:
        W = oracle.mpo_square(oracle.mpo_ising(1.0, 0.9))
    if c:
        W = W.astype(complex)
    E = ph.hermitian_env(rng, cL if side == "L" else cR, W.shape[0] if side == "L" else W.shape[1], c)
    out = gpu_env(side, E, M, W)
    assert relerr(out, oracle.env_update(side, E, M, W)) < TOL


@pytest.mark.parametrize("c", [False, True])
def test_env_large_vs_blas_oracle(cuda, c):
    chi, D = 512, 9
    rng = np.random.default_rng(3)
    M = np.asfortranarray(rng.standard_normal((2, chi, chi)) + (1j * rng.standard_normal((2, chi, chi)) if c else 0))
    W = oracle.mpo_square(oracle.mpo_ising(1.0, 1.1)).astype(complex if c else float)
    for side in ("L", "R"):
        E = ph.hermitian_env(rng, chi, D, c)
        assert relerr(gpu_env(side, E, M, W), rn.env_update_blas(side, E, M, W)) < TOL


def test_env_hermiticity_preserved(cuda):
    """A Hermitian-slice env stays Hermitian per slice after an update with a Hermitian MPO (size-independent)."""
    chi, D = 1024, 3
    rng = np.random.default_rng(8)
    M = np.asfortranarray(rng.standard_normal((2, chi, chi)) + 1j * rng.standard_normal((2, chi, chi)))
    W = oracle.mpo_ising(1.0, 0.6).astype(complex)
    E = ph.hermitian_env(rng, chi, D, True)
    out = gpu_env("L", E, M, W)
    for n in range(D):
        sl = out[:, :, n]
        assert np.linalg.norm(sl - sl.conj().T) <= 1e-12 * np.linalg.norm(sl)


def test_env_rejects_bad_shapes(cuda):
    rng = np.random.default_rng(1)
    M = np.asfortranarray(rng.standard_normal((2, 5, 6)))
    W = oracle.mpo_ising(1.0, 0.9)
    E = ph.hermitian_env(rng, 6, 3, False)  # wrong: L side needs chiL = 5
    with pytest.raises(hb.HeffError) as e:
        gpu_env("L", E, M, W)
    assert e.value.code == 1
