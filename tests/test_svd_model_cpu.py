"""Host model of the single-CTA Jacobi SVD used for splits of at most 64 columns (oracle.ref_numpy.jacobi_small_model,
the kernel's pairing, criterion, floor and rotation in its index maps) on the reference's own SVD inputs (the HDF5 test
matrices of tests/svd/main.cpp and the SVD bench's matrices, committed under tests/golden/reference_h5): singular
values within 1e-14 of LAPACK gesdd's largest, A V = G to rounding, V unitary, and convergence in at most 20 sweeps."""
import glob
import os

import numpy as np
import pytest

from dmrg_b200 import replay
from oracle import ref_numpy as rn

FIX = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_h5")


def small_cases():
    out = []
    for p in sorted(glob.glob(os.path.join(FIX, "svd*.h5"))):
        for d in replay.svd_dumps(p):
            if (d["A"].shape[1] + 31) // 32 * 32 <= 64:
                out.append(pytest.param(d["A"], id=f"{os.path.basename(p)}:{d['name']}"))
    return out


@pytest.mark.parametrize("A", small_cases())
def test_jacobi_small_model_on_reference_matrices(A):
    m, n = A.shape
    sig, G, V, sweeps = rn.jacobi_small_model(A)
    ref = np.linalg.svd(A, compute_uv=False)
    assert sweeps <= 20
    assert np.max(np.abs(sig - ref[: len(sig)])) <= 1e-14 * ref[0]
    assert np.linalg.norm(A @ V[:n, :] - G) <= 1e-13 * np.linalg.norm(A)
    assert np.linalg.norm(V.conj().T @ V - np.eye(V.shape[0])) <= 1e-13 * V.shape[0]


def test_round_robin_pairs_cover_every_pair_once():
    for n in (2, 8, 34, 64):
        seen = set()
        for step in range(n - 1):
            cols = [c for k in range(n // 2) for c in rn.round_robin_pair(n, step, k)]
            assert sorted(cols) == list(range(n))  # disjoint pairs covering all columns in each step
            seen |= {tuple(sorted(rn.round_robin_pair(n, step, k))) for k in range(n // 2)}
        assert len(seen) == n * (n - 1) // 2
