"""Generates the golden fixtures in tests/golden/ (run from the repository root:
``python tests/golden/make_golden.py``).

The reference (DMRG++) cannot be built in this environment and ships no golden
vectors for the H_eff path, so these fixtures pin the C oracle against
computations that do not share its code:

* ``contractions.npz`` -- seeded small inputs and the outputs of the numpy
  einsum restatement (oracle/ref_numpy.py), written from the index equations:
  matvec (both chiL>=chiR and chiL<chiR, one- and two-site, D=1/3/9, real and
  complex), expectation values, L/R environment updates, the dense H_eff matrix
  product, the two-site MPO merge and the MPO square.
* ``physics.json`` -- exact-diagonalisation ground energies and half-chain
  entropies of the random-field Ising chain (scipy), free-fermion energies
  (Lieb-Schultz-Mattis), the splitmix64 random fields used by the C++ side, and
  truncation-rule cases worked by hand from svd.cpp:257-280.
"""
import json
import os
import sys

import numpy as np

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), "..", ".."))
sys.path.insert(0, ROOT)

from oracle import physics as ph  # noqa: E402
from oracle import ref_numpy as rn  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))

MATVEC_CASES = [
    # (spin, chiL, chiR, D, complex, seed)
    (4, 5, 7, 3, False, 11),
    (4, 7, 5, 3, False, 12),
    (4, 6, 6, 9, False, 13),
    (4, 9, 4, 9, True, 14),
    (4, 4, 9, 3, True, 15),
    (2, 3, 8, 3, False, 16),
    (2, 8, 3, 9, True, 17),
    (4, 1, 1, 3, False, 18),
    (4, 1, 6, 1, True, 19),
    (4, 16, 16, 3, True, 20),
]
ENV_CASES = [
    # (chiL, chiR, D, complex, seed)
    (5, 7, 3, False, 31),
    (7, 4, 9, False, 32),
    (6, 6, 3, True, 33),
    (3, 8, 9, True, 34),
    (1, 2, 3, False, 35),
]


def main():
    arrays = {}
    for i, (S, cL, cR, D, c, seed) in enumerate(MATVEC_CASES):
        th, W, L, R = ph.heff_inputs(cL, D=D, cplx=c, seed=seed, chiR=cR, spin=S)
        y = rn.matvec_einsum(th, W, L, R)
        e = rn.expval_einsum(th, W, L, R)
        arrays[f"mv{i}_mps"] = th
        arrays[f"mv{i}_mpo"] = W
        arrays[f"mv{i}_envL"] = L
        arrays[f"mv{i}_envR"] = R
        arrays[f"mv{i}_res"] = np.asfortranarray(y)
        arrays[f"mv{i}_expval"] = np.array([e])
        if not c and S * cL * cR <= 256:
            H = np.einsum("axm,mnst,byn->txysab", L, W, R).reshape(S * cL * cR, S * cL * cR, order="F")
            arrays[f"mv{i}_dense"] = np.asfortranarray(H)
    for i, (cL, cR, D, c, seed) in enumerate(ENV_CASES):
        rng = np.random.default_rng(seed)
        M = rng.standard_normal((2, cL, cR)) + (1j * rng.standard_normal((2, cL, cR)) if c else 0)
        M = np.asfortranarray(M)
        EL = ph.hermitian_env(rng, cL, D, c)
        ER = ph.hermitian_env(rng, cR, D, c)
        W = ph.clib.mpo_ising(1.0, 0.8) if D == 3 else ph.clib.mpo_square(ph.clib.mpo_ising(1.0, 0.8))
        if c:
            W = W.astype(np.complex128)
        arrays[f"env{i}_M"] = M
        arrays[f"env{i}_L"] = EL
        arrays[f"env{i}_R"] = ER
        arrays[f"env{i}_W"] = np.asfortranarray(W)
        arrays[f"env{i}_outL"] = np.asfortranarray(rn.env_update_einsum("L", EL, M, W))
        arrays[f"env{i}_outR"] = np.asfortranarray(rn.env_update_einsum("R", ER, M, W))
    WA = np.zeros((3, 3, 2, 2), order="F")
    sx = np.array([[0, 1], [1, 0]])
    sz = np.array([[1, 0], [0, -1]])
    I2 = np.eye(2)
    h, J = 0.83, 1.0
    WA[0, 0] = I2
    WA[1, 0] = sz
    WA[2, 0] = -h * sx
    WA[2, 1] = -J * sz
    WA[2, 2] = I2
    WB = WA.copy()
    WB[2, 0] = -1.21 * sx
    arrays["mpo_ising_h083"] = WA
    arrays["mpo_merge"] = np.asfortranarray(rn.mpo_merge_einsum(WA, WB))
    arrays["mpo_square"] = np.asfortranarray(rn.mpo_square_einsum(WA))
    np.savez_compressed(os.path.join(OUT, "contractions.npz"), **arrays)

    phys = {"ed": [], "free_fermion": [], "fields": [], "truncation": []}
    for L, seed in ((8, 101), (10, 102), (12, 103)):
        hs = ph.random_fields(seed, L)
        e0, s = ph.ed_ground(hs)
        phys["ed"].append({"L": L, "seed": seed, "h": hs.tolist(), "E0": e0, "S_half": s})
    for L, seed in ((16, 201), (32, 202), (24, 203)):
        hs = ph.random_fields(seed, L)
        lev = ph.free_fermion_levels(hs)
        phys["free_fermion"].append({"L": L, "seed": seed, "h": hs.tolist(), "E0": -float(lev.sum()), "Emax": float(lev.sum())})
    for seed in (0, 1, 12345):
        phys["fields"].append({"seed": seed, "h": ph.random_fields(seed, 6).tolist()})
    # svd.cpp:257-280 worked by hand: errors[s] = ||S[s:]||, rank = #(errors >= lim) clipped to rank_max
    phys["truncation"] = [
        {"S": [0.8, 0.6], "rank_max": 0, "lim": 1e-12, "rank": 2},
        {"S": [0.9, 0.4, 1e-7, 1e-13], "rank_max": 0, "lim": 1e-12, "rank": 3},
        {"S": [0.9, 0.4, 1e-7, 1e-13], "rank_max": 2, "lim": 1e-12, "rank": 2},
        {"S": [0.7, 0.5, 0.4, 0.3], "rank_max": 0, "lim": 0.45, "rank": 3},
        {"S": [1.0, 0.0, 0.0], "rank_max": 0, "lim": 1e-12, "rank": 1},
    ]
    with open(os.path.join(OUT, "physics.json"), "w") as f:
        json.dump(phys, f, indent=1)
    print("wrote", os.path.join(OUT, "contractions.npz"), "and physics.json")


if __name__ == "__main__":
    main()
