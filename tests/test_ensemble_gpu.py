"""Disorder ensemble: independent fDMRG realisations overlapped on one GPU vs one at a time.

Bar: every realisation's energy is the same run alone and in the overlapped ensemble (to 1e-10; the kernels
reduce in a fixed order, so in practice bit-identical), and matches exact diagonalisation to 1e-10 where
chi_max covers the exact Schmidt rank (chi_max >= 2^(L/2)).
"""
import pytest

import dmrg_b200 as hb
from oracle import physics as ph

pytestmark = pytest.mark.gpu


def realisations(n, seed0=900):
    out = []
    for i in range(n):
        L = (8, 10, 12)[i % 3]
        chi = 2 ** (L // 2)
        out.append((ph.random_fields(seed0 + i, L), chi, i))
    return out


def test_ensemble_alone_vs_overlapped_and_exact(cuda):
    reals = realisations(18)
    r1, st1, t1 = hb.ensemble(reals, nthreads=1, sweeps=4)
    r8, st8, t8 = hb.ensemble(reals, nthreads=8, sweeps=4)
    assert all(s == 0 for s in st1) and all(s == 0 for s in st8)
    for (h, chi, seed), a, b in zip(reals, r1, r8):
        assert abs(a["energy"] - b["energy"]) <= 1e-10 * abs(a["energy"])
        e_ed, s_ed = ph.ed_ground(h)
        assert abs(a["energy"] - e_ed) < 1e-10
        assert abs(a["entropy_mid"] - s_ed) < 1e-8
    print(f"ensemble: one at a time {len(reals) / t1:.2f} realisations/s, 8 workers {len(reals) / t8:.2f} realisations/s")


def test_ensemble_mixed_sizes_match_single_driver(cuda):
    """Workspaces sized for the largest member serve smaller chains too (L=16 chi 64 beside L=8 chi 16)."""
    reals = [(ph.random_fields(7, 16), 64, 1), (ph.random_fields(8, 8), 16, 2), (ph.random_fields(9, 12), 32, 3)]
    res, st, _ = hb.ensemble(reals, nthreads=3, sweeps=6)
    assert all(s == 0 for s in st)
    for (h, chi, seed), r in zip(reals, res):
        single = hb.fdmrg(h, chi_max=chi, sweeps=6, seed=seed)
        assert abs(single["energy"] - r["energy"]) <= 1e-10 * abs(r["energy"])
    assert abs(res[0]["energy"] - ph.free_fermion_ground(reals[0][0])) < 1e-10
