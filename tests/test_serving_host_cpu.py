"""Host side of the serving workload and the library's Python MPO helper, without a GPU: the merged two-site Ising MPO
(and its uncompressed square) that serve_specs builds for every request equals the oracle's restatement of
IsingRandomField.cpp / MpoSite.cpp, and the bench's request stream has the configured shape (chi log-uniform in range,
about 70/30 real/complex, D in {3, 9}, Poisson arrivals in order)."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import dmrg_b200 as hb  # noqa: E402
from oracle import physics as ph  # noqa: E402


@pytest.mark.parametrize("D", [3, 9])
@pytest.mark.parametrize("cplx", [False, True])
def test_two_site_ising_mpo_matches_the_oracle(D, cplx):
    W = hb.two_site_ising_mpo(D, cplx, h1=0.8, h2=1.2)
    ref = ph.ising_two_site_mpo(0.8, 1.2, squared=(D == 9))
    assert W.shape == (D, D, 4, 4) and W.flags.f_contiguous
    assert W.dtype == (np.complex128 if cplx else np.float64)
    assert np.array_equal(np.real(W), ref)
    with pytest.raises(ValueError):
        hb.two_site_ising_mpo(4, False)


def test_serving_stream_shape():
    import bench

    specs = bench.serving_specs(2000, 64, 2048, 4.0, hb.PREC_MIXED, seed=7)
    chis = np.array([s["chi"] for s in specs])
    assert chis.min() >= 64 and chis.max() <= 2048
    # log-uniform: about half the requests below the geometric middle of the range
    assert abs(np.mean(chis < np.sqrt(64 * 2048)) - 0.5) < 0.05
    assert abs(np.mean([s["cplx"] for s in specs]) - 0.3) < 0.04
    assert set(s["D"] for s in specs) == {3, 9}
    arr = np.array([s["arrival"] for s in specs])
    assert arr[0] == 0.0 and np.all(np.diff(arr) >= 0)
    assert abs(len(specs) / arr[-1] - 4.0) < 0.4  # the Poisson rate
    assert all(s["precision"] == hb.PREC_MIXED and s["tol"] == 1e-10 for s in specs)
    assert len(set(s["seed"] for s in specs)) == len(specs)
