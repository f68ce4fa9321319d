"""Eigensolve server: admission by device-memory budget, concurrent requests, results identical alone and in the mix.

Bar: eigenvalues of a request answered in a concurrent mix equal those of the same request solved alone to
1e-10 relative (the kernels reduce in a fixed order, so in practice they are bit-identical), eigenvectors
agree to 1e-10 in norm.
"""
import numpy as np
import pytest
import torch

import dmrg_b200 as hb
from oracle import physics as ph

pytestmark = pytest.mark.gpu


def mpo_for(D, cplx):
    W = ph.ising_two_site_mpo(0.8, 1.2, squared=(D == 9))
    return W.astype(np.complex128 if cplx else np.float64)


@pytest.mark.parametrize("D,c", [(3, False), (3, True), (9, False), (9, True)])
def test_generated_envs_make_heff_hermitian(cuda, D, c):
    chiL, chiR = 5, 4
    L = hb.to_host(hb.make_env(chiL, D, c, seed=11, swap_base=3 if D == 9 else 0), (chiL, chiL, D))
    R = hb.to_host(hb.make_env(chiR, D, c, seed=12, swap_base=3 if D == 9 else 0), (chiR, chiR, D))
    W = mpo_for(D, c)
    H = np.einsum("axm,mnst,byn->txysab", L, W, R).reshape(4 * chiL * chiR, 4 * chiL * chiR, order="F")
    assert np.linalg.norm(H - H.conj().T) <= 1e-13 * np.linalg.norm(H)


REQS = [
    # chi, D, complex, precision, ritz
    (24, 3, False, hb.PREC_FP64, "SA"),
    (40, 9, False, hb.PREC_FP64, "SA"),
    (64, 3, True, hb.PREC_MIXED, "SA"),
    (96, 3, False, hb.PREC_MIXED, "SA"),
    (33, 9, True, hb.PREC_FP64, "SA"),
    (128, 3, True, hb.PREC_FP64, "SA"),
    (72, 9, False, hb.PREC_MIXED, "SA"),
    (16, 3, False, hb.PREC_FP64, "TARGET"),
]


def build(i, spec):
    chi, D, c, prec, ritz = spec
    envL = hb.make_env(chi, D, c, seed=100 + i, swap_base=3 if D == 9 else 0)
    envR = hb.make_env(chi, D, c, seed=200 + i, swap_base=3 if D == 9 else 0)
    th0 = hb.make_vector(4 * chi * chi, c, seed=300 + i)
    out = np.zeros(4 * chi * chi, dtype=np.complex128 if c else np.float64)
    torch.cuda.synchronize()  # device inputs must be complete when a request is submitted
    target = 0.0
    return hb.EigServer.request(mpo_for(D, c), envL, envR, 4, chi, chi, c, theta0=th0, ritz=ritz, target=target, tol=1e-10, precision=prec,
                                theta_out=out), out


def test_alone_vs_mix(cuda):
    # alone: one slot, one request at a time
    alone = []
    srv = hb.EigServer(hbm_budget_bytes=64 << 30, max_inflight=1)
    for i, spec in enumerate(REQS):
        req, out = build(i, spec)
        rid = srv.submit(req)
        r = srv.wait(rid, timeout=300)
        assert r["status"] == 0 and r["converged"] == 1, r
        alone.append((r, out.copy()))
    srv.close()
    # mix: four slots and a budget that holds only about two of the largest requests, all submitted at once
    reqs = [build(i, spec) for i, spec in enumerate(REQS)]
    sizes = sorted(hb.EigServer.request_bytes(r[0][0]) for r in reqs)
    budget = sizes[-1] + sizes[-2] + 1
    srv = hb.EigServer(hbm_budget_bytes=budget, max_inflight=4)
    ids = [srv.submit(r[0]) for r in reqs]
    got = [srv.wait(rid, timeout=300) for rid in ids]
    st = srv.stats()
    srv.close()
    assert st["completed"] == len(REQS) and st["failed"] == 0
    assert st["peak_bytes"] <= budget
    assert st["peak_inflight"] >= 2  # requests really overlapped
    assert st["p50_latency_s"] <= st["p99_latency_s"]
    for (ra, xa), r, (req, out) in zip(alone, got, reqs):
        assert r["status"] == 0 and r["converged"] == 1, r
        assert abs(r["eigval"] - ra["eigval"]) <= 1e-10 * max(1.0, abs(ra["eigval"]))
        assert np.linalg.norm(out - xa) <= 1e-10 * max(1.0, np.linalg.norm(xa))


def test_slot_arenas_are_reused_without_growth(cuda):
    """A slot keeps its device buffers from one request to the next: after one pass over a stream of sizes (real and
    complex, FP64 and mixed, D=3 and 9) a second pass over the same sizes grows no arena (no cudaMalloc/cudaFree, so
    no device-wide synchronisation), and its answers equal the first pass's bit for bit although every request now
    runs in buffers another request left behind."""
    srv = hb.EigServer(hbm_budget_bytes=64 << 30, max_inflight=1)
    first = []
    for i, spec in enumerate(REQS):
        req, out = build(i, spec)
        r = srv.wait(srv.submit(req), timeout=300)
        first.append((r, out.copy()))
    st1 = srv.stats()
    # the second pass runs the sizes in reverse order: the largest shapes first, then the small ones in big buffers
    for i in reversed(range(len(REQS))):
        req, out = build(i, REQS[i])
        r = srv.wait(srv.submit(req), timeout=300)
        r1, x1 = first[i]
        assert r["status"] == 0 and r1["status"] == 0
        assert r["eigval"] == r1["eigval"]
        assert np.array_equal(out, x1)
    st2 = srv.stats()
    srv.close()
    assert st1["arena_grows"] >= 1
    assert st2["arena_grows"] == st1["arena_grows"], (st1, st2)
    assert st2["arena_bytes"] == st1["arena_bytes"]
    assert st2["arena_bytes"] >= max(hb.EigServer.request_bytes(build(i, s)[0][0]) for i, s in enumerate(REQS)) - (4 << 20)


def test_over_budget_request_is_answered_with_oom(cuda):
    srv = hb.EigServer(hbm_budget_bytes=64 << 20, max_inflight=2)
    big, _ = build(0, (512, 3, True, hb.PREC_FP64, "SA"))
    small, _ = build(1, (8, 3, False, hb.PREC_FP64, "SA"))
    rb = srv.submit(big)
    rs = srv.submit(small)
    assert srv.wait(rb, timeout=60)["status"] == 3  # HEFF_OOM
    assert srv.wait(rs, timeout=120)["status"] == 0
    srv.close()


def test_server_matches_direct_eigensolve(cuda):
    chi = 48
    W = mpo_for(3, False)
    envL = hb.make_env(chi, 3, False, seed=5)
    envR = hb.make_env(chi, 3, False, seed=6)
    Lh, Rh = hb.to_host(envL, (chi, chi, 3)), hb.to_host(envR, (chi, chi, 3))
    op = hb.MatVecMPOS([W], Lh, Rh)
    e_direct, _ = op.eigs(tol=1e-12, mixed=False)
    op.close()
    srv = hb.EigServer(max_inflight=2)
    req, out = hb.EigServer.request(W, envL, envR, 4, chi, chi, False, tol=1e-12), None
    r = srv.wait(srv.submit(req), timeout=120)
    srv.close()
    assert abs(r["eigval"] - e_direct) < 1e-10 * abs(e_direct)
