"""CUDA-graph replay of the FP64 matvec (heff_op_set_graphs): on an operator with its own stream, the first product of a
shape runs as plain launches and is recorded; later products replay the graph with the input and output pointers
retargeted.  Every product must equal the plain launches' bit for bit, for fresh input/output pairs, across rebinds of
the shape (sweeps, server arenas), with the tail split of the GEMMs on, and inside eigensolves."""
import pytest
import torch

import dmrg_b200 as hb
from oracle import physics as ph

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("chi,chiR,D,c", [(24, 20, 3, False), (40, 40, 9, True), (64, 48, 3, False), (130, 128, 3, True)])
def test_graph_replay_matches_plain_launches(cuda, chi, chiR, D, c):
    th, W, L, R = ph.heff_inputs(chi, D=D, cplx=c, seed=chi + D, chiR=chiR)
    st = torch.cuda.Stream()
    opg = hb.MatVecMPOS([W], L, R, cplx=c, stream=st)
    opg.set_graphs(True)
    opp = hb.MatVecMPOS([W], L, R, cplx=c, stream=st)
    opp.set_graphs(False)
    dt = torch.complex128 if c else torch.float64
    n = th.size
    xs = [torch.randn(n, dtype=dt, device="cuda") for _ in range(5)]
    ys_g = [torch.full((n,), float("nan"), dtype=dt, device="cuda") for _ in range(5)]
    ys_p = [torch.empty(n, dtype=dt, device="cuda") for _ in range(5)]
    torch.cuda.synchronize()
    with torch.cuda.stream(st):
        for k in range(5):  # the first product records, the next four replay with new input/output pointers
            opg.MultAx(xs[k], ys_g[k])
            opp.MultAx(xs[k], ys_p[k])
    st.synchronize()
    for a, b in zip(ys_g, ys_p):
        assert torch.equal(a, b)
    opg.close()
    opp.close()


def test_graphs_through_eigensolves_and_sweeps(cuda):
    """Eigensolves on a streamed operator (graphs on) give the plain path's eigenvalue bit for bit, and a DMRG sweep on
    a stream (shapes rebound per bond) matches the run without a stream (the legacy stream keeps plain launches)."""
    th, W, L, R = ph.heff_inputs(48, D=3, cplx=False, seed=9, chiR=40)
    st = torch.cuda.Stream()
    x0 = hb.to_device(th)
    out = []
    for g in (True, False):
        op = hb.MatVecMPOS([W], L, R, stream=st)
        op.set_graphs(g)
        with torch.cuda.stream(st):
            e, r = op.eigs(x0=x0, tol=1e-12, mixed=False)
        st.synchronize()
        out.append((e, r["num_mv"]))
        op.close()
    assert out[0] == out[1]
    h = ph.random_fields(11, 12)
    r_stream = hb.fdmrg(h, chi_max=32, sweeps=4, stream=st)
    r_plain = hb.fdmrg(h, chi_max=32, sweeps=4)
    assert r_stream["energy"] == r_plain["energy"]
    assert abs(r_stream["energy"] - ph.free_fermion_ground(h)) < 1e-10
