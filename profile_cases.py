"""Small fixed workloads for profiler captures (ncu) of single kernels of the hot path.

    python profile_cases.py matvec --chi 1024 --dtype c128 --precision mixed --reps 3
    python profile_cases.py eigs --chi 1024 --dtype f64 --precision fp64
    python profile_cases.py matvec --chi 1024 --dtype c128 --engine int8 --reps 2
    python profile_cases.py fdmrg --L 16 --chi 32 --sweeps 1
    python profile_cases.py svd --chi 512 --reps 1

The matvec case builds the standalone two-site workload (theta[4,chi,chi], Hermitian-slice environments
generated on the device, merged two-site Ising MPO) and applies H_eff `reps` times after one warm-up
application, so `-s`/`-c` in ncu select launches deterministically: each application launches
permute + GEMM1 + mix + GEMM2 (FP64) or split + GEMM1 + mix + GEMM2 (mixed).
"""
import argparse
import sys

import numpy as np


def two_site_ising(D, cplx):
    def site(h):
        W = np.zeros((3, 3, 2, 2))
        sx = np.array([[0.0, 1.0], [1.0, 0.0]])
        sz = np.array([[1.0, 0.0], [0.0, -1.0]])
        W[0, 0] = np.eye(2)
        W[1, 0] = sz
        W[2, 0] = -h * sx
        W[2, 1] = -sz
        W[2, 2] = np.eye(2)
        return W

    def square(W):
        return np.einsum("mnsp,MNpt->mMnNst", W, W).reshape(9, 9, 2, 2, order="F")

    WA, WB = site(0.7), site(1.3)
    if D == 9:
        WA, WB = square(WA), square(WB)
    return [np.asfortranarray(W.astype(np.complex128 if cplx else np.float64)) for W in (WA, WB)]


def main(argv=None):
    import torch

    import dmrg_b200 as hb

    ap = argparse.ArgumentParser()
    ap.add_argument("case", choices=["matvec", "eigs", "fdmrg", "svd"])
    ap.add_argument("--L", type=int, default=16)
    ap.add_argument("--sweeps", type=int, default=1)
    ap.add_argument("--chi", type=int, default=1024)
    ap.add_argument("--D", type=int, default=3)
    ap.add_argument("--dtype", choices=["f64", "c128"], default="c128")
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="fp64")
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--engine", choices=["dmma", "int8"], default="dmma", help="engine of the FP64-accurate matvecs")
    a = ap.parse_args(argv)
    if a.case == "fdmrg":  # two-site ground-state sweeps of the random-field Ising chain, fixed fields in [0.5, 1.5)
        h = 0.5 + np.array([(((i * 0x9E3779B97F4A7C15) >> 11) % 1000003) / 1000003.0 for i in range(1, a.L + 1)])
        r = hb.fdmrg(h, chi_max=a.chi, sweeps=a.sweeps, seed=2)
        print("fdmrg", r["energy"], r["num_mv"], r["t_eig"], r["t_svd"], r["t_env"])
        return 0
    if a.case == "svd":  # truncated SVD of a two-site theta reshaped to (2 chi) x (2 chi), graded spectrum, rank_max chi
        n = 2 * a.chi
        g = torch.Generator(device="cuda").manual_seed(n)
        U, _ = torch.linalg.qr(torch.randn(n, n, device="cuda", dtype=torch.float64, generator=g))
        V, _ = torch.linalg.qr(torch.randn(n, n, device="cuda", dtype=torch.float64, generator=g))
        sv = torch.exp(-torch.arange(n, device="cuda", dtype=torch.float64) * (30.0 / n))
        A = ((U * sv) @ V.T).T.contiguous().reshape(-1)
        for _ in range(a.reps):
            _, S, _, k, err = hb.svd(A, n, n, rank_max=a.chi)
        torch.cuda.synchronize()
        print("svd ok", k, err, float(S[0]))
        return 0
    cplx = a.dtype == "c128"
    prec = hb.PREC_MIXED if a.precision == "mixed" else hb.PREC_FP64
    chi, D = a.chi, a.D
    swap = 3 if D == 9 else 0
    L = hb.to_host(hb.make_env(chi, D, cplx, seed=1, swap_base=swap), (chi, chi, D))
    R = hb.to_host(hb.make_env(chi, D, cplx, seed=2, swap_base=swap), (chi, chi, D))
    op = hb.MatVecMPOS(two_site_ising(D, cplx), L, R, cplx=cplx, precision=prec)
    if a.engine == "int8":
        op.set_fp64_engine(hb.FP64_INT8)
    x = hb.make_vector(op.rows(), cplx, seed=3)
    y = torch.empty_like(x)
    if a.case == "matvec":
        op.MultAx(x, y)
        torch.cuda.synchronize()
        for _ in range(a.reps):
            op.MultAx(x, y)
        torch.cuda.synchronize()
        print("matvec ok", float(torch.linalg.norm(y)))
    else:
        e, r = op.eigs(x0=x, tol=1e-12, mixed=(prec == hb.PREC_MIXED))
        print("eigs", e, r)
    op.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
