"""Benchmark of the H_eff hot path on B200 (one JSON line on rank 0).

Workload (the standalone two-site matvec microbenchmark): theta[4, chi, chi]
complex128 with N(0,1)+iN(0,1) entries, L/R environments [chi, chi, D] with
every D-slice Hermitian ((X + X^dagger)/2, X complex Gaussian), W = the merged
two-site random-field Ising MPO (D=3); chi = 1024.  Synthetic, seeded inputs.

* value     -- algorithmic TFLOP/s of the FP64 (complex128) matvec with inputs
               resident in HBM, CUDA-event timed per step; L2 flushed between steps.
* e2e       -- the same matvec through the C ABI with HOST buffers
               (heff_op_multax_host: H2D of theta, matvec, D2H of y) from pinned memory.
* roofline  -- the dominant kernel (the DMMA GEMM, two launches per matvec),
               achieved = its algorithmic FLOPs / its event-timed duration.
* cpu_baseline -- the reference's contraction sequence (contraction_tblis.cpp:277-290)
               restated with BLAS GEMMs (numpy/OpenBLAS, all host cores) on a bounded sample.

Multi-GPU: a single eigensolve does not shard ("replicas only"): under torchrun
every rank runs its own replica on its own GPU; value = total FLOPs / max time.
The extras (mixed precision, eigensolves, serving, ensemble) run at N=1 only.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

CHI = 1024
D = 3
SPIN = 4
METRIC = "H_eff matvec TFLOP/s (complex128 FP64 path, two-site, chi=1024, D=3)"
UNIT = "TFLOP/s"


def matvec_flops(S, cL, cR, DL, DR, cplx):
    f = 2.0 * S * cL * cL * cR * DL + 2.0 * cL * cR * S * DL * S * DR + 2.0 * S * cL * cR * cR * DR
    return 4.0 * f if cplx else f


def gemm_flops(S, cL, cR, DL, DR, cplx):
    f = 2.0 * S * cL * cL * cR * DL + 2.0 * S * cL * cR * cR * DR
    return 4.0 * f if cplx else f


def make_inputs(chi, D, cplx, seed):
    """Seeded synthetic inputs with the workload's shapes and distributions (no oracle code)."""
    rng = np.random.default_rng(seed)
    if cplx:
        theta = rng.standard_normal((SPIN, chi, chi)) + 1j * rng.standard_normal((SPIN, chi, chi))
    else:
        theta = rng.standard_normal((SPIN, chi, chi))

    def env():
        X = rng.standard_normal((chi, chi, D)) + (1j * rng.standard_normal((chi, chi, D)) if cplx else 0)
        return np.asfortranarray(0.5 * (X + np.conj(np.transpose(X, (1, 0, 2)))))

    L, R = env(), env()
    # merged two-site Ising MPO: W[m,n,s,s'] of two sites (h1=0.7, h2=1.3, J=1)
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

    WA, WB = site(0.7), site(1.3)
    X = np.einsum("mcst,cnuv->mnsutv", WA, WB)
    W = np.asfortranarray(X.reshape(3, 3, 4, 4, order="F"))
    if D == 9:
        raise ValueError("bench uses D=3")
    dt = np.complex128 if cplx else np.float64
    return np.asfortranarray(theta.astype(dt)), [WA.astype(dt), WB.astype(dt)], np.asfortranarray(L.astype(dt)), np.asfortranarray(R.astype(dt))


class ClockSampler:
    """nvidia-smi samples (200 ms) during the timed region."""

    FIELDS = "clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown," \
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[3:7]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(sm)}


SEED = 1  # seed of the headline workload's inputs (both arms)


def bench_config(ws):
    """The workload description both arms print (the reference arm times the same workload on the host cores)."""
    return {"workload": "standalone two-site H_eff matvec, theta[4,1024,1024] complex128, envs [1024,1024,3], Ising MPO D=3",
            "chi": CHI, "D": D, "spin": SPIN, "parallelism": "replicas" if ws > 1 else "none",
            "l2": "working set (theta 64 MB, envs 2 x 50 MB, intermediates 2 x 200 MB) larger than the 126 MB L2; the GPU arm "
                  "also writes a 256 MB buffer between timed steps"}


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for ln in f:
                if ln.startswith("model name"):
                    return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def cpu_reference_sample(chi, D, cplx, budget_s, seed=SEED, one_thread_s=0.0):
    """Time the reference's contraction sequence (BLAS restatement, oracle/ref_numpy.py) on the host."""
    from oracle import ref_numpy as rn

    theta, (WA, WB), L, R = make_inputs(chi, D, cplx, seed)
    X = np.einsum("mcst,cnuv->mnsutv", WA, WB)
    W = np.asfortranarray(X.reshape(WA.shape[0], WB.shape[1], 4, 4, order="F"))
    rn.matvec_blas(theta, W, L, R)  # warm-up (thread pool start, page faults)
    n, t0 = 0, time.perf_counter()
    while True:
        rn.matvec_blas(theta, W, L, R)
        n += 1
        el = time.perf_counter() - t0
        if el >= budget_s:
            break
    F = matvec_flops(SPIN, chi, chi, D, D, cplx)
    one = None
    try:
        from threadpoolctl import threadpool_info, threadpool_limits

        threads = max((p.get("num_threads", 1) for p in threadpool_info() if p.get("internal_api") in ("openblas", "mkl", "blis")), default=1)
        if one_thread_s > 0:
            with threadpool_limits(limits=1):
                n1, t1 = 0, time.perf_counter()
                while True:
                    rn.matvec_blas(theta, W, L, R)
                    n1 += 1
                    e1 = time.perf_counter() - t1
                    if e1 >= one_thread_s:
                        break
            one = {"value": F * n1 / e1 / 1e12, "cores": 1, "matvecs": n1, "seconds": e1}
    except ImportError:
        threads = os.cpu_count()
    return {"value": F * n / el / 1e12, "unit": UNIT, "cores": int(threads), "kind": "port", "matvecs": n, "seconds": el,
            "cpu_model": cpu_model(), "host_cpus": os.cpu_count(),
            "sample": f"{n} complex128 matvecs at chi={chi}, D={D} (full workload size), BLAS restatement of contraction_tblis.cpp:277-290",
            "one_thread": one}


def measure_mixed_and_eigs(hb, torch, op64, mpos, L, R, x, y, flush, stream, F):
    """Mixed-precision matvec (split-BF16 on tcgen05) and whole eigensolves, mixed vs FP64, on the same workload.

    Eigensolve: lowest eigenpair of H_eff (Hermitian: Hermitian-slice envs, Hermitian MPO slices), start vector
    theta, tolerance 1e-12 (||H x - E x|| <= 1e-12 ||H||); mixed = split-BF16 Krylov phase + FP64 Jacobi-Davidson
    refinement.  Wall-clock per solve with the device synchronised on both sides; one warm-up solve each."""
    opm = hb.MatVecMPOS(mpos, L, R, cplx=True, precision=hb.PREC_MIXED, stream=stream)
    ym = torch.empty_like(x)
    with torch.cuda.stream(stream):
        for _ in range(3):
            opm.MultAx(x, ym)
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(10)]
        for k, (a, b) in enumerate(evs):
            flush.fill_(float(k))
            a.record(stream)
            opm.MultAx(x, ym)
            b.record(stream)
        stream.synchronize()
        mixed_ms = sum(a.elapsed_time(b) for a, b in evs) / len(evs)
        op64.MultAx(x, y)
        stream.synchronize()
        rel = float(torch.linalg.norm(ym - y) / torch.linalg.norm(y))

        def solve(op, mixed):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            e, r = op.eigs(x0=x, tol=1e-12, mixed=mixed)
            torch.cuda.synchronize()
            return e, r, time.perf_counter() - t0

        solve(op64, False)
        solve(opm, True)
        s64 = [solve(op64, False) for _ in range(2)]
        smx = [solve(opm, True) for _ in range(2)]
        # the same matvec and solves with the FP64-accurate products emulated on the INT8 tensor cores
        op8 = hb.MatVecMPOS(mpos, L, R, cplx=True, stream=stream)
        op8.set_fp64_engine(hb.FP64_INT8)
        y8 = torch.empty_like(x)
        for _ in range(3):
            op8.MultAx(x, y8)
        ev8 = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(10)]
        for k, (a, b) in enumerate(ev8):
            flush.fill_(float(k))
            a.record(stream)
            op8.MultAx(x, y8)
            b.record(stream)
        stream.synchronize()
        i8_ms = sum(a.elapsed_time(b) for a, b in ev8) / len(ev8)
        rel8 = float(torch.linalg.norm(y8 - y) / torch.linalg.norm(y))
        solve(op8, False)
        s8 = [solve(op8, False) for _ in range(2)]
        opm.set_fp64_engine(hb.FP64_INT8)
        solve(opm, True)
        sm8 = [solve(opm, True) for _ in range(2)]
        op8.close()
    opm.close()
    t64 = statistics.median(t for _, _, t in s64)
    tmx = statistics.median(t for _, _, t in smx)
    t8 = statistics.median(t for _, _, t in s8)
    tm8 = statistics.median(t for _, _, t in sm8)
    e64, r64 = s64[-1][0], s64[-1][1]
    emx, rmx = smx[-1][0], smx[-1][1]
    int8 = {
        "path": "both GEMMs emulated in FP64 accuracy on the INT8 tensor cores (tcgen05 kind::i8): 7 signed 7-bit digit planes per "
                "operand row, equal-weight digit products folded into K, exact INT32 level sums, FP64 recombination",
        "matvec": {"tflops_fp64_equiv": F / (i8_ms / 1e3) / 1e12, "ms": i8_ms, "rel_err_vs_dmma": rel8, "speedup_vs_dmma": None},
        "eigensolves": {"fp64_int8_solves_per_s": 1.0 / t8, "mixed_int8_refinement_solves_per_s": 1.0 / tm8,
                        "abs_dE_fp64_int8": abs(s8[-1][0] - e64), "abs_dE_mixed_int8": abs(sm8[-1][0] - e64),
                        "speedup_fp64_int8_vs_dmma": t64 / t8, "speedup_mixed_int8_vs_dmma_fp64": t64 / tm8,
                        "converged": [s8[-1][1]["converged"], sm8[-1][1]["converged"]], "seconds": [t8, tm8]},
    }
    return {
        "int8_engine": int8,
        "mixed_matvec": {"tflops": F / (mixed_ms / 1e3) / 1e12, "ms": mixed_ms, "rel_err_vs_fp64": rel,
                         "speedup_vs_fp64_matvec": None, "path": "split-BF16 (hi+mid, 3 products) tcgen05 GEMMs, FP32 accumulation",
                         "flops": "algorithmic (dense FP64 count); the tensor cores execute 3x that in BF16"},
        "eigensolves": {"workload": "lowest eigenpair of the same H_eff, chi=1024 complex128, tol 1e-12", "fp64_solves_per_s": 1.0 / t64,
                        "mixed_solves_per_s": 1.0 / tmx, "speedup_mixed_vs_fp64": t64 / tmx, "abs_dE": abs(emx - e64), "E_fp64": e64,
                        "fp64_matvecs": r64["num_mv"], "mixed_split_matvecs": rmx["num_mv_mixed"], "mixed_fp64_matvecs": rmx["num_mv_fp64"],
                        "converged": [r64["converged"], rmx["converged"]], "seconds_fp64": t64, "seconds_mixed": tmx},
    }


def two_site_mpo(D, cplx):
    """Merged two-site Ising MPO (D=3) or merged uncompressed MPO squared (D=9), h = 0.8 / 1.2, J = 1."""
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
        X = np.einsum("mnsp,MNpt->mMnNst", W, W)
        return X.reshape(9, 9, 2, 2, order="F")

    WA, WB = site(0.8), site(1.2)
    if D == 9:
        WA, WB = square(WA), square(WB)
    X = np.einsum("mcst,cnuv->mnsutv", WA, WB)
    W = X.reshape(WA.shape[0], WB.shape[1], 4, 4, order="F")
    return np.asfortranarray(W.astype(np.complex128 if cplx else np.float64))


def host_matvec(th, W, L, R):
    """y = H_eff theta on the host in the reference's contraction order (contraction_tblis.cpp:277-290, chiL >= chiR):
    theta . envL over a, then . W over (m, s), then . envR over (b, n); numpy tensordot (BLAS)."""
    T1 = np.tensordot(th, L, axes=([1], [0]))  # [s, b, a', m]
    T2 = np.tensordot(T1, W, axes=([0, 3], [2, 0]))  # [b, a', n, s']
    y = np.tensordot(T2, R, axes=([0, 2], [0, 2]))  # [a', s', b']
    return np.asfortranarray(y.transpose(1, 0, 2))


def truncation_rank(S, rank_max, trunc_lim):
    """Rank rule of svd.cpp:257-280: keep singular values while the 2-norm of the discarded tail stays >= trunc_lim,
    at most rank_max; returns (rank, truncation error = norm of the discarded tail)."""
    S = np.asarray(S)
    tail = np.sqrt(np.cumsum((S[::-1] ** 2))[::-1])  # tail[k] = ||S[k:]||
    k = int(np.count_nonzero(tail >= trunc_lim))
    if rank_max > 0:
        k = min(k, rank_max)
    err = float(np.linalg.norm(S[k:])) if k < len(S) else 0.0
    return k, err


def measure_grid(hb, torch, stream, flush, chis=(256, 512, 1024, 2048), Ds=(3, 9), reps=5):
    """The precision-microbenchmark grid: the standalone two-site matvec (theta Gaussian, Hermitian-slice envs generated
    on the device, W = merged two-site Ising MPO for D=3 or its uncompressed square for D=9) at every chi and D, complex128
    and float64; FP64 on the DMMA engine, FP64 on the INT8 engine and mixed split-BF16, each CUDA-event timed over `reps`
    applications with the L2 flushed between them, and each compared with the host product in the reference's
    contraction order (host_matvec; rel. error ||y - y_host|| / ||y_host||)."""
    out = {}
    for cplx in (True, False):
        tag = "c128" if cplx else "f64"
        rows = {}
        for chi in chis:
            for D in Ds:
                W = two_site_mpo(D, cplx)
                sb = 3 if D == 9 else 0
                Ld = hb.make_env(chi, D, cplx, seed=1000 + chi + D, swap_base=sb)
                Rd = hb.make_env(chi, D, cplx, seed=2000 + chi + D, swap_base=sb)
                L = hb.to_host(Ld, (chi, chi, D))
                R = hb.to_host(Rd, (chi, chi, D))
                x = hb.make_vector(SPIN * chi * chi, cplx, seed=3000 + chi + D)
                th = hb.to_host(x, (SPIN, chi, chi))
                del Ld, Rd
                y_ref = host_matvec(th, W, L, R).ravel(order="F")
                nref = float(np.linalg.norm(y_ref))
                F = matvec_flops(SPIN, chi, chi, D, D, cplx)
                row = {"flops": F}

                def timed(op, name):
                    y = torch.empty_like(x)
                    with torch.cuda.stream(stream):
                        for _ in range(2):
                            op.MultAx(x, y)
                        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(reps)]
                        for k, (a, b) in enumerate(evs):
                            flush.fill_(float(k))
                            a.record(stream)
                            op.MultAx(x, y)
                            b.record(stream)
                        stream.synchronize()
                    ms = sum(a.elapsed_time(b) for a, b in evs) / reps
                    err = float(np.linalg.norm(y.cpu().numpy() - y_ref) / nref)
                    row[name] = {"ms": ms, "tflops": F / (ms / 1e3) / 1e12, "rel_err_vs_host": err}
                    return y

                op = hb.MatVecMPOS([W], L, R, cplx=cplx, stream=stream)
                op.set_profiling(True)
                op.stage_times(reset=True)
                timed(op, "fp64_dmma")
                st, cnt = op.stage_times(reset=True)
                op.set_profiling(False)
                row["fp64_dmma"]["stage_ms"] = [v / max(cnt, 1) for v in st]
                row["fp64_dmma"]["frac_of_nominal_40"] = row["fp64_dmma"]["tflops"] / 40.0
                op.set_fp64_engine(hb.FP64_INT8)
                timed(op, "fp64_int8")
                op.close()
                opm = hb.MatVecMPOS([W], L, R, cplx=cplx, precision=hb.PREC_MIXED, stream=stream)
                timed(opm, "mixed")
                opm.close()
                rows[f"chi{chi}_D{D}"] = row
                del x, L, R, th, y_ref
                torch.cuda.empty_cache()
        out[tag] = rows
    out["workload"] = ("two-site H_eff matvec theta[4,chi,chi] Gaussian, envs [chi,chi,D] Hermitian per slice (D=9: MPO-squared swap "
                       "symmetry), W = merged two-site Ising MPO (D=3) or its square (D=9); FLOPs are the dense algorithmic count; "
                       "rel_err_vs_host: against host_matvec, the contraction sequence of contraction_tblis.cpp:277-290 in numpy")
    return out


def measure_svd(hb, torch, chis=(512, 1024), reps=3):
    """Two-site SVD truncation at the split shape (2 chi) x (2 chi): a matrix with a Schmidt-like graded spectrum
    (singular values 1 .. 1e-13, geometric, random orthogonal factors), rank_max = chi, truncation limit 1e-12.
    Device one-sided Jacobi (heff_svd_d) vs LAPACK gesdd through numpy on all host cores (the routine the reference's
    svd::solver resolves to for this shape); singular values compared with gesdd's."""
    out = {}
    rng = np.random.default_rng(41)
    for chi in chis:
        n = 2 * chi
        Q1, _ = np.linalg.qr(rng.standard_normal((n, n)))
        Q2, _ = np.linalg.qr(rng.standard_normal((n, n)))
        sv = np.geomspace(1.0, 1e-13, n)
        A = np.asfortranarray((Q1 * sv) @ Q2.T)
        Ad = hb.to_device(A)
        hb.svd(Ad, n, n, rank_max=chi, trunc_lim=1e-12)
        torch.cuda.synchronize()
        tg = []
        for _ in range(reps):
            t0 = time.perf_counter()
            U, S, VT, k, terr = hb.svd(Ad, n, n, rank_max=chi, trunc_lim=1e-12)
            torch.cuda.synchronize()
            tg.append(time.perf_counter() - t0)
        tc = []
        for _ in range(2):
            t0 = time.perf_counter()
            Uc, Sc, VTc = np.linalg.svd(A, full_matrices=False)  # LAPACK ?gesdd
            kc, errc = truncation_rank(Sc, chi, 1e-12)
            tc.append(time.perf_counter() - t0)
        Sg = S.cpu().numpy()
        m = min(len(Sg), len(Sc))
        out[f"{n}x{n}"] = {"gpu_ms": 1e3 * statistics.median(tg), "cpu_gesdd_ms": 1e3 * min(tc), "speedup_vs_cpu": min(tc) / statistics.median(tg),
                           "rank_gpu": k, "rank_gesdd": kc, "max_sigma_err_rel_sigma_max": float(np.max(np.abs(Sg[:m] - Sc[:m])) / Sc[0]),
                           "trunc_err_gpu": terr, "trunc_err_gesdd": errc}
        del Ad, U, S, VT
    out["workload"] = "real (2chi)x(2chi), singular values geometric 1..1e-13, rank_max=chi, truncation limit 1e-12 (svd.cpp:257-280)"
    return out


def measure_svd_reference_matrices(hb, torch, reps=5):
    """The device SVD on the reference's own SVD inputs: the HDF5 test matrices of tests/svd/main.cpp:69-87 (normalised
    complex two-site states, truncation limit 1e-8) and the SVD bench's matrices (bench/svd/main.cpp:89-108, their
    rank_max and threshold), committed under tests/golden/reference_h5 and read through dmrg_b200.replay.  Per matrix:
    the median of `reps` device SVDs (heff_svd_z / heff_svd_d, host-synchronised) against LAPACK gesdd through numpy
    on the host cores with the same rank rule; ranks and singular values compared."""
    import glob

    from dmrg_b200 import replay

    rows = []
    files = sorted(glob.glob(os.path.join(ROOT, "tests", "golden", "reference_h5", "svd*.h5")))
    for path in files:
        for d in replay.svd_dumps(path):
            A = np.asfortranarray(d["A"].astype(np.complex128 if np.iscomplexobj(d["A"]) else np.float64))
            m, n = A.shape
            rmax, lim = d["rank_max"], d["truncation_lim"]
            Ad = hb.to_device(A)
            hb.svd(Ad, m, n, rmax, lim)
            torch.cuda.synchronize()
            tg = []
            for _ in range(reps):
                t0 = time.perf_counter()
                U, S, VT, k, err = hb.svd(Ad, m, n, rmax, lim)
                torch.cuda.synchronize()
                tg.append(time.perf_counter() - t0)
            tc = []
            for _ in range(reps):
                t0 = time.perf_counter()
                Sc = np.linalg.svd(A, compute_uv=False)  # LAPACK ?gesdd
                kc, _ = truncation_rank(Sc[np.nonzero(Sc)], rmax, lim)
                tc.append(time.perf_counter() - t0)
            Sg = S.cpu().numpy()
            rows.append({"name": f"{os.path.basename(path)}:{d['name']}", "shape": [m, n], "rank": k, "rank_gesdd": kc,
                         "gpu_ms": 1e3 * statistics.median(tg), "gesdd_ms": 1e3 * statistics.median(tc),
                         "max_sigma_err_rel": float(np.max(np.abs(Sg[:min(k, kc)] - Sc[:min(k, kc)])) / Sc[0]) if min(k, kc) else 0.0})
            del Ad, U, S, VT
    g = [r["gpu_ms"] for r in rows]
    c = [r["gesdd_ms"] for r in rows]
    return {"matrices": len(rows), "ranks_equal": all(r["rank"] == r["rank_gesdd"] for r in rows),
            "max_sigma_err_rel": max(r["max_sigma_err_rel"] for r in rows), "gpu_ms_median": statistics.median(g),
            "gesdd_ms_median": statistics.median(c), "per_matrix": rows,
            "workload": "the reference's SVD test and bench matrices (HDF5, 2x8 .. 138x90, complex and real), their truncation "
                        "limits and rank limits; device one-sided Jacobi vs numpy gesdd on the host cores"}


def measure_eigs_folded(hb, torch, chi=512):
    """Eigensolves at the excited-state configuration's shape: real H_eff with the merged uncompressed MPO squared
    (D=9) at chi_max=512, environments with the MPO-squared swap symmetry (generated on the device), lowest
    eigenpair to tol 1e-12; FP64 Krylov, FP64 Jacobi-preconditioned, and mixed (split-BF16 + FP64 refinement).
    One warm-up solve each, then the median of two."""
    W = two_site_mpo(9, False)
    L = hb.to_host(hb.make_env(chi, 9, False, seed=11, swap_base=3), (chi, chi, 9))
    R = hb.to_host(hb.make_env(chi, 9, False, seed=12, swap_base=3), (chi, chi, 9))
    op64 = hb.MatVecMPOS([W], L, R, cplx=False)
    opm = hb.MatVecMPOS([W], L, R, cplx=False, precision=hb.PREC_MIXED)
    x0 = hb.make_vector(op64.rows(), False, seed=13)

    def solve(op, **kw):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e, r = op.eigs(x0=x0, tol=1e-12, **kw)
        torch.cuda.synchronize()
        return e, r, time.perf_counter() - t0

    out = {}
    for name, op, kw in (("fp64", op64, {"mixed": False}), ("fp64_jacobi", op64, {"mixed": False, "precond": 1}), ("mixed", opm, {"mixed": True})):
        solve(op, **kw)
        runs = [solve(op, **kw) for _ in range(2)]
        t = statistics.median(r[2] for r in runs)
        e, r = runs[-1][0], runs[-1][1]
        out[name] = {"solves_per_s": 1.0 / t, "seconds": t, "E": e, "matvecs": r["num_mv"], "mixed_matvecs": r["num_mv_mixed"],
                     "converged": r["converged"]}
    op64.close()
    opm.close()
    out["workload"] = "lowest eigenpair, real H_eff, two-site MPO squared D=9, chi=512, tol 1e-12 (the folded-spectrum solve's shape)"
    out["speedup_mixed_vs_fp64"] = out["fp64"]["seconds"] / out["mixed"]["seconds"]
    out["abs_dE_mixed_vs_fp64"] = abs(out["mixed"]["E"] - out["fp64"]["E"])
    out["abs_dE_jacobi_vs_fp64"] = abs(out["fp64_jacobi"]["E"] - out["fp64"]["E"])
    return out


def measure_xdmrg(hb, L, chi, sweeps, one_site=False, seed=4242, offset=None, precision=None, jcb=128, max_mv=60000):
    """The excited-state configuration's sweep: random-field Ising chain (h ~ U[0.5,1.5] from splitmix64), energy
    density 0.5 (E_t = 0 for the symmetric spectrum, moved off the symmetric point by `offset`, a fraction of the level
    spacing), folded spectrum with the MPO squared, FP64, local solves preconditioned with 128-row Jacobi blocks and up
    to 60000 matvecs.  Reports the variance, the energy and, where the spectrum can be listed (L <= 20), the distance to
    the nearest exact eigenvalue (free-fermion levels E0 + sum of a subset of 2 Lambda_k)."""
    h = np.array(splitmix_fields(seed, L))
    B = np.diag(h) + np.diag(np.ones(L - 1), 1)
    lev = np.linalg.svd(B, compute_uv=False)
    off = offset if offset is not None else (1e-3 if L <= 14 else 1e-4)
    t0 = time.perf_counter()
    prec = hb.PREC_FP64 if precision is None else precision
    r = hb.xdmrg(h, 0.0 + off, one_site=one_site, chi_max=chi, sweeps=sweeps, eig_tol=1e-12, seed=1, jcb_blocksize=jcb,
                 eig_max_matvecs=max_mv, precision=prec)
    secs = time.perf_counter() - t0
    out = {"L": L, "chi_max": chi, "sweeps": sweeps, "one_site": one_site, "precision": "mixed" if prec == hb.PREC_MIXED else "fp64",
           "jacobi_block": jcb, "local_solve_matvec_limit": max_mv,
           "target": off, "variance": r["variance"], "mixed_matvecs": r["num_mv_mixed"],
           "energy": r["energy"], "chi_mid": r["chi_mid"], "matvecs": r["num_mv"], "unconverged_local_solves": r["unconverged_solves"],
           "seconds": secs, "objective_per_sweep": list(r["energy_per_sweep"][: r["sweeps_done"]])}
    if L <= 20:
        e = np.array([0.0])
        for x in lev:
            e = np.concatenate([e, e + 2 * x])
        out["distance_to_nearest_eigenvalue"] = float(np.min(np.abs(-lev.sum() + e - r["energy"])))
    return out


def serving_specs(n_req, chi_lo, chi_hi, rate, precision, seed=2024):
    """The serving stream's requests: Poisson arrivals at `rate`/s, chi log-uniform in [chi_lo, chi_hi], 70% float64 /
    30% complex128, D=3 (H, lowest eigenpair) or D=9 (MPO squared: lowest eigenpair of the folded operator) with equal
    probability, tol 1e-10, each request's environments and start vector seeded by its index."""
    rng = np.random.default_rng(seed)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, n_req))
    specs = []
    for i in range(n_req):
        chi = int(round(np.exp(rng.uniform(np.log(chi_lo), np.log(chi_hi)))))
        D = 3 if rng.uniform() < 0.5 else 9
        cplx = bool(rng.uniform() < 0.3)
        specs.append({"chi": chi, "D": D, "cplx": cplx, "seed": seed * 100003 + i, "precision": precision, "tol": 1e-10,
                      "arrival": float(arrivals[i] - arrivals[0])})
    return specs


def measure_serving(hb, torch, n_req, chi_lo, chi_hi, rate, precision, seed=2024, max_inflight=8):
    """The serving stream through one EigServer (hb.serve_specs): p50/p99 latency, solves/s, the server's peak
    concurrency and what its slot arenas hold."""
    specs = serving_specs(n_req, chi_lo, chi_hi, rate, precision, seed)
    resp, st_codes, secs, st = hb.serve_specs(specs, max_inflight=max_inflight, wait_timeout=1800)
    ok = sum(1 for c in st_codes if c == 0)
    return {"requests": n_req, "answered_ok": ok, "p50_latency_s": st["p50_latency_s"], "p99_latency_s": st["p99_latency_s"],
            "max_latency_s": st["max_latency_s"], "solves_per_s": st["solves_per_s"], "stream_seconds": secs,
            "p50_latency_from_arrival_s": st.get("p50_latency_from_arrival_s"), "p99_latency_from_arrival_s": st.get("p99_latency_from_arrival_s"),
            "peak_inflight": st["peak_inflight"], "peak_device_bytes": st["peak_bytes"], "arena_bytes": st["arena_bytes"],
            "arena_grows": st["arena_grows"], "arrival_rate_per_s": rate, "chi_range": [chi_lo, chi_hi],
            "chi_max_served": max(s["chi"] for s in specs), "eigvals_head": [r["eigval"] for r in resp[:4]]}


def splitmix_fields(seed, L, lo=0.5, hi=1.5):
    """h_i ~ U[lo, hi) from splitmix64 (the generator the library's sweep driver and tests share)."""
    m64 = (1 << 64) - 1
    st, out = seed & m64, []
    for _ in range(L):
        st = (st + 0x9E3779B97F4A7C15) & m64
        z = st
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & m64
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & m64
        z ^= z >> 31
        out.append(lo + (hi - lo) * ((z >> 11) * (1.0 / 9007199254740992.0)))
    return out


def measure_ensemble(hb, n, sweeps, nthreads, seed=77, serial_n=None):
    """The disorder ensemble: L uniform in {12,16,20,24}, chi_max uniform in {32,64,128,256}, h_i ~ U[0.5,1.5] per
    realisation seed, real FP64 two-site fDMRG; realisations/s of all n on overlapped workers, against one at a time on
    the first serial_n of them (default all: the same distribution, so the per-realisation rate compares), and the
    largest energy difference over the realisations both runs computed."""
    rng = np.random.default_rng(seed)
    reals = []
    for i in range(n):
        L = int(rng.choice([12, 16, 20, 24]))
        chi = int(rng.choice([32, 64, 128, 256]))
        reals.append((splitmix_fields(seed * 100003 + i, L), chi, i))
    ns = n if not serial_n else min(serial_n, n)
    r1, s1, t1 = hb.ensemble(reals[:ns], nthreads=1, sweeps=sweeps)
    rp, sp, tp = hb.ensemble(reals, nthreads=nthreads, sweeps=sweeps)
    dE = max(abs(a["energy"] - b["energy"]) for a, b in zip(r1, rp))
    return {"realisations": n, "one_at_a_time_sample": ns, "sweeps": sweeps, "workers": nthreads, "one_at_a_time_per_s": ns / t1,
            "overlapped_per_s": n / tp, "speedup": (t1 / ns) / (tp / n), "max_abs_dE_between_runs": dE,
            "ok": int(all(s == 0 for s in s1 + sp)),
            "workload": "L in {12,16,20,24}, chi_max in {32,64,128,256}, two-site fDMRG FP64, random-field Ising h~U[0.5,1.5]"}


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def reduce_max_over_ranks(values, dist=None):
    """Element-wise max of a list of floats over all ranks (NCCL reduces device tensors, gloo host ones)."""
    if dist is None:
        return [float(v) for v in values]
    import torch

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.cpu().tolist()]


def job_tflops(flops_per_step, steps_per_rank, world, max_ms):
    """Whole-job throughput: the work of all ranks divided by the slowest rank's time."""
    return world * flops_per_step * steps_per_rank / (max_ms / 1e3) / 1e12


def run_reference(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    budget = 4.0
    vals = []
    for _ in range(args.warmup):
        cpu_reference_sample(CHI, D, True, 1.0)
    for _ in range(args.steps):
        vals.append(cpu_reference_sample(CHI, D, True, budget))
    v = sum(x["value"] for x in vals) / len(vals)
    mv = sum(x["matvecs"] for x in vals)
    sec = sum(x["seconds"] for x in vals)
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * sec / mv, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c128",
            "data": "synthetic (seeded Gaussian theta, Hermitian-slice envs, Ising two-site MPO)", "config": bench_config(ws),
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": vals[0]["cores"], "kind": "port", "cpu_model": vals[0]["cpu_model"],
                             "sample": f"{mv} matvecs in {sec:.1f} s (each step ~{budget:.0f} s of BLAS restatement)"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="heff_b200", choices=["heff_b200", "reference"])
    ap.add_argument("--cpu-budget", type=float, default=12.0, help="seconds of CPU baseline sample")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="skip the mixed-precision, eigensolve and serving measurements")
    ap.add_argument("--no-serving", action="store_true", help="skip the serving-stream measurement")
    ap.add_argument("--serving-requests", type=int, default=120, help="requests of the mixed-precision serving stream")
    ap.add_argument("--serving-requests-fp64", type=int, default=60, help="requests of the FP64 serving stream (its first ones)")
    ap.add_argument("--serving-chi-max", type=int, default=2048)
    ap.add_argument("--serving-rate", type=float, default=4.0, help="Poisson arrival rate (requests/s)")
    ap.add_argument("--serving-only", action="store_true", help="run only the serving streams (after the headline matvec)")
    ap.add_argument("--xdmrg", default="", help="comma-separated L:chi:sweeps[:mixed|fp64[:jacobi block[:local matvec limit]]] "
                                                "excited-state sweeps to run after the headline matvec (e.g. 16:256:7,14:128:7:mixed,"
                                                "32:512:8:fp64:1:20000); not part of the default run")
    ap.add_argument("--ensemble-n", type=int, default=32, help="realisations in the ensemble sample")
    ap.add_argument("--ensemble-sweeps", type=int, default=4)
    ap.add_argument("--ensemble-serial-n", type=int, default=0, help="one-at-a-time sample (0: all realisations)")
    ap.add_argument("--ensemble-only", action="store_true", help="run only the ensemble (after the headline matvec)")
    ap.add_argument("--no-grid", action="store_true", help="skip the chi x D precision grid and the SVD timing")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    args.warmup = max(args.warmup, 3)

    import torch

    import dmrg_b200 as hb

    ws, rank, local = dist_env()
    if ws > 1:
        # the extras (mixed precision, eigensolves, serving, ensemble) are single-GPU measurements; replicas run
        # only the headline matvec so every rank takes the same collective steps in the same order
        args.no_extras = True
    torch.cuda.set_device(local)
    dist = None
    if ws > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))

    # CPU baseline first (rank 0, N=1 only), before any GPU work is timed
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        cpu = cpu_reference_sample(CHI, D, True, args.cpu_budget, one_thread_s=5.0)

    # FP64 peak reference: cuBLAS ZGEMM measured live (MEASURED_PEAKS.json has no FP64 entry)
    def zgemm_peak():
        n = 4096
        a = torch.randn(n, n, dtype=torch.complex128, device="cuda")
        b = torch.randn(n, n, dtype=torch.complex128, device="cuda")
        for _ in range(2):
            torch.matmul(a, b)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(5):
            torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        t = e0.elapsed_time(e1) / 5 / 1e3
        del a, b
        return 8.0 * n ** 3 / t / 1e12

    peak = zgemm_peak()

    theta, mpos, L, R = make_inputs(CHI, D, True, seed=SEED + rank)
    stream = torch.cuda.Stream()
    op = hb.MatVecMPOS(mpos, L, R, cplx=True, stream=stream)
    n = op.rows()
    x = hb.to_device(theta)
    y = torch.empty_like(x)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")  # 256 MB > 126 MB L2
    F = matvec_flops(SPIN, CHI, CHI, D, D, True)
    FG = gemm_flops(SPIN, CHI, CHI, D, D, True)

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            op.MultAx(x, y)
        stream.synchronize()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        op.set_profiling(True)
        op.stage_times(reset=True)
        clocks = ClockSampler(local)
        clocks.start()
        time.sleep(0.3)
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
        launches0 = int(hb.lib().heff_matvec_launches())
        for k in range(args.steps):
            flush.fill_(float(k))  # L2 flush outside the timed events
            evs[k][0].record(stream)
            op.MultAx(x, y)
            evs[k][1].record(stream)
        stream.synchronize()
        launches = int(hb.lib().heff_matvec_launches()) - launches0
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        step_ms = [a.elapsed_time(b) for a, b in evs]
        stage_ms, cnt = op.stage_times(reset=True)
        op.set_profiling(False)
        # e2e through the C ABI with host (pinned) buffers
        xh = torch.from_numpy(np.ascontiguousarray(theta.ravel(order="F"))).pin_memory()
        yh = torch.empty_like(xh).pin_memory()
        for _ in range(2):
            hb.lib().heff_op_multax_host(op.handle, hb.ptr(xh), hb.ptr(yh))
        t_e2e = []
        for _ in range(max(3, args.steps // 2)):
            flush.fill_(1.0)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            hb.check(hb.lib().heff_op_multax_host(op.handle, hb.ptr(xh), hb.ptr(yh)), "multax_host")
            t_e2e.append(time.perf_counter() - t0)
        clk = clocks.stop()
        extras = {} if (args.no_extras or args.serving_only) else measure_mixed_and_eigs(hb, torch, op, mpos, L, R, x, y, flush, stream, F)
    if args.ensemble_only:
        extras["ensemble"] = measure_ensemble(hb, args.ensemble_n, args.ensemble_sweeps, 32, serial_n=args.ensemble_serial_n)
    if args.xdmrg:
        runs = []
        for spec in args.xdmrg.split(","):
            f = spec.split(":")
            runs.append(measure_xdmrg(hb, int(f[0]), int(f[1]), int(f[2]), precision=hb.PREC_MIXED if f[3:4] == ["mixed"] else None,
                                      jcb=int(f[4]) if len(f) > 4 else 128, max_mv=int(f[5]) if len(f) > 5 else 60000))
        extras["xdmrg"] = runs
    if not args.no_extras and not args.no_serving:
        op.close()
        del x, y, flush
        torch.cuda.empty_cache()
        sv = {}
        for name, prec, nreq in (("mixed", hb.PREC_MIXED, args.serving_requests), ("fp64", hb.PREC_FP64, args.serving_requests_fp64)):
            if nreq > 0:
                sv[name] = measure_serving(hb, torch, nreq, 64, args.serving_chi_max, args.serving_rate, prec)
        sv["workload"] = ("bounded sample of the serving stream: Poisson arrivals, chi log-uniform, 70% f64 / 30% c128, D in {3, 9} "
                          "(D=9: MPO squared, folded-spectrum target), Hermitian seeded envs resident on the device, tol 1e-10")
        if "fp64" in sv and "mixed" in sv and sv["fp64"]["solves_per_s"] > 0:
            sv["mixed_vs_fp64_solves_per_s"] = sv["mixed"]["solves_per_s"] / sv["fp64"]["solves_per_s"]
        extras["serving"] = sv
        if not args.serving_only:
            extras["ensemble"] = measure_ensemble(hb, args.ensemble_n, args.ensemble_sweeps, 32,
                                                  serial_n=args.ensemble_serial_n)  # 32 workers: 21 /s vs 18.6 /s with 16
            extras["eigensolves_folded"] = measure_eigs_folded(hb, torch)
    if not args.no_extras and not args.no_grid and not args.serving_only:
        torch.cuda.empty_cache()
        gstream = torch.cuda.Stream()
        gflush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
        grid = measure_grid(hb, torch, gstream, gflush)
        extras["precision_grid"] = grid
        r = grid["f64"]["chi1024_D3"]["fp64_dmma"]
        FGr = gemm_flops(SPIN, CHI, CHI, D, D, False)
        gemm_ms_r = r["stage_ms"][1] + r["stage_ms"][3]
        extras["real_fp64_matvec"] = {
            "workload": "the same matvec in float64 (real Gaussian theta, real symmetric-slice envs), chi=1024, D=3",
            "ms": r["ms"], "tflops": r["tflops"], "frac_of_nominal_40": r["tflops"] / 40.0, "stage_ms": r["stage_ms"],
            "gemm_tflops": FGr / (gemm_ms_r / 1e3) / 1e12, "gemm_frac_of_nominal_40": FGr / (gemm_ms_r / 1e3) / 1e12 / 40.0,
            "rel_err_vs_host": r["rel_err_vs_host"]}
        del gflush
        torch.cuda.empty_cache()
        extras["svd"] = measure_svd(hb, torch)
        try:
            extras["svd_reference_matrices"] = measure_svd_reference_matrices(hb, torch)
        except Exception as e:  # a measurement extra never takes the headline line down
            extras["svd_reference_matrices"] = {"error": f"{type(e).__name__}: {e}"}

    tot_ms, e2e_t = reduce_max_over_ranks([sum(step_ms), statistics.median(t_e2e)], dist)
    ms_per_step = tot_ms / args.steps
    value = job_tflops(F, args.steps, ws, tot_ms)
    gemm_ms = (stage_ms[1] + stage_ms[3]) / max(cnt, 1)
    achieved = FG / (gemm_ms / 1e3) / 1e12
    traffic = None
    tf = os.path.join(ROOT, "profiles", "matvec_gemm_traffic.json")
    if os.path.exists(tf):
        try:
            traffic = json.load(open(tf)).get("bytes_per_matvec_both_gemm_launches")
        except Exception:
            traffic = None
    bytes_io = n * 16
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c128",
        "data": "synthetic (seeded Gaussian theta, Hermitian-slice envs, Ising two-site MPO)",
        "config": bench_config(ws),
        "roofline": {"bound": "tensor", "kernel": "gemm_f64_kernel (DMMA m16n8k4, 2 launches per matvec)", "achieved": achieved, "peak": peak,
                     "unit": "TFLOP/s", "frac": achieved / peak, "traffic": traffic,
                     "peak_source": "cuBLAS ZGEMM 4096^3 measured in this run (MEASURED_PEAKS.json has no FP64 entry)",
                     "frac_of_nominal_40": achieved / 40.0,
                     "flop_count": "achieved counts the algorithmic complex FLOPs (8 per complex multiply-add, as the reference "
                                   "computes); the kernel forms each complex product with 3 real DMMA products (3M), so the FP64 "
                                   "tensor work it executes is 3/4 of that",
                     "executed": 0.75 * achieved, "executed_frac": 0.75 * achieved / peak},
        "stage_ms": {"layout": stage_ms[0] / max(cnt, 1), "gemm1": stage_ms[1] / max(cnt, 1), "mix": stage_ms[2] / max(cnt, 1),
                     "gemm2": stage_ms[3] / max(cnt, 1)},
        "e2e": {"value": ws * F / e2e_t / 1e12, "unit": UNIT, "h2d_bytes_per_step": bytes_io, "d2h_bytes_per_step": bytes_io,
                "ms_per_step": e2e_t * 1e3, "api": "heff_op_multax_host (C ABI, pinned host buffers)"},
        "gpu_launches": launches,
        "clocks": clk,
        "cpu_baseline": cpu,
    }
    line.update(extras)
    if "mixed_matvec" in line:
        line["mixed_matvec"]["speedup_vs_fp64_matvec"] = ms_per_step / line["mixed_matvec"]["ms"]
    if "int8_engine" in line:
        line["int8_engine"]["matvec"]["speedup_vs_dmma"] = ms_per_step / line["int8_engine"]["matvec"]["ms"]
    if rank == 0:
        print(json.dumps(line), flush=True)
    op.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
