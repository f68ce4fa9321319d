"""Independent numpy restatements of the H_eff hot path.  TEST INFRASTRUCTURE ONLY.

* ``*_einsum``: one ``np.einsum`` per reference function, written from the
  index equations (not from the C loops) so that the two oracles cross-check.
* ``matvec_blas``: the reference's three-contraction sequence
  (contraction_tblis.cpp:277-290, both branches) with every contraction done
  as one BLAS GEMM (numpy -> OpenBLAS, multithreaded).  This is the timed CPU
  baseline of ``bench.py``: the same contractions and intermediate shapes as
  Eigen's ThreadPoolDevice path, through an optimised GEMM.
"""
import numpy as np


def matvec_einsum(mps, mpo, envL, envR):
    # y[s',a',b'] = sum L[a,a',m] mps[s,a,b] W[m,n,s,s'] R[b,b',n]
    return np.einsum("axm,sab,mnst,byn->txy", envL, mps, mpo, envR, optimize=True)


def matvec_multi_literal(mps, mpos, envL, envR):
    """The multi-MPO matrix_vector_product (contraction_tblis.cpp:307-420, Eigen path) restated step by step
    with tensordot (same result-dim order as Eigen's contract) and column-major reshapes.  mpos are
    unshuffled [m, n, s, s']; the reference first shuffles them {2,3,0,1} (:313-320)."""
    shf = [np.transpose(W, (2, 3, 0, 1)) for W in mpos]
    K = len(shf)

    def prod(fr, to):  # mpodimprod (:337-346)
        p = 1
        if to == 0:
            return p
        for idx in range(fr, to):
            if idx >= K:
                break
            p *= shf[idx].shape[1]
        return p

    shp6 = (prod(0, 1), prod(1, K), mps.shape[2], envL.shape[1], envL.shape[2], 1)
    t = np.tensordot(mps, envL, axes=([1], [0])).reshape(shp6, order="F").transpose(0, 1, 2, 3, 5, 4)  # :375
    for idx in range(K):  # :377-398
        mpo = shf[idx]
        shp6 = (prod(idx + 1, idx + 2), prod(idx + 2, K), t.shape[2], t.shape[3], prod(0, idx + 1), mpo.shape[3])
        t = np.tensordot(t, mpo, axes=([0, 5], [0, 2])).reshape(shp6, order="F")
    d0, d1, d2, d3 = t.shape[0] * t.shape[1] * t.shape[2], t.shape[3], t.shape[4], t.shape[5]
    out = np.tensordot(t.reshape((d0, d1, d2, d3), order="F"), envR, axes=([0, 3], [0, 2])).transpose(1, 0, 2)  # :415
    return np.asfortranarray(out)


def expansion_term_einsum(side, env, mps, mpo, alpha):
    """EnvBase::get_expansion_term(mps, mpo, alpha) (EnvBase.cpp:303-364), Eigen semantics restated:
    a contraction's result lists the free dims of the left operand, then of the right one.
      L (:311-333): B[a,a',m] . M[s,a,b] over (0,1) -> [a',m,s,b];  . W[m,n,s,s'] over ({1,2},{0,2}) -> [a',b,n,s'];
                    shuffle {3,0,1,2} -> [s',a',b,n];  reshape [spin, chiL, chiR*DR]
      R (:335-357): B[b,b',n] . M[s,a,b] over (0,2) -> [b',n,s,a];  . W over ({1,2},{1,2}) -> [b',a,m,s'];
                    shuffle {3,0,1,2} -> [s',b',a,m];  reshape [spin, chiL*DL, chiR] (memory order kept)
    alpha == 0 returns zeros (:319-322, :343-346)."""
    S, cL, cR = mps.shape
    DL, DR = mpo.shape[0], mpo.shape[1]
    if side == "L":
        Q = np.einsum("axm,sab,mnst->txbn", env, mps, mpo)
        shape = (S, cL, cR * DR)
    else:
        Q = np.einsum("byn,sab,mnst->tyam", env, mps, mpo)
        shape = (S, cL * DL, cR)
    if alpha == 0:
        return np.zeros(shape, dtype=Q.dtype, order="F")
    return np.asfortranarray(alpha * Q.reshape(shape, order="F"))


def diagonal_einsum(mps_shape, mpo, envL, envR):
    """MatVecMPOS::get_diagonal_new(0, ...) / get_matrix_element(I, I) (matvec_mpos.cpp:300-407):
    diag[s,a,b] = sum_{m,n} envL[a,a,m] W[m,n,s,s] envR[b,b,n], flattened column-major like the mps."""
    S, cL, cR = mps_shape
    lD = np.einsum("aam->am", envL)
    rD = np.einsum("bbn->bn", envR)
    wD = np.einsum("mnss->mns", mpo)
    return np.einsum("am,mns,bn->sab", lD, wD, rD).ravel(order="F")


def multpc(x, diag, shift):
    """MatVecMPOS::MultPc with jcbMaxBlockSize == 1 (matvec_mpos.cpp:1349-1364): x / (diag - shift)."""
    return x / (np.real(diag) - shift)


def expval_einsum(mps, mpo, envL, envR):
    y = matvec_einsum(mps, mpo, envL, envR)
    return np.vdot(mps.ravel(order="F"), y.ravel(order="F"))


def env_update_einsum(side, env, mps, mpo):
    if side == "L":
        # L'[b,b',n] = sum M[s,a,b] L[a,a',m] conj(M)[s',a',b'] W[m,n,s,s']
        return np.einsum("sab,axm,txc,mnst->bcn", mps, env, mps.conj(), mpo, optimize=True)
    # R'[a,a',m] = sum M[s,a,b] R[b,b',n] conj(M)[s',a',b'] W[m,n,s,s']
    return np.einsum("sab,bcn,tyc,mnst->aym", mps, env, mps.conj(), mpo, optimize=True)


def mpo_merge_einsum(WA, WB):
    mL, _, sA, tA = WA.shape
    _, mR, sB, tB = WB.shape
    X = np.einsum("mcst,cnuv->mnsutv", WA, WB)
    return X.reshape(mL, mR, sA * sB, tA * tB, order="F")


def mpo_square_einsum(W):
    D0, D1, d, _ = W.shape
    X = np.einsum("mnsp,MNpt->mMnNst", W, W.conj())
    return X.reshape(D0 * D0, D1 * D1, d, d, order="F")


def _mat(a, rows):
    """View a Fortran-ordered tensor as a (rows x rest) column-major matrix."""
    return a.reshape(rows, -1, order="F")


def matvec_blas(mps, mpo, envL, envR):
    """Reference contraction order with each step as one GEMM (see module doc)."""
    S, cL, cR = mps.shape
    DL, DR = mpo.shape[0], mpo.shape[1]
    if cL >= cR:
        # T1[s,b,a',m] = sum_a mps[s,a,b] L[a,a',m]
        mps_sba = np.asfortranarray(mps.transpose(0, 2, 1))  # [s,b,a]
        T1 = _mat(mps_sba, S * cR) @ _mat(envL, cL)  # [(s,b),(a',m)]
        T1 = T1.reshape(S, cR, cL, DL, order="F")
        # T2[b,a',n,s'] = sum_{m,s} T1[s,b,a',m] W[m,n,s,s']
        T1p = np.asfortranarray(T1.transpose(1, 2, 3, 0))  # [b,a',m,s]
        Wp = np.asfortranarray(mpo.transpose(0, 2, 1, 3))  # [m,s,n,s']
        T2 = _mat(T1p, cR * cL) @ _mat(Wp, DL * S)  # [(b,a'),(n,s')]
        T2 = T2.reshape(cR, cL, DR, S, order="F")
        # T3[a',s',b'] = sum_{b,n} T2[b,a',n,s'] R[b,b',n]
        T2p = np.asfortranarray(T2.transpose(1, 3, 0, 2))  # [a',s',b,n]
        Rp = np.asfortranarray(envR.transpose(0, 2, 1))  # [b,n,b']
        T3 = _mat(T2p, cL * S) @ _mat(Rp, cR * DR)  # [(a',s'),b']
        T3 = T3.reshape(cL, S, cR, order="F")
        return np.asfortranarray(T3.transpose(1, 0, 2))
    # T1[s,a,b',n] = sum_b mps[s,a,b] R[b,b',n]
    T1 = _mat(mps, S * cL) @ _mat(envR, cR)
    T1 = T1.reshape(S, cL, cR, DR, order="F")
    # T2[a,b',m,s'] = sum_{n,s} T1[s,a,b',n] W[m,n,s,s']
    T1p = np.asfortranarray(T1.transpose(1, 2, 3, 0))  # [a,b',n,s]
    Wp = np.asfortranarray(mpo.transpose(1, 2, 0, 3))  # [n,s,m,s']
    T2 = _mat(T1p, cL * cR) @ _mat(Wp, DR * S)
    T2 = T2.reshape(cL, cR, DL, S, order="F")
    # T3[b',s',a'] = sum_{a,m} T2[a,b',m,s'] L[a,a',m]
    T2p = np.asfortranarray(T2.transpose(1, 3, 0, 2))  # [b',s',a,m]
    Lp = np.asfortranarray(envL.transpose(0, 2, 1))  # [a,m,a']
    T3 = _mat(T2p, cR * S) @ _mat(Lp, cL * DL)
    T3 = T3.reshape(cR, S, cL, order="F")
    return np.asfortranarray(T3.transpose(1, 2, 0))


def env_update_blas(side, env, mps, mpo):
    """EnvBase::build_block with the reference's contraction order, each step one GEMM.

    L (EnvBase.cpp:109-112): X[a,m,s',b'] = L.contract(conj(M),{1},{1}); Y[a,b',n,s] = X.contract(W,{1,2},{0,3});
                             L'[b,b',n] = M.contract(Y,{0,1},{3,0})
    R (EnvBase.cpp:146-149): X[b,n,s',a'] = R.contract(conj(M),{1},{2}); Y[b,a',m,s] = X.contract(W,{1,2},{1,3});
                             R'[a,a',m] = M.contract(Y,{0,2},{3,0})"""
    d, cL, cR = mps.shape
    DL, DR = mpo.shape[0], mpo.shape[1]
    Mc = mps.conj()
    if side == "L":
        # X[(a,m),(s',b')] = sum_a' L[(a),(a'),m] conj(M)[s',a',b']
        Lp = np.asfortranarray(env.transpose(0, 2, 1))  # [a,m,a']
        Mp = np.asfortranarray(Mc.transpose(1, 0, 2))  # [a',s',b']
        X = _mat(Lp, cL * DL) @ _mat(Mp, cL)  # [(a,m),(s',b')]
        X = X.reshape(cL, DL, d, cR, order="F")
        # Y[(a,b'),(n,s)] = sum_{m,s'} X[a,m,s',b'] W[m,n,s,s']
        Xp = np.asfortranarray(X.transpose(0, 3, 1, 2))  # [a,b',m,s']
        Wp = np.asfortranarray(mpo.transpose(0, 3, 1, 2))  # [m,s',n,s]
        Y = _mat(Xp, cL * cR) @ _mat(Wp, DL * d)
        Y = Y.reshape(cL, cR, DR, d, order="F")
        # L'[b,(b',n)] = sum_{s,a} M[s,a,b] Y[a,b',n,s]
        Mq = np.asfortranarray(mps.transpose(2, 0, 1))  # [b,s,a]
        Yp = np.asfortranarray(Y.transpose(3, 0, 1, 2))  # [s,a,b',n]
        out = _mat(Mq, cR) @ _mat(Yp, d * cL)
        return out.reshape(cR, cR, DR, order="F")
    # R side
    Rp = np.asfortranarray(env.transpose(0, 2, 1))  # [b,n,b']
    Mp = np.asfortranarray(Mc.transpose(2, 0, 1))  # [b',s',a']
    X = _mat(Rp, cR * DR) @ _mat(Mp, cR)  # [(b,n),(s',a')]
    X = X.reshape(cR, DR, d, cL, order="F")
    Xp = np.asfortranarray(X.transpose(0, 3, 1, 2))  # [b,a',n,s']
    Wp = np.asfortranarray(mpo.transpose(1, 3, 0, 2))  # [n,s',m,s]
    Y = _mat(Xp, cR * cL) @ _mat(Wp, DR * d)
    Y = Y.reshape(cR, cL, DL, d, order="F")  # [b,a',m,s]
    Mq = np.asfortranarray(mps.transpose(1, 0, 2))  # [a,s,b]
    Yp = np.asfortranarray(Y.transpose(3, 0, 1, 2))  # [s,b,a',m]
    out = _mat(Mq, cL) @ _mat(Yp, d * cR)
    return out.reshape(cL, cL, DL, order="F")


def svd_truncated(A, rank_max=0, trunc_lim=1e-12):
    """svd::solver::do_svd_ptr for the two-site split: geauto resolves to LAPACK ?gesdd for
    rows*cols >= 256 (svd.cpp:127-140); numpy.linalg.svd calls the same LAPACK routine.  Then the
    rank rule of svd.cpp:257-280 on the nonzero singular values (svd_lapacke.cpp:453-458)."""
    from . import clib

    U, S, VT = np.linalg.svd(A, full_matrices=False)
    nz = int(np.count_nonzero(S))
    r, err = clib.truncation_rank(S[:nz], rank_max, trunc_lim)
    return U[:, :r], S[:r], VT[:r, :], r, err


def schmidt_multisite(theta, dL, dR, rank_max=0, trunc_lim=1e-12):
    """svd.h:189-220 (dR > 1 branch): reshape [dL,dR,chiL,chiR], shuffle {0,2,1,3}, SVD, S normalised,
    V = VT reshaped [k,dR,chiR] shuffled {1,0,2}."""
    S_, cL, cR = theta.shape
    T4 = theta.reshape(dL, dR, cL, cR, order="F").transpose(0, 2, 1, 3)
    A = np.asfortranarray(T4).reshape(dL * cL, dR * cR, order="F")
    U, S, VT, r, err = svd_truncated(A, rank_max, trunc_lim)
    Ut = U.reshape(dL, cL, r, order="F")
    V = VT.reshape(r, dR, cR, order="F").transpose(1, 0, 2)
    return np.asfortranarray(Ut), S / np.linalg.norm(S), np.asfortranarray(V), r, err


def matvec_flops(S, cL, cR, DL, DR, cplx=False):
    """Algorithmic real FLOPs of one H_eff matvec (dense, as the reference computes it).

    Stage A 2*S*cL*cL*cR*DL, stage B 2*cL*cR*(S*DL)*(S*DR), stage C 2*S*cL*cR*cR*DR;
    a complex multiply-add counts 8 real FLOPs (x4)."""
    f = 2.0 * S * cL * cL * cR * DL + 2.0 * cL * cR * S * DL * S * DR + 2.0 * S * cL * cR * cR * DR
    return 4.0 * f if cplx else f


def dmrg1_expansion_model(mpos, chi_max, sweeps, alpha0=1e-3, trunc_lim=1e-12, seed=0):
    """Host model of the one-site DMRG sweep with forward subspace expansion (the device driver, algorithm 2), in the
    driver's index maps, for small chains: site tensors M[i] [d, chi_i, chi_{i+1}], environments of the sites < i and
    > i, the expansion term of EnvBase::get_expansion_term (expansion_term_einsum; the R side read by its index meaning
    [s', b', (a, m)]), the enlarged-bond SVDs of expand_environment_1site (merge_expansion_term_PR / _PL), dense local
    eigensolves, and the mixing factor alpha0 halved every sweep and off for the last two.  Returns the energy of the
    last local solve per sweep and the final bond dimensions."""
    L = len(mpos)
    d = mpos[0].shape[2]
    rng = np.random.default_rng(seed)
    M = []
    for _ in range(L):
        v = rng.uniform(-0.5, 0.5, d)
        M.append((v / np.linalg.norm(v)).reshape(d, 1, 1))
    Le, Re = [None] * (L + 1), [None] * (L + 1)
    Le[0], Re[L - 1] = np.ones((1, 1, 1)), np.ones((1, 1, 1))

    def renv(i):
        Re[i] = env_update_einsum("R", Re[i + 1], M[i + 1], mpos[i + 1])

    def lenv(i):
        Le[i + 1] = env_update_einsum("L", Le[i], M[i], mpos[i])

    def svd(A, rmax):
        U, S, VT = np.linalg.svd(A, full_matrices=False)
        tail = np.sqrt(np.cumsum(S[::-1] ** 2))[::-1]
        k = max(1, min(int(np.count_nonzero(tail >= trunc_lim)), rmax))
        return U[:, :k], S[:k], VT[:k], k

    def solve(i):
        shape = M[i].shape
        n = int(np.prod(shape))
        H = np.stack([matvec_einsum(np.eye(n)[:, k].reshape(shape, order="F"), mpos[i], Le[i], Re[i]).ravel(order="F")
                      for k in range(n)], axis=1)
        w, v = np.linalg.eigh((H + H.T) / 2)
        M[i] = v[:, 0].reshape(shape, order="F")
        return w[0]

    def rows(T):  # [s, a, b] -> [a, (s, b)]
        return T.transpose(1, 0, 2).reshape(T.shape[1], -1, order="F")

    def unrows(X, k, cb):  # [a, (s, b)] -> [s, a, b]
        return X.reshape(k, d, cb, order="F").transpose(1, 0, 2)

    for i in range(L - 2, -1, -1):
        renv(i)
    energies = []
    E = None
    for sweep in range(sweeps):
        alpha = alpha0 * 2.0 ** (-sweep) if sweep + 2 < sweeps else 0.0
        for i in range(L - 1):
            if alpha > 0:
                _, ca, c = M[i].shape
                cb = M[i + 1].shape[2]
                P = expansion_term_einsum("R", Re[i + 1], M[i + 1], mpos[i + 1], alpha)
                DL = mpos[i + 1].shape[0]
                Psem = P.ravel(order="F").reshape(d, cb, c * DL, order="F").transpose(0, 2, 1)  # [s', (a, m), b']
                X = np.concatenate([rows(M[i + 1]), rows(Psem)], axis=0)
                U, S, VT, k = svd(X, min(d * ca, d * cb, chi_max))
                M[i] = ((M[i].reshape(d * ca, c, order="F") @ U[:c]) * S).reshape(d, ca, k, order="F")
                M[i + 1] = unrows(VT, k, cb)
                renv(i)
            E = solve(i)
            _, ca, c = M[i].shape
            cb = M[i + 1].shape[2]
            U, S, VT, k = svd(M[i].reshape(d * ca, c, order="F"), chi_max)
            S = S / np.linalg.norm(S)
            M[i] = U.reshape(d, ca, k, order="F")
            M[i + 1] = unrows((S[:, None] * VT) @ rows(M[i + 1]), k, cb)
            lenv(i)
        for i in range(L - 1, 0, -1):
            if alpha > 0:
                _, ca, c = M[i - 1].shape
                cb = M[i].shape[2]
                PL = expansion_term_einsum("L", Le[i - 1], M[i - 1], mpos[i - 1], alpha)
                X = np.concatenate([M[i - 1].ravel(order="F"), PL.ravel(order="F")]).reshape(d * ca, -1, order="F")
                U, S, VT, k = svd(X, min(d * ca, d * cb, chi_max))
                M[i - 1] = U.reshape(d, ca, k, order="F")
                M[i] = unrows((S[:, None] * VT[:, :c]) @ rows(M[i]), k, cb)
                lenv(i - 1)
            E = solve(i)
            _, c, cb = M[i].shape
            ca = M[i - 1].shape[1]
            U, S, VT, k = svd(rows(M[i]), chi_max)
            S = S / np.linalg.norm(S)
            M[i] = unrows(VT, k, cb)
            M[i - 1] = ((M[i - 1].reshape(d * ca, c, order="F") @ U) * S).reshape(d, ca, k, order="F")
            renv(i - 1)
        energies.append(E)
    return energies, [m.shape[2] for m in M[:-1]]


def gauss_jordan_inverse(A, floor_rel=1e-14):
    """Host model of the block-Jacobi inversion kernel (jcb_invert_kernel): in-place Gauss-Jordan elimination with
    partial (row) pivoting, lowest row on ties, pivots below floor_rel x max|A| floored to that value with their sign
    (counted), row interchanges undone as column interchanges in reverse order.  Returns (inverse, floored pivots)."""
    A = np.array(A, dtype=np.complex128 if np.iscomplexobj(A) else np.float64, copy=True)
    bs = A.shape[0]
    amax = float(np.max(np.abs(A))) if A.size else 0.0
    floor = floor_rel * (amax if amax > 0 else 1.0)
    perm = np.zeros(bs, dtype=int)
    floored = 0
    for k in range(bs):
        p = k + int(np.argmax(np.abs(A[k:, k])))
        perm[k] = p
        if p != k:
            A[[k, p], :] = A[[p, k], :]
        f = A[:, k].copy()
        f[k] = 0
        piv = A[k, k]
        if not abs(piv) >= floor:
            piv = (-floor if np.real(piv) < 0 else floor)
            floored += 1
        inv = 1.0 / piv
        A[k, :] *= inv
        A[k, k] = inv
        rowk = A[k, :].copy()
        for i in range(bs):
            if i == k:
                continue
            ai = A[i, :].copy()
            ai[k] = 0
            A[i, :] = ai - f[i] * rowk
    for k in range(bs - 1, -1, -1):
        p = perm[k]
        if p != k:
            A[:, [k, p]] = A[:, [p, k]]
    return A, floored


def round_robin_pair(n, step, k):
    """Pair k of step `step` in the circle-method tournament over n (even) columns: every pair once per n - 1 steps."""
    if k == 0:
        return n - 1, step
    return (step + k) % (n - 1), (step - k + (n - 1)) % (n - 1)


def jacobi_small_model(A, max_sweeps=60):
    """Host model of the single-CTA one-sided Jacobi SVD (jacobi_small_kernel) in its index maps: the columns padded
    to a multiple of 32 (zeros), the tournament over the n columns rounded up to even, steps of disjoint pairs; per
    pair the squared norms app, aqq and apq = a_p^H a_q, skipped unless |apq| > max(1e-300, floor,
    tol sqrt(app aqq)) with tol = max(1e-14, 8 eps sqrt(m)) and floor = m eps^2 max ||G_j||^2 of the previous sweep
    (0 in the first); else the Rutishauser-form rotation col_p' = col_p - s (conj(e) col_q + tau col_p),
    col_q' = col_q + s (e col_p - tau col_q) with e = apq / |apq|, applied to G and V; sweeps until one rotates
    nothing.  Returns (sigma descending over min(m, n), G, V, sweeps run)."""
    m, n = A.shape
    npad = (n + 31) // 32 * 32
    nc = min(npad, (n + 1) // 2 * 2)
    cplx = np.iscomplexobj(A)
    G = np.zeros((m, npad), dtype=np.complex128 if cplx else np.float64)
    G[:, :n] = A
    V = np.eye(npad, dtype=G.dtype)
    eps = 2.220446049250313e-16
    tol = max(1e-14, 8.0 * eps * np.sqrt(m))
    floor = 0.0
    sweeps = max_sweeps
    for sweep in range(max_sweeps):
        rotated = False
        for step in range(nc - 1):
            for k in range(nc // 2):
                p, q = round_robin_pair(nc, step, k)
                x, y = G[:, p].copy(), G[:, q].copy()
                app, aqq, apq = np.vdot(x, x).real, np.vdot(y, y).real, np.vdot(x, y)
                h = abs(apq)
                if h > 1e-300 and h > floor and h > tol * np.sqrt(app * aqq):
                    th = 0.5 * (aqq - app) / h
                    t = (1.0 if th >= 0 else -1.0) / (abs(th) + np.sqrt(1.0 + th * th))
                    c = 1.0 / np.sqrt(1.0 + t * t)
                    s = t * c
                    tau = s / (1.0 + c)
                    e = apq / h
                    ec = np.conj(e)
                    G[:, p] = x - s * (ec * y + tau * x)
                    G[:, q] = y + s * (e * x - tau * y)
                    vx, vy = V[:, p].copy(), V[:, q].copy()
                    V[:, p] = vx - s * (ec * vy + tau * vx)
                    V[:, q] = vy + s * (e * vx - tau * vy)
                    rotated = True
        gmax = float(np.max(np.sum(np.abs(G[:, :nc]) ** 2, axis=0)))
        if not rotated:
            sweeps = sweep + 1
            break
        floor = m * eps * eps * gmax
    sig = np.sort(np.linalg.norm(G, axis=0))[::-1]
    return sig[: min(m, n)], G, V, sweeps
