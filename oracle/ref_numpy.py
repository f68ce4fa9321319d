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


def matvec_flops(S, cL, cR, DL, DR, cplx=False):
    """Algorithmic real FLOPs of one H_eff matvec (dense, as the reference computes it).

    Stage A 2*S*cL*cL*cR*DL, stage B 2*cL*cR*(S*DL)*(S*DR), stage C 2*S*cL*cR*cR*DR;
    a complex multiply-add counts 8 real FLOPs (x4)."""
    f = 2.0 * S * cL * cL * cR * DL + 2.0 * cL * cR * S * DL * S * DR + 2.0 * S * cL * cR * cR * DR
    return 4.0 * f if cplx else f
