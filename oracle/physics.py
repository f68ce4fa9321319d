"""Independent physics answers and seeded synthetic inputs.  TEST INFRASTRUCTURE ONLY.

* ``splitmix64`` / ``uniform``: the documented generator shared with the C++
  library (heff_rng in dmrg_b200/csrc/host_util.hpp), so that both sides draw identical
  random fields h_i from the same seed.  (The reference draws with pcg64,
  math/rnd/rnd.cpp:46-57; pcg-cpp is absent, so its per-seed fields cannot be
  reproduced bit for bit.)
* ``ising_hamiltonian_sparse`` + ``ed_ground``: exact diagonalisation of
  H = -sum J sz_i sz_{i+1} - sum h_i sx_i (open chain).
* ``free_fermion_levels``: Lieb-Schultz-Mattis / Pfeuty solution of the open
  transverse-field Ising chain: E0 = -sum_k Lambda_k with Lambda_k the singular
  values of the L x L bidiagonal matrix (diag h_i, superdiag J_i); any
  eigenenergy is E0 + 2 sum_{k in S} Lambda_k.
* ``heff_inputs``: the standalone two-site matvec workload (theta[4,chi,chi],
  envs with every D-slice Hermitian, Ising two-site MPO or its square).
"""
import numpy as np

from . import clib

_M64 = (1 << 64) - 1


def splitmix64(state):
    """One step of splitmix64 (Steele, Lea, Flood 2014). Returns (new_state, output)."""
    state = (state + 0x9E3779B97F4A7C15) & _M64
    z = state
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & _M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & _M64
    return state, z ^ (z >> 31)


def uniform(seed, n, lo, hi):
    """n doubles in [lo, hi) from splitmix64 seeded with ``seed`` (53-bit mantissa)."""
    st = seed & _M64
    out = np.empty(n)
    for i in range(n):
        st, z = splitmix64(st)
        out[i] = lo + (hi - lo) * ((z >> 11) * (1.0 / 9007199254740992.0))
    return out


def random_fields(seed, L, h_lo=0.5, h_hi=1.5):
    return uniform(seed, L, h_lo, h_hi)


def ising_mpos(hs, J=1.0, eshift=0.0):
    """Site MPOs of the random-field Ising chain with edges applied (MpoSite.cpp:20-26)."""
    L = len(hs)
    mpos = []
    for i, h in enumerate(hs):
        W = clib.mpo_ising(J, h, eshift)
        if i == 0:
            W = clib.mpo_edge_left(W)
        if i == L - 1:
            W = clib.mpo_edge_right(W)
        mpos.append(W)
    return mpos


def ising_hamiltonian_sparse(hs, J=1.0):
    import scipy.sparse as sp

    L = len(hs)
    n = 1 << L
    idx = np.arange(n)
    # site i <-> bit i (site 0 = least significant); sz = +1 for bit 0
    bits = [(idx >> i) & 1 for i in range(L)]
    diag = np.zeros(n)
    for i in range(L - 1):
        zz = (1 - 2 * bits[i]) * (1 - 2 * bits[i + 1])
        diag -= J * zz
    rows, cols, vals = [idx], [idx], [diag]
    for i in range(L):
        rows.append(idx)
        cols.append(idx ^ (1 << i))
        vals.append(-hs[i] * np.ones(n))
    H = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(n, n))
    return H


def ed_ground(hs, J=1.0):
    """Ground energy and half-chain entanglement entropy by exact diagonalisation."""
    import scipy.sparse.linalg as sla

    H = ising_hamiltonian_sparse(hs, J)
    L = len(hs)
    if L <= 10:
        w, v = np.linalg.eigh(H.toarray())
        e0, psi = w[0], v[:, 0]
    else:
        w, v = sla.eigsh(H, k=1, which="SA", tol=1e-14, ncv=40)
        e0, psi = w[0], v[:, 0]
    # bipartition sites [0, L/2) | [L/2, L): index = low bits (sites < L/2) + high bits
    half = L // 2
    M = psi.reshape(1 << (L - half), 1 << half)  # rows: high sites, cols: low sites
    s = np.linalg.svd(M, compute_uv=False)
    p = s * s
    p = p[p > 0]
    return float(e0), float(-np.sum(p * np.log(p)))


def free_fermion_levels(hs, J=1.0):
    """Single-particle energies Lambda_k of the open TFIM (sorted ascending)."""
    L = len(hs)
    B = np.diag(np.asarray(hs, dtype=float))
    for i in range(L - 1):
        B[i, i + 1] = J
    return np.sort(np.linalg.svd(B, compute_uv=False))


def free_fermion_ground(hs, J=1.0):
    return -float(np.sum(free_fermion_levels(hs, J)))


def free_fermion_modes(hs, J=1.0):
    """Majorana normal modes of the open TFIM (Jordan-Wigner with sx_i = 1 - 2 n_i): H = (i/4) sum M_kl g_k g_l with
    M[a_i, b_i] = 2 h_i, M[b_i, a_{i+1}] = 2 J; returns (eps, W) with M = W blockdiag([[0, eps_k], [-eps_k, 0]]) W^T,
    eps_k = 2 Lambda_k >= 0 (real Schur form).  An eigenstate with mode occupations n_k has E = E0 + sum n_k eps_k."""
    import scipy.linalg as sla

    L = len(hs)
    M = np.zeros((2 * L, 2 * L))
    for i in range(L):
        M[2 * i, 2 * i + 1], M[2 * i + 1, 2 * i] = 2 * hs[i], -2 * hs[i]
        if i + 1 < L:
            M[2 * i + 1, 2 * i + 2], M[2 * i + 2, 2 * i + 1] = 2 * J, -2 * J
    T, W = sla.schur(M, output="real")
    eps = np.empty(L)
    for k in range(L):
        e = T[2 * k, 2 * k + 1]
        if e < 0:
            W[:, [2 * k, 2 * k + 1]] = W[:, [2 * k + 1, 2 * k]]
            e = -e
        eps[k] = e
    return eps, W


def free_fermion_schmidt(eps, W, occ, cut, keep=1 << 17):
    """Schmidt weights (squared singular values, descending, the largest `keep`) of the eigenstate with mode
    occupations `occ` across the bond after site `cut` - 1 (sites [0, cut) | [cut, L)): the eigenvalues +-nu_j of the
    restricted Majorana correlation matrix (Peschel, J. Phys. A 36, L205 (2003)) give the weights prod (1 +- nu_j)/2."""
    L = len(eps)
    G = np.zeros((2 * L, 2 * L))
    for k in range(L):
        v = 2.0 * occ[k] - 1.0
        G[2 * k, 2 * k + 1], G[2 * k + 1, 2 * k] = v, -v
    Gam = W @ G @ W.T
    nu = np.sort(np.abs(np.linalg.eigvals(Gam[: 2 * cut, : 2 * cut]).imag))[::2]
    p = np.array([1.0])
    for x in nu:
        p = np.concatenate([p * (1 + x) / 2, p * (1 - x) / 2])
        if p.size > keep:
            p = np.sort(p)[::-1][:keep]
    return np.sort(p)[::-1]


def bond_dimension_for_weight(p, weight):
    """Smallest number of Schmidt weights whose discarded tail sums to at most `weight`."""
    tail = np.cumsum(p[::-1])[::-1]
    return int(np.count_nonzero(tail > weight))


def hermitian_env(rng, chi, D, cplx):
    """[chi,chi,D] environment with every D-slice Hermitian: (X + X^dagger)/2, X Gaussian."""
    if cplx:
        X = rng.standard_normal((chi, chi, D)) + 1j * rng.standard_normal((chi, chi, D))
    else:
        X = rng.standard_normal((chi, chi, D))
    E = 0.5 * (X + np.conj(np.transpose(X, (1, 0, 2))))
    return np.asfortranarray(E)


def ising_two_site_mpo(h1=1.0, h2=1.0, J=1.0, squared=False):
    """Merged two-site bulk Ising MPO [3,3,4,4] or the merged uncompressed square [9,9,4,4]."""
    WA = clib.mpo_ising(J, h1)
    WB = clib.mpo_ising(J, h2)
    if squared:
        WA = clib.mpo_square(WA)
        WB = clib.mpo_square(WB)
    return clib.mpo_merge(WA, WB)


def heff_inputs(chi, D=3, cplx=True, seed=0, chiR=None, spin=4):
    """Seeded standalone two-site H_eff workload: theta [spin,chi,chiR] N(0,1)(+iN(0,1)),
    Hermitian envs, W = two-site Ising MPO (D=3) or its square (D=9)."""
    chiR = chi if chiR is None else chiR
    rng = np.random.default_rng(seed)
    if cplx:
        theta = rng.standard_normal((spin, chi, chiR)) + 1j * rng.standard_normal((spin, chi, chiR))
    else:
        theta = rng.standard_normal((spin, chi, chiR))
    theta = np.asfortranarray(theta)
    L = hermitian_env(rng, chi, D, cplx)
    R = hermitian_env(rng, chiR, D, cplx)
    if spin == 4 and D in (3, 9):
        W = ising_two_site_mpo(0.7, 1.3, squared=(D == 9))
    elif spin == 2 and D == 3:
        W = clib.mpo_ising(1.0, 0.9)
    elif spin == 2 and D == 9:
        W = clib.mpo_square(clib.mpo_ising(1.0, 0.9))
    else:
        W = np.asfortranarray(rng.standard_normal((D, D, spin, spin)))
        W = 0.5 * (W + W.transpose(0, 1, 3, 2))
    if spin != W.shape[2]:
        raise ValueError("spin dimension does not match the MPO")
    if cplx:
        W = W.astype(np.complex128)
    return theta, np.asfortranarray(W), L, R
