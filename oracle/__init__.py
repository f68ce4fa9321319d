"""CPU oracle for the H_eff hot path of DMRG++ (DavidAce/DMRG v3.5.0).

TEST INFRASTRUCTURE ONLY.  Nothing in the product package ``dmrg_b200`` imports
this module; it is loaded by ``tests/``, by ``__graft_entry__.smoke()`` (as the
checker) and by the ``cpu_baseline`` / ``--impl reference`` legs of
``bench.py``.

Parity status: UNPINNED against the reference's own outputs -- the reference
cannot be compiled here (Eigen 3.4.0, PRIMME, arpack-ng, LAPACKE and h5pp are
absent) and its tests hold no golden vectors for this path.  The C restatement
(``heff_oracle.c``) follows the reference's contraction sequences line by line;
it is pinned against an independent numpy restatement (:mod:`oracle.ref_numpy`),
the dense H_eff matrix, exact diagonalisation and the free-fermion solution of
the transverse-field Ising chain (:mod:`oracle.physics`).
"""
from .clib import (  # noqa: F401
    lib,
    matvec,
    expval,
    env_update,
    dense_heff,
    get_matrix,
    mpo_ising,
    mpo_edge_left,
    mpo_edge_right,
    mpo_merge,
    mpo_square,
    truncation_rank,
    entropy,
)
