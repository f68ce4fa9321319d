"""ctypes signatures of the C entry points beyond the matvec/operator core (see include/heff.h)."""
import ctypes

_P = ctypes.c_void_p
_I = ctypes.c_int
_I64 = ctypes.c_int64
_I64P = ctypes.POINTER(ctypes.c_int64)
_DP = ctypes.POINTER(ctypes.c_double)


class EigConfig(ctypes.Structure):
    """heff_eig_config (include/heff.h)."""

    _fields_ = [("ritz", ctypes.c_int), ("target", ctypes.c_double), ("tol", ctypes.c_double), ("max_basis", ctypes.c_int),
                ("min_basis", ctypes.c_int), ("max_matvecs", ctypes.c_int64), ("mixed", ctypes.c_int), ("mixed_tol", ctypes.c_double),
                ("inner_iters", ctypes.c_int), ("inner_tol", ctypes.c_double), ("seed", ctypes.c_int64), ("precond", ctypes.c_int)]


class EigResult(ctypes.Structure):
    """heff_eig_result (include/heff.h)."""

    _fields_ = [("eigval", ctypes.c_double), ("resnorm", ctypes.c_double), ("anorm", ctypes.c_double), ("seconds", ctypes.c_double),
                ("num_mv", ctypes.c_int64), ("num_mv_fp64", ctypes.c_int64), ("num_mv_mixed", ctypes.c_int64), ("num_mv_phase1", ctypes.c_int64),
                ("iters", ctypes.c_int), ("restarts", ctypes.c_int), ("refine_steps", ctypes.c_int), ("converged", ctypes.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class DmrgConfig(ctypes.Structure):
    """heff_dmrg_config (include/heff.h)."""

    _fields_ = [("L", ctypes.c_int), ("J", ctypes.c_double), ("h", _DP), ("chi_max", ctypes.c_int64), ("sweeps", ctypes.c_int),
                ("trunc_lim", ctypes.c_double), ("eig_tol", ctypes.c_double), ("ritz", ctypes.c_int), ("target", ctypes.c_double),
                ("precision", ctypes.c_int), ("seed", ctypes.c_int64), ("energy_shift_per_site", ctypes.c_double), ("algorithm", ctypes.c_int),
                ("precond", ctypes.c_int), ("fp64_engine", ctypes.c_int), ("expansion_alpha", ctypes.c_double),
                ("warmup_sweeps", ctypes.c_int), ("bond_min", ctypes.c_int64), ("jcb_blocksize", ctypes.c_int64),
                ("eig_max_matvecs", ctypes.c_int64)]


class DmrgResult(ctypes.Structure):
    """heff_dmrg_result (include/heff.h)."""

    _fields_ = [("energy", ctypes.c_double), ("entropy_mid", ctypes.c_double), ("trunc_err_max", ctypes.c_double), ("seconds", ctypes.c_double),
                ("t_eig", ctypes.c_double), ("t_svd", ctypes.c_double), ("t_env", ctypes.c_double), ("chi_mid", ctypes.c_int64),
                ("num_mv", ctypes.c_int64), ("num_mv_mixed", ctypes.c_int64), ("unconverged_solves", ctypes.c_int64), ("sweeps_done", ctypes.c_int),
                ("energy_per_sweep", ctypes.c_double * 64), ("variance", ctypes.c_double), ("svd_sweeps_max", ctypes.c_int)]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_ if k != "energy_per_sweep"}
        d["energy_per_sweep"] = list(self.energy_per_sweep)[: self.sweeps_done]
        return d


class ServerConfig(ctypes.Structure):
    _fields_ = [("hbm_budget_bytes", ctypes.c_size_t), ("max_inflight", ctypes.c_int), ("device", ctypes.c_int), ("max_basis", ctypes.c_int)]


class Request(ctypes.Structure):
    _fields_ = [("dtype", ctypes.c_int), ("spin", ctypes.c_int64), ("chiL", ctypes.c_int64), ("chiR", ctypes.c_int64), ("mpoL", ctypes.c_int64),
                ("mpoR", ctypes.c_int64), ("mpo", _P), ("envL", _P), ("envR", _P), ("env_where", ctypes.c_int), ("theta0", _P),
                ("ritz", ctypes.c_int), ("target", ctypes.c_double), ("tol", ctypes.c_double), ("precision", ctypes.c_int), ("theta_out", _P),
                ("fp64_engine", ctypes.c_int)]


class Response(ctypes.Structure):
    _fields_ = [("id", ctypes.c_int64), ("status", ctypes.c_int), ("converged", ctypes.c_int), ("eigval", ctypes.c_double),
                ("resnorm", ctypes.c_double), ("num_mv", ctypes.c_int64), ("num_mv_mixed", ctypes.c_int64), ("t_submit", ctypes.c_double),
                ("t_start", ctypes.c_double), ("t_done", ctypes.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class ServerStats(ctypes.Structure):
    _fields_ = [("completed", ctypes.c_int64), ("failed", ctypes.c_int64), ("queued", ctypes.c_int64), ("inflight", ctypes.c_int),
                ("peak_inflight", ctypes.c_int), ("peak_bytes", ctypes.c_size_t), ("p50_latency_s", ctypes.c_double),
                ("p99_latency_s", ctypes.c_double), ("max_latency_s", ctypes.c_double), ("solves_per_s", ctypes.c_double),
                ("arena_bytes", ctypes.c_size_t), ("arena_grows", ctypes.c_int64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


def declare(L, sig):
    sig(L, "heff_server_config_default", None, [ctypes.POINTER(ServerConfig)])
    sig(L, "heff_server_create", _I, [ctypes.POINTER(ServerConfig), ctypes.POINTER(_P)])
    sig(L, "heff_request_bytes", ctypes.c_size_t, [ctypes.POINTER(Request), _I])
    sig(L, "heff_server_submit", _I, [_P, ctypes.POINTER(Request), _I64P])
    sig(L, "heff_server_wait", _I, [_P, _I64, ctypes.c_double, ctypes.POINTER(Response)])
    sig(L, "heff_server_get_stats", _I, [_P, ctypes.POINTER(ServerStats)])
    sig(L, "heff_server_destroy", _I, [_P])
    sig(L, "heff_make_env", _I, [_I, _I64, _I64, _I64, ctypes.c_uint64, _P, _P])
    sig(L, "heff_make_vector", _I, [_I, _I64, ctypes.c_uint64, _P, _P])
    sig(L, "heff_op_device_error", _I, [_P, ctypes.POINTER(ctypes.c_int)])
    sig(L, "heff_op_diagonal", _I, [_P, _P])
    sig(L, "heff_op_get_matrix", _I, [_P, _P])
    for n in ("heff_matvec_multi_d", "heff_matvec_multi_z"):
        sig(L, n, _I, [_P, _P, _I64P, _I, ctypes.POINTER(_P), _I64P, _P, _I64P, _P, _I64P, _P])
    sig(L, "heff_dense_eig", _I, [_I, _I64, _P, _I64, _P, _P, _P])
    sig(L, "heff_op_multpc", _I, [_P, _P, _P, ctypes.c_double])
    sig(L, "heff_op_set_graphs", _I, [_P, _I])
    sig(L, "heff_op_set_jacobi_blocksize", _I, [_P, _I64])
    sig(L, "heff_op_jacobi_singular", _I, [_P, ctypes.POINTER(ctypes.c_int)])
    sig(L, "heff_gemm_bf16_f32", _I, [_P, _P, _P, _I64, _I64, _I64, _P])
    sig(L, "heff_gemm_i8_emu", _I, [_I, _P, _P, _P, _I64, _I64, _I64, _I, _P])
    sig(L, "heff_i8_set_tile_width", _I, [_I])
    sig(L, "heff_i8_tuned_shapes", _I, [])
    sig(L, "heff_matvec_launches", _I64, [])
    sig(L, "heff_gemm_set_tail_split", _I, [_I])
    sig(L, "heff_op_set_fp64_engine", _I, [_P, _I, _I])
    sig(L, "heff_ensemble_run", _I, [ctypes.POINTER(DmrgConfig), _I, _I, ctypes.POINTER(DmrgResult), ctypes.POINTER(ctypes.c_int), _DP])
    sig(L, "heff_dmrg_config_default", None, [ctypes.POINTER(DmrgConfig)])
    sig(L, "heff_dmrg_run", _I, [ctypes.POINTER(DmrgConfig), ctypes.POINTER(DmrgResult), _P])
    sig(L, "heff_eig_config_default", None, [ctypes.POINTER(EigConfig)])
    sig(L, "heff_eigs", _I, [_P, ctypes.POINTER(EigConfig), _P, _P, ctypes.POINTER(EigResult)])
    for n in ("heff_env_update_d", "heff_env_update_z"):
        sig(L, n, _I, [_I, _P, _P, _I64P, _P, _I64P, _P, _I64P, _P])
    for n in ("heff_expansion_term_d", "heff_expansion_term_z"):
        sig(L, n, _I, [_I, _P, _P, _I64P, _P, _I64P, _P, _I64P, ctypes.c_double, _P])
    for n in ("heff_svd_d", "heff_svd_z"):
        sig(L, n, _I, [_P, _I64, _I64, _I64, ctypes.c_double, _P, _P, _P, _I64P, _DP, _P])
    for n in ("heff_schmidt_d", "heff_schmidt_z"):
        sig(L, n, _I, [_P, _I64, _I64, _I64, _I64, _I64, ctypes.c_double, _P, _P, _P, _I64P, _DP, _P])
