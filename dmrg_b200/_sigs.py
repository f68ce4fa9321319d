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
                ("inner_iters", ctypes.c_int), ("inner_tol", ctypes.c_double), ("seed", ctypes.c_int64)]


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
                ("precision", ctypes.c_int), ("seed", ctypes.c_int64), ("energy_shift_per_site", ctypes.c_double)]


class DmrgResult(ctypes.Structure):
    """heff_dmrg_result (include/heff.h)."""

    _fields_ = [("energy", ctypes.c_double), ("entropy_mid", ctypes.c_double), ("trunc_err_max", ctypes.c_double), ("seconds", ctypes.c_double),
                ("t_eig", ctypes.c_double), ("t_svd", ctypes.c_double), ("t_env", ctypes.c_double), ("chi_mid", ctypes.c_int64),
                ("num_mv", ctypes.c_int64), ("num_mv_mixed", ctypes.c_int64), ("unconverged_solves", ctypes.c_int64), ("sweeps_done", ctypes.c_int),
                ("energy_per_sweep", ctypes.c_double * 64)]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_ if k != "energy_per_sweep"}
        d["energy_per_sweep"] = list(self.energy_per_sweep)[: self.sweeps_done]
        return d


def declare(L, sig):
    sig(L, "heff_op_device_error", _I, [_P, ctypes.POINTER(ctypes.c_int)])
    sig(L, "heff_gemm_bf16_f32", _I, [_P, _P, _P, _I64, _I64, _I64, _P])
    sig(L, "heff_dmrg_config_default", None, [ctypes.POINTER(DmrgConfig)])
    sig(L, "heff_dmrg_run", _I, [ctypes.POINTER(DmrgConfig), ctypes.POINTER(DmrgResult), _P])
    sig(L, "heff_eig_config_default", None, [ctypes.POINTER(EigConfig)])
    sig(L, "heff_eigs", _I, [_P, ctypes.POINTER(EigConfig), _P, _P, ctypes.POINTER(EigResult)])
    for n in ("heff_env_update_d", "heff_env_update_z"):
        sig(L, n, _I, [_I, _P, _P, _I64P, _P, _I64P, _P, _I64P, _P])
    sig(L, "heff_svd_d", _I, [_P, _I64, _I64, _I64, ctypes.c_double, _P, _P, _P, _I64P, _DP, _P])
    sig(L, "heff_schmidt_d", _I, [_P, _I64, _I64, _I64, _I64, _I64, ctypes.c_double, _P, _P, _P, _I64P, _DP, _P])
