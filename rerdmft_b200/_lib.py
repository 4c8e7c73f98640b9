"""ctypes binding of librr_ri.so (the in-tree CUDA library, C ABI in include/rr_ri.h).

There is no CPU fallback: if the library is missing or cannot be loaded every call raises.
"""
from __future__ import annotations

import ctypes
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "librr_ri.so"

RR_OK, RR_ERR_ARG, RR_ERR_CUDA, RR_ERR_SOLVER, RR_ERR_TIMEOUT, RR_ERR_NOMEM, RR_ERR_STATE, RR_ERR_UNSUPPORTED = range(8)
RR_MEM_HOST, RR_MEM_DEVICE = 0, 1
RR_PREC_FP64, RR_PREC_MIXED = 0, 1
RR_MO_NONREL_SPIN, RR_MO_COMPLEX = 0, 1

_i64 = ctypes.c_int64
_i32 = ctypes.c_int32
_vp = ctypes.c_void_p
_d = ctypes.c_double


class RrError(RuntimeError):
    """Raised when a librr_ri call returns a non-zero status (the reference throws
    std::runtime_error at the same points)."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"[rr error {code}] {msg}")
        self.code = code


class Opts(ctypes.Structure):
    _fields_ = [("mem", _i32), ("precision", _i32), ("stream", _vp), ("sync", _i32), ("incremental", _i32)]


class Timings(ctypes.Structure):
    _fields_ = [("total_ms", _d), ("recovery_ms", _d), ("half_transform_ms", _d), ("exchange_ms", _d),
                ("coulomb_ms", _d), ("epilogue_ms", _d), ("reserved", _d * 4)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}


class ScfOpts(ctypes.Structure):
    _fields_ = [("diis_size", _i32), ("max_iterations", _i32), ("energy_tolerance", _d),
                ("density_tolerance", _d), ("kramers_restricted", _i32), ("precision", _i32),
                ("mixed_switch", _d), ("mixing", _d)]


class AdamOptions(ctypes.Structure):
    _fields_ = [("learning_rate", _d), ("rate_factor", _d), ("beta1", _d), ("beta2", _d), ("epsilon", _d),
                ("base_iterations", _i32), ("iterations_increment", _i32), ("max_iterations_limit", _i32),
                ("reserved", _i32), ("gradient_tolerance", _d), ("energy_tolerance", _d)]


class AdamResult(ctypes.Structure):
    _fields_ = [("improved", _i32), ("gradient_converged", _i32), ("energy_converged", _i32),
                ("restart_requested", _i32), ("iterations", _i32), ("reserved", _i32), ("energy_start", _d),
                ("energy_best", _d), ("energy_difference", _d), ("max_gradient", _d), ("learning_rate", _d)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}


class ScfResult(ctypes.Structure):
    _fields_ = [("electronic_energy", _d), ("iterations", _i64), ("converged", _i64),
                ("mixed_iterations", _i64), ("fp64_iterations", _i64), ("seconds", _d),
                ("build_ms", _d), ("diis_ms", _d), ("density_ms", _d),
                ("orbital_energies", _vp), ("c_matrix", _vp), ("fock_matrix", _vp)]


class RankReport(ctypes.Structure):
    _fields_ = [("n_kept", _i64), ("n_dropped", _i64), ("smallest_kept", _d), ("largest_dropped", _d)]


class Basis(ctypes.Structure):
    """rr_basis: a flattened BasisFunction list (host arrays)."""
    _fields_ = [("n", _i64), ("center", _vp), ("lxyz", _vp), ("prim_offset", _vp), ("exponents", _vp),
                ("coefficients", _vp)]


class PairOp(ctypes.Structure):
    _fields_ = [("s", _vp), ("idx", _vp), ("w", _vp), ("row", _vp), ("post", _vp)]


class Restart(ctypes.Structure):
    _fields_ = [("method", ctypes.c_char_p), ("functional", ctypes.c_char_p), ("kind", ctypes.c_char_p),
                ("basis_fingerprint", ctypes.c_uint64), ("n_electrons", _i64), ("pnof_subspaces", _i64),
                ("pnof_coupling", _i64), ("n_core", _i64), ("jk_frozen_pairs", _i64), ("jk_active_pairs", _i64),
                ("total_energy", _d), ("orbitals_optimized", _i32), ("converged", _i32),
                ("occupations", _vp), ("n_occupations", _i64), ("gammas", _vp), ("n_gammas", _i64),
                ("amplitudes", _vp), ("n_amplitudes", _i64), ("complex_coefficients", _i32), ("rows", _i64),
                ("cols", _i64), ("coefficients", _vp), ("cas_electrons", _i64), ("cas_spinors", _i64),
                ("cas_state", _vp), ("n_cas_state", _i64)]


class BatchStats(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int64), ("launches_total", ctypes.c_int64),
                ("launches_setup", ctypes.c_int64), ("launches_max_iteration", ctypes.c_int64),
                ("grouped_instances_first", ctypes.c_int64), ("seconds", ctypes.c_double),
                ("autotune_seconds", ctypes.c_double), ("autotune_entries", ctypes.c_int64),
                ("build_ms", ctypes.c_double), ("diis_ms", ctypes.c_double), ("density_ms", ctypes.c_double),
                ("sp2_steps_max", ctypes.c_int64), ("host_wait_ms", ctypes.c_double),
                ("host_gemm_ms", ctypes.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class X2cInstance(ctypes.Structure):
    _fields_ = [("h", _vp), ("h_x2c", _vp), ("X", _vp), ("n_eff", _i64), ("S", _vp), ("P0", _vp),
                ("n_electrons", _i32), ("status", _i32), ("P_out", _vp), ("energy_history", _vp),
                ("result", ScfResult)]


_SIGS = {
    "rr_scf_run_x2c_batch": (ctypes.c_int, [ctypes.POINTER(X2cInstance), _i64, ctypes.POINTER(ScfOpts), _i32]),
    "rr_scf_run_x2c_grouped": (ctypes.c_int, [ctypes.POINTER(X2cInstance), _i64, ctypes.POINTER(ScfOpts),
                                              ctypes.POINTER(BatchStats)]),
    "rr_autotune_load": (ctypes.c_int, [ctypes.c_char_p]),
    "rr_autotune_save": (ctypes.c_int, [ctypes.c_char_p]),
    "rr_autotune_clear": (ctypes.c_int, []),
    "rr_autotune_entries": (_i64, []),
    "rr_adam_default_options": (ctypes.c_int, [ctypes.POINTER(AdamOptions)]),
    "rr_orbopt_create": (ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, ctypes.POINTER(AdamOptions),
                                        ctypes.POINTER(_vp)]),
    "rr_orbopt_destroy": (ctypes.c_int, [_vp]),
    "rr_orbopt_exclude_negative": (ctypes.c_int, [_vp, _i64]),
    "rr_orbopt_set_functional": (ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "rr_orbopt_jk": (ctypes.c_int, [_vp, _vp, _vp]),
    "rr_orbopt_info": (ctypes.c_int, [_vp, ctypes.POINTER(_i64), ctypes.POINTER(_i64), ctypes.POINTER(_i64)]),
    "rr_orbopt_run": (ctypes.c_int, [_vp, ctypes.POINTER(AdamResult)]),
    "rr_orbopt_energy": (ctypes.c_int, [_vp, ctypes.POINTER(_d)]),
    "rr_orbopt_gradient": (ctypes.c_int, [_vp, _vp]),
    "rr_orbopt_set_scales": (ctypes.c_int, [_vp, _vp]),
    "rr_orbopt_hessian_diagonal": (ctypes.c_int, [_vp, _vp]),
    "rr_orbopt_features": (ctypes.c_int, [_vp, _vp]),
    "rr_orbopt_state": (ctypes.c_int, [_vp, _vp, _vp, _vp]),
    "rr_mlp_create": (ctypes.c_int, [ctypes.c_uint64, ctypes.POINTER(_vp)]),
    "rr_mlp_destroy": (ctypes.c_int, [_vp]),
    "rr_mlp_train": (ctypes.c_int, [_vp, _vp, _vp, _i64, _i32, _i32, ctypes.c_float, ctypes.c_uint64, _vp]),
    "rr_mlp_predict": (ctypes.c_int, [_vp, _vp, _i64, _i32, _vp]),
    "rr_mlp_loss_and_grad": (ctypes.c_int, [_vp, _vp, _vp, _i64, ctypes.POINTER(ctypes.c_float), _vp]),
    "rr_mlp_get_params": (ctypes.c_int, [_vp, _vp]),
    "rr_mlp_set_params": (ctypes.c_int, [_vp, _vp]),
    "rr_test_adam_steps": (ctypes.c_int, [_i64, _i32, _i64, _d, _d, _d, _d, _vp, _vp]),
    "rr_test_rotation_matrix": (ctypes.c_int, [_i64, _vp, _vp]),
    "rr_test_rotation_matrix_complex": (ctypes.c_int, [_i64, _vp, _vp]),
    "rr_test_adam_run_quadratic": (ctypes.c_int, [_i64, _vp, _vp, _d, _vp, _i32, _vp, _vp, _vp, _vp, _vp]),
    "rr_last_error": (ctypes.c_char_p, []),
    "rr_version": (ctypes.c_int, []),
    "rr_ri_create": (ctypes.c_int, [_vp, _i64, _i64, _i32, ctypes.POINTER(_vp)]),
    "rr_ri_create_4c": (ctypes.c_int, [_vp, _vp, _i64, _i64, _i64, _i32, ctypes.POINTER(_vp)]),
    "rr_ri_destroy": (ctypes.c_int, [_vp]),
    "rr_canonical_orthogonalize": (ctypes.c_int, [_vp, _i64, _i32, _d, _vp, ctypes.POINTER(_i64),
                                                  ctypes.POINTER(RankReport), ctypes.POINTER(Opts)]),
    "rr_ri_three_center_tensor": (ctypes.c_int, [_vp, _i64, _i64, _vp, _i64, _vp, ctypes.POINTER(Opts)]),
    "rr_ri_transform_ao_legs": (ctypes.c_int, [_vp, _i64, _i64, _vp, _i64, _vp, ctypes.POINTER(Opts)]),
    "rr_restart_write": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(Restart)]),
    "rr_restart_read": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(Restart)]),
    "rr_restart_release": (ctypes.c_int, [ctypes.POINTER(Restart)]),
    "rr_restart_coefficients": (ctypes.c_int, [_vp, _i64, _i64, _vp, _i32, _vp, ctypes.POINTER(Opts)]),
    "rr_density_from_orbitals": (ctypes.c_int, [_vp, _i64, _i64, _vp, _i32, _vp, ctypes.POINTER(Opts)]),
    "rr_sigma_toolkit": (ctypes.c_int, [_vp, _i64, _i64, _i32, _vp, _vp, _vp, _vp, _vp, _vp, ctypes.POINTER(Opts)]),
    "rr_sigma_pair_contract": (ctypes.c_int, [_vp, _d, _i64, _i64, _i32, ctypes.POINTER(PairOp), ctypes.POINTER(PairOp),
                                              ctypes.POINTER(Opts)]),
    "rr_sigma_diag_contract": (ctypes.c_int, [_vp, _i64, _i64, _i32, _vp, _vp, _vp, ctypes.POINTER(Opts)]),
    "rr_sigma_accum_u": (ctypes.c_int, [_vp, _d, _i64, _i64, _i32, _vp, _vp, ctypes.POINTER(Opts)]),
    "rr_ri_create_raw": (ctypes.c_int, [_vp, _i64, _i64, _vp, _i64, _vp, _i64, _i32, ctypes.POINTER(_vp)]),
    "rr_int_aux_metric": (ctypes.c_int, [ctypes.POINTER(Basis), _vp, ctypes.POINTER(Opts)]),
    "rr_int_three_center_raw": (ctypes.c_int, [ctypes.POINTER(Basis), ctypes.POINTER(Basis), _vp,
                                               ctypes.POINTER(Opts)]),
    "rr_ri_create_basis": (ctypes.c_int, [ctypes.POINTER(Basis), ctypes.POINTER(Basis), _d, _vp, _i64,
                                          ctypes.POINTER(_vp), ctypes.POINTER(_i64), ctypes.POINTER(RankReport)]),
    "rr_test_boys": (ctypes.c_int, [_vp, _i64, _i32, _vp]),
    "rr_ri_info": (ctypes.c_int, [_vp, ctypes.POINTER(_i64), ctypes.POINTER(_i64), ctypes.POINTER(_i64)]),
    "rr_ri_sync": (ctypes.c_int, [_vp]),
    "rr_ri_fock_nonrel": (ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, _i64, _vp, ctypes.POINTER(Opts)]),
    "rr_ri_jk_occupied": (ctypes.c_int, [_vp, _vp, _i64, _vp, _vp, ctypes.POINTER(Opts)]),
    "rr_ri_coulomb_noalloc": (ctypes.c_int, [_vp, _vp, _vp, ctypes.POINTER(Opts)]),
    "rr_ri_fock_x2c": (ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, _i64, _vp, ctypes.POINTER(Opts)]),
    "rr_ri_two_electron_ukb": (ctypes.c_int, [_vp, _vp, _vp, _i64, _vp, _vp, ctypes.POINTER(Opts)]),
    "rr_ri_fock_rkb": (ctypes.c_int, [_vp, _vp, _vp, _i64, _vp, _vp, _i64, _vp, _vp, ctypes.POINTER(Opts)]),
    "rr_mo_build_nonrel": (ctypes.c_int, [_vp, _vp, ctypes.POINTER(_vp), ctypes.POINTER(Opts)]),
    "rr_mo_build_nonrel_into": (ctypes.c_int, [_vp, _vp, _vp, ctypes.POINTER(Opts)]),
    "rr_mo_build_ukb": (ctypes.c_int, [_vp, _vp, _i64, ctypes.POINTER(_vp), ctypes.POINTER(Opts)]),
    "rr_mo_hx_joint_hessian_diagonal": (ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, _i64, _vp, _vp, _vp, _vp, _vp,
                                                       ctypes.POINTER(Opts)]),
    "rr_mo_cas_two_electron": (ctypes.c_int, [_vp, _vp, _vp, ctypes.POINTER(Opts)]),
    "rr_mo_cas_cumulant_fock": (ctypes.c_int, [_vp, _i64, _vp, _vp, _vp, ctypes.POINTER(Opts)]),
    "rr_mo_cas_active_integrals": (ctypes.c_int, [_vp, _i64, _vp, _vp, ctypes.POINTER(Opts)]),
    "rr_mo_from_tensor": (ctypes.c_int, [_vp, _i64, _i64, _i32, _i32, ctypes.POINTER(_vp)]),
    "rr_mo_destroy": (ctypes.c_int, [_vp]),
    "rr_mo_info": (ctypes.c_int, [_vp, ctypes.POINTER(_i64), ctypes.POINTER(_i64), ctypes.POINTER(_i32)]),
    "rr_mo_copy_tensor": (ctypes.c_int, [_vp, _vp, ctypes.POINTER(Opts)]),
    "rr_mo_rotated": (ctypes.c_int, [_vp, _vp, ctypes.POINTER(_vp), ctypes.POINTER(Opts)]),
    "rr_mo_positive_block": (ctypes.c_int, [_vp, _i64, ctypes.POINTER(_vp), ctypes.POINTER(Opts)]),
    "rr_mo_embedded": (ctypes.c_int, [_vp, _vp, ctypes.POINTER(Opts)]),
    "rr_mo_eri": (ctypes.c_int, [_vp, _i64, _vp, _vp, ctypes.POINTER(Opts)]),
    "rr_mo_jkl": (ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, ctypes.POINTER(Opts)]),
    "rr_mo_hx_fock": (ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, ctypes.POINTER(Opts)]),
    "rr_scf_run_nonrel": (ctypes.c_int, [_vp, _vp, _vp, _i64, _vp, _vp, _i32, ctypes.POINTER(ScfOpts),
                                         ctypes.POINTER(ScfResult), _vp, _vp, ctypes.POINTER(Opts)]),
    "rr_scf_run_x2c": (ctypes.c_int, [_vp, _vp, _vp, _i64, _vp, _vp, _i32, ctypes.POINTER(ScfOpts),
                                      ctypes.POINTER(ScfResult), _vp, _vp, ctypes.POINTER(Opts)]),
    "rr_scf_run_dhf": (ctypes.c_int, [_vp, _vp, _vp, _i64, _vp, _vp, _vp, _i32, ctypes.POINTER(ScfOpts),
                                      ctypes.POINTER(ScfResult), _vp, _vp, ctypes.POINTER(Opts)]),
    "rr_ri_set_profiling": (ctypes.c_int, [_vp, _i32]),
    "rr_ri_get_timings": (ctypes.c_int, [_vp, ctypes.c_void_p]),
    "rr_kernel_launches": (ctypes.c_int64, []),
    "rr_test_gemm_f64": (ctypes.c_int, [_i64, _i64, _i64, _vp, _i64, _i64, _i32, _vp, _i64, _i64, _i32, _vp, _i64,
                                        _i64, _d, _d, _i64, _i32, _i32, _i32, _i32, _i32]),
    "rr_test_mixed_exchange": (ctypes.c_int, [_vp, _i64, _i64, _vp, _i64, _vp]),
    "rr_test_mixed_exchange_delta": (ctypes.c_int, [_vp, _i64, _i64, _vp, _vp, _i64, _vp]),
    "rr_test_j_passes": (ctypes.c_int, [_vp, _i64, _i64, _vp, _vp, _vp]),
    "rr_test_j_passes_packed": (ctypes.c_int, [_vp, _i64, _i64, _vp, _vp, _vp, _vp]),
    "rr_test_device_allocations": (ctypes.c_int64, []),
    "rr_test_half_transform": (ctypes.c_int, [_vp, _i64, _vp, _i64, _i64, _vp, _i32]),
    "rr_test_half_transform_time": (ctypes.c_int, [_vp, _i64, _vp, _i64, _i64, _vp, _i32, _i32, _vp]),
    "rr_test_wait_expiry": (ctypes.c_int, [ctypes.c_uint32, _i32, ctypes.POINTER(_i32), ctypes.POINTER(_d),
                                           ctypes.POINTER(_d)]),
}

_lib = None


def lib():
    """Loads librr_ri.so (raises if it is absent: there is no fallback path)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is not built; run `python -m rerdmft_b200.build`")
        L = ctypes.CDLL(str(LIB_PATH))
        for name, (res, args) in _SIGS.items():
            f = getattr(L, name, None)
            if f is None:
                continue
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(rc: int) -> None:
    if rc != RR_OK:
        raise RrError(rc, lib().rr_last_error().decode())


def opts(mem: int = RR_MEM_HOST, precision: int = RR_PREC_FP64, stream: int | None = None, sync: int = 1,
         incremental: int = 0) -> Opts:
    return Opts(mem, precision, stream, sync, incremental)
