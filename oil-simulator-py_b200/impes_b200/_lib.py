"""ctypes binding of libimpes_b200.so (the C ABI in include/impes_b200.h).

The shared library is built in-tree by ``csrc/build.py``.  There is no fallback:
if the library is missing or cannot be loaded, importing the compute modules
raises ``ImportError``.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libimpes_b200.so")

OK = 0
ERR_ARG, ERR_CUDA, ERR_NOT_CONVERGED, ERR_NAN, ERR_BAD_CSR = 1, 2, 3, 4, 5
ERR_COARSENING, ERR_OOM, ERR_TIMEOUT, ERR_SINGULAR, ERR_STATE = 6, 7, 8, 9, 10
NORM_EQUILIBRATED, NORM_JACOBI = 0, 1


class ImpesError(RuntimeError):
    """A non-zero status from the C ABI."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"[impes status {code}] {msg}")
        self.code = code


class NotConverged(ImpesError):
    pass


class AmgParams(C.Structure):
    _fields_ = [("theta", C.c_double), ("max_levels", C.c_int), ("coarsest_size", C.c_int),
                ("nullspace_dim", C.c_int), ("nullspace_blend", C.c_double),
                ("nullspace_reg", C.c_double), ("equilibration_threshold", C.c_double),
                ("tiebreak_seed", C.c_uint32), ("mixed_precision", C.c_int),
                ("p_max_elements", C.c_int), ("p_trunc_factor", C.c_double),
                ("smoother", C.c_int), ("cheb_lower", C.c_double), ("light_sweep_rows", C.c_int)]


class LevelDesc(C.Structure):
    _fields_ = [("n", C.c_int), ("nnz", C.c_int), ("p_cols", C.c_int), ("p_nnz", C.c_int),
                ("is_coarsest", C.c_int), ("col_index_bytes", C.c_int), ("col_row_relative", C.c_int),
                ("lanes", C.c_int * 6), ("layout", C.c_int * 2), ("fused_tail", C.c_int)]


class KrylovParams(C.Structure):
    _fields_ = [("tol", C.c_double), ("restart", C.c_int), ("max_iters", C.c_int),
                ("norm", C.c_int), ("precision", C.c_int), ("use_x0", C.c_int)]


class KrylovStats(C.Structure):
    _fields_ = [("iterations", C.c_int), ("restarts", C.c_int), ("converged", C.c_int),
                ("rel_res", C.c_double), ("true_rel_res", C.c_double)]


class ModelDesc(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
                ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double),
                ("mu_o", C.c_double), ("mu_w", C.c_double), ("mu_g", C.c_double),
                ("rho_o_ref", C.c_double), ("rho_w_ref", C.c_double), ("rho_g_ref", C.c_double),
                ("c_o", C.c_double), ("c_w", C.c_double), ("c_g", C.c_double), ("c_r", C.c_double),
                ("cf", C.c_double), ("relperm_model", C.c_int),
                ("nw", C.c_double), ("no", C.c_double), ("ng", C.c_double), ("now", C.c_double),
                ("nog", C.c_double), ("ko_end_w", C.c_double), ("ko_end_g", C.c_double),
                ("sw_cr", C.c_double), ("so_r", C.c_double), ("sg_cr", C.c_double),
                ("pc_scale", C.c_double), ("pc_exponent", C.c_double),
                ("pc_og_scale", C.c_double), ("pc_og_exponent", C.c_double),
                ("gravity", C.c_double), ("global_rate_scale", C.c_double),
                ("max_saturation_change", C.c_double), ("max_substeps", C.c_int),
                ("pvt_rows", C.c_int)]


class WellDesc(C.Structure):
    _fields_ = [("i", C.c_int), ("j", C.c_int), ("k", C.c_int), ("is_injector", C.c_int),
                ("control_bhp", C.c_int), ("value", C.c_double), ("well_index", C.c_double),
                ("injected_phase", C.c_int), ("surface_rate", C.c_int), ("surface_phase", C.c_int),
                ("limit_mask", C.c_int), ("limits", C.c_double * 4), ("has_bhp_min", C.c_int),
                ("bhp_min", C.c_double)]


class WellState(C.Structure):
    _fields_ = [("last_mode", C.c_int), ("has_q_total", C.c_int), ("last_q_total", C.c_double),
                ("has_surface_rates", C.c_int), ("surface_rates", C.c_double * 4)]


class SatStats(C.Structure):
    _fields_ = [("substeps", C.c_int), ("mass_balance", C.c_double * 6),
                ("component", C.c_double * 6)]


class AdjointStats(C.Structure):
    _fields_ = [("J", C.c_double), ("forward_iterations", C.c_longlong),
                ("adjoint_iterations", C.c_longlong), ("forward_ms", C.c_double),
                ("reverse_ms", C.c_double), ("checkpoints", C.c_int), ("recomputed_steps", C.c_int)]


class EnsembleMemberStats(C.Structure):
    _fields_ = [("status", C.c_int), ("steps_done", C.c_int), ("iterations", C.c_longlong),
                ("device_ms", C.c_double), ("worker", C.c_int)]


class Timing(C.Structure):
    _fields_ = [("count", C.c_longlong * 10), ("ms", C.c_double * 10), ("bytes", C.c_double * 10)]


PHASES = ("assemble", "saturation", "galerkin", "vcycle", "smooth_l0", "spmv_l0", "ortho", "solve",
          "smooth_wide", "tile_l0")

_P = C.c_void_p
_I = C.c_int
_D = C.c_double

# (name, argtypes)
_SIGNATURES = {
    "impes_last_error": ([], C.c_char_p),
    "impes_abi_version": ([], _I),
    "impes_amg_create": ([C.POINTER(_P), C.POINTER(AmgParams)], _I),
    "impes_amg_destroy": ([_P], _I),
    "impes_amg_setup": ([_P, _I, _I, _P, _P, _P, _P], _I),
    "impes_amg_update": ([_P, _P, _P], _I),
    "impes_amg_solve_vcycles": ([_P, _P, _P, _D, _I, C.POINTER(_I), C.POINTER(_D), _I, _P], _I),
    "impes_model_set_well_values": ([_P, _P, _I, _P], _I),
    "impes_pcg_solve": ([_I, _P, _P, _P, _P, _P, _D, _I, C.POINTER(_I), C.POINTER(_I), C.POINTER(_D), _P], _I),
    "impes_ensemble_run": ([_P, _P, _P, _P, _P, _P, _P, _I, _I, _D, C.POINTER(KrylovParams), _I,
                            _P, C.POINTER(_D)], _I),
    "impes_adjoint_num_producers": ([_P, C.POINTER(_I)], _I),
    "impes_adjoint_rates": ([_P, _P, _P, _P, _I, _D, C.POINTER(KrylovParams), _P, _P], _I),
    "impes_adjoint_gradient": ([_P, _P, _P, _P, _P, _P, _P, _I, _I, _D, C.POINTER(KrylovParams),
                                C.POINTER(KrylovParams), _P, _P, _P, _P, C.POINTER(AdjointStats), _P], _I),
    "impes_amg_solve_vcycles_noalloc": ([_P, _P, _P, _D, _I, C.POINTER(_I), C.POINTER(_D), _I, _P], _I),
    "impes_amg_apply": ([_P, _P, _P, _I, _D, _I, _P], _I),
    "impes_amg_vcycle_scaled": ([_P, _P, _P, _I, _P], _I),
    "impes_amg_fgmres": ([_P, _P, _P, C.POINTER(KrylovParams), C.POINTER(KrylovStats), _P], _I),
    "impes_amg_num_levels": ([_P, C.POINTER(_I)], _I),
    "impes_amg_level_info": ([_P, _I, C.POINTER(LevelDesc)], _I),
    "impes_amg_profile_levels": ([_P, _I, _I, C.POINTER(C.c_double), _P], _I),
    "impes_amg_step_graphs": ([_P, C.POINTER(C.c_int), C.POINTER(C.c_int)], _I),
    "impes_amg_level_export": ([_P, _I, _P, _P, _P, _P, _P, _P, _P, _P], _I),
    "impes_amg_equilibration": ([_P, _P, C.POINTER(_I), _P], _I),
    "impes_model_create": ([C.POINTER(_P), C.POINTER(ModelDesc), C.POINTER(WellDesc), _I, _P,
                            _P, _P, _P, _P, _P], _I),
    "impes_model_destroy": ([_P], _I),
    "impes_model_nnz": ([_P, C.POINTER(_I), C.POINTER(_I)], _I),
    "impes_csr_pattern": ([_P, _P, _P, _P], _I),
    "impes_well_cells": ([_P, _P], _I),
    "impes_model_export_static": ([_P, _P, _P, _P, _P, _P], _I),
    "impes_assemble": ([_P, _P, _P, _P, _D, _P, _P, _P], _I),
    "impes_saturation": ([_P, _P, _P, _P, _P, _D, C.POINTER(SatStats), _P], _I),
    "impes_step": ([_P, _P, _P, _P, _P, _P, _D, _I, C.POINTER(KrylovParams), _I,
                    C.POINTER(KrylovStats), C.POINTER(SatStats), _P], _I),
    "impes_model_balances": ([_P, C.POINTER(SatStats), _P], _I),
    "impes_model_reset_balances": ([_P, _P], _I),
    "impes_well_states": ([_P, C.POINTER(WellState), _P], _I),
    "impes_timing_enable": ([_I], _I),
    "impes_timing_collect": ([C.POINTER(Timing)], _I),
    "impes_kernel_launches": ([], C.c_ulonglong),
}

EXPORTED = tuple(_SIGNATURES)


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with python oil-simulator-py_b200/csrc/build.py")
    lib = C.CDLL(LIB_PATH)
    for name, (args, res) in _SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    return lib


lib = _load()


def check(status: int, what: str = ""):
    if status != OK:
        msg = lib.impes_last_error().decode(errors="replace")
        cls = NotConverged if status == ERR_NOT_CONVERGED else ImpesError
        raise cls(status, f"{what}: {msg}" if what else msg)


def ptr(t) -> int | None:
    """Device/host address of a contiguous torch tensor (None for None)."""
    if t is None:
        return None
    if not t.is_contiguous():
        raise ValueError("tensor must be contiguous")
    return t.data_ptr()


def timing_enable(on: bool = True):
    check(lib.impes_timing_enable(1 if on else 0), "impes_timing_enable")


def timing_collect() -> dict:
    """{phase: (launches, total ms, algorithmic bytes)} since the last collect."""
    t = Timing()
    check(lib.impes_timing_collect(C.byref(t)), "impes_timing_collect")
    return {name: (int(t.count[k]), float(t.ms[k]), float(t.bytes[k])) for k, name in enumerate(PHASES)}


def kernel_launches() -> int:
    return int(lib.impes_kernel_launches())


def stream_of(device=None) -> int:
    import torch
    return torch.cuda.current_stream(device).cuda_stream
