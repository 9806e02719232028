"""ctypes binding of the C ABI declared in include/cup_b200.h.

The CUDA library must exist in-tree (``cubismup_3d_b200/libcup_b200.so``);
there is no fallback of any kind: if it is missing, loading raises.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcup_b200.so")

CUP_OK = 0
CUP_ERR_ARG = 1
CUP_ERR_CUDA = 2
CUP_ERR_NONFINITE = 3
CUP_ERR_NOT_CONVERGED = 4
CUP_ERR_STATE = 5
CUP_ERR_TIMEOUT = 6

CUP_PREC_FP64 = 0
CUP_PREC_FP32_DC = 1
CUP_SCHEME_REF = 0
CUP_SCHEME_UPWIND3_RK2 = 1
CUP_WHERE_HOST = 0
CUP_WHERE_DEVICE = 1
CUP_FIELD_U, CUP_FIELD_V, CUP_FIELD_W, CUP_FIELD_P, CUP_FIELD_RHS = 0, 1, 2, 3, 4

ERROR_NAMES = {
    CUP_ERR_ARG: "CUP_ERR_ARG", CUP_ERR_CUDA: "CUP_ERR_CUDA", CUP_ERR_NONFINITE: "CUP_ERR_NONFINITE",
    CUP_ERR_NOT_CONVERGED: "CUP_ERR_NOT_CONVERGED", CUP_ERR_STATE: "CUP_ERR_STATE",
    CUP_ERR_TIMEOUT: "CUP_ERR_TIMEOUT",
}


class CupConfig(C.Structure):
    _fields_ = [
        ("bpdx", C.c_int), ("bpdy", C.c_int), ("bpdz", C.c_int),
        ("maxextent", C.c_double),
        ("nu", C.c_double), ("CFL", C.c_double), ("lambda_", C.c_double), ("DLM", C.c_double),
        ("uinf", C.c_double * 3),
        ("rampup", C.c_int),
        ("bImplicitPenalization", C.c_int),
        ("precision", C.c_int),
        ("scheme", C.c_int),
        ("dc_tol", C.c_double),
        ("dc_max_iter", C.c_int),
        ("dc_min_iter", C.c_int),
        ("device", C.c_int),
        ("z_halo", C.c_int),
    ]


class CupSphere(C.Structure):
    _fields_ = [
        ("radius", C.c_double),
        ("position", C.c_double * 3),
        ("enforcedVelocity", C.c_double * 3),
        ("bForcedInSimFrame", C.c_int * 3),
        ("bFixFrameOfRef", C.c_int * 3),
    ]


class CupSolveStats(C.Structure):
    _fields_ = [("n_solves", C.c_int), ("rel_residual", C.c_double)]


class CupStepStats(C.Structure):
    _fields_ = [
        ("dt", C.c_double), ("time", C.c_double), ("step", C.c_int),
        ("umax", C.c_double), ("kinetic_energy", C.c_double),
        ("force", C.c_double * 3), ("torque", C.c_double * 3),
        ("n_solves", C.c_int), ("rel_residual", C.c_double), ("n_unconverged", C.c_int),
        ("n_solves_total", C.c_longlong),
    ]


_dp = C.POINTER(C.c_double)
_H = C.c_void_p

# name -> (restype, argtypes); every symbol declared in include/cup_b200.h
SIGNATURES = {
    "cup_create": (C.c_int, [C.POINTER(CupConfig), C.POINTER(C.c_void_p)]),
    "cup_destroy": (C.c_int, [_H]),
    "cup_last_error": (C.c_char_p, [_H]),
    "cup_set_stream": (C.c_int, [_H, C.c_void_p]),
    "cup_sync": (C.c_int, [_H]),
    "cup_get_dims": (C.c_int, [_H, C.POINTER(C.c_int), _dp]),
    "cup_set_velocity": (C.c_int, [_H, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]),
    "cup_get_velocity": (C.c_int, [_H, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]),
    "cup_get_pressure": (C.c_int, [_H, C.c_void_p, C.c_int]),
    "cup_get_chi": (C.c_int, [_H, C.c_void_p, C.c_int]),
    "cup_get_rhs": (C.c_int, [_H, C.c_void_p, C.c_int]),
    "cup_field_ptr": (C.c_int, [_H, C.c_int, C.POINTER(C.c_void_p)]),
    "cup_blocks_to_global": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int]),
    "cup_global_to_blocks": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int]),
    "cup_add_sphere": (C.c_int, [_H, C.POINTER(CupSphere)]),
    "cup_create_obstacles": (C.c_int, [_H, C.c_double]),
    "cup_update_obstacles": (C.c_int, [_H, C.c_double]),
    "cup_get_sphere_motion": (C.c_int, [_H, _dp, _dp, _dp]),
    "cup_set_sphere_motion": (C.c_int, [_H, _dp, _dp, _dp]),
    "cup_set_graphs": (C.c_int, [_H, C.c_int]),
    "cup_prepare_run": (C.c_int, [_H, C.c_int, C.POINTER(C.c_int)]),
    "cup_set_sphere_position": (C.c_int, [_H, _dp]),
    "cup_get_sphere_position": (C.c_int, [_H, _dp]),
    "cup_set_uinf": (C.c_int, [_H, _dp]),
    "cup_get_obstacle_state": (C.c_int, [_H, _dp, _dp, _dp, _dp]),
    "cup_set_clock": (C.c_int, [_H, C.c_int, C.c_double]),
    "cup_max_velocity": (C.c_int, [_H, _dp]),
    "cup_calc_max_timestep": (C.c_int, [_H, _dp]),
    "cup_advect_diffuse": (C.c_int, [_H, C.c_double]),
    "cup_pressure_rhs": (C.c_int, [_H, C.c_double]),
    "cup_poisson_solve": (C.c_int, [_H, C.POINTER(CupSolveStats)]),
    "cup_grad_correct": (C.c_int, [_H, C.c_double]),
    "cup_poisson_buffer": (C.c_int, [_H, C.POINTER(C.c_void_p), C.POINTER(C.c_size_t), C.POINTER(C.c_size_t)]),
    "cup_poisson_reset": (C.c_int, [_H]),
    "cup_set_rhs": (C.c_int, [_H, C.c_void_p, C.c_int]),
    "cup_set_spectral_window": (C.c_int, [_H, C.c_int, C.c_int]),
    "cup_poisson_pass": (C.c_int, [_H, C.c_void_p, C.c_int]),
    "cup_pressure_projection": (C.c_int, [_H, C.c_double, C.POINTER(CupSolveStats)]),
    "cup_penalize": (C.c_int, [_H, C.c_double, _dp]),
    "cup_step": (C.c_int, [_H, C.c_double, C.POINTER(CupStepStats)]),
    "cup_run": (C.c_int, [_H, C.c_int, C.POINTER(CupStepStats)]),
    "cup_adjoint_step": (C.c_int, [_H, C.c_void_p, C.c_void_p, C.c_void_p, C.c_double, C.c_void_p, C.c_void_p,
                                   C.c_void_p]),
    "cup_get_velocity_raw": (C.c_int, [_H, C.c_void_p, C.c_void_p, C.c_void_p]),
    "cup_set_velocity_raw": (C.c_int, [_H, C.c_void_p, C.c_void_p, C.c_void_p]),
    "cup_poisson_solve_field": (C.c_int, [_H, C.c_void_p, C.c_void_p, C.c_int]),
    "cup_diagnostics": (C.c_int, [_H, _dp]),
    "cup_compute_dissipation": (C.c_int, [_H, _dp]),
    "cup_compute_forces": (C.c_int, [_H, _dp]),
    "cup_spectral_analysis": (C.c_int, [_H, _dp, _dp, C.c_int]),
    "cup_set_spectral_forcing": (C.c_int, [_H, C.c_double, C.c_double]),
    "cup_spectral_forcing": (C.c_int, [_H, C.c_double, _dp]),
    "cup_get_forcing_stats": (C.c_int, [_H, _dp]),
    "cup_debug_shift": (C.c_int, [_H, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]),
    "cup_max_velocity_noalloc": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_longlong, _dp, C.c_void_p,
                                           C.c_void_p]),
    "cup_dc_history": (C.c_int, [_H, _dp, C.c_int, C.POINTER(C.c_int)]),
    "cup_profile_enable": (C.c_int, [_H, C.c_int]),
    "cup_profile_report": (C.c_int, [_H, C.c_char_p, C.c_size_t, C.c_int]),
    "cup_adjoint_step_obstacle": (C.c_int, [_H, C.c_void_p, C.c_void_p, C.c_void_p, C.c_double, C.c_void_p,
                                            C.c_void_p, C.c_void_p, _dp, C.c_void_p, C.c_void_p]),
    "cup_set_chi": (C.c_int, [_H, C.c_void_p, C.c_int]),
    "cup_set_sphere_velocity": (C.c_int, [_H, _dp]),
    "cup_launch_count": (C.c_int, [_H, C.POINTER(C.c_longlong)]),
}

_lib = None


def lib():
    """Loads libcup_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -m cubismup_3d_b200.build` "
                "(nvcc, sm_100a). There is no fallback implementation.")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


class CupError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERROR_NAMES.get(code, code)}: {msg}")
        self.code = code


def check(code: int, handle=None, what: str = ""):
    if code == CUP_OK:
        return
    msg = what
    if handle:
        m = lib().cup_last_error(handle)
        if m:
            msg = f"{what}: {m.decode()}" if what else m.decode()
    if code == CUP_ERR_ARG:
        raise ValueError(f"CUP_ERR_ARG: {msg}")
    raise CupError(code, msg)
