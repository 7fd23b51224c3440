"""ctypes binding of ``libmgpcg_b200.so`` (declared in include/mgpcg_b200.h).

The library is the only compute path: importing this module raises if the
shared object is missing or does not export every entry point of the header.
There is no CPU or PyTorch fallback.
"""
import ctypes
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmgpcg_b200.so")
HEADER_PATH = os.path.join(HERE, "..", "include", "mgpcg_b200.h")

FLUID, AIR, SOLID = 0, 1, 2

MG_OK = 0
MG_E_BADARG = -1
MG_E_CUDA = -2
MG_E_UNBOUND = -3
MG_E_TOO_BIG = -4

SOLVE_CONVERGED, SOLVE_MAX_ITERS, SOLVE_NONFINITE, SOLVE_BAD_OPERATOR = 0, 1, 2, 3
STATUS_NAMES = {0: "converged", 1: "max_iters", 2: "nonfinite", 3: "bad_operator", 4: "timeout"}

STORE = {"f32": 0, "fp32": 0, "float32": 0, "f16": 1, "fp16": 1, "float16": 1, "bf16": 2, "bfloat16": 2}
STORE_BYTES = {0: 4, 1: 2, 2: 2}

FIELD_B, FIELD_X, FIELD_P, FIELD_AP, FIELD_R, FIELD_Z, FIELD_TYPE, FIELD_ADIAG, FIELD_AX = range(9)


class MGError(RuntimeError):
    """A negative status from the C library, with its error string."""

    def __init__(self, rc, where):
        super().__init__(f"{where} failed with status {rc}: {last_error()}")
        self.rc = rc


class PlanDesc(ctypes.Structure):
    _fields_ = [("dim", ctypes.c_int32), ("res", ctypes.c_int32 * 3), ("levels", ctypes.c_int32),
                ("pre_post", ctypes.c_int32), ("bottom", ctypes.c_int32), ("storage", ctypes.c_int32),
                ("refresh_every", ctypes.c_int32), ("flags", ctypes.c_int32)]


class SolveParams(ctypes.Structure):
    _fields_ = [("max_iters", ctypes.c_int32), ("warm_start", ctypes.c_int32), ("rel_tol", ctypes.c_double),
                ("abs_tol", ctypes.c_double), ("eps", ctypes.c_double)]


class SolveStats(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int32), ("iters", ctypes.c_int32), ("rTr0", ctypes.c_double),
                ("rTr", ctypes.c_double), ("bTb", ctypes.c_double)]


_vp = ctypes.c_void_p
_i32 = ctypes.c_int32
_f32 = ctypes.c_float
_f64 = ctypes.c_double
PLAN_STORED = 1
PLAN_DIRECT = 2

_SIGS = {
    "mg_plan_create": (ctypes.c_int, [ctypes.POINTER(PlanDesc), ctypes.POINTER(_vp)]),
    "mg_plan_destroy": (ctypes.c_int, [_vp]),
    "mg_plan_workspace_bytes": (ctypes.c_int64, [_vp]),
    "mg_plan_field": (ctypes.c_int, [_vp, _i32, _i32, _i32, ctypes.POINTER(ctypes.c_int64),
                                     ctypes.POINTER(ctypes.c_int64)]),
    "mg_plan_bind": (ctypes.c_int, [_vp, _vp]),
    "mg_initialize": (ctypes.c_int, [_vp, _vp]),
    "mg_set_cell_type": (ctypes.c_int, [_vp, _vp, _vp]),
    "mg_init_gridtype": (ctypes.c_int, [_vp, _i32, _vp]),
    "mg_fill_fluid": (ctypes.c_int, [_vp, _vp]),
    "mg_build_pressure_b": (ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, _f32, _f32, _f32, _i32, _f32, _vp]),
    "mg_build_pressure_A": (ctypes.c_int, [_vp, _i32, _vp, _f32, _i32, _f32, _vp]),
    "mg_add_rhs": (ctypes.c_int, [_vp, _vp, _f32, _vp]),
    "mg_build_psi_b": (ctypes.c_int, [_vp, _vp, _f32, _f32, _f32, _f32, _i32, _i32, _i32, _vp]),
    "mg_build_psi_A": (ctypes.c_int, [_vp, _vp, _f32, _i32, _i32, _i32, _vp]),
    "mg_galerkin_coarsen": (ctypes.c_int, [_vp, _i32, _f32, _vp]),
    "mg_build_psi_A_level": (ctypes.c_int, [_vp, _i32, _vp, _vp, _f32, _i32, _i32, _i32, _vp]),
    "mg_build_magnetic_b": (ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _f32, _f32, _f32, _f32, _vp]),
    "mg_build_potential_b": (ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, _vp]),
    "mg_build_potential_A": (ctypes.c_int, [_vp, _i32, _vp, _f64, _vp]),
    "mg_update_susceptibility": (ctypes.c_int, [_vp, _vp, _f64, _f32, _vp, _vp]),
    "mg_update_magnetic_field": (ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, _f32, _vp, _vp, _vp, _vp]),
    "mg_level_set_volume": (ctypes.c_int, [_vp, _vp, _f32, _vp, _vp]),
    "mg_volume_control": (ctypes.c_int, [_vp, _vp, _f32, _vp, _vp]),
    "mg_calc_surface_normal": (ctypes.c_int, [_vp, _i32, _vp, _f32, _vp, _vp]),
    "mg_calc_curvature": (ctypes.c_int, [_vp, _vp, _f32, _vp, _vp]),
    "mg_build_surface_tension_b": (ctypes.c_int, [_vp, _i32, _vp, _vp, _vp, _vp, _f64, _f64, _f64, _f64, _vp]),
    "mg_build_surface_tension_A": (ctypes.c_int, [_vp, _i32, _i32, _vp, _f64, _f64, _f64, _f64, _vp]),
    "mg_level_set_shape": (ctypes.c_int, [_i32, _vp, _vp, _f32, _i32, _vp, _vp, _i32, _vp]),
    "mg_apply_markers": (ctypes.c_int, [_i32, _vp, _vp, _vp, _i32, _vp]),
    "mg_init_boundary": (ctypes.c_int, [_i32, _vp, _vp, _vp]),
    "mg_level_set_redistance": (ctypes.c_int, [_i32, _vp, _vp, _vp, _vp, _f64, _i32, _vp]),
    "mg_level_set_propagate": (ctypes.c_int, [_i32, _vp, _vp, _vp, _vp, _f64, _i32, _vp]),
    "mg_level_set_markers_distance": (ctypes.c_int, [_i32, _vp, _vp, _vp, _vp, _i32, _f64, _i32, _vp]),
    "mg_level_set_target_minus": (ctypes.c_int, [_i32, _vp, _vp, _vp, _vp, _f64, _vp]),
    "mg_level_set_smooth": (ctypes.c_int, [_i32, _vp, _vp, _vp, _vp]),
    "mg_advect_quantity": (ctypes.c_int, [_i32, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _f32, _f32, _vp]),
    "mg_extrapolate_velocity": (ctypes.c_int, [_i32, _vp, _i32, _vp, _vp, _vp, _vp, _vp, _i32, _vp]),
    "mg_enforce_boundary": (ctypes.c_int, [_i32, _vp, _vp, _vp, _vp, _vp, _vp]),
    "mg_add_gravity": (ctypes.c_int, [_i32, _vp, _vp, _vp, _vp, _f64, _f64, _f64, _f32, _vp]),
    "mg_apply_pressure": (ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _f32, _f32, _i32, _f32, _vp]),
    "mg_apply_magnetic_force": (ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _f32, _f32, _f32,
                                               _vp]),
    "mg_plan_prepare": (ctypes.c_int, [_vp, _vp]),
    "mg_plan_prepare_declared": (ctypes.c_int, [_vp, ctypes.POINTER(_f32), _vp]),
    "mg_plan_prepare_declared_whole": (ctypes.c_int, [_vp, _vp]),
    "mg_pressure_solve_async": (ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, _f32, _f32, _f32, _i32, _f32,
                                               ctypes.c_void_p, _vp]),
    "mg_pressure_setup_async": (ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, _f32, _f32, _f32, _i32, _f32, _i32,
                                               _vp]),
    "mg_batch_create": (ctypes.c_int, [ctypes.POINTER(_vp), _i32, ctypes.POINTER(_vp)]),
    "mg_batch_destroy": (None, [_vp]),
    "mg_batch_workspace_bytes": (ctypes.c_int64, [_vp]),
    "mg_batch_bind": (ctypes.c_int, [_vp, _vp, _vp]),
    "mg_batch_solve_async": (ctypes.c_int, [_vp, ctypes.POINTER(SolveParams), _vp]),
    "mg_batch_launch_counts": (ctypes.c_int, [_vp, ctypes.POINTER(_i32), ctypes.POINTER(_i32)]),
    "mg_plan_operator_form": (ctypes.c_int, [_vp, _i32, ctypes.POINTER(_i32)]),
    "mg_plan_split": (ctypes.c_int, [_vp, _i32, ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(_i32)]),
    "mg_plan_steps": (ctypes.c_int, [_vp, _i32, ctypes.POINTER(ctypes.c_uint32)]),
    "mg_plan_grid": (ctypes.c_int, [_vp, _i32, ctypes.POINTER(ctypes.c_uint32)]),
    "mg_plan_sweep_kernel": (ctypes.c_int, [_vp, _i32, ctypes.POINTER(ctypes.c_uint32)]),
    "mg_plan_resident": (ctypes.c_int, [_vp, _i32, ctypes.POINTER(_i32), ctypes.POINTER(_i32)]),
    "mg_smooth": (ctypes.c_int, [_vp, _i32, _i32, _vp]),
    "mg_restrict": (ctypes.c_int, [_vp, _i32, _vp]),
    "mg_prolongate": (ctypes.c_int, [_vp, _i32, _vp]),
    "mg_v_cycle": (ctypes.c_int, [_vp, _vp]),
    "mg_compute_Ap": (ctypes.c_int, [_vp, _vp]),
    "mg_reduce": (ctypes.c_int, [_vp, _i32, _i32, ctypes.POINTER(ctypes.c_double), _vp]),
    "mg_pcg_solve": (ctypes.c_int, [_vp, ctypes.POINTER(SolveParams), ctypes.POINTER(SolveStats), _vp]),
    "mg_pcg_solve_async": (ctypes.c_int, [_vp, ctypes.POINTER(SolveParams), _vp]),
    "mg_pcg_stats": (ctypes.c_int, [_vp, ctypes.POINTER(SolveStats), _vp]),
    "mg_plan_launch_counts": (ctypes.c_int, [_vp, ctypes.POINTER(_i32), ctypes.POINTER(_i32)]),
    "mg_launch_stage": (ctypes.c_int, [_vp, _i32, _i32, _vp]),
    "mg_reduce_static": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_int64, _vp, _vp]),
    "mg_last_error": (ctypes.c_char_p, []),
    "mg_version": (ctypes.c_int32, []),
}

_lib = None


def header_entry_points():
    """Names of every function declared in include/mgpcg_b200.h."""
    with open(HEADER_PATH) as f:
        text = f.read()
    return sorted(set(re.findall(r"MG_API\s+[\w\s\*]*?\b(mg_\w+)\s*\(", text)))


def load():
    """Loads the library once; raises if it is missing or incomplete."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with build_lib.py (no fallback exists)")
    lib = ctypes.CDLL(LIB_PATH)
    missing = [n for n in header_entry_points() if not hasattr(lib, n)]
    if missing:
        raise ImportError(f"{LIB_PATH} lacks entry points {missing}")
    for name, (res, args) in _SIGS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def last_error() -> str:
    if _lib is None:
        return ""
    s = _lib.mg_last_error()
    return s.decode() if s else ""


def check(rc, where=""):
    if rc != MG_OK:
        raise MGError(rc, where)
    return rc


def ptr(t):
    """Device (or host) address of a tensor / array, or None."""
    if t is None:
        return None
    if hasattr(t, "data_ptr"):
        return t.data_ptr()
    return t.ctypes.data


def stream_ptr(device=None):
    import torch
    return torch.cuda.current_stream(device).cuda_stream
