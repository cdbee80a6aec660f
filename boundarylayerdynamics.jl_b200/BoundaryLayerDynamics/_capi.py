"""ctypes binding of the engine's C ABI (include/bld.h).

The library is the in-tree ``lib/libbld.so`` built by ``build.py``.  There is
no fallback: if the library or a CUDA device is missing, loading or creating a
model raises.
"""

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("BLD_LIBRARY") or os.path.join(os.path.dirname(HERE), "lib", "libbld.so")

BLD_OK = 0
BLD_ERR_INVALID_CONFIG = -1
BLD_ERR_OUT_OF_MEMORY = -2
BLD_ERR_DIVERGED = -3
BLD_ERR_UNSUPPORTED_BC = -4
BLD_ERR_CUDA = -5
BLD_ERR_TIMEOUT = -6
BLD_ERR_ARGUMENT = -7
BLD_ERR_NO_DEVICE = -8

BC_DIRICHLET, BC_NEUMANN = 0, 1
WALL_OTHER, WALL_ROUGH, WALL_FREESLIP = 0, 1, 2
FP64, MIXED = 0, 1
EULER, AB2, SSPRK22, SSPRK33 = 0, 1, 2, 3
DEALIAS_NONE, DEALIAS_QUADRATIC, DEALIAS_EXPLICIT = 0, 1, 2

_dp = C.POINTER(C.c_double)


class BldConfig(C.Structure):
    _fields_ = [
        ("n1", C.c_int32), ("n2", C.c_int32), ("n3", C.c_int32), ("members", C.c_int32),
        ("l1", C.c_double), ("l2", C.c_double), ("x3_min", C.c_double), ("x3_max", C.c_double),
        ("dx3_c", _dp), ("dx3_i", _dp), ("x3_c", _dp), ("x3_i", _dp),
        ("bc_kind", (C.c_int32 * 2) * 3), ("bc_value", (C.c_double * 2) * 3),
        ("wall_kind", C.c_int32 * 2), ("wall_z0", C.c_double * 2), ("wall_kappa", C.c_double * 2),
        ("advection", C.c_int32), ("adv_dealias", C.c_int32), ("adv_p1", C.c_int32), ("adv_p2", C.c_int32),
        ("diffusion", C.c_int32 * 3), ("diffusivity", C.c_double * 3),
        ("pressure", C.c_int32),
        ("source", C.c_int32 * 3), ("source_strength", C.c_double * 3),
        ("mean", C.c_int32 * 3), ("mean_value", C.c_double * 3),
        ("sgs", C.c_int32), ("sgs_dealias", C.c_int32), ("sgs_p1", C.c_int32), ("sgs_p2", C.c_int32),
        ("sgs_cs", C.c_double), ("sgs_wall_damping", C.c_int32), ("sgs_wall_damping_exponent", C.c_double),
        ("precision", C.c_int32), ("device", C.c_int32),
        ("member_cs", _dp), ("member_z0_lower", _dp), ("member_source1", _dp),
    ]


class BldInfo(C.Structure):
    _fields_ = [
        ("k1max", C.c_int32), ("k2max", C.c_int32), ("n3", C.c_int32), ("members", C.c_int32),
        ("modes_per_layer", C.c_int64), ("state_doubles", C.c_int64),
        ("adv_p1", C.c_int32), ("adv_p2", C.c_int32), ("adv_ref_p1", C.c_int32), ("adv_ref_p2", C.c_int32),
        ("sgs_p1", C.c_int32), ("sgs_p2", C.c_int32),
        ("device_bytes", C.c_int64), ("precision", C.c_int32),
    ]


class BldPhaseTimes(C.Structure):
    _fields_ = [
        ("inv_y_ms", C.c_double * 2), ("x_ms", C.c_double * 2), ("fwd_y_ms", C.c_double * 2),
        ("project_ms", C.c_double), ("linear_ms", C.c_double), ("launches_per_step", C.c_int32),
    ]


class BldProgress(C.Structure):
    _fields_ = [
        ("mean_velocity", C.c_double * 3), ("mean_ke", C.c_double), ("turbulent_ke", C.c_double),
        ("advective_timescale", C.c_double), ("wall_stress", (C.c_double * 2) * 2),
        ("grid_p1", C.c_int32), ("grid_p2", C.c_int32),
    ]


# exported symbols and their signatures (every declaration of include/bld.h)
SIGNATURES = {
    "bld_abi_version": (C.c_int32, []),
    "bld_status_string": (C.c_char_p, [C.c_int32]),
    "bld_last_error": (C.c_int32, [C.c_char_p, C.c_size_t]),
    "bld_create": (C.c_int32, [C.POINTER(BldConfig), C.POINTER(C.c_void_p)]),
    "bld_destroy": (None, [C.c_void_p]),
    "bld_get_info": (C.c_int32, [C.c_void_p, C.POINTER(BldInfo)]),
    "bld_set_state": (C.c_int32, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p]),
    "bld_get_state": (C.c_int32, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p]),
    "bld_compute_rates": (C.c_int32, [C.c_void_p, C.c_int32] + [C.c_void_p] * 6),
    "bld_apply_projections": (C.c_int32, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p]),
    "bld_evolve": (C.c_int32, [C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_int32]),
    "bld_prepare": (C.c_int32, [C.c_void_p]),
    "bld_step": (C.c_int32, [C.c_void_p, C.c_int64, C.c_double, C.c_int32]),
    "bld_compute_rates_device": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "bld_apply_projections_device": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "bld_state_device_ptr": (C.c_int32, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "bld_sync": (C.c_int32, [C.c_void_p]),
    "bld_set_field_physical": (C.c_int32, [C.c_void_p, C.c_int32, C.c_int32, C.c_void_p]),
    "bld_get_field_physical": (C.c_int32, [C.c_void_p, C.c_int32, C.c_int32, C.c_void_p]),
    "bld_set_field_centered": (C.c_int32, [C.c_void_p, C.c_int32, C.c_int32, C.c_void_p]),
    "bld_get_field_centered": (C.c_int32, [C.c_void_p, C.c_int32, C.c_int32, C.c_void_p]),
    "bld_profiles_start": (C.c_int32, [C.c_void_p, C.c_int32]),
    "bld_profiles_read": (C.c_int32, [C.c_void_p, C.c_int32, C.c_void_p]),
    "bld_profiles_sample": (C.c_int32, [C.c_void_p, C.c_int32, C.c_void_p]),
    "bld_get_stream": (C.c_int32, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "bld_step_async": (C.c_int32, [C.c_void_p, C.c_int64, C.c_double, C.c_int32]),
    "bld_stream_idle": (C.c_int32, [C.c_void_p, C.POINTER(C.c_int32)]),
    "bld_set_wait_limit": (C.c_int32, [C.c_int32, C.c_int64]),
    "bld_time_phases": (C.c_int32, [C.c_void_p, C.c_int32, C.c_int32, C.POINTER(BldPhaseTimes)]),
    "bld_ensemble_step": (C.c_int32, [C.c_void_p, C.c_int32, C.c_int64, C.c_double, C.c_int32]),
    "bld_set_active": (C.c_int32, [C.c_void_p, C.c_void_p]),
    "bld_set_member_params": (C.c_int32, [C.c_void_p, C.c_int32, C.c_double, C.c_double, C.c_double]),
    "bld_prepare_member": (C.c_int32, [C.c_void_p, C.c_int32]),
    "bld_get_diverged": (C.c_int32, [C.c_void_p, C.c_void_p]),
    "bld_describe": (C.c_int32, [C.c_void_p, C.c_char_p, C.c_size_t]),
    "bld_progress_stats": (C.c_int32, [C.c_void_p, C.c_int32, C.POINTER(BldProgress)]),
    "bld_init_random_field": (C.c_int32, [C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_int32,
                                          C.c_uint64]),
    "bld_project_noalloc": (C.c_int32, [C.c_int32, C.c_int32, C.c_int32] + [C.c_void_p] * 5
                            + [C.c_double, C.c_double, C.c_void_p, C.c_void_p]),
    "bld_ldlt_solve_device": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_int32, C.c_void_p]),
    "bld_ldlt_solve_real_device": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_int32, C.c_void_p]),
}

_lib = None


def load(path=None):
    """Load libbld.so (built in-tree); raises if it is missing."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError(f"libbld.so not found at {p}; run boundarylayerdynamics.jl_b200/build.py")
    lib = C.CDLL(p)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if lib.bld_abi_version() != 1:
        raise RuntimeError("libbld.so ABI version mismatch")
    if path is None:
        _lib = lib
    return lib


class BldError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(message)
        self.status = status


class DivergenceError(BldError):
    """``error("The simulation has diverged.")`` of rate! (src/BoundaryLayerDynamics.jl:156)."""


def check(status):
    if status == BLD_OK:
        return
    lib = load()
    buf = C.create_string_buffer(1024)
    lib.bld_last_error(buf, len(buf))
    msg = buf.value.decode(errors="replace") or lib.bld_status_string(status).decode()
    if status == BLD_ERR_DIVERGED:
        raise DivergenceError(status, "The simulation has diverged.")
    raise BldError(status, f"{lib.bld_status_string(status).decode()}: {msg}")
