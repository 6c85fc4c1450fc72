"""ctypes binding of ``libmhd_b200.so`` (C ABI in ``include/mhd_b200.h``).

The library is required: importing the engine on a machine without the
built library or without an sm_100 GPU raises, there is no CPU fallback.
"""

from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
LIB_PATH = os.path.join(PKG, "libmhd_b200.so")

MHD_OK = 0
ERRORS = {
    -1: "MHD_ERR_INVALID",
    -2: "MHD_ERR_CUDA",
    -3: "MHD_ERR_NOT_CONVERGED",
    -4: "MHD_ERR_NONFINITE",
    -5: "MHD_ERR_CAPACITY",
    -6: "MHD_ERR_NO_DEVICE",
    -7: "MHD_ERR_RELIST",
}
MHD_ERR_RELIST = -7

KERNELS = {"cubic": 0, "quintic": 1, "wendland_c2": 2, "wendland_c4": 3, "wendland_c6": 4, "gaussian": 5,
           "super_gaussian": 6}
PRECISIONS = {"fp64": 0, "fp32": 1}


class MhdError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class MhdParams(ctypes.Structure):
    _fields_ = [
        ("dim", ctypes.c_int32),
        ("kernel", ctypes.c_int32),
        ("iterate", ctypes.c_int32),
        ("min_iter", ctypes.c_int32),
        ("max_iter", ctypes.c_int32),
        ("precision", ctypes.c_int32),
        ("periodic", ctypes.c_int32 * 3),
        ("reserved", ctypes.c_int32),
        ("hfact", ctypes.c_double),
        ("gamma", ctypes.c_double),
        ("mu0", ctypes.c_double),
        ("av", ctypes.c_double),
        ("ac", ctypes.c_double),
        ("ar", ctypes.c_double),
        ("clean_speed", ctypes.c_double),
        ("clean_damp", ctypes.c_double),
        ("timestep_factor", ctypes.c_double),
        ("alpha_min", ctypes.c_double),
        ("alpha_max", ctypes.c_double),
        ("tf", ctypes.c_double),
        ("lo", ctypes.c_double * 3),
        ("hi", ctypes.c_double * 3),
    ]


class MhdRhsStats(ctypes.Structure):
    _fields_ = [
        ("density_passes", ctypes.c_int32),
        ("grid_rebuilds", ctypes.c_int32),
        ("n_unconverged", ctypes.c_int64),
        ("n_cells", ctypes.c_int64),
    ]


_lib = None
_state_type = None
STATE_FIELDS: list[str] = []
SORTED_FIELDS: list[str] = []

EXPORTS = (
    "mhd_abi_version", "mhd_state_field_count", "mhd_state_field_name", "mhd_sorted_field_count",
    "mhd_sorted_field_name", "mhd_ctx_create", "mhd_ctx_destroy", "mhd_ctx_set_params", "mhd_last_error",
    "mhd_launch_count", "mhd_cells_build", "mhd_density_iterate", "mhd_force_pass", "mhd_rhs", "mhd_timestep",
    "mhd_clock_set", "mhd_clock_get", "mhd_step_initialize", "mhd_step_stage1", "mhd_step_stage2",
    "mhd_corrector_predictor", "mhd_step", "mhd_timing_enable", "mhd_timing_read", "mhd_probe_fma_peak",
    "mhd_pair_counts", "mhd_list_counts", "mhd_timestep_noalloc", "mhd_neighbour_counts", "mhd_ctx_set_instances",
    "mhd_instance_count", "mhd_clock_set_all", "mhd_clock_get_all", "mhd_advance", "mhd_ctx_tune",
    "mhd_tangent_dirs", "mhd_tangent_sync", "mhd_tangent_rhs", "mhd_tangent_step", "mhd_tangent_magnetic_energy",
    "mhd_adjoint_field_count", "mhd_adjoint_field_name", "mhd_adjoint_forward", "mhd_adjoint_backward",
)
NOALLOC_MAX_N = 67108864
TIMING_KINDS = ("cells", "density", "prologue", "force", "dt", "integrate", "lists")


def load(path: str = LIB_PATH):
    """Load the library (once) and build the MhdState layout from its own field list."""
    global _lib, _state_type
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(f"{path} is missing: build it with `python pysph-mhd_b200/build.py`")
    lib = ctypes.CDLL(path)
    vp = ctypes.c_void_p
    lib.mhd_state_field_name.restype = ctypes.c_char_p
    lib.mhd_state_field_name.argtypes = [ctypes.c_int32]
    lib.mhd_sorted_field_name.restype = ctypes.c_char_p
    lib.mhd_sorted_field_name.argtypes = [ctypes.c_int32]
    lib.mhd_last_error.restype = ctypes.c_char_p
    lib.mhd_last_error.argtypes = [vp]
    lib.mhd_launch_count.restype = ctypes.c_int64
    lib.mhd_launch_count.argtypes = [vp]
    lib.mhd_ctx_create.argtypes = [ctypes.POINTER(MhdParams), ctypes.c_int64, ctypes.POINTER(vp)]
    lib.mhd_ctx_destroy.argtypes = [vp]
    lib.mhd_ctx_set_params.argtypes = [vp, ctypes.POINTER(MhdParams)]
    STATE_FIELDS[:] = [lib.mhd_state_field_name(i).decode() for i in range(lib.mhd_state_field_count())]
    SORTED_FIELDS[:] = [lib.mhd_sorted_field_name(i).decode() for i in range(lib.mhd_sorted_field_count())]
    _state_type = type("MhdState", (ctypes.Structure,), {"_fields_": [(f, vp) for f in STATE_FIELDS]})
    sp = ctypes.POINTER(_state_type)
    st = ctypes.POINTER(MhdRhsStats)
    i64, dbl, i32 = ctypes.c_int64, ctypes.c_double, ctypes.c_int32
    lib.mhd_cells_build.argtypes = [vp, sp, sp, i64, vp]
    lib.mhd_density_iterate.argtypes = [vp, sp, i64, st, vp]
    lib.mhd_force_pass.argtypes = [vp, sp, i64, vp]
    lib.mhd_rhs.argtypes = [vp, sp, sp, i64, st, vp]
    lib.mhd_timestep.argtypes = [vp, sp, i64, dbl, ctypes.POINTER(dbl), vp]
    lib.mhd_clock_set.argtypes = [vp, dbl, dbl, vp]
    lib.mhd_clock_get.argtypes = [vp, ctypes.POINTER(dbl), ctypes.POINTER(dbl), vp]
    lib.mhd_step_initialize.argtypes = [vp, sp, i64, vp]
    lib.mhd_step_stage1.argtypes = [vp, sp, i64, dbl, vp]
    lib.mhd_step_stage2.argtypes = [vp, sp, i64, dbl, vp]
    lib.mhd_corrector_predictor.argtypes = [vp, sp, i64, i32, dbl, dbl, vp]
    lib.mhd_step.argtypes = [vp, sp, sp, i64, dbl, st, vp]
    lib.mhd_timing_enable.argtypes = [vp, i32]
    lib.mhd_timing_read.argtypes = [vp, ctypes.POINTER(dbl), ctypes.POINTER(i64)]
    lib.mhd_probe_fma_peak.argtypes = [i32, ctypes.POINTER(dbl), vp]
    lib.mhd_pair_counts.argtypes = [vp, ctypes.POINTER(i64), ctypes.POINTER(i64), vp]
    lib.mhd_list_counts.argtypes = [vp, ctypes.POINTER(i64), ctypes.POINTER(i64), vp]
    lib.mhd_timestep_noalloc.argtypes = [vp, i64, dbl, dbl, vp, vp]
    lib.mhd_neighbour_counts.argtypes = [vp, sp, i64, vp, vp]
    lib.mhd_ctx_set_instances.argtypes = [vp, sp, i32, ctypes.POINTER(i64), dbl, vp]
    lib.mhd_instance_count.argtypes = [vp]
    lib.mhd_instance_count.restype = i32
    lib.mhd_clock_set_all.argtypes = [vp, ctypes.POINTER(dbl), ctypes.POINTER(dbl), vp]
    lib.mhd_clock_get_all.argtypes = [vp, ctypes.POINTER(dbl), ctypes.POINTER(dbl), vp]
    lib.mhd_advance.argtypes = [vp, sp, sp, i64, i32, i32, i32, vp]
    lib.mhd_ctx_tune.argtypes = [vp, i32, i32]
    dp = ctypes.POINTER(dbl)
    lib.mhd_tangent_sync.argtypes = [vp, sp, i64, vp]
    lib.mhd_tangent_rhs.argtypes = [vp, sp, i64, dp, vp]
    lib.mhd_tangent_step.argtypes = [vp, sp, i64, dbl, dp, vp]
    lib.mhd_tangent_magnetic_energy.argtypes = [vp, sp, i64, dp, vp]
    lib.mhd_adjoint_field_name.restype = ctypes.c_char_p
    lib.mhd_adjoint_field_name.argtypes = [i32]
    lib.mhd_adjoint_forward.argtypes = [vp, sp, i64, i32, dp, i32, vp, dp, vp]
    lib.mhd_adjoint_backward.argtypes = [vp, sp, i64, i32, dp, i32, vp, vp, dp, vp]
    _lib = lib
    return lib


def state_type():
    load()
    return _state_type


def check(rc: int, ctx=None):
    if rc != MHD_OK:
        msg = _lib.mhd_last_error(ctx).decode() if _lib is not None else ""
        raise MhdError(rc, msg)


def make_params(dim, kernel, hfact, gamma, mu0, av, ac, ar, clean_speed, clean_damp, timestep_factor, tf, lo, hi,
                periodic, iterate=True, alpha_min=0.0, alpha_max=1.0, precision="fp64", min_iter=2,
                max_iter=250) -> MhdParams:
    p = MhdParams()
    p.dim = int(dim)
    p.kernel = KERNELS[kernel] if isinstance(kernel, str) else int(kernel)
    p.iterate = 1 if iterate else 0
    p.min_iter = min_iter
    p.max_iter = max_iter
    p.precision = PRECISIONS[precision] if isinstance(precision, str) else int(precision)
    for a in range(3):
        p.periodic[a] = 1 if periodic[a] else 0
        p.lo[a] = float(lo[a])
        p.hi[a] = float(hi[a])
    p.hfact = hfact
    p.gamma = gamma
    p.mu0 = mu0
    p.av = av
    p.ac = ac
    p.ar = ar
    p.clean_speed = clean_speed
    p.clean_damp = clean_damp
    p.timestep_factor = timestep_factor
    p.alpha_min = alpha_min
    p.alpha_max = alpha_max
    p.tf = tf
    return p
