"""ctypes binding of libns3d_b200.so (the C ABI declared in include/ns3d_b200.h).

The library is loaded from this package directory.  There is no fallback: if
the library is missing, or no CUDA device is present, the calls fail loudly.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libns3d_b200.so")

NS3D_OK = 0
NS3D_PRIMITIVE, NS3D_CONSERVED, NS3D_RHS, NS3D_TEMPERATURE = 0, 1, 2, 3
NS3D_FP64, NS3D_MIXED = 0, 1

STATUS = {0: "NS3D_OK", -1: "NS3D_ERR_INVALID_ARG", -2: "NS3D_ERR_CONFIG", -3: "NS3D_ERR_OOM",
          -4: "NS3D_ERR_CUDA", -5: "NS3D_ERR_NONFINITE", -6: "NS3D_ERR_NO_DEVICE", -7: "NS3D_ERR_STATE",
          -8: "NS3D_ERR_DT", -9: "NS3D_ERR_TIMEOUT", -10: "NS3D_ERR_SIZE"}

# every entry point declared in include/ns3d_b200.h
EXPORTS = [
    "ns3d_params_default", "ns3d_status_string", "ns3d_create", "ns3d_destroy", "ns3d_last_error",
    "ns3d_field_dims", "ns3d_upload_primitives", "ns3d_initialize", "ns3d_set_interior_primitives", "ns3d_download",
    "ns3d_apply_boundary", "ns3d_compute_rhs", "ns3d_rk3_step", "ns3d_rk3_steps",
    "ns3d_compute_timestep", "ns3d_total_energy", "ns3d_diagnostics", "ns3d_residuals", "ns3d_time_advance",
    "ns3d_device_fields", "ns3d_set_stream", "ns3d_synchronize", "ns3d_last_launch_count",
    "ns3d_profile", "ns3d_profile_report", "ns3d_compute_timestep_noalloc", "ns3d_set_slab", "ns3d_rk3_stage",
    "ns3d_debug_face_vjp", "ns3d_debug_visc_vjp", "ns3d_debug_riemann", "ns3d_debug_wait_timeout",
    "ns3d_debug_mdcd_detector", "ns3d_vjp_rhs", "ns3d_vjp_rk3_step",
    "ns3d_adjoint_kinetic_energy", "ns3d_batch_create", "ns3d_batch_destroy", "ns3d_batch_last_error",
    "ns3d_batch_set_interior_primitives", "ns3d_batch_run", "ns3d_batch_autotune", "ns3d_batch_set_config",
    "ns3d_batch_query", "ns3d_batch_download",
]


class Params(C.Structure):
    _fields_ = [("gamma", C.c_double), ("Pr", C.c_double), ("Ma", C.c_double), ("Re", C.c_double),
                ("cfl", C.c_double), ("dt_fixed", C.c_double), ("mdcd_diss", C.c_double),
                ("mdcd_disp", C.c_double), ("sutherland_s", C.c_double), ("interpolation", C.c_int),
                ("riemann_solver", C.c_int), ("char_recon", C.c_int), ("bc", C.c_int * 6),
                ("precision", C.c_int), ("device", C.c_int), ("check_state", C.c_int),
                ("keep_rhs", C.c_int)]


class Grid(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("x0", C.c_double), ("y0", C.c_double),
                ("z0", C.c_double), ("Lx", C.c_double), ("Ly", C.c_double), ("Lz", C.c_double)]


class Ns3dError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


_lib = None


def load() -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is not built; run ns3d_wcns_b200.build.build()")
    lib = C.CDLL(LIB_PATH)
    dp = C.POINTER(C.c_double)
    h = C.c_void_p
    lib.ns3d_params_default.argtypes = [C.POINTER(Params)]
    lib.ns3d_params_default.restype = None
    lib.ns3d_status_string.restype = C.c_char_p
    lib.ns3d_status_string.argtypes = [C.c_int]
    lib.ns3d_create.argtypes = [C.POINTER(Params), C.POINTER(Grid), C.POINTER(h)]
    lib.ns3d_destroy.argtypes = [h]
    lib.ns3d_last_error.restype = C.c_char_p
    lib.ns3d_last_error.argtypes = [h]
    lib.ns3d_field_dims.argtypes = [h, C.POINTER(C.c_int)]
    lib.ns3d_upload_primitives.argtypes = [h, C.POINTER(dp)]
    lib.ns3d_set_interior_primitives.argtypes = [h, C.POINTER(dp)]
    lib.ns3d_initialize.argtypes = [h, C.c_int]
    lib.ns3d_download.argtypes = [h, C.c_int, C.POINTER(dp)]
    lib.ns3d_apply_boundary.argtypes = [h]
    lib.ns3d_compute_rhs.argtypes = [h]
    lib.ns3d_rk3_step.argtypes = [h, C.c_double]
    lib.ns3d_rk3_steps.argtypes = [h, C.c_int, C.c_double]
    lib.ns3d_compute_timestep.argtypes = [h, dp]
    lib.ns3d_total_energy.argtypes = [h, dp]
    lib.ns3d_diagnostics.argtypes = [h, dp]
    lib.ns3d_residuals.argtypes = [h, dp]
    lib.ns3d_time_advance.argtypes = [h, C.c_double, C.c_int, dp, C.POINTER(C.c_int)]
    lib.ns3d_device_fields.argtypes = [h, C.c_int, C.POINTER(C.c_void_p), C.POINTER(C.c_long)]
    lib.ns3d_set_stream.argtypes = [h, C.c_void_p]
    lib.ns3d_set_slab.argtypes = [h, C.c_int, C.c_int, C.c_double, C.c_int]
    lib.ns3d_rk3_stage.argtypes = [h, C.c_int, C.c_double]
    lib.ns3d_synchronize.argtypes = [h]
    lib.ns3d_last_launch_count.argtypes = [h, C.POINTER(C.c_long)]
    lib.ns3d_profile.argtypes = [h, C.c_int]
    lib.ns3d_profile_report.argtypes = [h, C.c_char_p, C.c_long]
    lib.ns3d_vjp_rhs.argtypes = [h, C.POINTER(dp), C.POINTER(dp)]
    lib.ns3d_vjp_rk3_step.argtypes = [h, C.c_double, C.POINTER(dp), C.POINTER(dp)]
    lib.ns3d_adjoint_kinetic_energy.argtypes = [h, C.c_int, C.c_double, C.c_int, dp, C.POINTER(dp), dp]
    lib.ns3d_batch_create.argtypes = [C.POINTER(Params), C.c_int, C.POINTER(Grid), dp, C.POINTER(h)]
    lib.ns3d_batch_destroy.argtypes = [h]
    lib.ns3d_batch_last_error.restype = C.c_char_p
    lib.ns3d_batch_last_error.argtypes = [h]
    lib.ns3d_batch_set_interior_primitives.argtypes = [h, C.c_int, C.POINTER(dp)]
    lib.ns3d_batch_run.argtypes = [h, C.c_int]
    lib.ns3d_batch_autotune.argtypes = [h, C.c_int, C.POINTER(C.c_int)]
    lib.ns3d_batch_set_config.argtypes = [h, C.c_int, C.c_int, C.c_int]
    lib.ns3d_batch_query.argtypes = [h, C.c_int, dp, C.POINTER(C.c_int), C.POINTER(C.c_int)]
    lib.ns3d_batch_download.argtypes = [h, C.c_int, C.POINTER(dp)]
    lib.ns3d_debug_face_vjp.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, dp, dp, dp, dp, dp]
    lib.ns3d_debug_visc_vjp.argtypes = [C.c_double, C.c_double, C.c_double, dp, dp, dp, dp, dp, dp]
    lib.ns3d_debug_riemann.argtypes = [C.c_int, C.c_int, C.c_double, dp, dp, dp]
    lib.ns3d_debug_wait_timeout.argtypes = [C.c_int, C.c_uint, C.POINTER(C.c_int)]
    lib.ns3d_debug_mdcd_detector.argtypes = [C.c_int, C.c_long, dp, C.POINTER(C.c_int)]
    lib.ns3d_compute_timestep_noalloc.argtypes = [C.POINTER(C.c_void_p), C.c_int, C.c_int, C.c_int, C.c_double,
                                                  C.c_double, C.c_double, C.c_void_p, C.c_void_p]
    _lib = lib
    return lib
