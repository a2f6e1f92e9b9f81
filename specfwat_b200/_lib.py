"""ctypes binding of ``libsem_b200.so`` (declarations in include/sem_b200.h).

The library is the product: there is no CPU fallback.  Loading fails with a
clear error when the in-tree library has not been built.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsem_b200.so")

SEM_OK = 0
SEM_ERR_NUMERIC = -6
STATUS = {
    0: "SEM_OK", -1: "SEM_ERR_ARG", -2: "SEM_ERR_CUDA", -3: "SEM_ERR_NOMEM",
    -4: "SEM_ERR_STATE", -5: "SEM_ERR_UNSUPPORTED", -6: "SEM_ERR_NUMERIC",
    -7: "SEM_ERR_NODEVICE",
}
SEM_STORE_FP32 = 0
SEM_STORE_FP16 = 1

# every entry point include/sem_b200.h declares
EXPORTS = (
    "sem_abi_version", "sem_last_error", "sem_device_info",
    "sem_prepare_mesh", "sem_release_mesh", "sem_mesh_info",
    "sem_prepare_timerun", "sem_release_run", "sem_run_bytes",
    "sem_set_sources", "sem_set_receivers", "sem_iterate_time",
    "sem_synchronize", "sem_get_seismograms", "sem_set_adjoint_sources",
    "sem_measure_l2", "sem_save_adjoint_kernels", "sem_sum_kernels",
    "sem_last_loop_ms", "sem_last_launch_count", "sem_set_observed",
    "sem_set_stream", "sem_sum_kernels_device", "sem_time_kernels",
    "sem_kernel_variants", "sem_measure_l2_noalloc",
    "sem_set_store_spill", "sem_store_info", "sem_mark", "sem_mark_done",
    "sem_mark_elapsed", "sem_lane_finish_async", "sem_lane_ready", "sem_lane_misfit",
    "sem_lane_move", "sem_set_sm_share",
    "sem_lane_store_bytes", "sem_lane_start_forward", "sem_lane_start_adjoint",
    "sem_advance", "sem_lane_status", "sem_lane_finish", "sem_fp32_fma_peak",
    "sem_smooth_pde", "sem_measure_waveform", "sem_measure_waveform_dev",
    "sem_set_approximate_hessian", "sem_save_hessian_kernel", "sem_sum_hessian",
    "sem_hessian_precond", "sem_depth_precond", "sem_set_injection",
    "sem_grid_project", "sem_grid_taper", "sem_grid_zprecond",
)
MEAS_MAX_BANDS = 4
SMOOTH_MAP_CUBE = 0
SMOOTH_MAP_REFERENCE = 1
L2_NOALLOC_MAX_RECEIVERS = 4096
L2_NOALLOC_MAX_STEPS = 32768


class SemError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{STATUS.get(code, code)}: {msg}")
        self.code = code


class MeshDesc(C.Structure):
    _fields_ = [
        ("nspec", C.c_int), ("nglob", C.c_int), ("index_base", C.c_int),
        ("ibool", C.POINTER(C.c_int)),
        ("xstore", C.POINTER(C.c_float)), ("ystore", C.POINTER(C.c_float)),
        ("zstore", C.POINTER(C.c_float)),
        ("xix_regular", C.c_float), ("jacobian_regular", C.c_float),
        ("irregular_element_number", C.POINTER(C.c_int)),
        ("kappastore", C.POINTER(C.c_float)), ("mustore", C.POINTER(C.c_float)),
        ("rhostore", C.POINTER(C.c_float)), ("rmass", C.POINTER(C.c_float)),
        ("rho_vp", C.POINTER(C.c_float)), ("rho_vs", C.POINTER(C.c_float)),
        ("num_abs_boundary_faces", C.c_int),
        ("abs_boundary_ispec", C.POINTER(C.c_int)),
        ("abs_boundary_ijk", C.POINTER(C.c_int)),
        ("abs_boundary_jacobian2Dw", C.POINTER(C.c_float)),
        ("abs_boundary_normal", C.POINTER(C.c_float)),
        ("nspec_irregular", C.c_int),
        ("xixstore", C.POINTER(C.c_float)), ("xiystore", C.POINTER(C.c_float)),
        ("xizstore", C.POINTER(C.c_float)), ("etaxstore", C.POINTER(C.c_float)),
        ("etaystore", C.POINTER(C.c_float)), ("etazstore", C.POINTER(C.c_float)),
        ("gammaxstore", C.POINTER(C.c_float)), ("gammaystore", C.POINTER(C.c_float)),
        ("gammazstore", C.POINTER(C.c_float)), ("jacobianstore", C.POINTER(C.c_float)),
    ]


class RunCfg(C.Structure):
    _fields_ = [("nev", C.c_int), ("nstep", C.c_int), ("dt", C.c_double),
                ("store_kind", C.c_int), ("use_graph", C.c_int),
                ("graph_steps", C.c_int), ("max_receivers", C.c_int),
                ("check_every", C.c_int), ("kernel_variant", C.c_int)]


class Source(C.Structure):
    _fields_ = [("x", C.c_double), ("y", C.c_double), ("z", C.c_double),
                ("Mrr", C.c_double), ("Mtt", C.c_double), ("Mpp", C.c_double),
                ("Mrt", C.c_double), ("Mrp", C.c_double), ("Mtp", C.c_double),
                ("f0", C.c_double), ("tshift", C.c_double)]


class MeasCfg(C.Structure):
    _fields_ = [("t0", C.c_double), ("obs_tbeg", C.c_double),
                ("obs_dt", C.c_double), ("obs_npts", C.c_int),
                ("nband", C.c_int), ("short_p", C.c_double * 4),
                ("long_p", C.c_double * 4), ("order", C.c_int),
                ("passes", C.c_int), ("pre_taper", C.c_double),
                ("win_taper", C.c_double), ("win_taper_type", C.c_int),
                ("weight", C.c_double), ("rotate", C.c_int),
                ("adj_norm", C.c_int)]


class SmoothCfg(C.Structure):
    _fields_ = [("sigma_h", C.c_double), ("sigma_v", C.c_double),
                ("distance_min", C.c_double), ("is_sph", C.c_int),
                ("mapping", C.c_int), ("nstep", C.c_int)]


class SmoothStats(C.Structure):
    _fields_ = [("nstep", C.c_int), ("fields_per_pass", C.c_int),
                ("cv", C.c_double), ("ch", C.c_double),
                ("distance_min", C.c_double), ("step_ms", C.c_double)]


class GridDesc(C.Structure):
    _fields_ = [("x0", C.c_double * 3), ("h", C.c_double * 3), ("n", C.c_int * 3),
                ("ngnod", C.c_int)]


class GridTaperCfg(C.Structure):
    _fields_ = [("h_suppress", C.c_double), ("h_buffer", C.c_double),
                ("v_suppress", C.c_double), ("v_buffer", C.c_double)]


_lib = None


def load():
    """Load the in-tree library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python -m specfwat_b200.build`"
            " (the CUDA solver has no CPU fallback)")
    L = C.CDLL(LIB_PATH)
    vp, ip, dp, fp = C.c_void_p, C.c_int, C.c_double, C.c_void_p
    sig = {
        "sem_abi_version": (C.c_int, []),
        "sem_last_error": (C.c_char_p, []),
        "sem_device_info": (C.c_int, [C.POINTER(C.c_int), C.POINTER(C.c_longlong),
                                      C.POINTER(C.c_int), C.POINTER(C.c_int)]),
        "sem_prepare_mesh": (C.c_int, [C.POINTER(MeshDesc), C.POINTER(vp)]),
        "sem_release_mesh": (C.c_int, [vp]),
        "sem_mesh_info": (C.c_int, [vp, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                    C.POINTER(C.c_int), C.POINTER(C.c_longlong)]),
        "sem_prepare_timerun": (C.c_int, [vp, C.POINTER(RunCfg), C.POINTER(vp)]),
        "sem_release_run": (C.c_int, [vp]),
        "sem_run_bytes": (C.c_longlong, [vp, C.POINTER(RunCfg)]),
        "sem_set_sources": (C.c_int, [vp, ip, C.POINTER(Source)]),
        "sem_set_receivers": (C.c_int, [vp, ip, ip, fp]),
        "sem_iterate_time": (C.c_int, [vp, ip, ip]),
        "sem_synchronize": (C.c_int, [vp]),
        "sem_get_seismograms": (C.c_int, [vp, ip, fp]),
        "sem_set_adjoint_sources": (C.c_int, [vp, ip, fp]),
        "sem_measure_l2": (C.c_int, [vp, ip, fp, dp, ip, C.POINTER(C.c_double)]),
        "sem_save_adjoint_kernels": (C.c_int, [vp, ip, fp]),
        "sem_sum_kernels": (C.c_int, [vp, fp]),
        "sem_last_loop_ms": (C.c_int, [vp, C.POINTER(C.c_double)]),
        "sem_last_launch_count": (C.c_int, [vp, C.POINTER(C.c_longlong)]),
        "sem_set_observed": (C.c_int, [vp, ip, fp]),
        "sem_set_stream": (C.c_int, [vp, vp]),
        "sem_sum_kernels_device": (C.c_int, [vp, vp]),
        "sem_time_kernels": (C.c_int, [vp, ip, ip, C.POINTER(C.c_double)]),
        "sem_kernel_variants": (C.c_int, [vp, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
        "sem_measure_l2_noalloc": (C.c_int, [vp, vp, ip, ip, dp, dp, ip, vp, vp, vp]),
        "sem_lane_store_bytes": (C.c_longlong, [vp, ip]),
        "sem_lane_start_forward": (C.c_int, [vp, ip, C.POINTER(Source), ip, fp, ip, ip]),
        "sem_lane_start_adjoint": (C.c_int, [vp, ip, fp, dp, ip, C.POINTER(C.c_double)]),
        "sem_advance": (C.c_int, [vp, ip]),
        "sem_lane_status": (C.c_int, [vp, ip, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                      C.POINTER(C.c_int)]),
        "sem_lane_finish": (C.c_int, [vp, ip, fp, fp, fp]),
        "sem_fp32_fma_peak": (C.c_int, [C.POINTER(C.c_double), C.POINTER(C.c_double)]),
        "sem_smooth_pde": (C.c_int, [vp, C.POINTER(SmoothCfg), ip, fp, fp, fp,
                                     C.POINTER(SmoothStats)]),
        "sem_measure_waveform": (C.c_int, [vp, ip, C.POINTER(MeasCfg), fp, fp, fp,
                                           fp, fp]),
        "sem_measure_waveform_dev": (C.c_int, [vp, ip, ip, dp, C.POINTER(MeasCfg), vp,
                                               vp, vp, vp, vp, vp]),
        "sem_set_approximate_hessian": (C.c_int, [vp, ip]),
        "sem_save_hessian_kernel": (C.c_int, [vp, ip, fp]),
        "sem_sum_hessian": (C.c_int, [vp, ip, fp]),
        "sem_hessian_precond": (C.c_int, [fp, C.c_longlong, ip, fp]),
        "sem_depth_precond": (C.c_int, [vp, fp, ip, ip, ip, fp]),
        "sem_set_injection": (C.c_int, [vp, ip, fp, fp, ip, ip, ip]),
        "sem_set_store_spill": (C.c_int, [vp, C.c_longlong]),
        "sem_mark": (C.c_int, [vp, C.POINTER(C.c_longlong)]),
        "sem_lane_finish_async": (C.c_int, [vp, ip, fp, fp, fp]),
        "sem_lane_ready": (C.c_int, [vp, ip, ip]),
        "sem_lane_move": (C.c_int, [vp, ip, ip]),
        "sem_set_sm_share": (C.c_int, [vp, ip, ip]),
        "sem_lane_misfit": (C.c_int, [vp, ip, fp]),
        "sem_mark_done": (C.c_int, [vp, C.c_longlong, ip]),
        "sem_mark_elapsed": (C.c_int, [vp, C.c_longlong, C.c_longlong,
                                       C.POINTER(C.c_double)]),
        "sem_grid_project": (C.c_int, [vp, C.POINTER(GridDesc), ip, fp, fp]),
        "sem_grid_taper": (C.c_int, [vp, C.POINTER(GridDesc), C.POINTER(GridTaperCfg), ip,
                                     fp, fp]),
        "sem_grid_zprecond": (C.c_int, [C.POINTER(GridDesc), fp, ip, ip, fp]),
        "sem_store_info": (C.c_int, [vp, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                     C.POINTER(C.c_int), C.POINTER(C.c_longlong),
                                     C.POINTER(C.c_longlong)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def check(rc):
    if rc != SEM_OK:
        msg = load().sem_last_error()
        raise SemError(rc, msg.decode() if msg else "")
    return rc
