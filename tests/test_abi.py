"""The C-ABI library loads without a GPU and exports every declared symbol."""
import os
import re

import pytest

from specfwat_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    inc = os.path.join(ROOT, "include")
    for fn in os.listdir(inc):
        if fn.endswith(".h"):
            text = open(os.path.join(inc, fn)).read()
            text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
            names |= set(re.findall(r"\b(sem_\w+)\s*\(", text))
    return names


def test_header_declares_entry_points():
    names = declared_symbols()
    assert {"sem_prepare_mesh", "sem_prepare_timerun", "sem_iterate_time",
            "sem_save_adjoint_kernels", "sem_measure_l2_noalloc"} <= names


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    for n in sorted(declared_symbols()):
        assert hasattr(lib, n), n
    assert set(_lib.EXPORTS) == declared_symbols()


def test_abi_version():
    assert _lib.load().sem_abi_version() == 2


def test_no_device_is_reported_not_crashed():
    lib = _lib.load()
    rc = lib.sem_device_info(None, None, None, None)
    if rc == 0:
        pytest.skip("a GPU is present")
    assert rc == -7
    assert b"CUDA" in lib.sem_last_error() or b"device" in lib.sem_last_error()


def test_argument_errors_without_device():
    """Pure host-side validation paths return SEM_ERR_ARG, not a crash."""
    import ctypes as C
    lib = _lib.load()
    assert lib.sem_prepare_mesh(None, None) == -1
    desc = _lib.MeshDesc()
    h = C.c_void_p()
    desc.nspec = 0
    assert lib.sem_prepare_mesh(C.byref(desc), C.byref(h)) == -1
    assert b"nspec" in lib.sem_last_error()
    assert lib.sem_iterate_time(None, 1, 0) == -1
    assert lib.sem_measure_l2_noalloc(None, None, 1, 1, 0.1, 0.0, 1, None,
                                      None, None) == -1


def test_entry_points_take_their_python_arguments():
    """Every entry point the Python layer calls with a raw array address or a
    ctypes reference accepts it (argument conversion happens before the
    call, so a null handle shows it without a device): each returns
    SEM_ERR_ARG for the null run instead of raising."""
    import ctypes as C
    import numpy as np
    L = _lib.load()
    f64 = np.zeros(4)
    f32 = np.zeros(4, np.float32)
    t = C.c_longlong()
    ms = C.c_double()
    i1, i2, i3 = C.c_int(), C.c_int(), C.c_int()
    b1, b2 = C.c_longlong(), C.c_longlong()
    calls = [
        lambda: L.sem_lane_misfit(None, 0, f64.ctypes.data),
        lambda: L.sem_lane_finish_async(None, 0, f32.ctypes.data, f64.ctypes.data, None),
        lambda: L.sem_lane_ready(None, 0, 0),
        lambda: L.sem_mark(None, C.byref(t)),
        lambda: L.sem_mark_done(None, 0, 0),
        lambda: L.sem_mark_elapsed(None, 0, 1, C.byref(ms)),
        lambda: L.sem_set_store_spill(None, -1),
        lambda: L.sem_store_info(None, C.byref(i1), C.byref(i2), C.byref(i3), C.byref(b1),
                                 C.byref(b2)),
        lambda: L.sem_lane_finish(None, 0, f32.ctypes.data, f64.ctypes.data, None),
        lambda: L.sem_lane_status(None, 0, C.byref(i1), C.byref(i2), C.byref(i3)),
    ]
    desc = _lib.GridDesc((C.c_double * 3)(0.0, 0.0, 0.0), (C.c_double * 3)(1.0, 1.0, 1.0),
                         (C.c_int * 3)(2, 2, 2), 8)
    bad = _lib.GridDesc((C.c_double * 3)(0.0, 0.0, 0.0), (C.c_double * 3)(0.0, 1.0, 1.0),
                        (C.c_int * 3)(2, 2, 2), 8)
    tap = _lib.GridTaperCfg(1.0, 1.0, 1.0, 1.0)
    z = np.zeros(2)
    calls += [
        lambda: L.sem_grid_project(None, C.byref(desc), 1, f32.ctypes.data, f32.ctypes.data),
        lambda: L.sem_grid_taper(None, C.byref(desc), C.byref(tap), 1, f32.ctypes.data, None),
        lambda: L.sem_grid_zprecond(C.byref(desc), z.ctypes.data, 1, 1, f32.ctypes.data),
        lambda: L.sem_grid_zprecond(C.byref(desc), z.ctypes.data, 2, 0, f32.ctypes.data),
        lambda: L.sem_grid_zprecond(C.byref(bad), z.ctypes.data, 2, 1, f32.ctypes.data),
    ]
    for k, call in enumerate(calls):
        assert call() == -1, k
