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
