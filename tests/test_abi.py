"""The C ABI library loads and exports every symbol include/e3d.h declares (CPU only)."""
import os
import re
import subprocess

from conftest import REPO

from euler3d_b200 import _lib


def header_functions():
    src = open(os.path.join(REPO, "include", "e3d.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(e3d_[a-z0-9_]+)\s*\(", src)))


def test_library_loads_and_exports_header():
    lib = _lib.lib()
    declared = header_functions()
    assert len(declared) >= 30
    for name in declared:
        assert hasattr(lib, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (e3d_\w+)", out))
    assert set(declared) <= exported
    # the Python binding covers the whole header
    assert set(declared) == set(_lib.SIGNATURES)


def test_version_and_error_text():
    lib = _lib.lib()
    assert b"sm_100a" in lib.e3d_version()
    import ctypes

    h = ctypes.c_void_p()
    rc = lib.e3d_case_load(b"/nonexistent/deck", None, ctypes.byref(h))
    assert rc == -2
    assert b"nonexistent" in lib.e3d_last_error()


def test_precision_constants_match_the_header():
    src = open(os.path.join(REPO, "include", "e3d.h")).read()
    for name, value in (("E3D_FP64", _lib.FP64), ("E3D_FP32", _lib.FP32), ("E3D_FP64_FMA", _lib.FP64_FMA),
                        ("E3D_FP32_DELTA", _lib.FP32_DELTA)):
        m = re.search(rf"#define {name} (\d+)", src)
        assert m and int(m.group(1)) == value, name
    lib = _lib.lib()
    assert lib.e3d_solver_set_precision(None, _lib.FP32_DELTA) == -1  # null solver: an error, not a crash
    assert b"null solver" in lib.e3d_last_error()
    assert lib.e3d_solver_set_precision(None, 7) == -1
