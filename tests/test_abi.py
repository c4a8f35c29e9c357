"""The C ABI surface, checked without a GPU: the in-tree library loads, exports
every function include/*.h declares, and fails cleanly without a device."""
import ctypes
import glob
import os
import re

import pytest

from tests.conftest import ROOT


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names |= set(re.findall(r"\b(ghost_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


def exported_symbols(path):
    import subprocess
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True, check=True).stdout
    return {line.split()[-1] for line in out.splitlines() if " T " in line}


def test_library_exports_every_declared_function():
    import ghost_b200
    from ghost_b200 import _lib
    lib = _lib.load()
    names = declared_functions()
    assert len(names) >= 30
    syms = exported_symbols(_lib.LIB_PATH)
    missing = [n for n in names if n not in syms]
    assert not missing, missing
    for n in names:
        getattr(lib, n)  # resolvable through ctypes
    assert set(_lib.SIGNATURES) <= set(names)


def test_errors_are_status_codes_not_exits():
    import torch
    if torch.cuda.is_available():
        pytest.skip("device present: covered by the gpu tests")
    from ghost_b200 import _lib
    lib = _lib.load()
    h = ctypes.c_void_p()
    assert lib.ghost_ctx_create(64, 64, 64, 1, 1, 1, 0, 8, ctypes.byref(h)) == 8  # GHOST_ERR_NODEV
    assert b"device" in lib.ghost_last_error_string()
    # argument validation comes before any device work
    assert lib.ghost_ctx_create(48, 64, 64, 1, 1, 1, 0, 8, ctypes.byref(h)) == 2  # size
    assert lib.ghost_ctx_create(64, 64, 64, 1, 1, 1, 0, 3, ctypes.byref(h)) == 1  # precision
    assert lib.ghost_derivk3(None, None, None, 1) == 1
    assert lib.ghost_fftp3d_destroy_plan(None) == 0


def test_python_mirror_raises_without_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("device present")
    from ghost_b200 import Ghost, GhostError
    with pytest.raises(GhostError):
        Ghost(32)


def test_fortran_binding_names_every_entry_point():
    text = open(os.path.join(ROOT, "ghost_b200", "fortran", "ghost_gpu.f90")).read()
    bound = set(re.findall(r'BIND\(C,\s*name="(ghost_[a-z0-9_]+)"\)', text))
    missing = [n for n in declared_functions() if n not in bound]
    assert not missing, missing
