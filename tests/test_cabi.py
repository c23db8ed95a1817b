"""The C ABI library: it builds, loads, and exports every declared symbol.

No GPU is touched here (no compute call is made)."""

import os
import re
import subprocess

import pytest

from tests.conftest import ROOT

HEADER = os.path.join(ROOT, "include", "pymatting_b200.h")


def header_functions():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"\b(pmb_[a-z0-9_]+)\s*\(", text)))


def exported():
    from pymatting_b200 import build
    path = build.build()
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True,
                         check=True).stdout
    return {ln.split()[-1] for ln in out.splitlines() if " T pmb_" in ln}


def test_library_loads():
    from pymatting_b200 import _ffi
    lib = _ffi.lib()
    assert lib.pmb_version() == 1
    assert lib.pmb_grid_pitch(1) == 32 and lib.pmb_grid_pitch(33) == 64


def test_header_symbols_are_exported():
    exp = exported()
    missing = [f for f in header_functions() if f not in exp]
    assert not missing, missing


def test_binding_covers_exports():
    from pymatting_b200 import _ffi
    exp = exported()
    assert set(_ffi.exported_symbols()) == exp


def test_header_declares_every_export():
    declared = set(header_functions())
    undeclared = sorted(exported() - declared)
    assert not undeclared, undeclared


def test_bad_arguments_fail_cleanly():
    """Argument checks run on the host and never reach a kernel."""
    import ctypes
    from pymatting_b200 import _ffi
    lib = _ffi.lib()
    h = ctypes.c_void_p()
    one = (ctypes.c_int * 1)(0)
    assert lib.pmb_stencil_create(1, one, one, 0, 2, 1, 1, 0.8, 64, ctypes.byref(h)) == -1
    assert "positive" in _ffi.last_error()
    hw = (ctypes.c_int * 1)(64)
    assert lib.pmb_stencil_create(1, hw, hw, 0, 2, 1, 1, 0.8, 1000, ctypes.byref(h)) == -1
    assert lib.pmb_cf_laplacian_ell(None, None, 4, 4, 1, 1e-7, None, 0.0, None, None, None,
                                    None) == -1
