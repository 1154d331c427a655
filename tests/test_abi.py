"""The C-ABI library loads and exports every entry point declared in include/*.h
(CPU only: no compute call is made)."""
import ctypes
import glob
import os
import re

import pytest

import emergence_b200 as E
from emergence_b200 import _abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"\b(emg_[a-z0-9_]+)\s*\(", src):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_the_uniform_api():
    names = declared_functions()
    for required in ("emg_uniform_create", "emg_uniform_step", "emg_uniform_dt_cfl", "emg_uniform_run_to",
                     "emg_uniform_download", "emg_uniform_totals", "emg_uniform_counters", "emg_uniform_destroy",
                     "emg_last_error"):
        assert required in names


def test_library_exports_every_declared_symbol():
    assert os.path.exists(_abi.LIB_PATH), "build the library first (python -m emergence_b200.build)"
    lib = ctypes.CDLL(_abi.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_bindings_cover_every_declared_symbol():
    missing = [n for n in declared_functions() if n not in _abi.SIGNATURES]
    assert not missing, missing


def test_version_and_error_strings_without_a_gpu():
    lib = _abi.lib()
    assert lib.emg_version().decode().count(".") == 2
    # invalid arguments are rejected before any device work
    h = ctypes.c_void_p()
    rc = lib.emg_uniform_create(None, None, None, None, None, 0, ctypes.byref(h))
    assert rc == 1 and b"null" in lib.emg_last_error()


def test_struct_layouts_match_the_header():
    assert ctypes.sizeof(_abi.EmgEos) == 40
    assert ctypes.sizeof(_abi.EmgMesh) == 80
    assert ctypes.sizeof(_abi.EmgBc) == 48
    assert ctypes.sizeof(_abi.EmgOpts) == 32
