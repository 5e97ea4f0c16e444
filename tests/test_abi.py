"""The C-ABI library loads and exports every symbol include/physgpu.h declares
(no compute calls: runs without a GPU)."""
import ctypes
import os
import re

import physgpu

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(REPO, "include", "physgpu.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(phys_[a-z0-9_]+)\s*\(", src)))


def test_header_and_binding_agree():
    assert declared_symbols() == sorted(physgpu.EXPORTED)


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(physgpu.LIB_PATH)
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_status_strings_without_device():
    lib = physgpu.load_library()
    assert lib.phys_status_string(0) == b"ok"
    assert lib.phys_status_string(physgpu.ERR_NONFINITE) == b"non-finite value"


def test_params_layout():
    assert ctypes.sizeof(physgpu.Params) == 40
    assert ctypes.sizeof(physgpu.Timings) == 88
