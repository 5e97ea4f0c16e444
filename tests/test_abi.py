"""The C-ABI library loads and exports every symbol include/physgpu.h declares
(no compute calls: runs without a GPU)."""
import ctypes
import os
import re

import pytest

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


def test_params_layout(tmp_path):
    """The ctypes mirrors match include/physgpu.h field by field (offsets
    printed by a C program compiled against the header)."""
    import os
    import shutil
    import subprocess
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    inc = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include")
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "physgpu.h"', "int main(void) {"]
    for cname, cls in (("phys_params", physgpu.Params), ("phys_timings", physgpu.Timings)):
        lines.append('printf("%s size %%zu\\n", sizeof(%s));' % (cname, cname))
        for f, _ in cls._fields_:
            lines.append('printf("%s %s %%zu\\n", offsetof(%s, %s));' % (cname, f, cname, f))
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run([cc, "-I", inc, str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {tuple(l.split()[:2]): int(l.split()[2]) for l in out if l.strip()}
    for cname, cls in (("phys_params", physgpu.Params), ("phys_timings", physgpu.Timings)):
        assert got[(cname, "size")] == ctypes.sizeof(cls)
        for f, _ in cls._fields_:
            assert got[(cname, f)] == getattr(cls, f).offset, (cname, f)
