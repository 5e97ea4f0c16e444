"""The C++ host layer (phys-rs_b200/host/physgpu.hpp): builds here; its port
of the reference's known-answer tests runs on the GPU."""
import os
import subprocess

import pytest

import oracle

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(REPO, "tests", "cpp", "test_host_systems.cpp")
OUT = os.path.join(REPO, "phys-rs_b200", "_build", "test_host_systems")
LIBDIR = os.path.join(REPO, "phys-rs_b200", "lib")


def build():
    oracle.build()
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    cmd = ["g++", "-O2", "-std=c++17", "-Wall", "-Wextra", SRC, "-o", OUT,
           "-L" + LIBDIR, "-lphysgpu", "-Wl,-rpath," + LIBDIR,
           "-L" + os.path.join(REPO, "oracle"), "-l:liboracle.so",
           "-Wl,-rpath," + os.path.join(REPO, "oracle")]
    subprocess.run(cmd, check=True)
    return OUT


def test_host_layer_builds():
    assert os.path.exists(build())


@pytest.mark.gpu
def test_host_layer_reference_kats_on_gpu():
    exe = build()
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.strip().endswith("ok (0 failures)")
