"""The C++ drop-in facade (include/ocu/opencurrent.h): it compiles against the C ABI on any
machine, and on a B200 the reference-style test program (tests/cpp/facade_test.cpp) passes."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "facade_test.cpp")
LIBDIR = os.path.join(ROOT, "opencurrent_b200")
OUT = os.path.join(ROOT, "_build", "facade_test")


def build_facade_test():
    gxx = shutil.which("g++") or "/usr/bin/g++"
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    cmd = [gxx, "-std=c++17", "-O1", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), SRC,
           "-L", LIBDIR, "-locu_b200", f"-Wl,-rpath,{LIBDIR}", "-o", OUT]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    return OUT


def test_facade_compiles():
    build_facade_test()
    assert os.path.exists(OUT)


@pytest.mark.gpu
def test_facade_program_passes_on_gpu():
    exe = build_facade_test()
    r = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and "FACADE OK" in r.stdout, r.stdout + r.stderr
