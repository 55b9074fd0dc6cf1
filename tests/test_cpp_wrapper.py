"""The header-only C++ layer (include/kp_transport.hpp), compiled with g++
against the shared library like a reference build would: host-only parts on
CPU, a small forward solve on the GPU."""
import os
import shutil
import subprocess

import pytest

from meshcases import AMR_BOX

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "kratos_polrad_b200")
SRC = os.path.join(ROOT, "tests", "cpp", "wrapper_check.cpp")

pytestmark = pytest.mark.skipif(
    shutil.which("g++") is None or not os.path.exists(os.path.join(LIBDIR, "libkp_b200.so")),
    reason="g++ or the library missing")


@pytest.fixture(scope="module")
def program(tmp_path_factory):
    d = tmp_path_factory.mktemp("cpp")
    exe = d / "wrapper_check"
    subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                    SRC, "-L", LIBDIR, "-lkp_b200", f"-Wl,-rpath,{LIBDIR}", "-o", str(exe)],
                   check=True)
    ini = d / "mesh.ini"
    ini.write_text(AMR_BOX.to_ini())
    return str(exe), str(ini)


def test_host_parts(program):
    exe, ini = program
    r = subprocess.run([exe, "host", ini], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.count("OK ") == 6, r.stdout


@pytest.mark.gpu
def test_gpu_forward(program):
    exe, ini = program
    r = subprocess.run([exe, "gpu", ini], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "OK forward emitted=20000" in r.stdout and r.stdout.count("OK ") == 2, r.stdout
