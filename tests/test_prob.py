"""The user problem entry (include/kp_prob.hpp): prob::run called by the
supplied main with the command line, prob::cmd merging the input files in
order (user/probgen.cpp:8-16, main.cpp:7-13).  Host-only: no GPU."""
import ctypes
import os
import shutil
import subprocess

import pytest

from kratos_polrad_b200 import Mesh, _lib
from meshcases import AMR_BOX

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "kratos_polrad_b200")
SRC = os.path.join(ROOT, "tests", "cpp", "prob_check.cpp")

pytestmark = pytest.mark.skipif(
    shutil.which("g++") is None or not os.path.exists(os.path.join(LIBDIR, "libkp_b200.so")),
    reason="g++ or the library missing")


@pytest.fixture(scope="module")
def program(tmp_path_factory):
    d = tmp_path_factory.mktemp("prob")
    exe = d / "prob_check"
    subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                    SRC, "-L", LIBDIR, "-lkp_b200", f"-Wl,-rpath,{LIBDIR}", "-o", str(exe)],
                   check=True)
    return str(exe), d


def test_later_files_override_earlier(program):
    exe, d = program
    base = d / "base.ini"
    base.write_text(AMR_BOX.to_ini() + "\n[particle]\nn_par = 100\nstep_max = 50\n")
    over = d / "over.ini"
    over.write_text("[particle]\nn_par = 2000   # this file's value wins\n\n[device]\nseed_rng = 5\n")
    r = subprocess.run([exe, str(base), str(over)], capture_output=True, text=True, timeout=60,
                       env=dict(os.environ, TMPDIR=str(d)))
    assert r.returncode == 0, r.stdout + r.stderr
    m = Mesh(AMR_BOX)
    assert (f"OK n_par=2000 step_max=50 seed_rng=5 n_blocks={m.n_blocks} "
            f"max_level={m.max_level} cells={m.n_cells}") in r.stdout, r.stdout
    # one file is read as it is
    r1 = subprocess.run([exe, str(base)], capture_output=True, text=True, timeout=60)
    assert r1.returncode == 0 and "OK n_par=100 step_max=50 seed_rng=7" in r1.stdout, r1.stdout


def test_no_input_file_is_refused(program):
    exe, _ = program
    r = subprocess.run([exe], capture_output=True, text=True, timeout=60)
    assert r.returncode != 0 and "No input file." in r.stderr


def test_merge_reports_a_missing_file(tmp_path):
    paths = (ctypes.c_char_p * 2)(str(tmp_path / "missing.ini").encode(), None)
    st = _lib.lib.kp_ini_merge(1, paths, str(tmp_path / "out.ini").encode())
    assert st == _lib.KP_ERR_CONFIG
    assert b"cannot read the input file" in _lib.lib.kp_last_error()
