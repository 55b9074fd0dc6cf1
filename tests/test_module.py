"""The radiation module layer (include/kp_module.hpp) with a user generator
(include/kp_generate.cuh), as a user problem would use them.

tests/cpp/module_check.cu reads the reference's [particle] / [device] keys,
enrolls its own __device__ packet generator, runs n_cycle_stp cycles and
saves the run in the reference's container.  On CPU the keys and the
enrolment are checked; on the GPU the saved tallies and flux field must
equal the C restatement's, fed the packets the generator made (read back per
cycle), bit for bit.
"""
import dataclasses
import os
import shutil
import subprocess

import numpy as np
import pytest

from meshcases import AMR_BOX

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "kratos_polrad_b200")
SRC = os.path.join(ROOT, "tests", "cpp", "module_check.cu")
NVCC = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"

pytestmark = pytest.mark.skipif(
    not os.path.exists(NVCC) or not os.path.exists(os.path.join(LIBDIR, "libkp_b200.so")),
    reason="nvcc or the library missing")

PARTICLE = """
[particle]
n_par = 1500
step_max = 100000
n_hv = 2
n_cycle_stp = 2
n_th = 128
f_par = 0.5

[device]
seed_rng = 11
"""


@pytest.fixture(scope="module")
def program(tmp_path_factory):
    d = tmp_path_factory.mktemp("module")
    exe = d / "module_check"
    subprocess.run([NVCC, "-std=c++17", "-O2", "-gencode", "arch=compute_100a,code=sm_100a",
                    "-Xcompiler", "-Wall", "-I", os.path.join(ROOT, "include"), SRC,
                    "-L", LIBDIR, "-lkp_b200", f"-Xlinker=-rpath,{LIBDIR}", "-o", str(exe)],
                   check=True)
    ini = d / "problem.ini"
    ini.write_text(AMR_BOX.to_ini() + PARTICLE)
    return str(exe), str(ini), d


def test_module_reads_keys_and_enrolls(program):
    exe, ini, _ = program
    r = subprocess.run([exe, "host", ini], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert ("OK keys n_par=1500 step_max=100000 n_hv=2 n_cycle_stp=2 n_th=128 f_par=0.5 "
            "seed_rng=11 output=1 max_round=16") in r.stdout, r.stdout
    assert "OK enrolled" in r.stdout


def test_module_defaults_without_keys(program, tmp_path):
    """Keys left out take the reference's defaults (generate_par.h:36-41,
    radiation.h:26, driver.cpp:18, device.cpp:69)."""
    exe, _, _ = program
    ini = tmp_path / "bare.ini"
    ini.write_text(AMR_BOX.to_ini())
    r = subprocess.run([exe, "host", str(ini)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert ("OK keys n_par=1 step_max=100 n_hv=1 n_cycle_stp=1 n_th=64 f_par=1 seed_rng=7 "
            "output=1 max_round=16") in r.stdout, r.stdout


@pytest.mark.gpu
def test_module_run_matches_restatement(program):
    from kratos_polrad_b200 import Mesh, bio
    from kratos_polrad_b200.transport import PACKET_INIT_DTYPE, TransportConfig
    from oracle import port
    from transport_cases import cell_centers, oracle_inputs
    exe, ini, d = program
    mesh = Mesh(AMR_BOX)
    c = cell_centers(mesh)
    rng = np.random.default_rng(12)
    ext = 1.5 + 5.0 * np.exp(-((c - 0.5) ** 2).sum(1) / (2 * 0.1 ** 2))
    alb = rng.uniform(0.6, 0.97, mesh.n_cells)
    sig = np.stack([ext * alb, ext * (1 - alb)], 1).astype(np.float32)
    sig.tofile(d / "sigma.bin")
    r = subprocess.run([exe, "gpu", ini, str(d)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "OK module packets_done=3000 pool=0" in r.stdout, r.stdout
    tables = np.fromfile(d / "tables.bin", PACKET_INIT_DTYPE).reshape(2, 1500)
    assert (tables["w"] >= 0.5).all()
    assert np.allclose(np.linalg.norm(tables["d"], axis=-1), 1, atol=1e-6)
    # the same run restated: the keys and settings of module_check.cu
    cfg = TransportConfig(n_packets=1500, sources=[], seed=11, max_steps=100000, image_n=32,
                          inclination_deg=60.0, image_center=(0.5, 0.5, 0.5),
                          image_half_width=0.87, image_batch_n=4, n_mu_bins=8, mu_lo=-1.0,
                          mu_hi=1.0, w_min=0.05, fx_shift=32, flux_fx_shift=24, flux=True)
    tab, grid, gn, cells = oracle_inputs(mesh, cfg)
    want = None
    for cyc in range(2):
        cc = dataclasses.replace(cfg, packet_offset=1500 * cyc, packets=tables[cyc])
        o = port.transport(tab, sig, grid, gn, cc, cells, flux=True)
        want = o if want is None else {k: want[k] + o[k] for k in
                                       ("mu", "image", "image_batch", "counters", "flux")}
    got = bio.load_solution(str(d / "run.bin"))
    assert got["packets_done"] == 3000
    for k in ("mu", "image", "image_batch", "flux"):
        np.testing.assert_array_equal(got[k].astype(np.int64), want[k], err_msg=k)
    np.testing.assert_array_equal(got["counters"].astype(np.int64),
                                  want["counters"].astype(np.int64))
    # the rad_t flux field per block: n_hv components, the tally in the first
    with bio.BinaryFile(str(d / "run.bin")) as f:
        cpb = mesh.cells_per_block
        for b in (0, mesh.n_blocks - 1):
            assert f.as_array(f"block_{b}|rad_flx_flux_n_int", "i")[0] == 2
            fld = f.as_array(f"block_{b}|rad_flx_flux_field", "f").reshape(cpb, 2)
            np.testing.assert_array_equal(
                fld[:, 0], (want["flux"][b * cpb:(b + 1) * cpb] * 2.0 ** -24).astype(np.float32))
            assert (fld[:, 1] == 0).all()


@pytest.mark.gpu
def test_module_keep_pool_matches_restatement(program):
    """comm_mode() keep_pool: with step_max = 25 most packets outlive their
    cycle, wait in the pool and go on in the next; drained after the cycles,
    the run equals the restatement of the same packets walked to the end
    (at most 100000 segments), bit for bit."""
    from kratos_polrad_b200 import Mesh, bio
    from kratos_polrad_b200.transport import PACKET_INIT_DTYPE, TransportConfig
    from oracle import port
    from transport_cases import cell_centers, oracle_inputs
    exe, _, d = program
    ini = d / "pool.ini"
    ini.write_text(AMR_BOX.to_ini() + PARTICLE.replace("step_max = 100000", "step_max = 25"))
    mesh = Mesh(AMR_BOX)
    c = cell_centers(mesh)
    rng = np.random.default_rng(12)
    ext = 1.5 + 5.0 * np.exp(-((c - 0.5) ** 2).sum(1) / (2 * 0.1 ** 2))
    alb = rng.uniform(0.6, 0.97, mesh.n_cells)
    sig = np.stack([ext * alb, ext * (1 - alb)], 1).astype(np.float32)
    sig.tofile(d / "sigma.bin")
    r = subprocess.run([exe, "pool", str(ini), str(d)], capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "OK module packets_done=3000 pool=0" in r.stdout, r.stdout
    kept = [int(line.split()[-2]) for line in r.stdout.splitlines()
            if line.startswith("OK pool after cycle")]
    assert len(kept) == 2 and min(kept) > 100, r.stdout
    tables = np.fromfile(d / "tables_pool.bin", PACKET_INIT_DTYPE).reshape(2, 1500)
    cfg = TransportConfig(n_packets=1500, sources=[], seed=11, max_steps=100000, image_n=32,
                          inclination_deg=60.0, image_center=(0.5, 0.5, 0.5),
                          image_half_width=0.87, image_batch_n=4, n_mu_bins=8, mu_lo=-1.0,
                          mu_hi=1.0, w_min=0.05, fx_shift=32, flux_fx_shift=24, flux=True)
    tab, grid, gn, cells = oracle_inputs(mesh, cfg)
    want = None
    for cyc in range(2):
        cc = dataclasses.replace(cfg, packet_offset=1500 * cyc, packets=tables[cyc])
        o = port.transport(tab, sig, grid, gn, cc, cells, flux=True)
        want = o if want is None else {k: want[k] + o[k] for k in
                                       ("mu", "image", "image_batch", "counters", "flux")}
    got = bio.load_solution(str(d / "run_pool.bin"))
    for k in ("mu", "image", "image_batch", "flux"):
        np.testing.assert_array_equal(got[k].astype(np.int64), want[k], err_msg=k)
    np.testing.assert_array_equal(got["counters"].astype(np.int64),
                                  want["counters"].astype(np.int64))
