"""Binary container of the reference's binary_io: byte-identical writer,
reader of both reference writers, solution save/load and restart (CPU)."""
import dataclasses
import os
import sys
import types

import numpy as np
import pytest

from kratos_polrad_b200 import KPError, Mesh, bio
from meshcases import AMR_BOX
from oracle import port, refharness

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
sys.path.insert(0, GOLDEN)
from make_golden import bio_entries  # noqa: E402

has_ref = pytest.mark.skipif(not refharness.available(2), reason="oracle/_ref not built")


def test_writer_reproduces_reference_file(tmp_path):
    """Same entries -> the bytes binary_io::base_t::save wrote (golden)."""
    p = tmp_path / "o.bin"
    bio.write(str(p), bio_entries())
    assert p.read_bytes() == open(os.path.join(GOLDEN, "bio_reference.bin"), "rb").read()


@pytest.mark.parametrize("name", ["bio_reference.bin", "bio_reference_py.bin"])
def test_reader_reads_reference_files(name):
    with bio.BinaryFile(os.path.join(GOLDEN, name)) as f:
        ent = dict(bio_entries())
        assert sorted(f.tags) == sorted(ent)
        for tag, a in ent.items():
            assert f.hmap[tag] == (a.nbytes, a.dtype.itemsize)
            np.testing.assert_array_equal(f.read(tag, a.dtype), a)
        assert f.as_array("alpha", "f").dtype == np.dtype("<f4")


@has_ref
def test_writer_matches_reference_live(tmp_path):
    rng = np.random.default_rng(3)
    ent = [(f"t{rng.integers(1000)}|{k}", rng.random(rng.integers(1, 50)).astype(dt))
           for k, dt in enumerate([np.float32, np.float64, np.int8, np.int16, np.uint64] * 4)]
    a, b = tmp_path / "ref.bin", tmp_path / "ours.bin"
    refharness.bio_write(str(a), ent)
    bio.write(str(b), ent)
    assert a.read_bytes() == b.read_bytes()
    for tag, arr in ent:                        # and the reference reads ours
        data, unit = refharness.bio_read(str(b), tag)
        assert unit == arr.dtype.itemsize and data == arr.tobytes()


def test_repeated_tag_keeps_last_and_errors(tmp_path):
    p = str(tmp_path / "x.bin")
    bio.write(p, [("a", np.int32([1])), ("a", np.int32([7, 8]))])
    with bio.BinaryFile(p) as f:
        np.testing.assert_array_equal(f.read("a", np.int32), [7, 8])
        with pytest.raises(KPError, match="cannot find tag"):
            f["b"]
    with pytest.raises(KPError, match="Cannot open file"):
        bio.BinaryFile(str(tmp_path / "missing.bin"))
    (tmp_path / "bad.bin").write_bytes(b"\x05" + b"\x00" * 20)
    with pytest.raises(KPError, match="Inconsistent size_t"):
        bio.BinaryFile(str(tmp_path / "bad.bin"))
    # a truncated file: header promises data the file lacks
    good = open(p, "rb").read()
    (tmp_path / "cut.bin").write_bytes(good[:-3])
    with pytest.raises(KPError, match="beyond the file"):
        bio.BinaryFile(str(tmp_path / "cut.bin"))


def _tallies(out):
    return types.SimpleNamespace(**{k: out[k] for k in ("mu", "image", "image_batch", "counters")})


@pytest.mark.skipif(not port.available(), reason="oracle not built")
def test_save_load_and_restart(tmp_path):
    """Half the packets, save, load, the other half from packets_done: the
    summed int64 tallies equal one run over all packets."""
    from transport_cases import case, run_oracle
    mesh, sig, t = case("amr_point")
    t = dataclasses.replace(t, n_record=0, n_packets=800)
    half = dataclasses.replace(t, n_packets=400)
    first = run_oracle(mesh, sig, half)
    flux = np.random.default_rng(1).random(mesh.n_cells).astype(np.float32)
    grads = (np.arange(mesh.n_cells, dtype=np.float64), -np.arange(mesh.n_cells, dtype=np.float64))
    p = str(tmp_path / "run.bin")
    bio.save_solution(p, mesh, sig, _tallies(first), half, grads=grads, flux=flux)
    s = bio.load_solution(p)
    assert s["packets_done"] == 400 and s["config"]["seed"] == t.seed
    np.testing.assert_array_equal(s["sigma"], sig)
    np.testing.assert_array_equal(s["grad_sca"], grads[0])
    second = run_oracle(mesh, s["sigma"], dataclasses.replace(half, packet_offset=s["packets_done"]))
    full = run_oracle(mesh, sig, t)
    for k in ("mu", "image", "image_batch"):
        np.testing.assert_array_equal(s[k] + second[k], full[k])
    np.testing.assert_array_equal(s["counters"] + second["counters"], full["counters"])
    # per-block tags as block_t::write and rad_t::write name them
    with bio.BinaryFile(p) as f:
        lev, reg = mesh.blocks()
        b = mesh.n_blocks - 1
        np.testing.assert_array_equal(f.as_array(f"block_{b}|i_logic", "i"), reg[b])
        assert f.as_array(f"block_{b}|level", "i")[0] == lev[b]
        cpb = mesh.cells_per_block
        np.testing.assert_array_equal(f.as_array(f"block_{b}|rad_flx_flux_field", "f"),
                                      flux[b * cpb:])
        np.testing.assert_array_equal(f.as_array(f"block_{b}|rad_flx_flux_n_cell", "i"), mesh.nc)


@has_ref
def test_reference_reads_solution_file(tmp_path):
    mesh = Mesh(AMR_BOX)
    flux = np.linspace(0, 1, mesh.n_cells, dtype=np.float32)
    p = str(tmp_path / "s.bin")
    bio.save_solution(p, mesh, flux=flux)
    data, unit = refharness.bio_read(p, "block_3|rad_flx_flux_field")
    cpb = mesh.cells_per_block
    assert unit == 4 and data == flux[3 * cpb:4 * cpb].tobytes()


@pytest.mark.skipif(not port.available(), reason="oracle not built")
def test_flux_tally_restart(tmp_path):
    """The transport's path-length flux tally is saved raw (int64) and as the
    rad_t flux field per block; a restart adds up to one run, bit for bit."""
    from transport_cases import case, oracle_inputs
    mesh, sig, t = case("amr_point")
    t = dataclasses.replace(t, n_record=0, n_packets=600, flux=True, flux_fx_shift=24)
    half = dataclasses.replace(t, n_packets=300)
    tab, grid, gn, cells = oracle_inputs(mesh, t)
    first = port.transport(tab, sig, grid, gn, half, cells, flux=True)
    p = str(tmp_path / "flux.bin")
    tal = types.SimpleNamespace(**{k: first[k] for k in ("mu", "image", "image_batch",
                                                         "counters", "flux")})
    bio.save_solution(p, mesh, sig, tal, half)
    s = bio.load_solution(p)
    second = port.transport(tab, sig, grid, gn, dataclasses.replace(half, packet_offset=300),
                            cells, flux=True)
    full = port.transport(tab, sig, grid, gn, t, cells, flux=True)
    np.testing.assert_array_equal(s["flux"] + second["flux"], full["flux"])
    with bio.BinaryFile(p) as f:
        cpb = mesh.cells_per_block
        b = 7
        np.testing.assert_array_equal(
            f.as_array(f"block_{b}|rad_flx_flux_field", "f"),
            (first["flux"][b * cpb:(b + 1) * cpb] * 2.0 ** -24).astype(np.float32))
