"""Golden fixtures of the reference's own geometric walk (tests/golden/*.npz,
made by tests/golden/make_golden.py from the reference compiled for the
host): the product's block tables, the oracle restatement and the GPU walk
must reproduce them bit for bit, with no reference build present."""
import glob
import os

import numpy as np
import pytest

from kratos_polrad_b200 import Mesh
from oracle import port

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "trace_*.npz")))
IDS = [os.path.basename(p)[6:-4] for p in GOLDEN]


def load(path, tmp_path):
    g = dict(np.load(path))
    ini = tmp_path / "mesh.ini"
    ini.write_text(str(g["ini"]))
    mesh = Mesh(ini_path=str(ini))
    pl, pr = mesh.blocks()
    key = {(int(l), *map(int, r)): i for i, (l, r) in enumerate(zip(pl, pr))}
    perm = np.array([key[(int(l), *map(int, r))] for l, r in zip(g["ref_levels"], g["ref_regions"])])
    return g, mesh, perm                               # perm: reference id -> product id


def dense(g, mesh, perm, name):
    """Sparse fixture flux (reference block order) as a dense product-order array."""
    a = np.zeros(mesh.n_cells, g[name].dtype)
    a[g["flux_idx"]] = g[name]
    cpb = mesh.cells_per_block
    return a.reshape(-1, cpb)[np.argsort(perm)].reshape(-1)


def test_fixtures_present():
    assert len(GOLDEN) >= 5


@pytest.mark.parametrize("path", GOLDEN, ids=IDS)
def test_tables_match_golden(path, tmp_path):
    g, mesh, perm = load(path, tmp_path)
    assert sorted(perm.tolist()) == list(range(mesh.n_blocks))
    xf0, dx0, vol0, pb = mesh.geometry(4 if int(g["precision"]) == 1 else 8)
    np.testing.assert_array_equal(xf0[perm], g["xf0"])
    np.testing.assert_array_equal(dx0[perm], g["dx0"])
    np.testing.assert_array_equal(vol0[perm], g["vol0"])
    np.testing.assert_array_equal(pb[perm], g["phybnd"])
    ids, sh, dl = mesh.neighbors()
    rid = g["nb_ids"]
    np.testing.assert_array_equal(ids[perm], np.where(rid >= 0, perm[np.maximum(rid, 0)], -1))
    np.testing.assert_array_equal(dl[perm], g["nb_dlvl"])
    coarse = np.repeat(g["nb_dlvl"] < 0, 8, axis=1)
    np.testing.assert_array_equal(np.where(coarse, sh[perm], 0), np.where(coarse, g["nb_shift"], 0))


def _mapped_ib(g, perm):
    rib = g["out_ib"]
    return np.where(rib >= 0, perm[np.maximum(rib, 0)], rib)


@pytest.mark.skipif(not port.available(), reason="oracle not built")
@pytest.mark.parametrize("path", GOLDEN, ids=IDS)
def test_oracle_matches_golden(path, tmp_path):
    g, mesh, perm = load(path, tmp_path)
    prec = int(g["precision"])
    o = port.trace(port.Tables.from_mesh(mesh, 4 if prec == 1 else 8), 4 if prec == 1 else 8,
                   g["in_x"], g["in_dir"], g["in_cell"], perm[g["in_ib"]], g["in_proper"],
                   g["in_steps"], fx_shift=int(g["fx_shift"]))
    np.testing.assert_array_equal(o["x"], g["out_x"])
    np.testing.assert_array_equal(o["cell"], g["out_cell"])
    np.testing.assert_array_equal(o["ib"], _mapped_ib(g, perm))
    np.testing.assert_array_equal(o["step"], g["out_step"])
    np.testing.assert_array_equal(o["todo"], g["out_todo"])
    np.testing.assert_array_equal(o["flux_fx"], dense(g, mesh, perm, "flux_fx"))
    np.testing.assert_array_equal(o["flux"], dense(g, mesh, perm, "flux"))   # same sequential order


@pytest.mark.gpu
@pytest.mark.parametrize("path", GOLDEN, ids=IDS)
def test_gpu_walk_matches_golden(path, tmp_path):
    import torch
    from kratos_polrad_b200 import PacketPool, trace
    g, mesh, perm = load(path, tmp_path)
    tdt = torch.float32 if int(g["precision"]) == 1 else torch.float64
    dev = torch.device("cuda")
    T = lambda a, dt=None: torch.tensor(a, dtype=dt, device=dev)
    pool = PacketPool(T(g["in_x"], tdt), T(g["in_dir"], tdt), T(g["in_cell"]),
                      T(perm[g["in_ib"]].astype(np.int32)), T(g["in_proper"], tdt), T(g["in_steps"]))
    flux = trace(mesh, pool, "fixed", int(g["fx_shift"]))
    torch.cuda.synchronize()
    assert mesh.status() == 0
    np.testing.assert_array_equal(pool.x.cpu().numpy().astype(np.float64), g["out_x"])
    np.testing.assert_array_equal(pool.cell.cpu().numpy(), g["out_cell"])
    np.testing.assert_array_equal(pool.ib.cpu().numpy(), _mapped_ib(g, perm))
    np.testing.assert_array_equal(pool.step.cpu().numpy(), g["out_step"])
    np.testing.assert_array_equal(pool.todo.cpu().numpy().astype(np.int32), g["out_todo"])
    np.testing.assert_array_equal(flux.cpu().numpy(), dense(g, mesh, perm, "flux_fx"))


SPH = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "sph_walk_*.npz")))


def load_sph(path, tmp_path):
    g = dict(np.load(path))
    ini = tmp_path / "sph.ini"
    ini.write_text(str(g["ini"]))
    mesh = Mesh(ini_path=str(ini), spherical=True)
    pl, pr = mesh.blocks()
    key = {(int(l), *map(int, r)): i for i, (l, r) in enumerate(zip(pl, pr))}
    perm = np.array([key[(int(l), *map(int, r))] for l, r in zip(g["ref_levels"], g["ref_regions"])])
    return g, mesh, perm


@pytest.mark.parametrize("path", SPH, ids=[os.path.basename(p)[:-4] for p in SPH])
def test_sph_tables_match_golden(path, tmp_path):
    g, mesh, perm = load_sph(path, tmp_path)
    P = 4 if int(g["precision"]) == 1 else 8
    xf0, dx0, vol0, pb = mesh.geometry(P)
    for a, b in ((xf0, "xf0"), (dx0, "dx0"), (vol0, "vol0"), (pb, "phybnd")):
        np.testing.assert_array_equal(a[perm], g[b], err_msg=b)
    rf, vol = mesh.geometry_sph(P)
    np.testing.assert_array_equal(rf[perm], g["r_faces"])
    cpb = mesh.cells_per_block
    np.testing.assert_array_equal(vol.reshape(-1, cpb)[perm].reshape(-1), g["volumes"])
    ids, _, dl = mesh.neighbors()
    rid = g["nb_ids"]
    np.testing.assert_array_equal(ids[perm], np.where(rid >= 0, perm[np.maximum(rid, 0)], -1))
    np.testing.assert_array_equal(dl[perm], g["nb_dlvl"])


@pytest.mark.gpu
@pytest.mark.parametrize("path", SPH, ids=[os.path.basename(p)[:-4] for p in SPH])
def test_gpu_sph_walk_matches_golden(path, tmp_path):
    """The reference's host-compiled spherical walk differs from the device's
    only through cosf/sinf/acosf/atan2f rounding: nearly every packet ends in
    the same state."""
    import torch
    from kratos_polrad_b200 import PacketPool
    from kratos_polrad_b200.walk import trace_sph
    g, mesh, perm = load_sph(path, tmp_path)
    tdt = torch.float32 if int(g["precision"]) == 1 else torch.float64
    dev = torch.device("cuda")
    T = lambda a, dt=None: torch.tensor(a, dtype=dt, device=dev)
    pool = PacketPool(T(g["in_x"], tdt), T(g["in_dir"], tdt), T(g["in_cell"]),
                      T(perm[g["in_ib"]].astype(np.int32)), T(g["in_proper"], tdt),
                      T(g["in_steps"]))
    xc = T(g["in_x_car"], tdt)
    trace_sph(mesh, pool, xc, "fixed", 16)
    torch.cuda.synchronize()
    assert mesh.status() & ~2 == 0
    rib = g["out_ib"]
    same = ((pool.cell.cpu().numpy() == g["out_cell"]).all(1)
            & (pool.ib.cpu().numpy() == np.where(rib >= 0, perm[np.maximum(rib, 0)], rib))
            & (pool.step.cpu().numpy() == g["out_step"])
            & (pool.todo.cpu().numpy().astype(np.int32) == g["out_todo"]))
    assert same.mean() >= 0.95, same.mean()
