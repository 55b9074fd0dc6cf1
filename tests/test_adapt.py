"""Runtime refinement: adapted meshes vs the reference's static refinement
(host), flags from the coefficients, field remapping and transport on an
adapted mesh (GPU)."""
import dataclasses

import numpy as np
import pytest

from kratos_polrad_b200 import KPError, Mesh
from kratos_polrad_b200.mesh import MeshConfig, RefineRegion
from meshcases import AMR_BOX, AMR_PERIODIC, THREE_LEVEL
from oracle import refharness

CASES = {"amr_box": AMR_BOX, "amr_periodic": AMR_PERIODIC, "three_level": THREE_LEVEL}


def leaf_config(base: MeshConfig, mesh: Mesh) -> MeshConfig:
    """The static configuration with one refine box (the block's centre
    point) per leaf above level 0 of `mesh`."""
    lev, reg = mesh.blocks()
    xf0, dx0, _, _ = mesh.geometry(8)
    nc = np.array(mesh.nc)
    boxes = []
    for b in np.nonzero(lev > 0)[0]:
        c = tuple(xf0[b] + 0.5 * nc * dx0[b])
        boxes.append(RefineRegion(int(lev[b]), c, c))
    return dataclasses.replace(base, refine=boxes)


def random_flags(mesh, rng, p_refine=0.12, p_coarsen=0.5):
    lev, _ = mesh.blocks()
    f = np.zeros(mesh.n_blocks, np.int32)
    f[(rng.random(mesh.n_blocks) < p_refine) & (lev < 3)] = 1
    f[(rng.random(mesh.n_blocks) < p_coarsen) & (lev > 0) & (f == 0)] = -1
    return f


def same_tables(a: Mesh, b: Mesh):
    la, ra = a.blocks()
    lb, rb = b.blocks()
    np.testing.assert_array_equal(la, lb)
    np.testing.assert_array_equal(ra, rb)
    for x, y in zip(a.geometry(8), b.geometry(8)):
        np.testing.assert_array_equal(x, y)
    for x, y in zip(a.neighbors(), b.neighbors()):
        np.testing.assert_array_equal(x, y)


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("seed", [0, 1])
def test_adapted_equals_static_refinement(name, seed):
    """Adapting equals building the leaf set statically (same block order)."""
    base = CASES[name]
    m = Mesh(base)
    a = m.adapt(random_flags(m, np.random.default_rng(seed)))
    assert a.n_blocks != m.n_blocks
    same_tables(a, Mesh(leaf_config(base, a)))


@pytest.mark.skipif(not refharness.available(2), reason="oracle/_ref not built")
@pytest.mark.parametrize("name", sorted(CASES))
def test_adapted_tables_match_reference(name):
    """...and the reference's own tree/meshgen/proxy code builds the same
    blocks and neighbour tables from those refine boxes."""
    base = CASES[name]
    m = Mesh(base)
    a = m.adapt(random_flags(m, np.random.default_rng(7)))
    a = a.adapt(random_flags(a, np.random.default_rng(8)))          # twice
    ref = refharness.RefMesh(leaf_config(base, a).to_ini(), 2)
    assert ref.n_blocks == a.n_blocks
    pl, pr = a.blocks()
    rl, rr = ref.blocks()
    key = {(int(l), *map(int, r)): i for i, (l, r) in enumerate(zip(pl, pr))}
    perm = np.array([key[(int(l), *map(int, r))] for l, r in zip(rl, rr)])
    pxf, pdx, pvol, ppb = a.geometry(8)
    rxf, rdx, rvol, rpb = ref.geometry()
    np.testing.assert_array_equal(pxf[perm], rxf)
    np.testing.assert_array_equal(pdx[perm], rdx)
    np.testing.assert_array_equal(ppb[perm], rpb)
    pid, psh, pdl = a.neighbors()
    rid, rsh, rdl = ref.neighbors()
    np.testing.assert_array_equal(pid[perm], np.where(rid >= 0, perm[np.maximum(rid, 0)], -1))
    np.testing.assert_array_equal(pdl[perm], rdl)
    coarse = np.repeat(rdl < 0, 8, axis=1)
    np.testing.assert_array_equal(np.where(coarse, psh[perm], 0), np.where(coarse, rsh, 0))


def test_zero_flags_keep_the_mesh():
    m = Mesh(THREE_LEVEL)
    same_tables(m, m.adapt(np.zeros(m.n_blocks, np.int32)))


def test_coarsening_needs_whole_family_and_balance():
    m = Mesh(THREE_LEVEL)                      # has level-2 blocks
    lev, reg = m.blocks()
    # coarsening only part of a family does nothing
    fam = np.nonzero(lev == 2)[0][:3]
    f = np.zeros(m.n_blocks, np.int32)
    f[fam] = -1
    same_tables(m, m.adapt(f))
    # coarsening every level-1 block while level-2 blocks remain keeps the
    # level-1 blocks the 2:1 balance needs
    f = np.where(lev == 1, -1, 0).astype(np.int32)
    a = m.adapt(f)
    la, _ = a.blocks()
    assert la.max() == 2 and (la == 1).sum() > 0
    # coarsening everything, repeatedly, comes down to the root blocks
    flat = m
    for _ in range(3):
        flat = flat.adapt(np.full(flat.n_blocks, -1, np.int32))
    assert flat.max_level == 0 and flat.n_blocks == 8 ** 3


def test_errors():
    m = Mesh(AMR_BOX)
    with pytest.raises(ValueError):
        m.adapt(np.zeros(m.n_blocks + 1, np.int32))
    # refining one deepest block again and again ends in a clear error (the
    # finest-level lookup grid or the level limit), not in a crash
    deep = m
    with pytest.raises(KPError, match="too large|exceed 20"):
        for _ in range(25):
            lev, _ = deep.blocks()
            f = np.zeros(deep.n_blocks, np.int32)
            f[np.argmax(lev)] = 1
            deep = deep.adapt(f)


# ---------------------------------------------------------------- GPU

def _octant_remap(src_mesh, dst_mesh, field):
    """float32 restatement of kp_mesh_remap."""
    xf0, dx0, _, _ = dst_mesh.geometry(8)
    nc = np.array(dst_mesh.nc)
    k, j, i = np.meshgrid(np.arange(nc[2]), np.arange(nc[1]), np.arange(nc[0]), indexing="ij")
    cells = np.stack([i.ravel(), j.ravel(), k.ravel()], 1)
    idx = []
    for s in range(8):
        off = np.array([0.75 if (s >> a) & 1 else 0.25 for a in range(3)])
        x = (xf0[:, None, :] + (cells[None] + off) * dx0[:, None, :]).reshape(-1, 3)
        ib, cell = src_mesh.locate(x)
        idx.append(ib * src_mesh.cells_per_block + cell[:, 0] + nc[0] * (cell[:, 1] + nc[1] * cell[:, 2]))
    idx = np.stack(idx, 1)
    same = (idx == idx[:, :1]).all(1)
    out = field[idx[:, 0]].astype(np.float32).copy()
    acc = field[idx[:, 0]].astype(np.float32)
    for s in range(1, 8):
        acc = (acc + field[idx[:, s]]).astype(np.float32)
    out[~same] = (acc[~same] * np.float32(0.125)).astype(np.float32)
    return out


@pytest.mark.gpu
def test_flags_remap_and_transport_on_adapted_mesh():
    import torch
    from kratos_polrad_b200.transport import Tallies, forward
    from transport_cases import case
    mesh, sig, t = case("amr_point")
    mesh.set_sigma(sig)
    tau_r, tau_c = 0.25, 0.05
    flags = mesh.flag_tau(tau_r, tau_c).cpu().numpy()
    # numpy restatement of the flags
    _, dx0, _, _ = mesh.geometry(8)
    dxm = dx0.max(1).astype(np.float32)
    ext = (sig[:, 0] + sig[:, 1]).astype(np.float32).reshape(mesh.n_blocks, -1)
    v = (ext * dxm[:, None]).astype(np.float32).max(1)
    np.testing.assert_array_equal(flags, np.where(v > tau_r, 1, np.where(v < tau_c, -1, 0)))
    assert (flags == 1).any() and (flags == -1).any()
    fine = mesh.adapt(flags)
    s_dev = torch.tensor(sig, device="cuda")
    s_fine = mesh.remap_to(fine, s_dev)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(s_fine.cpu().numpy(), _octant_remap(mesh, fine, sig))
    assert fine.status() == 0
    # refine-then-back copies exactly where nothing was coarsened
    back = fine.remap_to(mesh, s_fine).cpu().numpy()
    np.testing.assert_array_equal(back, _octant_remap(fine, mesh, s_fine.cpu().numpy()))
    # the transport runs on the adapted mesh
    fine.set_sigma(s_fine)
    tt = dataclasses.replace(t, n_record=0, n_packets=20000)
    tal = forward(fine, tt, Tallies(tt))
    torch.cuda.synchronize()
    c = tal.counts()
    assert fine.status() == 0 and c["emitted"] == tt.n_packets and c["lost"] == 0
    assert c["escaped"] + c["absorbed"] + c["capped"] == tt.n_packets
