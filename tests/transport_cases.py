"""Small transport cases shared by the CPU and GPU tests."""
import numpy as np

from kratos_polrad_b200 import Mesh
from kratos_polrad_b200.transport import (EMIT_ISOTROPIC, EMIT_UP_UNIFORM, PHASE_HG_POL,
                                          PHASE_RAYLEIGH, SOURCE_PLANE_BASE, SOURCE_POINT,
                                          Source, TransportConfig, packet_array)
from meshcases import AMR_BOX, AMR_PERIODIC
from kratos_polrad_b200.mesh import MeshConfig
from oracle import port


def cell_centers(mesh):
    xf0, dx0, _, _ = mesh.geometry(8)
    nc = mesh.nc
    k, j, i = np.meshgrid(np.arange(nc[2]), np.arange(nc[1]), np.arange(nc[0]), indexing="ij")
    idx = np.stack([i.ravel(), j.ravel(), k.ravel()], 1) + 0.5     # x fastest
    return (xf0[:, None, :] + idx[None] * dx0[:, None, :]).reshape(-1, 3)


def case(name):
    """Returns (mesh, sigma2 [n_cells, 2] float32, TransportConfig)."""
    if name == "slab":
        cfg = MeshConfig((0, 0, 0), (32, 32, 16), (32, 32, 16), (8, 8, 8), (True, True, False))
        mesh = Mesh(cfg)
        sig = np.zeros((mesh.n_cells, 2), np.float32)
        sig[:, 0] = 2.0 / 16                                   # vertical tau = 2
        t = TransportConfig(n_packets=3000, sources=[Source(SOURCE_PLANE_BASE, EMIT_UP_UNIFORM)],
                            seed=1, n_mu_bins=10, mu_lo=0.0, mu_hi=1.0, n_record=3000)
    elif name == "amr_point":
        mesh = Mesh(AMR_BOX)
        c = cell_centers(mesh)
        r2 = ((c - 0.5) ** 2).sum(1)
        rho = 1 + 40 * np.exp(-r2 / (2 * 0.08 ** 2))
        rng = np.random.default_rng(2)
        alb = np.exp(rng.uniform(np.log(0.5), np.log(0.99), mesh.n_cells))
        ext = 3.0 * rho / rho.mean()
        sig = np.stack([ext * alb, ext * (1 - alb)], 1).astype(np.float32)
        t = TransportConfig(n_packets=2000, sources=[Source(SOURCE_POINT, EMIT_ISOTROPIC, (0.5, 0.5, 0.5))],
                            seed=2, image_n=32, inclination_deg=60.0, image_center=(0.5, 0.5, 0.5),
                            image_half_width=0.87, w_min=0.05, image_batch_n=4, n_mu_bins=8, mu_lo=-1, mu_hi=1,
                            n_record=2000)
    elif name == "hg_multi":
        mesh = Mesh(AMR_PERIODIC)
        c = cell_centers(mesh)
        rng = np.random.default_rng(5)
        ext = 0.5 + rng.random(mesh.n_cells)
        sig = np.stack([0.9 * ext, 0.1 * ext], 1).astype(np.float32)
        srcs = [Source(SOURCE_POINT, EMIT_ISOTROPIC, tuple(p))
                for p in [(-0.3, 0.2, 1.1), (0.7, -1.5, 2.2), (0.0, 1.9, 0.6), (0.26, 0.55, 1.55)]]
        t = TransportConfig(n_packets=1500, sources=srcs, seed=7, stream_id=3, phase=PHASE_HG_POL,
                            hg_g=0.6, pol_max=0.5, image_n=24, inclination_deg=35.0, azimuth_deg=20.0,
                            image_center=(0, 0, 1.5), image_half_width=2.5, w_min=0.02,
                            n_mu_bins=16, mu_lo=-1, mu_hi=1, n_record=1500, max_scatter=200,
                            tau_peel_max=20.0)
    elif name == "table":
        # a user generator's packets: a ring of emitters with directions,
        # weights and polarization of its own; half give their block, half
        # are located on the device; half peel off toward the observer
        mesh = Mesh(AMR_BOX)
        c = cell_centers(mesh)
        rng = np.random.default_rng(8)
        ext = 2.0 + 6.0 * np.exp(-((c - 0.5) ** 2).sum(1) / (2 * 0.1 ** 2))
        alb = rng.uniform(0.6, 0.95, mesh.n_cells)
        sig = np.stack([ext * alb, ext * (1 - alb)], 1).astype(np.float32)
        n = 1500
        ang = rng.uniform(0, 2 * np.pi, n)
        x = np.stack([0.5 + 0.2 * np.cos(ang), 0.5 + 0.2 * np.sin(ang),
                      rng.uniform(0.3, 0.7, n)], 1)
        d = rng.normal(size=(n, 3))
        d /= np.linalg.norm(d, axis=1, keepdims=True)
        pol = np.zeros((n, 3))
        pol[::3, 0] = 0.4
        pol[1::3, 1] = -0.3
        ib, _ = mesh.locate(x)
        ib = np.where(np.arange(n) % 2 == 0, ib, -1)
        table = packet_array(x, d, w=rng.uniform(0.5, 2.0, n), stokes=pol, ib=ib,
                             peel_I=np.where(np.arange(n) % 2 == 0, 1 / (4 * np.pi), 0.0))
        t = TransportConfig(n_packets=n, sources=[], seed=9, image_n=32, inclination_deg=45.0,
                            azimuth_deg=30.0, image_center=(0.5, 0.5, 0.5), image_half_width=0.87,
                            w_min=0.05, image_batch_n=4, n_mu_bins=8, mu_lo=-1, mu_hi=1,
                            n_record=n, packets=table)
    else:
        raise KeyError(name)
    return mesh, sig, t


def to_device(t):
    """The cfg with its packet table (if any) copied to the GPU."""
    import dataclasses
    from kratos_polrad_b200.transport import packet_table
    if t.packets is None or hasattr(t.packets, "data_ptr"):
        return t
    return dataclasses.replace(t, packets=packet_table(t.packets))


def run_oracle(mesh, sig, t, deposits=0):
    tab = port.Tables.from_mesh(mesh, 8)
    lev, reg = mesh.blocks()
    root = [mesh.nc[a] and int(round((mesh.x_max[a] - mesh.x_min[a]) /
                                     (port.Tables.from_mesh(mesh, 8).dx0[0, a] * mesh.nc[a] * 2 ** lev[0])))
            for a in range(3)]
    grid, n = port.lookup_grid(lev, reg, root)
    cells = []
    for s in t.sources:
        if s.kind == SOURCE_POINT:
            ib, cell = mesh.locate(np.array([s.pos]))
            cells.append((ib[0], cell[0]))
        else:
            cells.append((0, (0, 0, 0)))
    return port.transport(tab, sig, grid, n, t, cells, deposits=deposits)


def oracle_inputs(mesh, t):
    """Tables, lookup grid and located source cells for the oracle."""
    tab = port.Tables.from_mesh(mesh, 8)
    lev, reg = mesh.blocks()
    root = [int(round((mesh.x_max[a] - mesh.x_min[a]) / (tab.dx0[0, a] * mesh.nc[a] * 2 ** lev[0])))
            for a in range(3)]
    grid, n = port.lookup_grid(lev, reg, root)
    cells = []
    for s in t.sources:
        if s.kind == SOURCE_POINT:
            ib, cell = mesh.locate(np.array([s.pos]))
            cells.append((ib[0], cell[0]))
        else:
            cells.append((0, (0, 0, 0)))
    return tab, grid, n, cells


def run_oracle_adjoint(mesh, sig, t, adj_img, grad_shift=24, abs_sum=False, fp64=False):
    tab, grid, n, cells = oracle_inputs(mesh, t)
    return port.adjoint(tab, sig, grid, n, t, cells, adj_img, grad_shift, abs_sum, fp64)
