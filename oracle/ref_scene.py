"""Bench scenes built on the reference's own mesh code (test infrastructure).

The CPU arm of the benchmark must not lean on the product: it builds the
clump scene's blocks, geometry and neighbour tables with the reference's
tree/meshgen/proxy code compiled for the host (oracle/_ref/libkpref_p2.so,
via refharness), takes the scene's coefficients and transport configuration
from kratos_polrad_b200.problems (plain data, no library), and runs the C
restatement of the transport (port.transport) on those tables.  The product
library is never loaded.
"""
from __future__ import annotations

import math

import numpy as np

from . import port, refharness


def cell_centres(tab: port.Tables) -> np.ndarray:
    """Cell-centre coordinates [n_cells, 3], block-id order, x fastest."""
    nc = tab.nc
    k, j, i = np.meshgrid(np.arange(nc[2]), np.arange(nc[1]), np.arange(nc[0]), indexing="ij")
    idx = np.stack([i.ravel(), j.ravel(), k.ravel()], 1) + 0.5
    return (tab.xf0[:, None, :] + idx[None] * tab.dx0[:, None, :]).reshape(-1, 3)


def root_blocks(tab: port.Tables, levels) -> list:
    """Root blocks per axis, from the block spacing of the coarsest block."""
    b = int(np.argmin(levels))
    return [int(round(tab.lbox[a] / (tab.dx0[b, a] * tab.nc[a] * 2 ** int(levels[b]))))
            for a in range(3)]


def locate(tab: port.Tables, levels, regs, x) -> tuple:
    """(block id, cell[3]) of point x: the leaf whose region key holds x's
    logical coordinate at its level (floor, clamped to the domain), then the
    cell by floor((x - xf0) / dx0), clamped to the block."""
    roots = root_blocks(tab, levels)
    keys = {(int(l), *map(int, r)): b for b, (l, r) in enumerate(zip(levels, regs))}
    lo = tab.xlim[0]
    for lev in sorted(set(int(v) for v in levels)):
        k = []
        for a in range(3):
            n = roots[a] << lev
            f = math.floor((x[a] - lo[a]) / tab.lbox[a] * n)
            k.append(min(max(f, 0), n - 1))
        b = keys.get((lev, *k))
        if b is not None:
            cell = [min(max(int(math.floor((x[a] - tab.xf0[b, a]) / tab.dx0[b, a])), 0),
                        tab.nc[a] - 1) for a in range(3)]
            return b, cell
    raise ValueError(f"point {x} lies in no block")


def clump(n_packets: int):
    """The 2-level AMR clump of the benchmark on the reference's meshgen:
    (tables, sigma2, lookup grid, its shape, cfg, source cells)."""
    from kratos_polrad_b200 import problems
    mcfg, sigma_of, cfg = problems.clump_spec(n_packets=n_packets)
    ref = refharness.RefMesh(mcfg.to_ini(), 2)
    tab = port.Tables.from_ref(ref)
    levels, regs = ref.blocks()
    sigma2 = sigma_of(cell_centres(tab))
    grid, gn = port.lookup_grid(levels, regs, root_blocks(tab, levels))
    cells = [locate(tab, levels, regs, s.pos) for s in cfg.sources]
    return tab, sigma2, grid, gn, cfg, cells
