"""Straight-line walks of the polarized transport against the reference's own
walk (photon::cart_t::proc compiled from the reference sources, PRECISION=2).

With zero coefficients a packet never interacts: the transport walk is the
geometric walk of the reference, and its path-length flux tally is the
reference's rad_t::flx estimator (modules/particle/radiation/photon.h:73-83).
The reference walks every packet from the same start: the source position,
the packet's direction (read back from its record), the source cell.

The reference's walk parts from the straight line whenever geo_loc_t::fix
(modules/particle/types/particle_base.h:117-126) shifts a cached face without
moving the cell index.  That happens after a coarse-to-fine hand-off into the
upper half of a coarse cell (proxy.h:111-117 picks the lower fine cell), and
after a periodic crossing toward -x whose face coordinate equals the domain's
lower limit (regulate, particle_base.h:37-56, wraps only x < x_min, so the
packet keeps x = x_min while its index moves to the far end).  The restated
walk (oracle kpo_trace_ex, pinned bit for bit to the reference here) counts
these shifts per packet.  Packets without one must take the transport's walk
exactly: same segments, same exit point, same flux.
"""
from __future__ import annotations

import dataclasses

import numpy as np

from kratos_polrad_b200 import Mesh
from kratos_polrad_b200.transport import EMIT_ISOTROPIC, SOURCE_POINT, Source, TransportConfig
from meshcases import AMR_BOX, SLAB, THREE_LEVEL
from oracle import port, refharness
from test_trace_gpu import perm_ref_to_prod

# mesh, source position (inside a cell, on no face), segment budget
STRAIGHT = {
    "slab": (SLAB, (45.3172, 77.8915, 23.4567), 4096),
    "amr_box": (AMR_BOX, (0.2113, 0.3187, 0.2561), 4096),        # rays enter the refined box
    "three_level": (THREE_LEVEL, (0.9513, 1.0371, 0.9822), 600),  # periodic: every ray is capped
}
FLUX_SHIFT = 32
N_PACKETS = 4000
# Per-cell bar for the flux of the packets that walk alike: the deposits
# differ in the last bits (the kernel multiplies by 1/dir and 1/volume, the
# reference divides), so a cell may differ by a few fixed-point units.
FLUX_RTOL = 1e-8
FLUX_ATOL_UNITS = 128          # 2^-25 in flux units at scale 2^32


def setup(name):
    mc, pos, steps = STRAIGHT[name]
    mesh = Mesh(mc)
    cfg = TransportConfig(n_packets=N_PACKETS, sources=[Source(SOURCE_POINT, EMIT_ISOTROPIC, pos)],
                          seed=11, n_record=N_PACKETS, max_steps=steps, flux=True,
                          flux_fx_shift=FLUX_SHIFT)
    sig = np.zeros((mesh.n_cells, 2), np.float32)
    return mesh, sig, cfg


def reference_walks(name, mesh, rec):
    """Walks the packets of `rec` (their directions) from the source with the
    reference; returns the reference's output, the restated walk's fix counts
    and the start arrays."""
    mc, pos, steps = STRAIGHT[name]
    ref = refharness.RefMesh(mc.to_ini(), 2)
    perm = perm_ref_to_prod(mesh, ref)
    inv = np.argsort(perm)
    ib, cell = mesh.locate(np.array([pos]))
    n = len(rec)
    start = (np.tile(pos, (n, 1)), rec["d"].astype(np.float64), np.tile(cell[0], (n, 1)),
             np.full(n, inv[ib[0]]), np.ones(n), np.full(n, steps, np.int32))
    r = ref.trace(*start, fx_shift=FLUX_SHIFT)
    q = port.trace(port.Tables.from_ref(ref), 8, *start, fx_shift=FLUX_SHIFT)
    for k in ("x", "cell", "ib", "step", "todo", "flux_fx"):
        np.testing.assert_array_equal(q[k], r[k], err_msg=f"restated walk vs reference: {k}")
    return ref, perm, r, q["fix"], start


def compare_walks(name, mesh, rec, r, fix):
    """Per-packet comparison; returns the mask of packets without fix shifts
    (every one of them must agree) and a summary."""
    mc, _, steps = STRAIGHT[name]
    escaped = rec["status"] == 1
    # the reference's budget does not count the segment that leaves the
    # domain (photon.h:111-121 breaks before decrementing)
    ref_segments = steps - r["step"] + escaped
    same_steps = rec["n_steps"] == ref_segments
    # both end on the boundary face an escaping packet leaves through
    dx = np.abs(rec["x"] - r["x"])
    clean = fix == 0
    bad = clean & ~(same_steps & (dx.max(1) <= 1e-9))
    assert not bad.any(), (f"{name}: {bad.sum()} packets without a fix shift walk differently, "
                           f"e.g. packet {np.nonzero(bad)[0][:5]}")
    summary = dict(packets=len(rec), fix_packets=int((~clean).sum()),
                   fix_alike=int((~clean & same_steps).sum()),
                   clean_max_dx=float(dx[clean].max()) if clean.any() else 0.0)
    return clean, summary


def clean_runs(clean):
    """Contiguous [start, end) packet-index runs of the clean packets."""
    idx = np.nonzero(clean)[0]
    if len(idx) == 0:
        return []
    cut = np.nonzero(np.diff(idx) != 1)[0] + 1
    starts = np.concatenate([[0], cut])
    ends = np.concatenate([cut, [len(idx)]])
    return [(int(idx[s]), int(idx[e - 1]) + 1) for s, e in zip(starts, ends)]


def reference_clean_flux(ref, start, clean):
    return ref.trace(*(a[clean] for a in start), fx_shift=FLUX_SHIFT)["flux_fx"]


def oracle_clean_flux(mesh, sig, cfg, clean):
    """The C restatement's flux over the clean packets (run by runs)."""
    from transport_cases import oracle_inputs
    tab, grid, gn, cells = oracle_inputs(mesh, cfg)
    out = np.zeros(mesh.n_cells, np.int64)
    for a, b in clean_runs(clean):
        c = dataclasses.replace(cfg, packet_offset=cfg.packet_offset + a, n_packets=b - a,
                                n_record=0)
        out += port.transport(tab, sig, grid, gn, c, cells, flux=True)["flux"]
    return out


def compare_flux(mesh, perm, prod_flux, ref_flux):
    """prod_flux in product block order, ref_flux in the reference's."""
    cpb = mesh.cells_per_block
    a = np.asarray(prod_flux, np.int64).reshape(-1, cpb)[perm].reshape(-1)
    b = np.asarray(ref_flux, np.int64)
    d = np.abs(a - b)
    tol = np.maximum(FLUX_ATOL_UNITS, FLUX_RTOL * np.abs(b))
    bad = d > tol
    assert not bad.any(), f"{bad.sum()} cells beyond the bar, worst {d.max()} units"
    assert (b != 0).sum() > 1000, "too few cells visited to compare"
    return dict(cells=int((b != 0).sum()), cells_differing=int((d > 0).sum()),
                max_units=int(d.max()), max_rel=float((d / np.maximum(np.abs(b), 1)).max()))
