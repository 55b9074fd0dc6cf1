"""Generates the golden fixtures of the geometric walk from the reference's
own code compiled for the host (oracle/_ref: tree_t, meshgen, proxy_base_t
::setup and photon::cart_t::proc built from the reference sources).

Each fixture holds the reference's block tables and the final packet states
and flux sums of a seeded packet set, in the reference's block order, so
tests can pin the product tables, the oracle restatement and the GPU walk
without the reference present.  Run from the repository root after
`make -C oracle ref REF=<reference tree>`:

    python tests/golden/make_golden.py [reference tree]

It also writes two binary-container fixtures, one with the reference's C++
binary_io and one with its Python writer (visual/binary_io.py).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.dirname(HERE)]

from kratos_polrad_b200 import Mesh                      # noqa: E402
from meshcases import CASES                              # noqa: E402
from oracle import refharness                            # noqa: E402

FIXTURES = [("amr_box", 1), ("amr_periodic", 1), ("amr_periodic", 2), ("three_level", 2),
            ("slab", 1)]
N_PACKETS, BUDGET, FX_SHIFT = 256, 120, 30


def packets(mesh, n, ftype, seed):
    """Seeded packets: random interior points and directions, plus axis-aligned
    and in-plane directions, starts on a cell face and short budgets."""
    rng = np.random.default_rng(seed)
    lo, hi = np.array(mesh.x_min), np.array(mesh.x_max)
    x = (lo + rng.random((n, 3)) * (hi - lo)).astype(ftype)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    d = d.astype(ftype)
    k = n // 8
    d[:k, :] = 0
    d[:k, 0] = np.where(rng.random(k) < 0.5, 1, -1)
    d[k:2 * k, 2] = 0
    xf0, dx0, _, _ = mesh.geometry(4 if ftype == np.float32 else 8)
    ib, cell = mesh.locate(x.astype(np.float64))
    m = slice(2 * k, 3 * k)
    x[m, 1] = (xf0[ib[m], 1] + cell[m, 1] * dx0[ib[m], 1]).astype(ftype)
    ib, cell = mesh.locate(x.astype(np.float64))
    proper = rng.random(n).astype(ftype) + ftype(0.5)
    steps = np.full(n, BUDGET, np.int32)
    steps[3 * k:4 * k] = rng.integers(0, 40, k)
    return x, d, cell, ib, proper, steps


def make(name, precision):
    cfg = CASES[name]
    ftype = np.float32 if precision == 1 else np.float64
    mesh = Mesh(cfg)
    ref = refharness.RefMesh(cfg.to_ini(), precision)
    rl, rr = ref.blocks()
    pl, pr = mesh.blocks()
    key = {(int(l), *map(int, r)): i for i, (l, r) in enumerate(zip(pl, pr))}
    perm = np.array([key[(int(l), *map(int, r))] for l, r in zip(rl, rr)])   # ref -> product
    inv = np.argsort(perm)
    x, d, cell, ib, proper, steps = packets(mesh, N_PACKETS, ftype, seed=100 + precision)
    ib_ref = inv[ib].astype(np.int32)
    r = ref.trace(x, d, cell, ib_ref, proper, steps, fx_shift=FX_SHIFT)
    xf0, dx0, vol0, pb = ref.geometry()
    ids, sh, dl = ref.neighbors()
    xlim, lbox, per = ref.box()
    nz = np.nonzero((r["flux"] != 0) | (r["flux_fx"] != 0))[0]
    out = dict(ini=np.array(cfg.to_ini()), precision=np.int32(precision),
               ref_levels=rl, ref_regions=rr, xf0=xf0, dx0=dx0, vol0=vol0, phybnd=pb,
               nb_ids=ids, nb_shift=sh, nb_dlvl=dl, xlim=xlim, lbox=lbox, periodic=per,
               in_x=x, in_dir=d, in_cell=cell.astype(np.int32), in_ib=ib_ref, in_proper=proper,
               in_steps=steps, fx_shift=np.int32(FX_SHIFT),
               out_x=r["x"], out_cell=r["cell"], out_ib=r["ib"], out_step=r["step"],
               out_todo=r["todo"], flux_idx=nz.astype(np.int32), flux=r["flux"][nz],
               flux_fx=r["flux_fx"][nz])
    path = os.path.join(HERE, f"trace_{name}_p{precision}.npz")
    np.savez_compressed(path, **out)
    return path, os.path.getsize(path)


def bio_entries():
    """Entries of the binary-container fixtures: unsorted tags (the writer
    sorts them), every unit size the transport stores, a block-key tag."""
    rng = np.random.default_rng(12)
    return [("zeta|tally", rng.integers(-2 ** 40, 2 ** 40, 24, dtype=np.int64)),
            ("block_10|level", np.int32([2])),
            ("block_2|i_logic", np.int32([1, 0, 3])),
            ("alpha", rng.random(7).astype(np.float32)),
            ("kp|grad", rng.normal(size=5)),
            ("kp|config", np.frombuffer(b'{"seed": 4}', np.uint8))]


def make_bio(reference_tree):
    """bio_reference.bin: the reference's C++ binary_io::base_t; bio_reference_py.bin:
    the reference's Python writer (visual/binary_io.py), which keeps insertion order."""
    ent = bio_entries()
    p1 = os.path.join(HERE, "bio_reference.bin")
    refharness.bio_write(p1, ent)
    sys.path.insert(0, os.path.join(reference_tree, "visual"))
    from binary_io import binary_io as py_writer        # the reference's own reader/writer
    p2 = os.path.join(HERE, "bio_reference_py.bin")
    w = py_writer(p2)
    for tag, a in ent:
        w.cache(tag, a)
    w.save()
    return [(p, os.path.getsize(p)) for p in (p1, p2)]


# Spherical-polar fixture: r in [1, 3] geometric, theta [0.4, 2.7], phi periodic,
# 16^3 cells in 8^3 blocks with one refined box.
SPH_INI = """[mesh]
x_min = 1.0 0.4 0.0
x_max = 3.0 2.7 6.283185307179586
n_cell_global = 16 16 16
n_cell_block = 8 8 8
r_ratio = -1.0

[boundary]
kinds = outflow outflow outflow outflow periodic periodic

[refine_region_00000]
level = 1
x_min = 1.5 1.2 1.0
x_max = 1.8 1.5 2.0
"""


def make_sph(precision, n=256, budget=120):
    """Reference tables and photon::sph_t walk of seeded packets."""
    ftype = np.float32 if precision == 1 else np.float64
    ref = refharness.RefMeshSph(SPH_INI, precision)
    rng = np.random.default_rng(300 + precision)
    lo, hi = np.array([1.0, 0.4, 0.0]), np.array([3.0, 2.7, 2 * np.pi])
    pad = np.array([0.02, 0.05, 0.0]) * (hi - lo)
    x = lo + pad + rng.random((n, 3)) * (hi - lo - 2 * pad)
    r, th, ph = x[:, 0], x[:, 1], x[:, 2]
    xc = np.stack([r * np.sin(th) * np.cos(ph), r * np.sin(th) * np.sin(ph), r * np.cos(th)], 1)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    import tempfile
    from kratos_polrad_b200 import Mesh
    with tempfile.NamedTemporaryFile("w", suffix=".ini", delete=False) as f:
        f.write(SPH_INI)
    prod = Mesh(ini_path=f.name, spherical=True)
    os.unlink(f.name)
    rl, rr = ref.blocks()
    pl, pr = prod.blocks()
    key = {(int(l), *map(int, q)): i for i, (l, q) in enumerate(zip(pl, pr))}
    inv = np.argsort(np.array([key[(int(l), *map(int, q))] for l, q in zip(rl, rr)]))
    ib, cell = prod.locate(x)
    x, xc, d = x.astype(ftype), xc.astype(ftype), d.astype(ftype)
    proper = (rng.random(n) + 0.5).astype(ftype)
    steps = np.full(n, budget, np.int32)
    out = ref.trace(x, xc, d, cell, inv[ib], proper, steps, fx_shift=16)
    xf0, dx0, vol0, pb = ref.geometry()
    rf, vol = ref.geometry_sph()
    ids, sh, dl = ref.neighbors()
    path = os.path.join(HERE, f"sph_walk_p{precision}.npz")
    np.savez_compressed(path, ini=np.array(SPH_INI), precision=np.int32(precision),
                        ref_levels=rl, ref_regions=rr, xf0=xf0, dx0=dx0, vol0=vol0, phybnd=pb,
                        r_faces=rf, volumes=vol, nb_ids=ids, nb_dlvl=dl,
                        in_x=x, in_x_car=xc, in_dir=d, in_cell=cell.astype(np.int32),
                        in_ib=inv[ib].astype(np.int32), in_proper=proper, in_steps=steps,
                        out_x=out["x"], out_x_car=out["x_car"], out_cell=out["cell"],
                        out_ib=out["ib"], out_step=out["step"], out_todo=out["todo"])
    return path, os.path.getsize(path)


if __name__ == "__main__":
    if not refharness.available(1):
        sys.exit("oracle/_ref not built: make -C oracle ref REF=<reference tree>")
    # the reference checkout: argument, $KP_REFERENCE_SRC, or a "reference"
    # directory beside this repository
    ref_tree = (sys.argv[1] if len(sys.argv) > 1 else os.environ.get(
        "KP_REFERENCE_SRC", os.path.join(os.path.dirname(ROOT), "reference")))
    for name, prec in FIXTURES:
        print(*make(name, prec))
    for p in make_bio(ref_tree):
        print(*p)
    for prec in (1, 2):
        print(*make_sph(prec))
