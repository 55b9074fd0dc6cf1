"""Geometric walk on the GPU vs the reference's own cart_t::proc on the host.

Per-packet final state (position, cell, block, remaining budget, todo) and the
int64 fixed-point flux must be bit-identical; the float-atomic flux must agree
with the reference's sequential float sum to within the reordering bound
n_deposits * eps * sum|deposit| per cell.
"""
import numpy as np
import pytest
import torch

from kratos_polrad_b200 import Mesh, PacketPool, trace
from oracle import refharness
from meshcases import CASES

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not refharness.available(1), reason="oracle/_ref not built")]


def make_packets(mesh, n, ftype, seed, budget=4000):
    rng = np.random.default_rng(seed)
    lo, hi = np.array(mesh.x_min), np.array(mesh.x_max)
    x = (lo + rng.random((n, 3)) * (hi - lo)).astype(ftype)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    d = d.astype(ftype)
    # axis-aligned and in-plane directions exercise the dir == 0 branches
    k = n // 8
    d[:k, :] = 0
    d[:k, 0] = np.where(rng.random(k) < 0.5, 1, -1)
    d[k:2 * k, 2] = 0
    # some packets start exactly on a cell face
    xf0, dx0, _, _ = mesh.geometry(4 if ftype == np.float32 else 8)
    ib, cell = mesh.locate(x.astype(np.float64))
    m = slice(2 * k, 3 * k)
    x[m, 1] = (xf0[ib[m], 1] + cell[m, 1] * dx0[ib[m], 1]).astype(ftype)
    ib, cell = mesh.locate(x.astype(np.float64))
    proper = rng.random(n).astype(ftype) + ftype(0.5)
    steps = np.full(n, budget, np.int32)
    steps[3 * k:4 * k] = rng.integers(0, 40, k)          # budgets that run out
    return x, d, cell, ib, proper, steps


def perm_ref_to_prod(prod, ref):
    pl, pr = prod.blocks()
    rl, rr = ref.blocks()
    key = {(int(l), *map(int, r)): i for i, (l, r) in enumerate(zip(pl, pr))}
    return np.array([key[(int(l), *map(int, r))] for l, r in zip(rl, rr)])


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("precision", [1, 2])
def test_trace_bit_exact(name, precision):
    cfg = CASES[name]
    ftype = np.float32 if precision == 1 else np.float64
    tdt = torch.float32 if precision == 1 else torch.float64
    mesh = Mesh(cfg)
    ref = refharness.RefMesh(cfg.to_ini(), precision)
    perm = perm_ref_to_prod(mesh, ref)              # ref id -> prod id
    inv = np.argsort(perm)                          # prod id -> ref id
    n = 4096
    x, d, cell, ib, proper, steps = make_packets(mesh, n, ftype, seed=11 + precision)
    r = ref.trace(x, d, cell, inv[ib], proper, steps, fx_shift=32)

    dev = torch.device("cuda")
    pool = PacketPool(torch.tensor(x, dtype=tdt, device=dev), torch.tensor(d, dtype=tdt, device=dev),
                      torch.tensor(cell, device=dev), torch.tensor(ib, device=dev),
                      torch.tensor(proper, dtype=tdt, device=dev), torch.tensor(steps, device=dev))
    flux = trace(mesh, pool, "fixed", 32)
    torch.cuda.synchronize()
    assert mesh.status() == 0
    np.testing.assert_array_equal(pool.x.cpu().numpy().astype(np.float64), r["x"])
    np.testing.assert_array_equal(pool.cell.cpu().numpy(), r["cell"])
    rib = r["ib"]
    np.testing.assert_array_equal(pool.ib.cpu().numpy(), np.where(rib >= 0, perm[np.maximum(rib, 0)], rib))
    np.testing.assert_array_equal(pool.step.cpu().numpy(), r["step"])
    np.testing.assert_array_equal(pool.todo.cpu().numpy().astype(np.int32), r["todo"])
    cpb = mesh.cells_per_block
    ref_fx = r["flux_fx"].reshape(-1, cpb)[inv].reshape(-1)     # prod block order
    np.testing.assert_array_equal(flux.cpu().numpy(), ref_fx)

    # float atomics: same deposits in another order
    pool2 = PacketPool(torch.tensor(x, dtype=tdt, device=dev), torch.tensor(d, dtype=tdt, device=dev),
                       torch.tensor(cell, device=dev), torch.tensor(ib, device=dev),
                       torch.tensor(proper, dtype=tdt, device=dev), torch.tensor(steps, device=dev))
    fl = trace(mesh, pool2, "float").cpu().numpy().astype(np.float64)
    ref_f = r["flux"].reshape(-1, cpb)[inv].reshape(-1)
    # Reordered float sums: deposits can have either sign (the reference's
    # get_dl may pick a negative distance), so the bound scales with the
    # field's magnitude: 2^12 ulps of max|flux| per cell.
    eps = np.finfo(ftype).eps
    atol = 2.0 ** 12 * eps * np.abs(ref_f).max()
    np.testing.assert_allclose(fl, ref_f, rtol=0, atol=atol)
    np.testing.assert_allclose(fl.sum(), ref_f.sum(), rtol=1e-5 if precision == 1 else 1e-12)


@pytest.mark.gpu
def test_trace_skips_removed_packets():
    cfg = CASES["slab"]
    mesh = Mesh(cfg)
    dev = torch.device("cuda")
    x, d, cell, ib, proper, steps = make_packets(mesh, 256, np.float64, seed=3)
    todo = torch.full((256,), -3, dtype=torch.int8, device=dev)
    pool = PacketPool(torch.tensor(x, device=dev), torch.tensor(d, device=dev),
                      torch.tensor(cell, device=dev), torch.tensor(ib, device=dev),
                      torch.tensor(proper, device=dev), torch.tensor(steps, device=dev), todo)
    flux = trace(mesh, pool, "fixed")
    assert int(flux.abs().sum()) == 0
    assert torch.equal(pool.x.cpu(), torch.tensor(x))
