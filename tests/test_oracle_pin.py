"""Pins the C restatement oracle to the reference's own code (both on CPU).

The walk of oracle/kp_oracle.c, fed the reference harness's block tables,
must reproduce the reference's cart_t::proc bit for bit: final positions,
cells, blocks, budgets, todo flags, float flux sums and int64 flux sums.
"""
import numpy as np
import pytest

from kratos_polrad_b200 import Mesh
from oracle import port, refharness
from meshcases import CASES
from test_trace_gpu import make_packets, perm_ref_to_prod

pytestmark = pytest.mark.skipif(not (refharness.available(1) and port.available()),
                                reason="oracle libraries not built")


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("precision", [1, 2])
def test_port_matches_reference(name, precision):
    cfg = CASES[name]
    ftype = np.float32 if precision == 1 else np.float64
    mesh = Mesh(cfg)
    ref = refharness.RefMesh(cfg.to_ini(), precision)
    inv = np.argsort(perm_ref_to_prod(mesh, ref))
    x, d, cell, ib, proper, steps = make_packets(mesh, 2048, ftype, seed=5 + precision)
    r = ref.trace(x, d, cell, inv[ib], proper, steps, fx_shift=30)
    o = port.trace(port.Tables.from_ref(ref), 4 if precision == 1 else 8,
                   x, d, cell, inv[ib], proper, steps, fx_shift=30)
    for k in ("x", "cell", "ib", "step", "todo", "flux", "flux_fx"):
        np.testing.assert_array_equal(o[k], r[k], err_msg=k)


@pytest.mark.parametrize("name", ["amr_periodic", "three_level"])
def test_port_on_product_tables(name):
    """The product's tables drive the restatement to the same result."""
    cfg = CASES[name]
    mesh = Mesh(cfg)
    ref = refharness.RefMesh(cfg.to_ini(), 2)
    perm = perm_ref_to_prod(mesh, ref)
    inv = np.argsort(perm)
    x, d, cell, ib, proper, steps = make_packets(mesh, 1024, np.float64, seed=9)
    a = port.trace(port.Tables.from_mesh(mesh, 8), 8, x, d, cell, ib, proper, steps)
    b = port.trace(port.Tables.from_ref(ref), 8, x, d, cell, inv[ib], proper, steps)
    np.testing.assert_array_equal(a["x"], b["x"])
    np.testing.assert_array_equal(np.where(a["ib"] >= 0, inv[np.maximum(a["ib"], 0)], a["ib"]), b["ib"])
    cpb = mesh.cells_per_block
    np.testing.assert_array_equal(a["flux_fx"].reshape(-1, cpb)[perm], b["flux_fx"].reshape(-1, cpb))
