"""Host-side pieces of bench.py's JSON line (no GPU): the per-kernel DRAM
traffic read from the committed ncu summary, the algorithmic bytes of a
solve, and the workload description."""
import importlib.util
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench_module", os.path.join(ROOT, "bench.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def test_traffic_of_both_kernels_from_the_profile():
    b = _bench()
    t = b.ncu_traffic(10_000_000)
    assert set(t) == {"k_forward", "k_peel"}
    assert all(v > 1e9 for v in t.values())          # the queue streams through DRAM
    assert b.ncu_traffic(1_000_000) is None           # captured at 1e7 packets only


def test_algorithmic_bytes_of_a_solve():
    b = _bench()
    c = {"steps": 10, "peel_steps": 5, "hops": 2, "deposits": 3, "emitted": 1}
    assert b.algorithmic_bytes(c) == 8 * 15 + 8 * 2 + 32 * 3 + 128


def test_workload_names_the_configuration():
    from kratos_polrad_b200 import scenes
    b = _bench()
    _, _, cfg = scenes.clump_amr(n_packets=10)
    w = b.workload_config(cfg, 10_000_000)
    assert w["workload"] == "clump_amr_2level" and w["packets_per_gpu"] == 10_000_000
    assert w["l2"].startswith("flushed")


@pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libkpref_p2.so")),
                    reason="reference walk not built")
def test_reference_arm_does_not_load_the_product():
    """The CPU arm builds its scene on the reference's own mesh code and runs
    the restatement: in a fresh process, libkp_b200.so is never mapped, and
    the scene equals the product's (same blocks, coefficients, source cell)."""
    code = ("import sys; sys.path.insert(0, %r)\n"
            "from oracle import ref_scene\n"
            "tab, sig, grid, gn, cfg, cells = ref_scene.clump(1000)\n"
            "maps = open('/proc/self/maps').read()\n"
            "assert 'libkp_b200' not in maps, 'product library mapped'\n"
            "assert 'libkpref_p2' in maps\n"
            "import numpy as np\n"
            "np.save(sys.argv[1], np.concatenate([sig.ravel().astype(np.float64), "
            "tab.xf0.ravel(), [cells[0][0]], cells[0][1]]))\n" % ROOT)
    import subprocess
    import tempfile
    with tempfile.TemporaryDirectory() as d:
        out = os.path.join(d, "scene.npy")
        r = subprocess.run([sys.executable, "-c", code, out], capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        got = np.load(out)
    from kratos_polrad_b200 import scenes
    mesh, sig, cfg = scenes.clump_amr(n_packets=1000)
    ib, cell = mesh.locate([cfg.sources[0].pos])
    xf0, _, _, _ = mesh.geometry(8)
    want = np.concatenate([sig.ravel().astype(np.float64), xf0.ravel(), [ib[0]], cell[0]])
    np.testing.assert_array_equal(got, want)


def test_tangential_polarization_about_sources():
    """A centrosymmetric pattern drawn around two source positions reads its
    own degree about them, and about the image centre much less."""
    import numpy as np
    from kratos_polrad_b200 import scenes
    n, p = 64, 0.1
    cen = np.array([[-10.0, 12.0], [9.0, -14.0]])
    c = (np.arange(n) + 0.5) - n / 2
    Y, X = np.meshgrid(c, c, indexing="ij")
    d2 = (Y[..., None] - cen[:, 0]) ** 2 + (X[..., None] - cen[:, 1]) ** 2
    near = cen[d2.argmin(-1)]
    phi = np.arctan2(X - near[..., 1], Y - near[..., 0])
    img = np.zeros((n, n, 4))
    img[..., 0] = 1.0
    img[..., 1] = -p * np.cos(2 * phi)
    img[..., 2] = p * np.sin(2 * phi)
    assert abs(scenes.tangential_polarization(img, cen) - p) < 1e-12
    assert abs(scenes.tangential_polarization(img)) < 0.5 * p


def test_source_pixels_match_the_peel_off_projection():
    """A source at the image centre sits at offset 0; one displaced along the
    image's vertical axis (+z at inclination 90) moves up by its offset over
    the pixel size."""
    import numpy as np
    from kratos_polrad_b200 import scenes
    from kratos_polrad_b200.config import SOURCE_POINT, Source, TransportConfig
    cfg = TransportConfig(n_packets=1, sources=[Source(SOURCE_POINT, 0, (0.5, 0.5, 0.5)),
                                               Source(SOURCE_POINT, 0, (0.5, 0.5, 0.75))],
                          inclination_deg=90.0, image_center=(0.5, 0.5, 0.5), image_half_width=0.5)
    px = scenes.source_pixels(cfg, 64)
    np.testing.assert_allclose(px[0], [0, 0], atol=1e-12)
    np.testing.assert_allclose(px[1], [0.25 * 64, 0], atol=1e-9)
