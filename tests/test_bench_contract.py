"""Host-side pieces of bench.py's JSON line (no GPU): the per-kernel DRAM
traffic read from the committed ncu summary, the algorithmic bytes of a
solve, and the workload description."""
import importlib.util
import os

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
