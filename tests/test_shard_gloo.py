"""Multi-rank sharding on CPU: two gloo ranks, each solving its packet range
with the C restatement, reduce to the single-process tallies bit for bit.

This covers the host logic of the multi-GPU path (packet ranges, the int64
tally all-reduce, the scene split and gather of batched solves); on GPUs the
same functions run with NCCL and the transport kernel in place of the
restatement."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from kratos_polrad_b200 import shard
from oracle import port

pytestmark = pytest.mark.skipif(not port.available(), reason="oracle not built")

KEYS = ("mu", "image", "image_batch", "counters")


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _init(rank, world, port_no):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port_no)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))


def _as_tensors(out):
    return [torch.from_numpy(np.ascontiguousarray(out[k]).view(np.int64).copy()) for k in KEYS]


def _packets_worker(rank, world, port_no, weak, name):
    import sys
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    from transport_cases import case, run_oracle
    _init(rank, world, port_no)
    try:
        mesh, sig, t = case(name)
        t = t.__class__(**{**t.__dict__, "n_record": 0, "n_packets": 600})
        mine = _as_tensors(run_oracle(mesh, sig, shard.shard_config(t, rank, world, weak)))
        shard.reduce_tallies(mine)
        if rank == 0:
            n_all = t.n_packets * world if weak else t.n_packets
            full = _as_tensors(run_oracle(mesh, sig, t.__class__(**{**t.__dict__,
                                                                   "n_packets": n_all})))
            for k, a, b in zip(KEYS, mine, full):
                assert torch.equal(a, b), k
            assert int(mine[3][7]) == n_all                      # KP_CNT_EMITTED
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("weak", [True, False])
def test_sharded_packets_reduce_to_single_run(weak):
    mp.spawn(_packets_worker, args=(2, _free_port(), weak, "amr_point"), nprocs=2, join=True)


def _scenes_worker(rank, world, port_no):
    import sys
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    from transport_cases import case, run_oracle
    _init(rank, world, port_no)
    try:
        mesh, sig, t = case("slab")
        n_scenes = 5
        scenes = [(t.__class__(**{**t.__dict__, "n_record": 0, "n_packets": 200 + 50 * k,
                                  "stream_id": k}), (1.0 + 0.3 * k) * sig)
                  for k in range(n_scenes)]
        lo, hi = shard.scene_range(n_scenes, rank, world)
        local = torch.stack([torch.from_numpy(run_oracle(mesh, s, c)["mu"]) for c, s in scenes[lo:hi]])
        got = shard.gather_scene_tallies(local, n_scenes, rank, world)
        if rank == 0:
            want = torch.stack([torch.from_numpy(run_oracle(mesh, s, c)["mu"]) for c, s in scenes])
            assert torch.equal(got, want)
        else:
            assert got is None
    finally:
        dist.destroy_process_group()


def test_scene_split_gathers_every_scene():
    mp.spawn(_scenes_worker, args=(2, _free_port()), nprocs=2, join=True)


def test_packet_ranges_cover_ids_once():
    for n, world in [(10, 3), (7, 7), (5, 8), (0, 2), (1_000_003, 4)]:
        spans = [shard.packet_range(n, r, world, weak=False) for r in range(world)]
        assert sum(c for _, c in spans) == n
        assert all(spans[r][0] + spans[r][1] == spans[r + 1][0] for r in range(world - 1))
        assert max(c for _, c in spans) - min(c for _, c in spans) <= 1
    assert shard.packet_range(100, 3, 4) == (300, 100)
    with pytest.raises(ValueError):
        shard.packet_range(10, 4, 4)
