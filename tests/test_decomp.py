"""Domain-decomposed solves: block partition and record exchange (CPU, gloo),
and ranks emulated on one GPU against the replicated solve (bit for bit)."""
import dataclasses
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from kratos_polrad_b200 import Mesh, decomp
from meshcases import AMR_BOX, THREE_LEVEL


@pytest.mark.parametrize("cfg", [AMR_BOX, THREE_LEVEL])
@pytest.mark.parametrize("n", [1, 2, 3, 8])
def test_partition_covers_blocks_evenly(cfg, n):
    m = Mesh(cfg)
    owner = decomp.partition_blocks(m, n)
    counts = np.bincount(owner, minlength=n)
    assert owner.shape == (m.n_blocks,) and counts.sum() == m.n_blocks
    assert counts.max() - counts.min() <= 1


def test_partition_is_spatially_compact():
    """Z-order runs: a rank's blocks touch each other far more than random."""
    m = Mesh(AMR_BOX)
    owner = decomp.partition_blocks(m, 4)
    ids, _, _ = m.neighbors()
    same = [(owner[b] == owner[n]) for b in range(m.n_blocks) for n in ids[b] if n >= 0]
    assert np.mean(same) > 0.6


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _exchange_worker(rank, world, port):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        def rec(src, dst, k):          # record k from src to dst
            return torch.full((decomp.WALK_BYTES,), (src * 7 + dst * 3 + k) % 251, dtype=torch.uint8)
        sizes = [[(s + 2 * d) % 3 for d in range(world)] for s in range(world)]   # [src][dst]
        parts = [torch.stack([rec(rank, d, k) for k in range(sizes[rank][d])])
                 if sizes[rank][d] else torch.empty((0, decomp.WALK_BYTES), dtype=torch.uint8)
                 for d in range(world)]
        got = decomp.exchange(parts, decomp.WALK_BYTES)
        want = [rec(s, rank, k) for s in range(world) for k in range(sizes[s][rank])]
        want = torch.stack(want) if want else torch.empty((0, decomp.WALK_BYTES), dtype=torch.uint8)
        assert torch.equal(got, want)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_exchange_delivers_every_record(world):
    mp.spawn(_exchange_worker, args=(world, _free_port()), nprocs=world, join=True)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["amr_point", "hg_multi", "slab", "table"])
@pytest.mark.parametrize("n_ranks", [2, 3])
def test_emulated_ranks_equal_replicated_solve(name, n_ranks):
    from kratos_polrad_b200.transport import Tallies, forward
    from transport_cases import case, to_device
    mesh, sig, t = case(name)
    t = to_device(dataclasses.replace(t, n_record=0))
    mesh.set_sigma(sig)
    ref = forward(mesh, t, Tallies(t))
    torch.cuda.synchronize()
    got, rounds = decomp.solve_emulated(mesh, sig, t, n_ranks, chunk=t.n_packets // 3 + 1)
    torch.cuda.synchronize()
    assert mesh.status() == 0 and rounds > 1
    for k in ("mu", "image", "image_batch", "counters"):
        assert torch.equal(getattr(got, k), getattr(ref, k)), k


@pytest.mark.gpu
def test_queue_overflow_is_reported():
    from transport_cases import case
    mesh, sig, t = case("amr_point")
    t = dataclasses.replace(t, n_record=0)
    with pytest.raises(RuntimeError, match="overflow"):
        decomp.solve_emulated(mesh, sig, t, 2, peel_factor=0, min_cap=1)
    assert mesh.status() == 0          # the flag was read and cleared


@pytest.mark.gpu
@pytest.mark.parametrize("n_ranks", [2, 3])
def test_emulated_ranks_flux_tally(n_ranks):
    """Each rank tallies the path-length flux of its own blocks; put together
    they equal the replicated solve's flux bit for bit."""
    from kratos_polrad_b200.transport import Tallies, forward
    from transport_cases import case
    mesh, sig, t = case("amr_point")
    t = dataclasses.replace(t, n_record=0, flux=True, flux_fx_shift=24)
    mesh.set_sigma(sig)
    ref = forward(mesh, t, Tallies(t, n_cells=mesh.n_cells))
    torch.cuda.synchronize()
    got, rounds = decomp.solve_emulated(mesh, sig, t, n_ranks, chunk=t.n_packets // 3 + 1)
    torch.cuda.synchronize()
    assert mesh.status() == 0 and rounds > 1
    assert int(ref.flux.sum()) > 0
    assert torch.equal(got.flux, ref.flux)
    assert torch.equal(got.image, ref.image)
