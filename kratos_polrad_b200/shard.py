"""Multi-GPU sharding of a solve: one process per GPU, packets partitioned by id.

Packets are independent and every random number is keyed by (seed, global
packet id), so a contiguous packet-id range per rank reproduces the
single-GPU solve: the int64 fixed-point tallies of the ranks sum, in any
order, to the single-GPU tallies bit for bit (one all-reduce of int64 sums at
the end of a solve).  Float tallies (KP_TALLY_FLOAT) sum to the same value up
to float rounding.  This replaces the reference's packet migration between
ranks (modules/particle/boundary/comm.h:118-239): with the mesh replicated
on every GPU, no packet ever changes rank.

Batched solves split the scene list instead (contiguous scene ranges, no
collective in the data path) and gather the per-scene tallies on one rank.
"""
from __future__ import annotations

import dataclasses

import torch
import torch.distributed as dist


def packet_range(n_packets: int, rank: int, world: int, weak: bool = True):
    """(packet_offset, n_packets) of this rank.

    weak=True: every rank solves ``n_packets`` packets, rank r taking ids
    [r n, (r + 1) n) (fixed work per GPU).  weak=False: the ``n_packets`` ids
    are cut into ``world`` contiguous ranges whose sizes differ by at most
    one (fixed total work)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside world of {world}")
    if n_packets < 0:
        raise ValueError("negative packet count")
    if weak:
        return rank * n_packets, n_packets
    q, r = divmod(n_packets, world)
    start = rank * q + min(rank, r)
    return start, q + (1 if rank < r else 0)


def shard_config(cfg, rank: int, world: int, weak: bool = True):
    """The rank's TransportConfig: same seed and sources, its own packet range
    (added to the configuration's own packet_offset)."""
    off, n = packet_range(cfg.n_packets, rank, world, weak)
    return dataclasses.replace(cfg, packet_offset=cfg.packet_offset + off, n_packets=n)


def reduce_tallies(tensors, group=None):
    """Sums the tally tensors over the ranks in place (one all-reduce each;
    a no-op without an initialised process group or with one rank)."""
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size(group) == 1:
        return tensors
    for t in tensors:
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return tensors


def scene_range(n_scenes: int, rank: int, world: int):
    """Contiguous [start, stop) of the scenes this rank solves in a batched run."""
    start, n = packet_range(n_scenes, rank, world, weak=False)
    return start, start + n


def gather_scene_tallies(local: torch.Tensor, n_scenes: int, rank: int, world: int, dst: int = 0,
                         group=None):
    """Collects per-scene tallies ``local`` [scenes of this rank, ...] into
    [n_scenes, ...] on rank ``dst`` (returns None on the other ranks)."""
    if world == 1:
        return local
    counts = [scene_range(n_scenes, r, world) for r in range(world)]
    width = max(b - a for a, b in counts)
    pad = torch.zeros((width,) + tuple(local.shape[1:]), dtype=local.dtype, device=local.device)
    pad[: local.shape[0]] = local
    bufs = [torch.empty_like(pad) for _ in range(world)] if rank == dst else None
    dist.gather(pad, bufs, dst=dst, group=group)
    if rank != dst:
        return None
    return torch.cat([b[: hi - lo] for b, (lo, hi) in zip(bufs, counts)], 0)
