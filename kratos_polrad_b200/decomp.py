"""Domain-decomposed solves: packets migrate between ranks that each own part
of the blocks (for meshes whose coefficients do not fit one GPU).

Replaces the reference's off-rank packet registration and MPI exchange loop
(modules/particle/boundary/comm.h:118-239): every rank holds the block
tables of the whole mesh (about 100 B per block) and the coefficients of its
own blocks only.  A solve runs in rounds (``kp_transport_forward_dd``): each
rank processes the records it received (walks, peel-off rays) and, in the
first round, its share of the emissions, and writes every ray that crosses
into another rank's block to that rank's out-queue; the queues are then
exchanged, one all-to-all per record kind, until no rank holds a record.
Each packet's arithmetic is that of the replicated solve, so the int64
tallies summed over the ranks equal ``transport.forward``'s bit for bit.

``solve_emulated`` runs the ranks one after another on one GPU and moves the
queues with device copies; ``solve_distributed`` runs one rank per process
(NCCL, or gloo on CPU for the exchange alone).
"""
from __future__ import annotations

import ctypes
import dataclasses

import numpy as np
import torch

from . import _lib
from ._lib import call, ptr
from .transport import CTallies, CTransportCfg, TALLY_FIXED, Tallies, TransportConfig

WALK_BYTES = 128          # KP_DD_WALK_BYTES
PEEL_BYTES = 96           # KP_DD_PEEL_BYTES
ST_QUEUE_FULL = 1 << 2


class CDDRound(ctypes.Structure):
    _fields_ = [("rank", ctypes.c_int), ("n_ranks", ctypes.c_int),
                ("owner", ctypes.c_void_p), ("block_local", ctypes.c_void_p),
                ("sigma_local", ctypes.c_void_p),
                ("in_walk", ctypes.c_void_p), ("n_in_walk", ctypes.c_longlong),
                ("in_peel", ctypes.c_void_p), ("n_in_peel", ctypes.c_longlong),
                ("emit", ctypes.c_int),
                ("out_walk", ctypes.c_void_p), ("out_walk_rank", ctypes.c_void_p),
                ("cap_walk", ctypes.c_longlong),
                ("out_peel", ctypes.c_void_p), ("out_peel_rank", ctypes.c_void_p),
                ("cap_peel", ctypes.c_longlong),
                ("out_count", ctypes.c_void_p)]


_lib.register("kp_transport_forward_dd", [ctypes.c_void_p, ctypes.POINTER(CTransportCfg),
                                          ctypes.POINTER(CDDRound), ctypes.POINTER(CTallies),
                                          ctypes.c_void_p])


def _morton(level, reg, max_level):
    """Morton key of each block's lower corner at the finest level."""
    pos = reg.astype(np.int64) << (max_level - level)[:, None]
    key = np.zeros(len(level), np.int64)
    for bit in range(21):
        for a in range(3):
            key |= ((pos[:, a] >> bit) & 1) << (3 * bit + a)
    return key


def partition_blocks(mesh, n_ranks: int) -> np.ndarray:
    """Owner rank of every block: contiguous runs of a Morton (Z-order) curve
    over the blocks, with block counts differing by at most one (every block
    has the same number of cells)."""
    if n_ranks < 1:
        raise ValueError("n_ranks must be positive")
    lev, reg = mesh.blocks()
    order = np.argsort(_morton(lev, reg, int(lev.max())), kind="stable")
    owner = np.empty(mesh.n_blocks, np.int32)
    for r, chunk in enumerate(np.array_split(order, n_ranks)):
        owner[chunk] = r
    return owner


class Rank:
    """One rank of a decomposed solve: its coefficients, queues and tallies.

    One out-queue per record kind, each record tagged with its destination
    rank (sorted by destination after the round), sized per round from that
    round's work: every incoming walk or emission leaves at most once, and
    the peel-off rays leaving are bounded by `peel_factor` per walk plus the
    incoming ones; a round that overflows raises (its records are
    incomplete), asking for a larger factor."""

    def __init__(self, mesh, sigma2, owner, rank: int, n_ranks: int, cfg: TransportConfig,
                 peel_factor: int = 16, min_cap: int = 4096, device="cuda"):
        if cfg.n_record:
            raise ValueError("records are not kept in decomposed solves")
        self.mesh, self.cfg, self.rank, self.n_ranks = mesh, cfg, rank, n_ranks
        self.peel_factor, self.min_cap = int(peel_factor), int(min_cap)
        owner = np.asarray(owner, np.int32)
        mine = np.nonzero(owner == rank)[0]
        loc = np.full(mesh.n_blocks, -1, np.int32)
        loc[mine] = np.arange(len(mine), dtype=np.int32)
        cpb = mesh.cells_per_block
        s = torch.as_tensor(np.asarray(sigma2, np.float32)).reshape(mesh.n_blocks, cpb, 2)
        self.sigma_local = s[torch.as_tensor(mine, dtype=torch.long)].reshape(-1, 2).to(device)
        self.owner = torch.as_tensor(owner, device=device)
        self.loc = torch.as_tensor(loc, device=device)
        self.device = device
        self.cap_walk = self.cap_peel = 0
        self.out_walk = self.out_peel = self.out_walk_rank = self.out_peel_rank = None
        self.out_count = torch.zeros(2, dtype=torch.int64, device=device)
        self.in_walk = torch.empty((0, WALK_BYTES), dtype=torch.uint8, device=device)
        self.in_peel = torch.empty((0, PEEL_BYTES), dtype=torch.uint8, device=device)
        # the flux tally (cfg.flux) holds this rank's own blocks, local order
        self.mine = mine
        self.tallies = Tallies(cfg, device=device, n_cells=len(mine) * cpb)
        self.tallies.flux_blocks = mine

    def _ensure(self, cap_walk, cap_peel):
        if cap_walk > self.cap_walk:
            self.cap_walk = int(cap_walk)
            self.out_walk = torch.empty((self.cap_walk, WALK_BYTES), dtype=torch.uint8,
                                        device=self.device)
            self.out_walk_rank = torch.empty(self.cap_walk, dtype=torch.int32, device=self.device)
        if cap_peel > self.cap_peel:
            self.cap_peel = int(cap_peel)
            self.out_peel = torch.empty((self.cap_peel, PEEL_BYTES), dtype=torch.uint8,
                                        device=self.device)
            self.out_peel_rank = torch.empty(self.cap_peel, dtype=torch.int32, device=self.device)

    def _split(self, rec, dest, n):
        """Records [:n] grouped by destination rank (stable)."""
        d = dest[:n].to(torch.int64)
        order = torch.sort(d, stable=True).indices
        grouped = rec[:n][order]
        counts = torch.bincount(d, minlength=self.n_ranks).cpu().tolist()
        return list(torch.split(grouped, counts))

    def round(self, emit_offset: int = 0, emit_n: int = 0, stream=None):
        """Runs one round, emitting (this rank's share of) packets
        [emit_offset, emit_offset + emit_n) of the configuration; returns
        (walks, peels): lists over destination ranks of uint8 record tensors."""
        items = self.in_walk.shape[0] + emit_n
        self._ensure(max(self.min_cap, items),
                     max(self.min_cap, self.peel_factor * items + self.in_peel.shape[0]))
        self.out_count.zero_()
        cfg = dataclasses.replace(self.cfg, packet_offset=self.cfg.packet_offset + emit_offset,
                                  n_packets=emit_n)
        if self.cfg.packets is not None and emit_n > 0:   # this round's table entries
            cfg.packets = self.cfg.packets[emit_offset:emit_offset + emit_n]
        r = CDDRound()
        r.rank, r.n_ranks = self.rank, self.n_ranks
        r.owner, r.block_local, r.sigma_local = ptr(self.owner), ptr(self.loc), ptr(self.sigma_local)
        r.in_walk, r.n_in_walk = ptr(self.in_walk), self.in_walk.shape[0]
        r.in_peel, r.n_in_peel = ptr(self.in_peel), self.in_peel.shape[0]
        r.emit = int(emit_n > 0)
        r.out_walk, r.out_walk_rank, r.cap_walk = (ptr(self.out_walk), ptr(self.out_walk_rank),
                                                   self.cap_walk)
        r.out_peel, r.out_peel_rank, r.cap_peel = (ptr(self.out_peel), ptr(self.out_peel_rank),
                                                   self.cap_peel)
        r.out_count = ptr(self.out_count)
        s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
        call("kp_transport_forward_dd", self.mesh.handle, ctypes.byref(cfg.to_c()),
             ctypes.byref(r), ctypes.byref(self.tallies.to_c()), s)
        nw, npl = (int(v) for v in self.out_count.cpu().tolist())
        full = self.mesh.status() & ST_QUEUE_FULL          # read (and clear) always
        if full or nw > self.cap_walk or npl > self.cap_peel:
            raise RuntimeError(f"rank {self.rank}: out-queue overflow (walks {nw} of "
                               f"{self.cap_walk}, peel-off rays {npl} of {self.cap_peel}); "
                               "raise peel_factor")
        return (self._split(self.out_walk, self.out_walk_rank, nw),
                self._split(self.out_peel, self.out_peel_rank, npl))


def _sum_tallies(ranks):
    mesh = ranks[0].mesh
    out = Tallies(ranks[0].cfg, device=ranks[0].tallies.mu.device, n_cells=mesh.n_cells)
    for rk in ranks:
        for name in ("mu", "image", "image_batch", "counters"):
            getattr(out, name).add_(getattr(rk.tallies, name))
        if out.flux is not None:      # ranks own disjoint blocks
            cpb = mesh.cells_per_block
            idx = torch.as_tensor(rk.mine, dtype=torch.long, device=out.flux.device)
            out.flux.view(-1, cpb)[idx] = rk.tallies.flux.view(-1, cpb)
    return out


def _chunks(n_packets, chunk):
    return [(o, min(chunk, n_packets - o)) for o in range(0, n_packets, chunk)]


def solve_emulated(mesh, sigma2, cfg: TransportConfig, n_ranks: int, owner=None,
                   chunk: int = 1 << 22, peel_factor: int = 16, min_cap: int = 4096,
                   max_rounds: int = 100_000):
    """All ranks on the current GPU, one after another per round; queues move
    by device copies.  Packets are emitted `chunk` per round.  Returns (summed
    Tallies, rounds)."""
    owner = partition_blocks(mesh, n_ranks) if owner is None else np.asarray(owner, np.int32)
    ranks = [Rank(mesh, sigma2, owner, r, n_ranks, cfg, peel_factor, min_cap)
             for r in range(n_ranks)]
    emits = _chunks(cfg.n_packets, max(1, int(chunk)))
    for rounds in range(max_rounds):
        off, n = emits[rounds] if rounds < len(emits) else (0, 0)
        outs = [rk.round(off, n) for rk in ranks]
        moved = 0
        for d, rk in enumerate(ranks):
            rk.in_walk = torch.cat([o[0][d] for o in outs]).contiguous()
            rk.in_peel = torch.cat([o[1][d] for o in outs]).contiguous()
            moved += rk.in_walk.shape[0] + rk.in_peel.shape[0]
        if moved == 0 and rounds + 1 >= len(emits):
            return _sum_tallies(ranks), rounds + 1
    raise RuntimeError("decomposed solve did not finish")


def exchange(parts, record_bytes: int, group=None):
    """All-to-all of per-destination record tensors (uint8 [n, record_bytes]
    each, one per rank): returns the records this rank receives, in source
    rank order.  Two collectives: the counts, then the records."""
    import torch.distributed as dist
    dev = parts[0].device
    send_n = torch.tensor([p.shape[0] for p in parts], dtype=torch.int64, device=dev)
    recv_n = torch.empty_like(send_n)
    dist.all_to_all_single(recv_n, send_n, group=group)
    send = torch.cat(parts).contiguous().view(-1)
    rn = recv_n.cpu().tolist()
    recv = torch.empty(sum(rn) * record_bytes, dtype=torch.uint8, device=dev)
    dist.all_to_all_single(recv, send, [n * record_bytes for n in rn],
                           [p.shape[0] * record_bytes for p in parts], group=group)
    return recv.view(-1, record_bytes)


def solve_distributed(mesh, sigma2, cfg: TransportConfig, owner=None, chunk: int = 1 << 22,
                      peel_factor: int = 16, max_rounds: int = 100_000, group=None):
    """One rank per process (torch.distributed initialised; NCCL on GPUs).
    Every rank takes the same collective steps each round: two all-to-alls
    per record kind and one all-reduce of the records left.  Returns (this
    rank's Tallies summed over all ranks, rounds).  The flux tally (cfg.flux)
    is not summed: it holds this rank's own blocks (``tallies.flux_blocks``,
    local order)."""
    import torch.distributed as dist
    rank, n = dist.get_rank(group), dist.get_world_size(group)
    owner = partition_blocks(mesh, n) if owner is None else np.asarray(owner, np.int32)
    rk = Rank(mesh, sigma2, owner, rank, n, cfg, peel_factor)
    emits = _chunks(cfg.n_packets, max(1, int(chunk)))
    for rounds in range(max_rounds):
        off, m = emits[rounds] if rounds < len(emits) else (0, 0)
        walks, peels = rk.round(off, m)
        rk.in_walk = exchange(walks, WALK_BYTES, group)
        rk.in_peel = exchange(peels, PEEL_BYTES, group)
        left = torch.tensor([rk.in_walk.shape[0] + rk.in_peel.shape[0]], dtype=torch.int64,
                            device=rk.in_walk.device)
        dist.all_reduce(left, group=group)
        if int(left.item()) == 0 and rounds + 1 >= len(emits):
            for name in ("mu", "image", "image_batch", "counters"):
                dist.all_reduce(getattr(rk.tallies, name), group=group)
            return rk.tallies, rounds + 1
    raise RuntimeError("decomposed solve did not finish")
