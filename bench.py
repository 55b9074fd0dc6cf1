#!/usr/bin/env python
"""Benchmark of the polarized photon-packet transport (packet-steps/s).

Workload: the static 2-level AMR clump scene (root 128^3 in 16^3 blocks,
refined x2 where the density exceeds 3x its mean; Gaussian clump peak 100,
FWHM 0.1 box; centre-to-edge extinction depth 5; albedo log-uniform in
[0.5, 0.99], seed 2; 1e7 packets from a central isotropic point source;
128x128 peel-off I/Q/U/V image; int64 fixed-point tallies).  A step is one
forward solve of all packets.  Packet-steps are walk segments plus peel-off
segments (reported separately).

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Under torchrun each rank solves its own 1e7 packets (its own packet-id
range: weak scaling) and the int64 tallies are summed with one NCCL
all-reduce per step.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import dataclasses
import math
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "packet-steps/s (walk + peel-off segments), 2-level AMR clump, 1e7 packets"
UNIT = "packet-steps/s"
L2_FLUSH_BYTES = 512 << 20      # > 126 MB L2


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--packets", type=float, default=1e7)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--peel-order", default="auto", choices=["auto", "queue", "cell"],
                   help="--workload large: the order the peel-off queue is marched in "
                        "(kp_mesh_peel_order; auto sorts by starting cell on this scene)")
    p.add_argument("--workload", default="clump",
                   choices=["clump", "batched", "diff", "large", "decomp", "trace", "sph",
                            "refine", "bio", "resume"])
    p.add_argument("--budget", type=int, default=256,
                   help="resume workload: walk segments per packet and call")
    return p.parse_args()


def workload_config(cfg, n_packets):
    return {"workload": "clump_amr_2level", "root_cells": "128^3", "block_cells": "16^3",
            "levels": 2, "tau_edge": 5.0, "albedo": "log-uniform [0.5,0.99] seed 2",
            "packets_per_gpu": int(n_packets), "source": "central isotropic point",
            "image": f"{cfg.image_n}x{cfg.image_n} IQUV peel-off, inclination "
                     f"{cfg.inclination_deg:g} deg", "tallies": "int64 fixed point",
            "l2": "flushed between timed steps (512 MiB write)"}


class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons while the timed region runs."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index, self.proc, self.lines = index, None, []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [v.strip() for v in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def ncu_traffic(n_packets):
    """DRAM bytes (read + write) of the two launches of one solve, per kernel,
    from the committed ncu summary (profiles/k_forward_clump_traffic.txt),
    when it was captured on this packet count, else None."""
    p = os.path.join(ROOT, "profiles", "k_forward_clump_traffic.txt")
    try:
        kv = {}
        for ln in open(p):
            if "=" in ln and not ln.lstrip().startswith("#"):
                k, v = ln.split("=", 1)
                kv[k.strip()] = float(v)
        if int(kv["packets"]) != int(n_packets):
            return None
        return {k: kv[k + ".dram_read_bytes"] + kv[k + ".dram_write_bytes"]
                for k in ("k_forward", "k_peel")}
    except (OSError, KeyError, ValueError):
        return None


def algorithmic_bytes(c):
    """Bytes the solve must move: 8 B of (sigma_sca, sigma_abs) per walk or
    peel-off segment, 8 B per block hand-off, 32 B (int64 IQUV) per tally
    deposit, and a 64-byte packet state written at emission and read at the
    end (2 x 64 B per packet)."""
    return (8 * (c["steps"] + c["peel_steps"]) + 8 * c["hops"] + 32 * c["deposits"]
            + 128 * c["emitted"])


def cpu_baseline(mesh, sigma2, cfg, budget_s=20.0, threads=None):
    """Times the oracle's C restatement on the host cores over a bounded
    sample of the same workload (packets 0..n of the same scene), on the
    product mesh's tables."""
    from oracle import port
    tab = port.Tables.from_mesh(mesh, 8)
    lev, reg = mesh.blocks()
    roots = [int(round((mesh.x_max[a] - mesh.x_min[a]) / (tab.dx0[0, a] * mesh.nc[a] * 2 ** lev[0])))
             for a in range(3)]
    grid, gn = port.lookup_grid(lev, reg, roots)
    cells = []
    for s in cfg.sources:
        ib, cell = mesh.locate([s.pos])
        cells.append((ib[0], cell[0]))
    return cpu_baseline_tables(tab, sigma2, grid, gn, cfg, cells, budget_s, threads)


def cpu_baseline_tables(tab, sigma2, grid, gn, cfg, cells, budget_s=20.0, threads=None):
    """The restatement timed on the host cores over a bounded sample
    (packets 0..n of the scene), sized to about budget_s of CPU work."""
    from oracle import port
    threads = threads or os.cpu_count() or 1
    # calibrate on a small sample, then size the timed sample to the budget
    probe = dataclasses.replace(cfg, n_packets=2000, n_record=0)
    t0 = time.perf_counter()
    port.transport(tab, sigma2, grid, gn, probe, cells)
    per_pkt = (time.perf_counter() - t0) / 2000
    chunk = max(50, int(budget_s / per_pkt / threads / 4))
    n_chunks = threads * 4

    def work(k):
        c = dataclasses.replace(cfg, n_packets=chunk, packet_offset=k * chunk, n_record=0)
        return port.transport(tab, sigma2, grid, gn, c, cells)["counters"]

    t0 = time.perf_counter()
    with cf.ThreadPoolExecutor(threads) as ex:
        outs = list(ex.map(work, range(n_chunks)))
    dt = time.perf_counter() - t0
    tot = sum(o.astype(float) for o in outs)
    steps = float(tot[0] + tot[1])
    return {"value": steps / dt, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{chunk * n_chunks} packets (ids 0..{chunk * n_chunks - 1}) of the same scene, "
                      f"{steps:.3g} packet-steps in {dt:.1f} s"}


def run_reference(args, rank, world):
    """--impl reference: the CPU implementation of this path on the host cores.

    The reference has no scattering physics for this workload, so the timed
    CPU implementation is the oracle's restatement (kind "port").  The scene
    is built on the reference's own tree/meshgen/proxy code (oracle/_ref);
    this arm never loads the product library."""
    if rank != 0:
        return
    from oracle import ref_scene
    tab, sigma2, grid, gn, cfg, cells = ref_scene.clump(int(args.packets))
    vals = []
    for k in range(args.warmup + args.steps):
        cb = cpu_baseline_tables(tab, sigma2, grid, gn, cfg, cells, budget_s=8.0)
        if k >= args.warmup:
            vals.append(cb["value"])
    v = statistics.mean(vals)
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64 positions / f32 Stokes",
            "data": "synthetic", "config": workload_config(cfg, args.packets),
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": cb["cores"], "kind": "port",
                             "sample": cb["sample"],
                             "tables": "built by the reference's tree/meshgen/proxy code "
                                       "(oracle/_ref/libkpref_p2.so)"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def measure_batched(steps, warmup, clocks=None):
    """The 256-scene batched solve (scenes.batched_cubes: uniform cubes with
    sides from {16,32,48,64,96}, tau log-uniform [0.1,20], albedo uniform
    [0.3,1], seed 3, 1e5-1e6 packets in proportion to tau, 32-bin mu tallies)
    in one autotuned, graph-replayed persistent launch, against sequential
    single-scene launches of the same packets (same tallies, bit for bit).
    Under torchrun each rank solves a contiguous range of the scenes (no
    collective in the data path); the per-scene tallies are gathered on rank
    0 (the other ranks report gathered_scenes None)."""
    import contextlib
    import torch
    from kratos_polrad_b200 import scenes, shard
    from kratos_polrad_b200.batch import Batch
    from kratos_polrad_b200.transport import Tallies, forward
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    sc_all, cfg = scenes.batched_cubes()
    lo, hi = shard.scene_range(len(sc_all), rank, world)
    sc = sc_all[lo:hi]
    for mesh, sig, *_ in sc:
        mesh.set_sigma(sig)
    b = Batch([(m, n, sid, src) for m, _, n, sid, src in sc])
    tune = b.autotune(cfg, fraction=0.05)
    s = torch.cuda.Stream()
    cnt = torch.zeros(10, dtype=torch.int64, device="cuda")
    mu = b.new_mu(cfg)
    with torch.cuda.stream(s):
        for _ in range(warmup):
            mu.zero_()
            b.forward(cfg, mu=mu, graph=True, stream=s.cuda_stream)
    s.synchronize()
    times = []
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    with (clocks if clocks is not None else contextlib.nullcontext()):
        for k in range(steps):
            mu.zero_()
            cnt.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            with torch.cuda.stream(s):
                e0.record(s)
                b.forward(cfg, mu=mu, counters=cnt, graph=True, stream=s.cuda_stream)
                e1.record(s)
            s.synchronize()
            times.append(e0.elapsed_time(e1))
    red = torch.tensor([statistics.mean(times)], dtype=torch.float64, device="cuda")
    shard_max(red)
    batched_ms = float(red.item())
    shard.reduce_tallies([cnt])
    c = cnt.cpu().numpy()
    n_steps = int(c[0] + c[1])
    mu_all = shard.gather_scene_tallies(mu, len(sc_all), rank, world)
    # sequential plain launches of the same scenes
    seq_mu = torch.zeros_like(mu)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    cfgs = [dataclasses.replace(cfg, n_packets=n, stream_id=sid, sources=[src])
            for (_, _, n, sid, src) in sc]
    tals = [Tallies(cc) for cc in cfgs]
    for (mesh, *_), cc, tl in zip(sc, cfgs, tals):          # warm-up
        forward(mesh, cc, tl)
    torch.cuda.synchronize()
    for tl in tals:
        tl.zero_()
    e0.record()
    for (mesh, *_), cc, tl in zip(sc, cfgs, tals):
        forward(mesh, cc, tl)
    e1.record()
    torch.cuda.synchronize()
    red = torch.tensor([e0.elapsed_time(e1)], dtype=torch.float64, device="cuda")
    shard_max(red)
    seq_ms = float(red.item())
    for k, tl in enumerate(tals):
        seq_mu[k] = tl.mu
    differs = torch.tensor([0 if torch.equal(seq_mu, mu) else 1], dtype=torch.int64, device="cuda")
    shard_max(differs)                                   # any rank whose scenes differ
    return {"value": n_steps / (batched_ms / 1e3), "unit": UNIT, "ms_per_step": batched_ms,
            "steps": steps, "warmup": warmup,
            "config": {"workload": "batched_cubes_256", "scenes": len(sc_all),
                       "packets": int(sum(n for _, _, n, _, _ in sc_all)),
                       "cells": int(sum(m.n_cells for m, *_ in sc_all)),
                       "tallies": "int64 fixed point",
                       "launch": "one persistent launch replayed from a CUDA graph",
                       "split": "contiguous scene ranges per rank, tallies gathered on rank 0"},
            # rank 0 holds every scene's tallies, the others none
            "gathered_scenes": None if mu_all is None else int(mu_all.shape[0]),
            "autotune": tune,
            "sequential_ms": seq_ms, "sequential_value": n_steps / (seq_ms / 1e3),
            "batched_over_sequential": seq_ms / batched_ms,
            "tallies_identical_to_sequential": bool(differs.item() == 0)}


def run_batched(args):
    """--workload batched: the batched solve on its own JSON line."""
    rank, world, local = _init_ranks()
    clk = ClockSampler(local)
    r = measure_batched(args.steps, args.warmup, clk)
    if rank == 0:
        line = {"metric": "packet-steps/s, 256-scene batched solve", "value": r["value"],
                "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": r["ms_per_step"], "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64 positions / f32 Stokes", "data": "synthetic",
                "config": r["config"],
                **{k: r[k] for k in ("gathered_scenes", "autotune", "sequential_ms",
                                     "sequential_value", "batched_over_sequential",
                                     "tallies_identical_to_sequential")},
                "clocks": clk.summary()}
        print(json.dumps(line), flush=True)
    _finish_ranks(world)


def _init_ranks():
    """(rank, world, local rank); initialises NCCL under torchrun."""
    import torch
    import torch.distributed as dist
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(local)
    if world > 1 and not dist.is_initialized():
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    return rank, world, local


def _finish_ranks(world):
    import torch.distributed as dist
    if world > 1 and dist.is_initialized():
        dist.barrier()
        dist.destroy_process_group()


def shard_max(t):
    """In-place max over the ranks (no-op with one rank)."""
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t


def _timed(fn):
    import torch
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    out = fn()
    e1.record()
    torch.cuda.synchronize()
    return out, e0.elapsed_time(e1)


def _gradient_check(mesh, sig, cfg, g_img, rng, n_check=1_200_000_000, n_batch=20, n_dirs=8,
                    n_cells=16, n_cell_check=50_000_000, h=0.1):
    """Paired batch-means comparison of the path-replay gradient with
    common-random-number central differences of the same estimator.

    The functional is F = sum over packets of <a, image contribution> with
    a = g_img / max|g_img| (the loss linearised at the forward solution).
    Packets [0, n_check) are cut into n_batch ranges; on each range the
    adjoint and the differences use the same packets.

    Blob directions (the 2% bar): Gaussian density blobs of radius 0.08 box
    (both coefficients scaled by 1 +- h phi, albedo unchanged; h = 0.1: the
    differences' noise comes from the packets whose paths the perturbation
    changes, a fraction that grows like h, so their standard error falls
    like h^-1/2 while the central difference's bias grows like h^2).  Their
    centres are the points of a 16^3 grid over the box with the largest
    |dF/d blob| (at least 0.15 box apart), that derivative taken from a
    gradient of other packets (ids from 5e9), so that the choice does not
    favour the checked estimate; large derivatives keep the differences'
    relative noise low.  For each: the difference's mean, its batch-means standard
    error, and the adjoint's relative difference from it; a direction passes
    when that is within 2% and the standard error is within 1%.
    Single cells (a z-score check, too noisy for a 2% bar): n_cells cells
    among the 2000 of largest |dF/dsigma_sca| (sigma_sca +- 10%), on the
    first n_cell_check packets."""
    import numpy as np
    import torch
    from kratos_polrad_b200 import scenes
    from kratos_polrad_b200.adjoint import gradients
    from kratos_polrad_b200.transport import Tallies, forward
    a = (g_img / g_img.abs().max()).float().contiguous()
    a64 = a.double()
    mesh.set_sigma(sig)
    sel = dataclasses.replace(cfg, n_packets=20_000_000, packet_offset=5_000_000_000, n_record=0)
    gs_sel, ga_sel = gradients(mesh, sel, a, 24)
    g_sel = gs_sel.cpu().numpy()
    xc = scenes.cell_centers(mesh)
    xc_d = torch.tensor(xc, device="cuda", dtype=torch.float64)
    w_sel = (gs_sel.double() * torch.tensor(sig[:, 0], device="cuda", dtype=torch.float64)
             + ga_sel.double() * torch.tensor(sig[:, 1], device="cuda", dtype=torch.float64))
    lo, hi = xc.min(0), xc.max(0)
    grid = np.stack(np.meshgrid(*[np.linspace(lo[k], hi[k], 16) for k in range(3)],
                                indexing="ij"), -1).reshape(-1, 3)
    blob = np.array([float((w_sel * torch.exp(-((xc_d - torch.tensor(c, device="cuda")) ** 2)
                                              .sum(1) / (2 * 0.08 ** 2))).sum()) for c in grid])
    centres = []
    for k in np.argsort(-np.abs(blob)):   # blob centres at least 0.15 box apart
        if all(np.linalg.norm(grid[k] - c) > 0.15 for c in centres):
            centres.append(grid[k])
        if len(centres) == n_dirs:
            break
    order = np.argsort(-np.abs(g_sel))
    phis = [np.exp(-((xc - c) ** 2).sum(1) / (2 * 0.08 ** 2)) for c in centres]
    cells = rng.choice(order[:2000], n_cells, replace=False)
    sig_d = torch.tensor(sig, device="cuda", dtype=torch.float64)
    phi_d = torch.tensor(np.stack(phis, 1), device="cuda", dtype=torch.float64)
    cells_d = torch.tensor(cells, device="cuda")

    def ranges(n_total):
        nb = n_total // n_batch
        return [dataclasses.replace(cfg, n_packets=nb, packet_offset=b * nb, n_record=0)
                for b in range(n_batch)]

    cb, cc = ranges(n_check), ranges(n_cell_check)
    adj_b = np.zeros((n_batch, n_dirs))
    adj_c = np.zeros((n_batch, n_cells))
    for b in range(n_batch):
        gs, ga = gradients(mesh, cb[b], a, 24)
        adj_b[b] = ((gs * sig_d[:, 0])[:, None] * phi_d
                    + (ga * sig_d[:, 1])[:, None] * phi_d).sum(0).cpu().numpy()
        adj_c[b] = gradients(mesh, cc[b], a, 24)[0][cells_d].cpu().numpy()

    def scores(s2, ranges_):
        mesh.set_sigma(s2)
        out = []
        for c in ranges_:
            tal = forward(mesh, c, Tallies(c))
            out.append(float((tal.image.double() * a64).sum()) * tal.scale())
        return np.array(out)

    fd_b = np.zeros_like(adj_b)
    fd_c = np.zeros_like(adj_c)
    for k, phi in enumerate(phis):
        sp = (sig * (1 + h * phi)[:, None]).astype(np.float32)
        sm = (sig * (1 - h * phi)[:, None]).astype(np.float32)
        fd_b[:, k] = (scores(sp, cb) - scores(sm, cb)) / (2 * h)
    for j, cell in enumerate(cells):
        sp, sm = sig.copy(), sig.copy()
        sp[cell, 0] *= 1.1
        sm[cell, 0] *= 0.9
        fd_c[:, j] = (scores(sp, cc) - scores(sm, cc)) / (float(sp[cell, 0]) - float(sm[cell, 0]))
    mesh.set_sigma(sig)
    sq = np.sqrt(n_batch)
    fd_mean, fd_se = fd_b.mean(0), fd_b.std(0, ddof=1) / sq
    adj_mean = adj_b.mean(0)
    rel = np.abs(adj_mean - fd_mean) / np.abs(fd_mean)
    rel_se = fd_se / np.abs(fd_mean)
    d = adj_b - fd_b
    zb = d.mean(0) / (d.std(0, ddof=1) / sq)
    dc = adj_c - fd_c
    zc = dc.mean(0) / (dc.std(0, ddof=1) / sq)
    ok = (rel <= 0.02) & (rel_se <= 0.01)
    return {"packets": n_check, "batches": n_batch, "h": h,
            "blob_directions": {"n": n_dirs, "fd": [float(v) for v in fd_mean],
                                "fd_rel_std_err": [round(float(v), 5) for v in rel_se],
                                "adjoint": [float(v) for v in adj_mean],
                                "rel_diff": [round(float(v), 5) for v in rel],
                                "max_rel_diff": float(rel.max()),
                                "within_2pct_with_se_below_1pct": int(ok.sum()),
                                "paired_z": [round(float(v), 2) for v in zb]},
            "cells": {"n": n_cells, "packets": n_cell_check,
                      "frac_abs_z_below_3": float(np.mean(np.abs(zc) < 3)),
                      "mean_z2": float(np.mean(zc ** 2)), "max_abs_z": float(np.abs(zc).max())},
            "note": "adjoint vs common-random-number central differences on the same packets "
                    "(paired batch means); blob centres chosen from other packets"}


def run_diff(args):
    """Differentiable workload: 96^3 lognormal field (std of ln rho 1.0,
    k^-11/3, seed 4), albedo 0.9, Rayleigh, 64x64 Q/U image at 60 deg; loss =
    L2 distance (Q, U) to the image of the field perturbed by 5% Gaussian
    noise.  Times the forward and the path-replay gradient of 1e8 packets,
    then checks the gradient against common-random-number central differences
    (blob directions and single cells, paired batch means)."""
    import numpy as np
    import torch
    from kratos_polrad_b200 import scenes
    from kratos_polrad_b200.adjoint import TransportImage
    n_pk = int(args.packets) if args.packets != 1e7 else 100_000_000
    mesh, sig, cfg, _ = scenes.lognormal_cube(n_packets=n_pk)
    rng = np.random.default_rng(4)
    sig_t = (sig * (1 + 0.05 * rng.normal(size=sig.shape))).astype(np.float32)
    dev = torch.device("cuda")
    with torch.no_grad():
        target = TransportImage.apply(torch.tensor(sig_t[:, 0], device=dev, dtype=torch.float64),
                                      torch.tensor(sig_t[:, 1], device=dev, dtype=torch.float64),
                                      mesh, cfg)

    def loss_of(s):
        img = TransportImage.apply(s[:, 0], s[:, 1], mesh, cfg)
        return ((img - target)[..., 1:3] ** 2).sum(), img

    s = torch.tensor(sig, device=dev, dtype=torch.float64)
    for _ in range(max(1, args.warmup)):
        x = s.clone().requires_grad_(True)
        loss_of(x)[0].backward()
    x = s.clone().requires_grad_(True)
    with ClockSampler(0) as clk:
        (L, img), t_fwd = _timed(lambda: loss_of(x))
        _, t_bwd = _timed(lambda: L.backward())
    g = x.grad[:, 0].detach().cpu().numpy()
    g_img = torch.zeros_like(img)
    g_img[..., 1:3] = 2 * (img.detach() - target)[..., 1:3]
    check = None if args.no_cpu_baseline else _gradient_check(mesh, sig, cfg, g_img, rng)
    line = {"metric": "path-replay gradient, 96^3 lognormal, Q/U image loss", "unit": "ms",
            "value": t_bwd, "higher_is_better": False, "n_gpus": 1,
            "config": {"workload": "lognormal_96_diff", "packets": n_pk, "cells": mesh.n_cells},
            "forward_ms": t_fwd, "gradient_ms": t_bwd, "gradient_cost_vs_forward": t_bwd / t_fwd,
            "gradient_check": check, "clocks": clk.summary()}
    print(json.dumps(line), flush=True)


def run_decomp(args):
    """Domain-decomposed solve of the clump scene: the blocks split over 4
    ranks (Z-order runs), each holding only its own coefficients, emulated one
    after another on this GPU with the out-queues moved by device copies;
    against the replicated solve of the same packets (tallies must agree bit
    for bit).  Under torchrun each process is one rank (NCCL all-to-all)."""
    import torch
    import torch.distributed as dist
    from kratos_polrad_b200 import decomp, scenes, shard
    from kratos_polrad_b200.transport import Tallies, forward
    rank, world, _ = _init_ranks()
    n_pk = int(args.packets)
    mesh, sig, cfg = scenes.clump_amr(n_packets=n_pk)
    mesh.set_sigma(sig)
    ref = forward(mesh, cfg, Tallies(cfg))
    torch.cuda.synchronize()
    _, t_rep = _timed(lambda: forward(mesh, cfg, Tallies(cfg)))
    n_ranks = 4 if world == 1 else world
    if world == 1:
        decomp.solve_emulated(mesh, sig, dataclasses.replace(cfg, n_packets=min(n_pk, 100_000)),
                              n_ranks)
        (tal, rounds), t_dd = _timed(lambda: decomp.solve_emulated(mesh, sig, cfg, n_ranks))
    else:
        dist.barrier()
        (tal, rounds), t_dd = _timed(lambda: decomp.solve_distributed(mesh, sig, cfg))
        t = torch.tensor([t_dd], dtype=torch.float64, device="cuda")
        shard_max(t)
        t_dd = float(t.item())
        shard.reduce_tallies([ref.image, ref.mu, ref.image_batch, ref.counters])
    same = all(bool(torch.equal(getattr(tal, k), getattr(ref, k)))
               for k in ("mu", "image", "image_batch", "counters"))
    c = tal.counts()
    if rank == 0:
        line = {"metric": "packet-steps/s, decomposed clump solve", "unit": UNIT,
                "value": (c["steps"] + c["peel_steps"]) / (t_dd / 1e3), "higher_is_better": True,
                "n_gpus": world, "config": {"workload": "clump_amr_2level_decomposed",
                                            "packets": n_pk, "ranks": n_ranks,
                                            "ranks_emulated_on_one_gpu": world == 1,
                                            "blocks": mesh.n_blocks},
                "rounds": rounds, "decomposed_ms": t_dd, "replicated_ms": t_rep,
                "tallies_identical_to_replicated": same}
        print(json.dumps(line), flush=True)
    _finish_ranks(world)


def _walk_bench(args, spherical):
    """Reference-semantics walks (kp_trace: cart_t::proc; kp_trace_sph:
    sph_t::proc) on GPU against the reference's own code compiled for the
    host (oracle/_ref).  Packets start uniformly in the domain with
    isotropic directions and walk to its boundary or for 4096 steps, one
    int64 path-length flux deposit per step.  Per precision (float_t of the
    reference's PRECISION=1 and 2): device time of the walk (pool restored
    before each step, outside the timed region), the final states of a
    sample against the reference's (identical packets), and the reference
    on all host cores over that sample."""
    import os
    import time
    import numpy as np
    import torch
    from kratos_polrad_b200 import Mesh, PacketPool, scenes
    from kratos_polrad_b200.walk import TO_KEEP, trace as gpu_trace, trace_sph as gpu_trace_sph
    from oracle import refharness
    two_pi = 2 * math.pi
    if spherical:
        from kratos_polrad_b200.mesh import MeshConfig, RefineRegion
        mcfg = MeshConfig((0.5, 0.4, 0.0), (2.5, 2.7, two_pi), (64, 64, 128), (16, 16, 16),
                          (False, False, True),
                          [RefineRegion(1, (1.0, 1.0, 2.0), (1.6, 1.8, 3.6)),
                           RefineRegion(2, (1.1, 1.2, 2.5), (1.3, 1.4, 3.0))])
        ratio = 1.0
        mesh = Mesh(mcfg, spherical=True, r_ratio=ratio)
        ini = mcfg.to_ini().replace("[boundary]", f"r_ratio = {ratio!r}\n\n[boundary]", 1)
        name, metric = "trace_sph", "packet-steps/s, spherical-polar walk (sph_t::proc)"
    else:
        mcfg = scenes.clump_mesh_config()
        mesh = Mesh(mcfg)
        ini = mcfg.to_ini()
        name, metric = "trace_clump_mesh", "packet-steps/s, reference-semantics walk (cart_t::proc)"
    n = int(args.packets) if args.packets != 1e7 else 1 << 23
    dev = torch.device("cuda")
    lo, hi = np.array(mcfg.x_min, float), np.array(mcfg.x_max, float)
    per = {}
    for prec in (1, 2):
        ftype, tdt = (np.float32, torch.float32) if prec == 1 else (np.float64, torch.float64)
        rng = np.random.default_rng(17 + prec)
        pad = np.array([0.01, 0.05, 0.0]) * (hi - lo) if spherical else np.zeros(3)
        x = lo + pad + rng.random((n, 3)) * (hi - lo - 2 * pad)
        d = rng.normal(size=(n, 3))
        d /= np.linalg.norm(d, axis=1, keepdims=True)
        x, d = x.astype(ftype), d.astype(ftype)
        ib, cell = mesh.locate(x.astype(np.float64))
        proper = (rng.random(n) + 0.5).astype(ftype)
        # a finite budget: a few packets of the spherical walk stall at cell
        # corners (the reference's own walk does the same) until it runs out
        steps = np.full(n, 4096, np.int32)
        T = lambda a, dt=None: torch.tensor(a, dtype=dt, device=dev)
        orig = [T(x, tdt), T(d, tdt), T(cell), T(ib), T(proper, tdt), T(steps)]
        pool = PacketPool(*[o.clone() for o in orig])
        if spherical:
            r, th, ph = (x[:, k].astype(np.float64) for k in range(3))
            xc = np.stack([r * np.sin(th) * np.cos(ph), r * np.sin(th) * np.sin(ph), r * np.cos(th)], 1)
            xc0 = T(xc.astype(ftype), tdt)
            x_car = xc0.clone()
        flux = torch.zeros(mesh.n_cells, dtype=torch.int64, device=dev)

        def restore():
            for dst, src in zip((pool.x, pool.dir, pool.cell, pool.ib, pool.proper, pool.step), orig):
                dst.copy_(src)
            pool.todo.fill_(TO_KEEP)
            if spherical:
                x_car.copy_(xc0)
            flux.zero_()

        def walk():
            if spherical:
                gpu_trace_sph(mesh, pool, x_car, "fixed", 16, flux)
            else:
                gpu_trace(mesh, pool, "fixed", 32, flux)

        for _ in range(max(1, args.warmup)):
            restore(); walk()
        torch.cuda.synchronize()
        ms = []
        for _ in range(args.steps):
            restore()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(); walk(); e1.record()
            torch.cuda.synchronize()
            ms.append(e0.elapsed_time(e1))
        status = mesh.status()
        done = int((orig[5].long() - pool.step.long()).sum())
        value = done / (statistics.mean(ms) / 1e3)
        # the reference on the host: a sample of the same packets, all cores
        entry = {"value": value, "ms": statistics.mean(ms), "steps": done, "status": status}
        if refharness.available(prec):
            ref = (refharness.RefMeshSph if spherical else refharness.RefMesh)(ini, prec)
            pl, pr = mesh.blocks()
            rl, rr = ref.blocks()
            key = {(int(l), *map(int, q)): i for i, (l, q) in enumerate(zip(pl, pr))}
            perm = np.array([key[(int(l), *map(int, q))] for l, q in zip(rl, rr)])
            inv = np.argsort(perm)
            cores = os.cpu_count() or 1
            refharness.deposits_outside(prec)          # reset the harness's count
            m = min(n, 1 << 17)
            for it in range(3):                 # grow the sample to about 1.5 s
                sel = slice(0, m)
                t0 = time.perf_counter()
                if spherical:
                    rres = ref.trace(x[sel], xc[sel], d[sel], cell[sel], inv[ib[sel]], proper[sel],
                                     steps[sel], fx_shift=16, n_threads=cores)
                else:
                    rres = ref.trace(x[sel], d[sel], cell[sel], inv[ib[sel]], proper[sel],
                                     steps[sel], fx_shift=32, n_threads=cores)
                dt = time.perf_counter() - t0
                if dt >= 1.0 or m == n or it == 2:
                    break
                m = min(n, int(m * 1.5 / max(dt, 1e-3)))
            rib = rres["ib"]
            # the same walk: cells, blocks, steps and end flags; positions are
            # bit-identical for the Cartesian walk and within the float
            # transcendentals' ulps for the spherical one (cos/sin/acos/atan2)
            walk = ((pool.cell[:m].cpu().numpy() == rres["cell"]).all(1)
                    & (pool.ib[:m].cpu().numpy() == np.where(rib >= 0, perm[np.maximum(rib, 0)], rib))
                    & (pool.step[:m].cpu().numpy() == rres["step"])
                    & (pool.todo[:m].cpu().numpy().astype(np.int32) == rres["todo"]))
            xs = pool.x[:m].cpu().numpy().astype(np.float64)
            bit = walk & (xs == rres["x"]).all(1)
            rel = np.abs(xs[walk] - rres["x"][walk]) / np.maximum(np.abs(rres["x"][walk]), 1e-6)
            rsteps = int((steps[:m].astype(np.int64) - rres["step"]).sum())
            entry["parity"] = {"packets": m, "same_walk": float(walk.mean()),
                               "bit_identical_final_state": float(bit.mean()),
                               "position_rel_diff_q99_same_walk": float(np.quantile(rel, 0.99))
                               if rel.size else 0.0,
                               "reference_deposits_beyond_flux_pool_skipped":
                                   refharness.deposits_outside(prec)}
            entry["cpu_baseline"] = {"value": rsteps / dt, "unit": "packet-steps/s", "cores": cores,
                                     "kind": "reference",
                                     "sample": f"packets 0..{m - 1} of the same set, {rsteps:.3g} "
                                               f"packet-steps in {dt:.2f} s"}
        per[str(prec)] = entry
    line = {"metric": metric, "unit": "packet-steps/s", "value": per["1"]["value"],
            "higher_is_better": True, "n_gpus": 1,
            "config": {"workload": name, "packets": n, "blocks": mesh.n_blocks,
                       "cells": mesh.n_cells, "budget": "to the domain boundary, at most 4096 steps",
                       "flux": "int64 fixed point", "value_precision": "PRECISION=1 (float_t float)"},
            "precisions": per}
    print(json.dumps(line), flush=True)


def run_refine(args):
    """Runtime refinement of the clump scene: per-block flags from the
    extinction depth across a cell (device), the refined and coarsened mesh
    with 2:1 balance and neighbour tables (host), its upload, and the
    coefficients carried onto it (device)."""
    import time
    import torch
    from kratos_polrad_b200 import scenes
    mesh, sig, cfg = scenes.clump_amr(n_packets=1)
    mesh.set_sigma(sig)
    dev = torch.device("cuda")
    src = torch.tensor(sig, device=dev)
    ev = lambda: torch.cuda.Event(enable_timing=True)
    res = {}
    for k in range(max(1, args.warmup) + args.steps):
        e0, e1, e2, e3 = ev(), ev(), ev(), ev()
        e0.record()
        flags = mesh.flag_tau(0.1, 0.02)
        e1.record()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        fine = mesh.adapt(flags)
        t1 = time.perf_counter()
        fine.upload()
        torch.cuda.synchronize()
        t2 = time.perf_counter()
        e2.record()
        dst = mesh.remap_to(fine, src)
        e3.record()
        torch.cuda.synchronize()
        if k >= max(1, args.warmup):
            for key, v in (("flag_ms", e0.elapsed_time(e1)), ("adapt_host_ms", (t1 - t0) * 1e3),
                           ("upload_ms", (t2 - t1) * 1e3), ("remap_ms", e2.elapsed_time(e3))):
                res.setdefault(key, []).append(v)
    f = flags.cpu().numpy()
    out = {k: statistics.mean(v) for k, v in res.items()}
    total = sum(out.values())
    line = {"metric": "runtime refinement step, 2-level AMR clump", "unit": "ms", "value": total,
            "higher_is_better": False, "n_gpus": 1,
            "config": {"workload": "refine_clump", "blocks": mesh.n_blocks, "cells": mesh.n_cells,
                       "tau_refine": 0.1, "tau_coarsen": 0.02},
            "flagged_refine": int((f > 0).sum()), "flagged_coarsen": int((f < 0).sum()),
            "blocks_after": fine.n_blocks, "cells_after": fine.n_cells, **out,
            "remap_cells_per_s": fine.n_cells / (out["remap_ms"] / 1e3),
            "finite": bool(torch.isfinite(dst).all()),
            # the remap copies where a new cell lies in one old cell and
            # averages octants elsewhere: the field's range is kept
            "range_kept": bool(dst.min() >= src.min() and dst.max() <= src.max())}
    print(json.dumps(line), flush=True)


def run_bio(args):
    """The binary container (the reference's binary_io format): a clump
    solution (block keys, per-block flux fields, coefficients, tallies,
    config) written and read back, byte sizes and rates, values checked."""
    import tempfile
    import time
    import numpy as np
    import torch
    from kratos_polrad_b200 import bio, scenes
    from kratos_polrad_b200.transport import forward
    mesh, sig, cfg = scenes.clump_amr(n_packets=1_000_000)
    mesh.set_sigma(sig)
    tal = forward(mesh, cfg)
    torch.cuda.synchronize()
    flux = (sig[:, 0].astype(np.float64) + sig[:, 1])
    wr, rd, ok = [], [], True
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "solution.bin")
        for k in range(max(1, args.warmup) + args.steps):
            t0 = time.perf_counter()
            bio.save_solution(path, mesh, sig, tal, cfg, flux=flux)
            t1 = time.perf_counter()
            got = bio.load_solution(path)
            t2 = time.perf_counter()
            if k >= max(1, args.warmup):
                wr.append(t1 - t0)
                rd.append(t2 - t1)
            ok = ok and np.array_equal(got["sigma"], sig) and np.array_equal(
                got["image"], tal.image.cpu().numpy())
        size = os.path.getsize(path)
    line = {"metric": "binary container write + read, clump solution", "unit": "MB/s",
            "value": size / 1e6 / statistics.mean(wr), "higher_is_better": True, "n_gpus": 1,
            "config": {"workload": "bio_clump", "bytes": size, "blocks": mesh.n_blocks},
            "write_ms": statistics.mean(wr) * 1e3, "read_ms": statistics.mean(rd) * 1e3,
            "read_mb_per_s": size / 1e6 / statistics.mean(rd), "values_equal": bool(ok)}
    print(json.dumps(line), flush=True)


def run_resume(args):
    """Resumable calls: the clump solve carried out in calls with a step budget
    of `--budget` walk segments per packet and call (kp_transport_forward_resume;
    the packets still walking are written out and resumed by the next call)
    against one uninterrupted solve of the same packets: device time of all
    the calls, their number, the packets carried between calls, and the
    tallies compared."""
    import torch
    from kratos_polrad_b200 import scenes
    from kratos_polrad_b200.transport import Tallies, forward, forward_resume
    n_pk = int(args.packets)
    mesh, sigma2, cfg = scenes.clump_amr(n_packets=n_pk)
    mesh.set_sigma(sigma2)
    rest = dataclasses.replace(cfg, n_packets=0)

    def budgeted(tal):
        tal, out = forward_resume(mesh, cfg, args.budget, tallies=tal)
        calls, carried = 1, int(out.shape[0])
        while out.shape[0] > 0 and calls < 10000:
            tal, out = forward_resume(mesh, rest, args.budget, resumed=out, tallies=tal)
            calls += 1
            carried += int(out.shape[0])
        return tal, calls, carried, int(out.shape[0])

    full = Tallies(cfg)
    forward(mesh, cfg, full)                     # warm-up of both forms
    budgeted(Tallies(cfg))
    torch.cuda.synchronize()
    full.zero_()
    _, t_full = _timed(lambda: forward(mesh, cfg, full))
    (tal, calls, carried, left), t_res = _timed(lambda: budgeted(Tallies(cfg)))
    assert mesh.status() == 0
    same = all(torch.equal(getattr(tal, k), getattr(full, k))
               for k in ("image", "image_batch", "mu", "counters"))
    c = full.counts()
    steps = c["steps"] + c["peel_steps"]
    print(json.dumps({"metric": "packet-steps/s, clump solve in budgeted calls", "unit": UNIT,
                      "value": steps / (t_res / 1e3), "higher_is_better": True, "n_gpus": 1,
                      "config": {"workload": "clump_amr_2level_resumed", "packets": n_pk,
                                 "step_budget": args.budget},
                      "calls": calls, "packets_carried": carried, "packets_left": left,
                      "ms_budgeted": t_res, "ms_one_solve": t_full,
                      "cost_vs_one_solve": t_res / t_full,
                      "tallies_equal_one_solve": same}), flush=True)


def run_large(args):
    """Large workload: 256^3 root, 3 levels on a lognormal field (std of ln
    rho 1.5, seed 5; ~2e7 cells, 166 MB of coefficients: beyond L2), HG g=0.6
    with polarization, 64 random point sources, 256^2 IQUV image; one forward
    solve and one path-replay gradient of `--packets` packets (default 1e9)."""
    import numpy as np
    import torch
    from kratos_polrad_b200 import scenes
    from kratos_polrad_b200.adjoint import adjoint
    from kratos_polrad_b200.transport import Tallies, forward
    n_pk = int(args.packets) if args.packets != 1e7 else 1_000_000_000
    mesh, sig, cfg = scenes.large_amr(n_packets=n_pk)
    mesh.set_sigma(sig)
    from kratos_polrad_b200.mesh import PEEL_ORDER_AUTO, PEEL_ORDER_CELL, PEEL_ORDER_QUEUE
    mesh.set_peel_order({"auto": PEEL_ORDER_AUTO, "queue": PEEL_ORDER_QUEUE,
                         "cell": PEEL_ORDER_CELL}[args.peel_order])
    warm = dataclasses.replace(cfg, n_packets=min(n_pk, 2_000_000))
    forward(mesh, warm)
    torch.cuda.synchronize()
    tal = Tallies(cfg)
    with ClockSampler(0) as clk:
        _, t_fwd = _timed(lambda: forward(mesh, cfg, tal))
    c = tal.counts()
    bimg = tal.image_batch.cpu().numpy() * tal.scale()
    p_tan, rel = scenes.batch_rel_error(bimg)
    # tangential polarization about the nearest source's image position:
    # linear in Q, U (unbiased batch means), positive for the scattered
    # light's pattern around each source
    p_loc, rel_loc = scenes.batch_rel_error(bimg, scenes.source_pixels(cfg, bimg.shape[1]))
    # the image-integrated linear polarization fraction sqrt(Q^2+U^2)/I, and
    # the intensity-weighted mean degree of the coarse pixels, with their
    # batch-means relative std-errors
    from kratos_polrad_b200.transport import batch_std_error
    p_int, rel_int = batch_std_error(bimg.sum((1, 2)))
    deg = np.array([np.sqrt(b[..., 1] ** 2 + b[..., 2] ** 2).sum() / b[..., 0].sum()
                    for b in bimg])
    p_deg = float(np.sqrt(bimg.sum(0)[..., 1] ** 2 + bimg.sum(0)[..., 2] ** 2).sum()
                  / bimg.sum(0)[..., 0].sum())
    rel_deg = float(deg.std(ddof=1) / np.sqrt(len(deg)) / p_deg)
    g_img = torch.randn((cfg.image_n, cfg.image_n, 4), device="cuda",
                        generator=torch.Generator(device="cuda").manual_seed(5))
    acnt = torch.zeros(10, dtype=torch.int64, device="cuda")
    _, t_adj = _timed(lambda: adjoint(mesh, cfg, g_img, 24, acnt))
    ac = acnt.cpu().numpy()
    line = {"metric": "packet-steps/s, 3-level AMR lognormal, 64 sources", "unit": UNIT,
            "value": (c["steps"] + c["peel_steps"]) / (t_fwd / 1e3), "higher_is_better": True,
            "n_gpus": 1, "config": {"workload": "large_amr_3level", "packets": n_pk,
                                    "blocks": mesh.n_blocks, "cells": mesh.n_cells,
                                    "sigma_MB": sig.nbytes / 1e6, "image": cfg.image_n,
                                    "peel_order": args.peel_order},
            "forward_ms": t_fwd, "counts": c, "pol_tangential": p_tan, "pol_rel_std_err": rel,
            "pol_tangential_about_sources": p_loc, "pol_tangential_about_sources_rel_std_err": rel_loc,
            # the std-error falls like packets^-1/2: packets (and forward time at
            # this rate) for 1% on the statistic about the sources
            "pol_packets_for_1pct": n_pk * (rel_loc / 0.01) ** 2,
            "pol_forward_s_for_1pct": t_fwd / 1e3 * (rel_loc / 0.01) ** 2,
            "pol_integrated": p_int, "pol_integrated_rel_std_err": rel_int,
            "pol_mean_degree_coarse": p_deg, "pol_mean_degree_rel_std_err": rel_deg,
            "adjoint_ms": t_adj, "adjoint_cost_vs_forward": t_adj / t_fwd,
            "adjoint_packet_steps_per_s": float(ac[0] + ac[1]) / (t_adj / 1e3),
            "clocks": clk.summary()}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.workload == "batched":
        return run_batched(args)
    if args.workload == "diff":
        return run_diff(args)
    if args.workload == "large":
        return run_large(args)
    if args.workload == "decomp":
        return run_decomp(args)
    if args.workload in ("trace", "sph"):
        return _walk_bench(args, args.workload == "sph")
    if args.workload == "refine":
        return run_refine(args)
    if args.workload == "bio":
        return run_bio(args)
    if args.workload == "resume":
        return run_resume(args)
    if args.impl == "reference":     # host cores only: rank 0 runs, the others exit
        run_reference(args, int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)))
        return
    import torch
    import torch.distributed as dist
    rank, world, local = _init_ranks()

    from kratos_polrad_b200 import scenes, shard
    from kratos_polrad_b200._lib import call, ptr
    from kratos_polrad_b200.transport import Tallies, forward
    dev = torch.device("cuda", local)
    n_pk = int(args.packets)
    mesh, sigma2, cfg = scenes.clump_amr(n_packets=n_pk)
    cfg = shard.shard_config(cfg, rank, world, weak=True)
    mesh.set_sigma(sigma2)
    tal = Tallies(cfg)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    rank_counts = torch.zeros(10, dtype=torch.int64, device=dev)

    def allreduce():
        rank_counts.copy_(tal.counters)               # this rank's own counts
        shard.reduce_tallies([tal.image, tal.mu, tal.image_batch, tal.counters])

    for _ in range(args.warmup):
        tal.zero_()
        forward(mesh, cfg, tal)
        allreduce()
    torch.cuda.synchronize()
    assert mesh.status() == 0

    # ---- device-timed region: K solves, L2 flushed before each ----
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    kev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.steps)]
    # recorded by the library between the walk and the peel-off kernel
    mid = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    for e in mid:
        e.record()                      # creates the CUDA event
    counts = []
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        for k in range(args.steps):
            tal.zero_()
            flush.fill_(float(k))
            ev[k][0].record()
            kev[k][0].record()
            call("kp_transport_split_event", mid[k].cuda_event)
            forward(mesh, cfg, tal)
            kev[k][1].record()
            allreduce()
            ev[k][1].record()
            counts.append(tal.counters.clone())
        torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    step_ms = [a.elapsed_time(b) for a, b in ev]
    call("kp_transport_split_event", None)
    kern_ms = [a.elapsed_time(b) for a, b in kev]
    walk_ms = statistics.mean(a.elapsed_time(m) for (a, _), m in zip(kev, mid))
    peel_ms = statistics.mean(m.elapsed_time(b) for (_, b), m in zip(kev, mid))
    t_local = sum(step_ms) / 1e3
    t = torch.tensor([t_local], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    t_max = float(t.item())
    c = {k: int(v) for k, v in zip(tal.counts().keys(), counts[-1].cpu().numpy())}
    if world > 1:   # counters were all-reduced: whole-job totals already
        job_steps = (c["steps"] + c["peel_steps"]) * args.steps
    else:
        job_steps = sum(int(x[0]) + int(x[1]) for x in (cc.cpu().numpy() for cc in counts))
    value = job_steps / t_max

    # quality: batch-means relative std-error of the tangential polarization
    scale = 2.0 ** -cfg.fx_shift
    p_tan, rel_err = scenes.batch_rel_error(tal.image_batch.cpu().numpy() * scale)

    # roofline of the transport kernel (per launch, this rank)
    c_rank = {k: int(v) for k, v in zip(tal.counts().keys(), rank_counts.cpu().numpy())}
    kern_s = statistics.mean(kern_ms) / 1e3
    peak, peak_kind = measured_peak()
    ach = algorithmic_bytes(c_rank) / kern_s / 1e9
    traffic = ncu_traffic(n_pk)
    roofline = {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s",
                "frac": ach / peak, "peak_source": peak_kind,
                "kernel": "k_forward + k_peel (the two launches of one solve)",
                "traffic": sum(traffic.values()) if traffic else None,
                "algorithmic_bytes": algorithmic_bytes(c_rank),
                "kernel_ms": statistics.mean(kern_ms),
                "kernels": {"k_forward": {"ms": walk_ms, "share": walk_ms / (walk_ms + peel_ms),
                                          "traffic": traffic and traffic["k_forward"]},
                            "k_peel": {"ms": peel_ms, "share": peel_ms / (walk_ms + peel_ms),
                                       "traffic": traffic and traffic["k_peel"]}}}

    # ---- adjoint: gradient of an image loss, cost relative to one forward ----
    from kratos_polrad_b200.adjoint import adjoint as run_adjoint
    adj_img = torch.randn((cfg.image_n, cfg.image_n, 4), device=dev, generator=torch.Generator(
        device=dev).manual_seed(7))
    adj_cnt = torch.zeros(10, dtype=torch.int64, device=dev)
    run_adjoint(mesh, cfg, adj_img, 24, adj_cnt)
    torch.cuda.synchronize()
    adj_ms = []
    for k in range(max(1, min(args.steps, 3))):
        adj_cnt.zero_()
        flush.fill_(float(k))
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a0.record()
        run_adjoint(mesh, cfg, adj_img, 24, adj_cnt)
        a1.record()
        torch.cuda.synchronize()
        adj_ms.append(a0.elapsed_time(a1))
    ac = adj_cnt.cpu().numpy()
    # the gradient of a taped forward solve (an autograd step): forward with
    # the tape kept, then the adjoint from the tape; gradients checked equal
    g_full = run_adjoint(mesh, cfg, adj_img, 24)
    tape_fwd_ms, tape_adj_ms, tape_same = [], [], True
    tal_t = Tallies(cfg)
    for k in range(max(1, min(args.steps, 3))):
        tal_t.zero_()
        flush.fill_(float(k))
        t0, t1, t2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        t0.record()
        forward(mesh, cfg, tal_t, tape=True)
        t1.record()
        g_tape = run_adjoint(mesh, cfg, adj_img, 24, tape_id=tal_t.tape_id)
        t2.record()
        torch.cuda.synchronize()
        tape_fwd_ms.append(t0.elapsed_time(t1))
        tape_adj_ms.append(t1.elapsed_time(t2))
        tape_same = tape_same and tal_t.tape_id > 0 and all(
            torch.equal(x, y) for x, y in zip(g_tape, g_full))
    adjoint_info = {"ms_per_solve": statistics.mean(adj_ms),
                    "cost_vs_forward": statistics.mean(adj_ms) / statistics.mean(kern_ms),
                    "packet_steps_per_s": float(ac[0] + ac[1]) / (statistics.mean(adj_ms) / 1e3),
                    "note": "two replays per packet (measure, deposit); same packets as the forward",
                    "taped": {"forward_ms": statistics.mean(tape_fwd_ms),
                              "gradient_ms": statistics.mean(tape_adj_ms),
                              "gradients_equal_full_adjoint": tape_same,
                              "note": "forward with its peel-off rays kept, then the adjoint "
                                      "from them (autograd step)"}}

    # ---- the path-length flux tally (rad_t::flx): same solves with it on ----
    fcfg = dataclasses.replace(cfg, flux=True, flux_fx_shift=20)
    ftal = Tallies(fcfg, n_cells=mesh.n_cells)
    forward(mesh, fcfg, ftal)
    torch.cuda.synchronize()
    flux_ms = []
    for k in range(max(1, min(args.steps, 3))):
        ftal.zero_()
        flush.fill_(float(k))
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record()
        forward(mesh, fcfg, ftal)
        f1.record()
        torch.cuda.synchronize()
        flux_ms.append(f0.elapsed_time(f1))
    fc = ftal.counts()
    flux_same = all(torch.equal(getattr(ftal, n), getattr(tal, n)) for n in ("image", "mu"))
    flux_info = {"ms_per_solve": statistics.mean(flux_ms),
                 "cost_vs_forward": statistics.mean(flux_ms) / statistics.mean(kern_ms),
                 "algorithmic_bytes": algorithmic_bytes(fc) + 8 * fc["steps"],
                 "achieved_gbs": (algorithmic_bytes(fc) + 8 * fc["steps"])
                 / (statistics.mean(flux_ms) / 1e3) / 1e9,
                 "cells_visited": int((ftal.flux != 0).sum()),
                 "other_tallies_unchanged": flux_same,
                 "note": "int64 w*dl/volume per walk segment (scale 2^20); +8 B per walk "
                         "segment (read + write of the cell's tally)"}
    assert mesh.status() == 0

    # ---- the batched solve (256 scenes), its own numbers ----
    batched_info = measure_batched(max(1, min(args.steps, 3)), 1)

    # ---- end to end through the C ABI with host buffers ----
    import ctypes
    n_cells = mesh.n_cells
    h_sigma = torch.from_numpy(sigma2.reshape(-1)).pin_memory()
    h_img = torch.empty_like(tal.image, device="cpu").pin_memory()
    h_mu = torch.empty_like(tal.mu, device="cpu").pin_memory()
    h_cnt = torch.empty_like(tal.counters, device="cpu").pin_memory()
    d_sig = ctypes.c_void_p()
    call("kp_mesh_sigma_ptr", mesh.handle, ctypes.byref(d_sig))
    s = torch.cuda.current_stream().cuda_stream
    e2e_ev = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
    h2d = h_sigma.numel() * 4
    d2h = (h_img.numel() + h_mu.numel() + h_cnt.numel()) * 8
    e2e_steps = 0
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e2e_ms = 0.0
    for k in range(args.steps):
        tal.zero_()
        flush.fill_(float(k))
        e2e_ev[0].record()
        call("kp_memcpy_async", d_sig.value, ptr(h_sigma), h2d, s)
        forward(mesh, cfg, tal)
        allreduce()
        call("kp_memcpy_async", ptr(h_img), ptr(tal.image), h_img.numel() * 8, s)
        call("kp_memcpy_async", ptr(h_mu), ptr(tal.mu), h_mu.numel() * 8, s)
        call("kp_memcpy_async", ptr(h_cnt), ptr(tal.counters), h_cnt.numel() * 8, s)
        e2e_ev[1].record()
        torch.cuda.synchronize()
        e2e_ms += e2e_ev[0].elapsed_time(e2e_ev[1])
        e2e_steps += int(h_cnt[0]) + int(h_cnt[1])
    t2 = torch.tensor([e2e_ms / 1e3], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t2, op=dist.ReduceOp.MAX)
    e2e_value = e2e_steps / float(t2.item())

    out = None
    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            cpu = cpu_baseline(mesh, sigma2, cfg)
        out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
               "steps": args.steps, "warmup": args.warmup,
               "ms_per_step": t_max * 1e3 / args.steps, "higher_is_better": True,
               "scaling": "weak", "vs_baseline": None, "dtype": "f64 positions / f32 Stokes",
               "data": "synthetic", "config": workload_config(cfg, n_pk),
               "walk_steps_per_solve": c_rank["steps"], "peel_steps_per_solve": c_rank["peel_steps"],
               "pol_tangential": p_tan, "pol_rel_std_err": rel_err,
               "roofline": roofline, "cpu_baseline": cpu,
               "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d,
                       "d2h_bytes_per_step": d2h},
               "adjoint": adjoint_info, "flux_tally": flux_info, "batched": batched_info,
               # per solve: the extinction refresh, the walk and (with an
               # image) the peel-off march
               "gpu_launches": args.steps * (3 if cfg.image_n > 0 else 2),
               "clocks": clk.summary()}
        print(json.dumps(out), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
