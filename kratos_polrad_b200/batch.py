"""Batched solves: many independent scenes in one persistent launch.

Host mirror of ``kp_batch_*`` (include/kp_transport.h).  A scene's packets
in a batched launch are the same packets as a single-scene
``transport.forward`` of that scene with the same seed and stream id.
"""
from __future__ import annotations

import ctypes

import torch

from . import _lib
from ._lib import call, ptr
from .transport import CSource, CTransportCfg, TALLY_FIXED, TransportConfig

c_void_p = ctypes.c_void_p


class CScene(ctypes.Structure):
    _fields_ = [("mesh", c_void_p), ("n_packets", ctypes.c_longlong),
                ("stream_id", ctypes.c_uint32), ("source", CSource)]


class CTuneResult(ctypes.Structure):
    _fields_ = [("threads", ctypes.c_int), ("lane_batch", ctypes.c_int), ("grid_pct", ctypes.c_int),
                ("sample_ms", ctypes.c_float), ("sample_packets", ctypes.c_longlong)]


_lib.register("kp_batch_create", [ctypes.c_int, ctypes.POINTER(CScene), ctypes.POINTER(c_void_p)])
_lib.register("kp_batch_destroy", [c_void_p])
_lib.register("kp_batch_refresh_sigma", [c_void_p, c_void_p])
_lib.register("kp_batch_status", [c_void_p, c_void_p, ctypes.POINTER(ctypes.c_uint)])
_lib.register("kp_batch_forward", [c_void_p, ctypes.POINTER(CTransportCfg), c_void_p, c_void_p,
                                   c_void_p])
_lib.register("kp_batch_graph_launch", [c_void_p, ctypes.POINTER(CTransportCfg), c_void_p,
                                        c_void_p, c_void_p])
_lib.register("kp_batch_autotune", [c_void_p, ctypes.POINTER(CTransportCfg), ctypes.c_double,
                                    c_void_p, c_void_p, ctypes.POINTER(CTuneResult)])


class Batch:
    """``scenes``: list of (mesh, n_packets, stream_id, Source)."""

    def __init__(self, scenes):
        arr = (CScene * len(scenes))()
        for k, (mesh, n, sid, src) in enumerate(scenes):
            arr[k].mesh = mesh.handle
            arr[k].n_packets = int(n)
            arr[k].stream_id = int(sid)
            arr[k].source.kind, arr[k].source.emit = int(src.kind), int(src.emit)
            for a in range(3):
                arr[k].source.pos[a] = float(src.pos[a])
        h = c_void_p()
        call("kp_batch_create", len(scenes), arr, ctypes.byref(h))
        self.handle = h
        self.n_scenes = len(scenes)
        self.meshes = [s[0] for s in scenes]
        self.n_packets = [int(s[1]) for s in scenes]

    def close(self):
        if self.handle:
            call("kp_batch_destroy", self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def new_mu(self, cfg: TransportConfig):
        dt = torch.int64 if cfg.tally_mode == TALLY_FIXED else torch.float32
        return torch.zeros((self.n_scenes, cfg.n_batches, cfg.n_mu_bins, 4), dtype=dt, device="cuda")

    def forward(self, cfg: TransportConfig, mu=None, counters=None, graph=False, stream=None):
        if mu is None:
            mu = self.new_mu(cfg)
        c = cfg.to_c()
        s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
        name = "kp_batch_graph_launch" if graph else "kp_batch_forward"
        call(name, self.handle, ctypes.byref(c), ptr(mu), ptr(counters), s)
        return mu

    def autotune(self, cfg: TransportConfig, fraction=0.05, stream=None) -> dict:
        scratch = self.new_mu(cfg)
        r = CTuneResult()
        s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
        call("kp_batch_autotune", self.handle, ctypes.byref(cfg.to_c()), fraction, ptr(scratch),
             s, ctypes.byref(r))
        return {"threads": r.threads, "lane_batch": r.lane_batch, "grid_pct": r.grid_pct,
                "sample_ms": r.sample_ms, "sample_packets": r.sample_packets}

    def refresh_sigma(self, stream=None):
        call("kp_batch_refresh_sigma", self.handle, stream)

    def status(self, stream=None) -> int:
        f = ctypes.c_uint()
        call("kp_batch_status", self.handle, stream, ctypes.byref(f))
        return f.value
