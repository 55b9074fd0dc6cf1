"""Batched multi-scene launch: each scene's tallies equal a single-scene solve
of that scene (same seed and stream id), bit for bit; CUDA-graph replay and
autotuned launch shapes give the same tallies."""
import dataclasses

import pytest
import torch

from kratos_polrad_b200 import scenes
from kratos_polrad_b200.batch import Batch
from kratos_polrad_b200.transport import Tallies, forward

pytestmark = pytest.mark.gpu


def _setup():
    sc, cfg = scenes.batched_cubes(n_scenes=5, sides=(16, 32, 48), packets=(300, 3000), seed=11)
    for mesh, sig, *_ in sc:
        mesh.set_sigma(sig)
    b = Batch([(m, n, sid, src) for m, _, n, sid, src in sc])
    return sc, cfg, b


def test_batch_equals_single_scene_solves():
    sc, cfg, b = _setup()
    mu = b.forward(cfg)
    torch.cuda.synchronize()
    assert b.status() == 0
    for k, (mesh, _, n, sid, src) in enumerate(sc):
        c = dataclasses.replace(cfg, n_packets=n, stream_id=sid, sources=[src])
        ref = forward(mesh, c, Tallies(c))
        torch.cuda.synchronize()
        assert torch.equal(mu[k], ref.mu), k


def test_graph_replay_and_autotune_keep_results():
    sc, cfg, b = _setup()
    ref = b.forward(cfg)
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        g1 = b.forward(cfg, graph=True, stream=s.cuda_stream)
        g2 = b.new_mu(cfg)
        b.forward(cfg, mu=g2, graph=True, stream=s.cuda_stream)   # new buffer: re-capture
        b.forward(cfg, mu=g2, graph=True, stream=s.cuda_stream)   # replay: accumulates
    s.synchronize()
    assert torch.equal(g1, ref)
    assert torch.equal(g2, 2 * ref)
    tune = b.autotune(cfg, fraction=0.2)
    assert tune["threads"] in (128, 256) and tune["lane_batch"] > 0
    again = b.forward(cfg)
    torch.cuda.synchronize()
    assert torch.equal(again, ref)
