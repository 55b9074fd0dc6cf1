"""The C-ABI library loads without a GPU and exports every declared symbol."""
import ctypes

from kratos_polrad_b200 import _lib


def test_every_header_symbol_is_exported():
    names = _lib.header_symbols()
    assert "kp_transport_forward" in names and "kp_trace" in names
    missing = [n for n in names if not hasattr(_lib.lib, n)]
    assert not missing, missing


def test_abi_version_and_error_channel():
    assert _lib.lib.kp_abi_version() == _lib.ABI_VERSION == 2
    # a failing call reports a status and a message, without touching a GPU
    st = _lib.lib.kp_mesh_create(None, None)
    assert st == _lib.KP_ERR_ARG
    assert b"null" in _lib.lib.kp_last_error()


def test_bad_mesh_config_is_refused():
    d = _lib.MeshDesc()
    for a in range(3):
        d.x_min[a], d.x_max[a] = 0.0, 1.0
        d.n_cell_global[a], d.n_cell_block[a] = 30, 16       # not divisible
    h = ctypes.c_void_p()
    st = _lib.lib.kp_mesh_create(ctypes.byref(d), ctypes.byref(h))
    assert st == _lib.KP_ERR_CONFIG
    assert b"indivisible" in _lib.lib.kp_last_error()


def test_peel_order_is_checked():
    """kp_mesh_peel_order takes the three orders and refuses others
    (KP_ERR_CONFIG); it only sets the mesh's choice."""
    from meshcases import AMR_BOX
    from kratos_polrad_b200 import Mesh
    from kratos_polrad_b200.mesh import PEEL_ORDER_AUTO, PEEL_ORDER_CELL, PEEL_ORDER_QUEUE
    m = Mesh(AMR_BOX)
    for order in (PEEL_ORDER_QUEUE, PEEL_ORDER_CELL, PEEL_ORDER_AUTO):
        assert _lib.lib.kp_mesh_peel_order(m.handle, order) == _lib.KP_OK
    for bad in (2, -2):
        assert _lib.lib.kp_mesh_peel_order(m.handle, bad) == _lib.KP_ERR_CONFIG
        assert b"unknown peel-off order" in _lib.lib.kp_last_error()
    assert _lib.lib.kp_mesh_peel_order(None, 0) == _lib.KP_ERR_ARG


def test_tape_entry_points_refuse_without_a_taped_solve():
    """A mesh that never ran a taped solve has tape id 0, and the adjoint of
    tape 0 (or of any id) is refused before any device work."""
    from meshcases import AMR_BOX
    from kratos_polrad_b200 import Mesh
    from kratos_polrad_b200.transport import EMIT_ISOTROPIC, SOURCE_POINT, Source, TransportConfig
    m = Mesh(AMR_BOX)
    assert m.tape_id() == 0
    cfg = TransportConfig(n_packets=10, sources=[Source(SOURCE_POINT, EMIT_ISOTROPIC, (0.5, 0.5, 0.5))],
                          image_n=8)
    c = cfg.to_c()
    for tid in (0, 1):
        st = _lib.lib.kp_transport_adjoint_tape(m.handle, tid, ctypes.byref(c), None, 24,
                                                None, None, None, None)
        assert st == _lib.KP_ERR_CONFIG
        assert b"no taped solve" in _lib.lib.kp_last_error()


def test_resume_arguments_are_checked_before_device_work():
    """kp_transport_forward_resume refuses a budget below 1, missing queues
    and overlapping in/out queues (KP_ERR_ARG), before touching a GPU."""
    from meshcases import AMR_BOX
    from kratos_polrad_b200 import Mesh
    from kratos_polrad_b200.transport import (CResume, EMIT_ISOTROPIC, SOURCE_POINT, Source,
                                              TransportConfig)
    from kratos_polrad_b200.config import CTallies
    m = Mesh(AMR_BOX)
    c = TransportConfig(n_packets=10, sources=[Source(SOURCE_POINT, EMIT_ISOTROPIC,
                                                      (0.5, 0.5, 0.5))]).to_c()
    t = CTallies()
    buf = (ctypes.c_ubyte * (128 * 8))()
    cnt = ctypes.c_ulonglong(0)
    base = ctypes.addressof(buf)

    def run(**kw):
        r = CResume()
        r.in_, r.n_in, r.out, r.cap_out = None, 0, base, 4
        r.out_count, r.step_budget = ctypes.addressof(cnt), 10
        for k, v in kw.items():
            setattr(r, k, v)
        st = _lib.lib.kp_transport_forward_resume(m.handle, ctypes.byref(c), ctypes.byref(r),
                                                  ctypes.byref(t), None)
        return st, _lib.lib.kp_last_error()

    st, msg = run(step_budget=0)
    assert st == _lib.KP_ERR_ARG and b"step_budget" in msg
    st, msg = run(out_count=None)
    assert st == _lib.KP_ERR_ARG and b"null queue" in msg
    st, msg = run(n_in=3)                       # in is null
    assert st == _lib.KP_ERR_ARG and b"null queue" in msg
    st, msg = run(in_=base + 128 * 2, n_in=3)   # overlaps out[2:4]
    assert st == _lib.KP_ERR_ARG and b"overlap" in msg


def test_resume_python_rejects_a_malformed_queue():
    """forward_resume checks the resumed queue's type and shape before any
    call (a CPU tensor of the wrong width here)."""
    import pytest
    import torch
    from meshcases import AMR_BOX
    from kratos_polrad_b200 import Mesh
    from kratos_polrad_b200.transport import (EMIT_ISOTROPIC, SOURCE_POINT, Source, Tallies,
                                              TransportConfig, forward_resume)
    cfg = TransportConfig(n_packets=10, sources=[Source(SOURCE_POINT, EMIT_ISOTROPIC,
                                                        (0.5, 0.5, 0.5))])
    tal = Tallies(cfg, device="cpu")
    with pytest.raises(ValueError, match="packet states"):
        forward_resume(Mesh(AMR_BOX), cfg, 10, resumed=torch.zeros((4, 64), dtype=torch.uint8),
                       tallies=tal)
