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
