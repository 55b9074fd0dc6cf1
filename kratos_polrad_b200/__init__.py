"""kratos_polrad_b200: B200-native Monte-Carlo photon-packet transport.

Python mirror of the C ABI in include/kp_transport.h (the product is the
in-tree shared library libkp_b200.so; importing fails loudly without it).
"""
from ._lib import KPError, lib  # noqa: F401  (loads libkp_b200.so)
from .mesh import Mesh, MeshConfig, RefineRegion  # noqa: F401
from .trace import PacketPool, trace  # noqa: F401

__all__ = ["KPError", "Mesh", "MeshConfig", "RefineRegion", "PacketPool", "trace"]
