"""kratos_polrad_b200: B200-native Monte-Carlo photon-packet transport.

Python mirror of the C ABI in include/kp_transport.h.  The product is the
in-tree shared library libkp_b200.so: every module that calls it (mesh,
transport, walk, adjoint, batch, decomp, bio) loads it on import and fails
loudly without it.  ``config`` (plain set-up types) and ``problems`` (the
synthetic problem set-ups as data) load nothing, so that other
implementations of the path can be handed the same inputs.
"""
_EXPORTS = {"KPError": "._lib", "lib": "._lib", "Mesh": ".mesh", "MeshConfig": ".config",
            "RefineRegion": ".config", "PacketPool": ".walk", "trace": ".walk"}

__all__ = sorted(_EXPORTS)


def __getattr__(name):
    if name in _EXPORTS:
        import importlib
        value = getattr(importlib.import_module(_EXPORTS[name], __name__), name)
        globals()[name] = value
        return value
    raise AttributeError(f"module {__name__!r} has no attribute {name!r}")
