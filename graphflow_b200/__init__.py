"""graphflow_b200: B200-native transform-batch hot path of graphFlow (tile flattening, dense and
hash classify, exact slot planning, scatter, and the particle/photon transform bodies) behind a
C ABI (include/graphflow_b200.h). This Python package is the binding used by the tests and the
benchmark; it loads the in-tree native library and has no CPU fallback."""
from . import capi  # noqa: F401

__all__ = ["capi"]
