"""B200 core/accessory distance library: Python helpers above the C ABI.

``capi``   ctypes binding of include/sketchlib_b200.h (requires the built .so)
``synth``  seeded synthetic sketch populations
"""
from . import capi, synth  # noqa: F401

__all__ = ["capi", "synth"]
