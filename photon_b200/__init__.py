"""photon_b200: a B200-native wavefront path tracer that is a drop-in for Photon's GPU renderer.

The product is the CUDA library libphoton_wavefront.so behind the C ABI of
include/photon_wavefront.h; `photon_b200.native` binds it with ctypes and mirrors Photon's
GpuRenderer interface. `photon_b200.abi` holds the ctypes structures.
"""
from . import abi  # noqa: F401

__all__ = ["abi", "native"]
