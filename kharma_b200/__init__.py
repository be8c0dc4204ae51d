"""kharma_b200: B200-native (sm_100a) per-step GRMHD path for KHARMA.

The product is libkhb.so (kharma_b200/lib, C ABI in include/khb.h); this package binds it with
ctypes and provides the host-side pieces a KHARMA user needs to drive it: block options
(spec), initial states (problems) and a device block with the reference step/timestep
sequencing (block).
"""
from .spec import BlockSpec, FloorSpec, mhdmodes_spec, torus_spec  # noqa: F401

__all__ = ["BlockSpec", "FloorSpec", "mhdmodes_spec", "torus_spec"]
