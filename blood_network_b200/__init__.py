"""B200-native AMG-preconditioned CG for vessel-network pressure systems.

The product is the C ABI library ``lib/libamg_b200.so`` (declared in
``include/amg_b200.h``); this package holds its CUDA sources (``csrc/``), the
ctypes binding (``amg``), the seeded network generator (``network``) and the
build step (``build``).
"""
from .network import Network, vascular_network, make_config, CONFIGS  # noqa: F401

__all__ = ["Network", "vascular_network", "make_config", "CONFIGS"]
