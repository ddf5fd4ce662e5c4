"""superlite_b200 -- SuperLite's per-timestep hot path on NVIDIA B200 (sm_100a).

The product is the CUDA library libslg.so (C ABI in include/slg.h, kernels in
csrc/); this package builds it (build.py), binds it (capi.py) and exposes the
reference's routine names (api.HotPath).  workloads.py makes the seeded
synthetic inputs of the benchmark configurations.
"""
from .api import HotPath, PACKET_DTYPE  # noqa: F401
from .capi import SlgError  # noqa: F401

__all__ = ["HotPath", "PACKET_DTYPE", "SlgError"]
