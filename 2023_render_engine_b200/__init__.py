"""B200-native rendering core (sm_100a) behind the reference renderer's hot-path API.

The CUDA library (lib/librt_b200.so) is the product; this package loads it through
ctypes (`_native`), wraps contexts and scenes (`core`) and provides the seeded
synthetic scenes used by tests and benchmarks (`scenes`).
"""
from . import scenes  # noqa: F401

__all__ = ["scenes", "core", "_native"]
