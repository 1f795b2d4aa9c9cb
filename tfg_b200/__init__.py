"""B200-native path-tracing hot path with a neural radiance cache.

The product is the native library ``libtfgpt.so`` (C ABI in
``include/tfg_pt.h``); this package binds it and provides the seeded
synthetic scenes and the host-side call sequence.
"""
from . import scenes, structs  # noqa: F401
from ._lib import TfgError, lib  # noqa: F401

__all__ = ["scenes", "structs", "lib", "TfgError"]
