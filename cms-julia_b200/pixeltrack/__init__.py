"""B200-native pixel reconstruction chain (host side).

The reconstruction runs in libpxl_b200.so (hand-written sm_100a CUDA behind the
C ABI of include/pxl.h); this package binds it with ctypes and mirrors the
reference's producer interface. Import fails loudly if the library is missing.
"""
from . import _native
from ._native import (STAGE_ALL, STAGE_CLASSIFY, STAGE_DIGIS, STAGE_FIT, STAGE_HITS, STAGE_TUPLES,
                      STAGE_VERTICES)
from .chain import PRODUCTS, PixelChain, TrackExport, batch_params, default_params, extended_params

__all__ = ["PixelChain", "TrackExport", "default_params", "extended_params", "batch_params", "PRODUCTS", "STAGE_ALL", "STAGE_DIGIS", "STAGE_HITS",
           "STAGE_TUPLES", "STAGE_FIT", "STAGE_CLASSIFY", "STAGE_VERTICES", "native_library"]


def native_library():
    """Loads (or returns) the CUDA library; raises when it is not built."""
    return _native.lib()
