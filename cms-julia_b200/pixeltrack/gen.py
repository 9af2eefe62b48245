"""Seeded synthetic inputs (native generator libpxlgen.so).

Event modes follow the benchmark configurations:
  MODE_SINGLE  one vertex with ``ntracks`` helix tracks, no noise (small CPU case)
  MODE_PU      ``pu`` vertices, Poisson(30) tracks each, 1e-4 noise, 1% inefficiency
  MODE_UNIFORM pileup drawn uniformly in [0, pu] per event
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _native
from .formats import CONDITION_FILES

MODE_SINGLE, MODE_PU, MODE_UNIFORM = 0, 1, 2


def conditions() -> dict[str, bytes]:
    g = _native.gen()
    ptrs = [ctypes.c_void_p() for _ in range(5)]
    sizes = [ctypes.c_size_t() for _ in range(5)]
    args = []
    for p, s in zip(ptrs, sizes):
        args += [ctypes.byref(p), ctypes.byref(s)]
    rc = g.pxlgen_conditions(*args)
    if rc != 0:
        raise RuntimeError("pxlgen_conditions failed")
    out = {}
    for name, p, s in zip(CONDITION_FILES, ptrs, sizes):
        out[name] = ctypes.string_at(p.value, s.value)
        g.pxlgen_free(p)
    return out


def events(n_events: int, mode: int = MODE_PU, pu: float = 50.0, ntracks: int = 100, seed: int = 1,
           threads: int = 0) -> tuple[np.ndarray, np.ndarray]:
    """Returns (blob as uint8 array, event offsets uint64[n_events+1]) in raw.bin layout."""
    g = _native.gen()
    blob = ctypes.c_void_p()
    nb = ctypes.c_size_t()
    offs = np.zeros(n_events + 1, dtype=np.uint64)
    rc = g.pxlgen_events(seed, n_events, mode, float(pu), ntracks, threads, ctypes.byref(blob), ctypes.byref(nb),
                         offs.ctypes.data_as(ctypes.c_void_p))
    if rc != 0:
        raise RuntimeError("pxlgen_events failed")
    arr = np.frombuffer(ctypes.string_at(blob.value, nb.value), dtype=np.uint8).copy()
    g.pxlgen_free(blob)
    return arr, offs


def fit_tracks(n_tracks: int, seed: int = 1, threads: int = 0) -> dict[str, np.ndarray]:
    """Seeded fit workload: hits (H, 3) float64, ge (H, 6) float32 global covariances,
    offsets (n+1,) int32, module (H,) int16 (-1 off the pixel layers), truth (n, 5)
    float64 = (phi0, d0, q/pT, cot(theta), z0) at generation."""
    g = _native.gen()
    cap = 8 * n_tracks
    hits = np.zeros((cap, 3), np.float64)
    ge = np.zeros((cap, 6), np.float32)
    offs = np.zeros(n_tracks + 1, np.int32)
    mod = np.zeros(cap, np.int16)
    truth = np.zeros((n_tracks, 5), np.float64)
    vp = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    nh = g.pxlgen_fit_tracks(seed, n_tracks, threads, vp(hits), vp(ge), vp(offs), vp(mod), vp(truth))
    if nh < 0:
        raise RuntimeError("pxlgen_fit_tracks failed")
    return {"hits": hits[:nh], "ge": ge[:nh], "offsets": offs, "module": mod[:nh], "truth": truth}


def module_positions() -> np.ndarray:
    """Centres (1856, 3) of the synthetic geometry's modules, in cm."""
    out = np.zeros((1856, 3), np.float64)
    _native.gen().pxlgen_module_positions(out.ctypes.data_as(ctypes.c_void_p))
    return out
