"""Test infrastructure: Python handle of the CPU oracle (oracle/_lib/liboracle.so).

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg use this
module, as the checker of the CUDA chain. It exposes the oracle's products
under the same names as pixeltrack.chain.PRODUCTS.
"""
from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_lib" / "liboracle.so"

DTYPES = {
    "words": np.uint32, "xx": np.int16, "yy": np.int16, "adc": np.int32, "module_ind": np.int16, "clus": np.int32,
    "pdigi": np.uint32, "raw_id_arr": np.uint32, "module_start": np.uint32, "clus_in_module": np.uint32,
    "module_id": np.uint32, "clus_module_start": np.uint32, "xl": np.float32, "yl": np.float32,
    "xerr": np.float32, "yerr": np.float32, "xg": np.float32, "yg": np.float32, "zg": np.float32, "rg": np.float32,
    "iphi": np.int16, "charge": np.uint32, "xsize": np.int16, "ysize": np.int16, "det_ind": np.int16,
    "hits_layer_start": np.uint32, "phi_off": np.uint32, "phi_bins": np.uint32, "agc": np.float32,
    "cells": np.int32, "cell_neighbors": np.uint32, "cell_tracks": np.uint32, "outer_hit_of_cell": np.uint32,
    "tuple_off": np.uint32, "tuple_hits": np.uint32, "det_hits": np.uint16, "quality": np.uint8,
    "tm_off": np.uint32, "tm_bins": np.uint32, "pt": np.float32, "eta": np.float32, "chi2": np.float32,
    "state": np.float32, "cov": np.float32, "fitted": np.uint8, "hit_to_tuple_off": np.uint32,
    "hit_to_tuple_bins": np.uint32, "idv": np.int16, "zv": np.float32, "wv": np.float32, "vchi2": np.float32,
    "ptv2": np.float32, "ndof": np.int32, "sort_ind": np.uint16, "errors": np.uint32,
}
COUNT_NAMES = ("n_words", "n_modules", "n_clusters", "n_hits", "n_cells", "n_tuples", "n_tuple_hits", "nv_final",
               "n_vtx_tracks", "flags", "n_errors", "n_tracks")

# Per-event capacities of the extended mode (hits, doublets, tuples, fits per multiplicity,
# list columns): no pileup-200 event of the synthetic generator reaches them. The reference's
# own values (48K hits, 458,752 doublets, 32K tuples, 24K fits, 64K columns) are the default.
EXTENDED_CAPS = {"hits": 256 * 1024, "doublets": 4 * 1024 * 1024, "tuples": 256 * 1024,
                 "fits_per_mult": 256 * 1024, "columns": 4 * 1024 * 1024}

_lib = None


def build() -> Path:
    """Compiles the oracle with its Makefile (g++ only)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        _lib = ctypes.CDLL(str(LIB))
        V = ctypes.c_void_p
        _lib.orc_ctx_create.restype = V
        _lib.orc_ctx_create.argtypes = [V, ctypes.c_size_t] * 5
        _lib.orc_ctx_destroy.argtypes = [V]
        _lib.orc_set_caps.argtypes = [V] + [ctypes.c_uint32] * 5
        _lib.orc_run_event.restype = ctypes.c_int32
        _lib.orc_run_event.argtypes = [V, V, ctypes.c_size_t, ctypes.c_int32]
        _lib.orc_counts.argtypes = [V, V]
        _lib.orc_get.restype = ctypes.c_int64
        _lib.orc_get.argtypes = [V, ctypes.c_char_p, V, ctypes.c_int64]
        _lib.orc_clusterize_digis.argtypes = [V, V, V, V, ctypes.c_int32, V, V, V, V, V, ctypes.c_int32]
        _lib.orc_bl_fit.restype = ctypes.c_int32
        _lib.orc_bl_fit.argtypes = [V, V, ctypes.c_int32, ctypes.c_double, V, V, V, V, V, V]
        _lib.orc_bl_chi2_grad_fwd.restype = ctypes.c_double
        _lib.orc_bl_chi2_grad_fwd.argtypes = [V, V, ctypes.c_int32, ctypes.c_double, V]
        _lib.orc_riemann_fit.restype = ctypes.c_int32
        _lib.orc_riemann_fit.argtypes = [V, V, ctypes.c_int32, ctypes.c_double, V, V, V]
        _lib.orc_bl_fit_batch.restype = ctypes.c_double
        _lib.orc_bl_fit_batch.argtypes = [V, V, V, ctypes.c_int32, ctypes.c_double, ctypes.c_int32, V, V]
        _lib.orc_run_batch.restype = ctypes.c_double
        _lib.orc_run_batch.argtypes = [V, V, V, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, V]
    return _lib


class Oracle:
    """caps: per-event capacities (keys of EXTENDED_CAPS), the reference's when None."""

    def __init__(self, conds: dict[str, bytes], caps: dict[str, int] | None = None):
        self._l = lib()
        names = ("cablingMap.bin", "fedIds.bin", "gain.bin", "cpefast.bin", "beamspot.bin")
        self._bufs = [conds[n] for n in names]
        args = []
        for b in self._bufs:
            args += [ctypes.cast(ctypes.c_char_p(b), ctypes.c_void_p), len(b)]
        self._h = self._l.orc_ctx_create(*args)
        if not self._h:
            raise RuntimeError("oracle: bad conditions")
        if caps:
            self._l.orc_set_caps(self._h, *(int(caps.get(k, 0)) for k in ("hits", "doublets", "tuples",
                                                                            "fits_per_mult", "columns")))

    def close(self):
        if self._h:
            self._l.orc_ctx_destroy(self._h)
            self._h = None

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass

    def run_event(self, raw: bytes | np.ndarray, stages: int = 63) -> int:
        buf = np.ascontiguousarray(np.frombuffer(raw, np.uint8) if isinstance(raw, (bytes, bytearray)) else raw,
                                   dtype=np.uint8)
        return self._l.orc_run_event(self._h, buf.ctypes.data, buf.nbytes, stages)

    def counts(self) -> dict[str, int]:
        out = (ctypes.c_uint32 * len(COUNT_NAMES))()
        self._l.orc_counts(self._h, out)
        return dict(zip(COUNT_NAMES, list(out)))

    def get(self, name: str) -> np.ndarray:
        n = self._l.orc_get(self._h, name.encode(), None, 0)
        if n < 0:
            raise KeyError(name)
        a = np.empty(int(n), dtype=DTYPES[name])
        if n:
            self._l.orc_get(self._h, name.encode(), a.ctypes.data, a.nbytes)
        return a

    def run_batch(self, blob: np.ndarray, offsets: np.ndarray, threads: int, stages: int = 63,
                  counts: bool = False):
        blob = np.ascontiguousarray(blob, np.uint8)
        offsets = np.ascontiguousarray(offsets, np.uint64)
        n = len(offsets) - 1
        cnt = np.zeros((n, len(COUNT_NAMES)), np.uint32) if counts else None
        dt = self._l.orc_run_batch(self._h, blob.ctypes.data, offsets.ctypes.data, n, threads, stages,
                                   cnt.ctypes.data if counts else None)
        return (dt, cnt) if counts else dt


def clusterize_digis(id_, x, y, adc, charge_cut: bool = True) -> dict[str, np.ndarray]:
    l = lib()
    n = len(id_)
    id_ = np.ascontiguousarray(id_, np.uint16)
    x = np.ascontiguousarray(x, np.int16)
    y = np.ascontiguousarray(y, np.int16)
    adc = np.ascontiguousarray(adc, np.int32)
    ms = np.zeros(2001, np.uint32)
    cim = np.zeros(2000, np.uint32)
    mid = np.zeros(2000, np.uint32)
    clus = np.zeros(n, np.int32)
    ido = np.zeros(n, np.uint16)
    l.orc_clusterize_digis(id_.ctypes.data, x.ctypes.data, y.ctypes.data, adc.ctypes.data, n, ms.ctypes.data,
                           cim.ctypes.data, mid.ctypes.data, clus.ctypes.data, ido.ctypes.data, int(charge_cut))
    return {"module_start": ms, "clus_in_module": cim, "module_id": mid, "clus": clus, "id": ido}


def bl_fit(hits: np.ndarray, ge: np.ndarray, B: float) -> dict:
    """hits: (3, N) float64, ge: (6, N) float32 (column per hit)."""
    l = lib()
    h = np.ascontiguousarray(np.asarray(hits, np.float64).T)   # column-major 3xN == row-major N x 3
    g = np.ascontiguousarray(np.asarray(ge, np.float32).T)
    n = h.shape[0]
    st = np.zeros(5)
    cv = np.zeros(15)
    c2 = np.zeros(2)
    pt = np.zeros(1)
    eta = np.zeros(1)
    ff = np.zeros(4)
    rc = l.orc_bl_fit(h.ctypes.data, g.ctypes.data, n, B, st.ctypes.data, cv.ctypes.data, c2.ctypes.data,
                      pt.ctypes.data, eta.ctypes.data, ff.ctypes.data)
    return {"rc": rc, "state": st, "cov": cv, "chi2_line": c2[0], "chi2_circle": c2[1], "pt": pt[0], "eta": eta[0],
            "fast_fit": ff}


def bl_fit_batch(hits: np.ndarray, ge: np.ndarray, offsets: np.ndarray, B: float, threads: int = 1):
    """FP64 fits of a track collection: hits (H, 3) float64, ge (H, 6) float32, offsets
    (n+1,) int32. Returns (state (n, 5), pt (n,), elapsed seconds)."""
    l = lib()
    h = np.ascontiguousarray(hits, np.float64)
    g = np.ascontiguousarray(ge, np.float32)
    o = np.ascontiguousarray(offsets, np.int32)
    n = len(o) - 1
    st = np.zeros((n, 5))
    pt = np.zeros(n)
    dt = l.orc_bl_fit_batch(h.ctypes.data, g.ctypes.data, o.ctypes.data, n, B, threads, st.ctypes.data, pt.ctypes.data)
    return st, pt, dt


def bl_chi2_grad_fwd(hits: np.ndarray, ge: np.ndarray, B: float):
    """chi2_line + chi2_circle of one track and its gradient (N, 3) with respect to the hits
    (forward-mode dual numbers through the reference formulation). hits (N, 3), ge (N, 6)."""
    h = np.ascontiguousarray(hits, np.float64)
    g = np.ascontiguousarray(ge, np.float32)
    grad = np.zeros_like(h)
    c = lib().orc_bl_chi2_grad_fwd(h.ctypes.data, g.ctypes.data, h.shape[0], B, grad.ctypes.data)
    return c, grad


def riemann_fit(hits: np.ndarray, ge: np.ndarray, B: float) -> dict:
    """Riemann helix fit of one track: hits (N, 3) float64, ge (N, 6) float32. state =
    (phi, d0, q/pT, cot(theta), zip)."""
    h = np.ascontiguousarray(hits, np.float64)
    g = np.ascontiguousarray(ge, np.float32)
    st = np.zeros(5)
    c2 = np.zeros(2)
    pt = np.zeros(1)
    rc = lib().orc_riemann_fit(h.ctypes.data, g.ctypes.data, h.shape[0], B, st.ctypes.data, c2.ctypes.data, pt.ctypes.data)
    return {"rc": rc, "state": st, "chi2_circle": c2[0], "chi2_line": c2[1], "pt": pt[0]}
