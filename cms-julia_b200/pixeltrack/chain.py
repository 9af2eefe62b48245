"""Host-side handle of a reconstruction context (one CUDA context object of
libpxl_b200.so): runs single events or batches and copies products out in the
reference's layouts."""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _native
from ._native import PxlConditions, PxlEventCounts, PxlParams, check
from .formats import CONDITION_FILES

# product ids and element types (enum PxlProduct in include/pxl.h)
PRODUCTS: dict[str, tuple[int, type]] = {
    "xx": (1, np.int16), "yy": (2, np.int16), "adc": (3, np.int32), "module_ind": (4, np.int16),
    "clus": (5, np.int32), "pdigi": (6, np.uint32), "raw_id_arr": (7, np.uint32),
    "module_start": (10, np.uint32), "clus_in_module": (11, np.uint32), "module_id": (12, np.uint32),
    "clus_module_start": (13, np.uint32),
    "xl": (20, np.float32), "yl": (21, np.float32), "xerr": (22, np.float32), "yerr": (23, np.float32),
    "xg": (24, np.float32), "yg": (25, np.float32), "zg": (26, np.float32), "rg": (27, np.float32),
    "iphi": (28, np.int16), "charge": (29, np.uint32), "xsize": (30, np.int16), "ysize": (31, np.int16),
    "det_ind": (32, np.int16), "hits_layer_start": (33, np.uint32), "phi_off": (34, np.uint32),
    "phi_bins": (37, np.uint32), "phi_bins16": (35, np.uint16), "agc": (36, np.float32),
    "cells": (40, np.int32), "cell_neighbors": (41, np.uint32), "cell_tracks": (42, np.uint32),
    "outer_hit_of_cell": (43, np.uint32), "tuple_multiplicity": (44, np.uint32),
    "tuple_off": (50, np.uint32), "tuple_hits": (67, np.uint32), "tuple_hits16": (51, np.uint16),
    "det_hits": (52, np.uint16),
    "quality": (53, np.uint8), "chi2": (54, np.float32), "eta": (55, np.float32), "pt": (56, np.float32),
    "state": (57, np.float32), "cov": (58, np.float32), "fitted": (59, np.uint8),
    "idv": (60, np.int16), "zv": (61, np.float32), "wv": (62, np.float32), "vchi2": (63, np.float32),
    "ptv2": (64, np.float32), "ndof": (65, np.int32), "sort_ind": (66, np.uint16), "errors": (70, np.uint32),
}


@dataclass
class EventCounts:
    n_words: int
    n_modules: int
    n_clusters: int
    n_hits: int
    n_doublets: int
    n_tuples: int
    n_tuple_hits: int
    n_vertices: int
    n_vertex_tracks: int
    warnings: int
    n_errors: int
    n_fits_fp64: int


def default_params(**kw) -> PxlParams:
    p = PxlParams()
    check(_native.lib().pxl_params_default(ctypes.byref(p)), "pxl_params_default")
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def extended_params(**kw) -> PxlParams:
    """The reference's parameters with the extended per-event capacities (pxl_params_extended)."""
    p = PxlParams()
    check(_native.lib().pxl_params_extended(ctypes.byref(p)), "pxl_params_extended")
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def batch_params(n_events: int, words_per_event: int = 64_000, hits_per_event_avg: int = 16_000,
                 doublets_per_event_avg: int = 160_000, tuples_per_event_avg: int = 12_000, extended: bool = False,
                 **kw) -> PxlParams:
    """Buffer sizes for a batch of n_events with the given per-event averages; the per-event
    semantic capacities stay at the reference's values, or take the extended ones."""
    make = extended_params if extended else default_params
    return make(max_events=n_events, max_words=n_events * words_per_event,
                max_hits=n_events * hits_per_event_avg, max_doublets=n_events * doublets_per_event_avg,
                max_tuples=n_events * tuples_per_event_avg, **kw)


class PixelChain:
    """One reconstruction context on one GPU."""

    def __init__(self, conditions: dict[str, bytes], params: PxlParams | None = None):
        self._lib = _native.lib()
        self._cond_bufs = [conditions[n] for n in CONDITION_FILES]
        c = PxlConditions()
        for name, buf in zip(("cabling_map", "fed_ids", "gain", "cpe", "beamspot"), self._cond_bufs):
            setattr(c, name, ctypes.cast(ctypes.c_char_p(buf), ctypes.c_void_p))
            setattr(c, name + "_bytes", len(buf))
        self.params = params if params is not None else default_params()
        h = ctypes.c_void_p()
        check(self._lib.pxl_ctx_create(ctypes.byref(c), ctypes.byref(self.params), ctypes.byref(h)), "pxl_ctx_create")
        self._h = h
        self._keep: list = []
        self._slot_keep: list = [None] * _native.INPUT_SLOTS

    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            self._lib.pxl_ctx_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):  # pragma: no cover - best effort
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ---- running
    def run_event(self, raw_event: bytes | np.ndarray, stages: int = _native.STAGE_ALL) -> int:
        buf = np.ascontiguousarray(np.frombuffer(raw_event, dtype=np.uint8) if isinstance(raw_event, (bytes, bytearray))
                                   else raw_event, dtype=np.uint8)
        self._keep = [buf]
        check(self._lib.pxl_event_run(self._h, buf.ctypes.data, buf.nbytes, stages, None), "pxl_event_run")
        return self.sync()

    def continue_stages(self, stages: int) -> int:
        check(self._lib.pxl_event_continue(self._h, stages, None), "pxl_event_continue")
        return self.sync()

    def run_batch(self, blob: np.ndarray, offsets: np.ndarray, stages: int = _native.STAGE_ALL,
                  sync: bool = True) -> int:
        blob = np.ascontiguousarray(blob, dtype=np.uint8)
        offsets = np.ascontiguousarray(offsets, dtype=np.uint64)
        self._keep = [blob, offsets]
        n = len(offsets) - 1
        check(self._lib.pxl_batch_run(self._h, blob.ctypes.data, offsets.ctypes.data, n, 0, stages, None),
              "pxl_batch_run")
        return self.sync() if sync else 0

    def run_batch_device(self, blob_ptr: int, offsets_ptr: int, n_events: int, stages: int = _native.STAGE_ALL,
                         stream: int | None = None) -> None:
        """Batch already in device memory (pointers to the blob and its uint64 offsets)."""
        check(self._lib.pxl_batch_run(self._h, blob_ptr, offsets_ptr, n_events, 1, stages, stream),
              "pxl_batch_run")

    def stage_batch(self, blob: np.ndarray, offsets: np.ndarray, stream: int | None = None) -> None:
        blob = np.ascontiguousarray(blob, dtype=np.uint8)
        offsets = np.ascontiguousarray(offsets, dtype=np.uint64)
        self._keep = [blob, offsets]
        check(self._lib.pxl_batch_stage(self._h, blob.ctypes.data, offsets.ctypes.data, len(offsets) - 1, stream),
              "pxl_batch_stage")

    def capture_graph(self, stages: int = _native.STAGE_ALL) -> None:
        check(self._lib.pxl_graph_capture(self._h, stages), "pxl_graph_capture")

    def launch_graph(self, stream: int | None = None) -> None:
        check(self._lib.pxl_graph_launch(self._h, stream), "pxl_graph_launch")

    def stage_slot(self, slot: int, blob: np.ndarray, offsets: np.ndarray, stream: int | None = None) -> None:
        """Enqueues the copy of a batch into input slot `slot` on `stream` (pxl_slot_stage).
        blob should be pinned host memory and must stay unchanged until the copy ends."""
        blob = np.ascontiguousarray(blob, dtype=np.uint8)
        offsets = np.ascontiguousarray(offsets, dtype=np.uint64)
        self._slot_keep[slot] = [blob, offsets]
        check(self._lib.pxl_slot_stage(self._h, slot, blob.ctypes.data, offsets.ctypes.data, len(offsets) - 1,
                                       stream), "pxl_slot_stage")

    def launch_slot(self, slot: int, stream: int | None = None) -> None:
        """Replays input slot `slot`'s graph once its copy has ended (pxl_slot_launch)."""
        check(self._lib.pxl_slot_launch(self._h, slot, stream), "pxl_slot_launch")

    def results_async(self, host_ptr: int, max_events: int, stream: int | None = None) -> int:
        return check(self._lib.pxl_results_async(self._h, host_ptr, max_events, stream), "pxl_results_async")

    def export_async(self, out: "TrackExport", stream: int | None = None, copy_stream: int | None = None) -> None:
        """Compacted loose tracks and vertices of the last run into `out`'s pinned host arrays,
        one copy per array (pxl_export_async); read `out` after copy_stream reaches the copies."""
        check(self._lib.pxl_export_async(self._h, ctypes.byref(out.desc), stream, copy_stream), "pxl_export_async")

    def validate_counts(self, expected: np.ndarray) -> tuple[int, np.ndarray]:
        """CountValidator over the last run's events (pxl_validate_counts): expected (n, 5) =
        modules, digis, clusters, tracks, vertices per event (formats.read_counts layout).
        Returns (good events, per-event status: failed-check bits | N(track) << 8)."""
        x = np.ascontiguousarray(expected, dtype=np.uint32).reshape(-1, 5)
        st = np.zeros(len(x), np.uint32)
        good = check(self._lib.pxl_validate_counts(self._h, x.ctypes.data, len(x), st.ctypes.data),
                     "pxl_validate_counts")
        return good, st

    def sync(self) -> int:
        return check(self._lib.pxl_sync(self._h), "pxl_sync")

    def graph_kernel_nodes(self) -> int:
        return check(self._lib.pxl_graph_kernel_nodes(self._h), "pxl_graph_kernel_nodes")

    def profile(self, on: bool = True) -> None:
        check(self._lib.pxl_profile_enable(self._h, int(on)), "pxl_profile_enable")

    def profile_read(self) -> list[tuple[str, float]]:
        ms = (ctypes.c_float * 128)()
        names = (ctypes.c_char_p * 128)()
        n = check(self._lib.pxl_profile_read(self._h, ms, names, 128), "pxl_profile_read")
        return [(names[i].decode(), ms[i]) for i in range(n)]

    def autotune(self, candidates=(4, 8, 16, 32, 64, 128, -2, -8), reps: int = 2) -> dict[str, int]:
        """Chooses the launch shape of each tunable stage on the staged batch (pxl_autotune):
        c > 0 a static grid of c blocks per event, c < 0 a persistent work queue of virtual
        blocks of -c loop strides."""
        cand = (ctypes.c_int32 * len(candidates))(*candidates)
        out = (ctypes.c_int32 * len(_native.TUNE_STAGES))()
        check(self._lib.pxl_autotune(self._h, cand, len(candidates), reps, out), "pxl_autotune")
        return dict(zip(_native.TUNE_STAGES, list(out)))

    # ---- products
    def counts(self, event: int = 0) -> EventCounts:
        c = PxlEventCounts()
        check(self._lib.pxl_event_counts(self._h, event, ctypes.byref(c)), "pxl_event_counts")
        return EventCounts(**{f: getattr(c, f) for f, _ in PxlEventCounts._fields_})

    def product(self, name: str, event: int = 0) -> np.ndarray:
        pid, dt = PRODUCTS[name]
        n = self._lib.pxl_copy_product(self._h, event, pid, None, 0)
        if n < 0:
            raise RuntimeError(f"product {name} unavailable ({n})")
        out = np.empty(int(n), dtype=dt)
        if n:
            got = self._lib.pxl_copy_product(self._h, event, pid, out.ctypes.data, out.nbytes)
            if got < 0:
                raise RuntimeError(f"product {name} copy failed ({got})")
        return out

    def clusterize_digis(self, id_: np.ndarray, x: np.ndarray, y: np.ndarray, adc: np.ndarray,
                         charge_cut: bool = True) -> dict[str, np.ndarray]:
        n = len(id_)
        id_ = np.ascontiguousarray(id_, dtype=np.uint16)
        x = np.ascontiguousarray(x, dtype=np.int16)
        y = np.ascontiguousarray(y, dtype=np.int16)
        adc = np.ascontiguousarray(adc, dtype=np.int32)
        ms = np.zeros(2001, np.uint32)
        cim = np.zeros(2000, np.uint32)
        mid = np.zeros(2000, np.uint32)
        clus = np.zeros(n, np.int32)
        ido = np.zeros(n, np.uint16)
        check(self._lib.pxl_clusterize_digis(self._h, id_.ctypes.data, x.ctypes.data, y.ctypes.data, adc.ctypes.data,
                                             n, int(charge_cut), ms.ctypes.data, cim.ctypes.data, mid.ctypes.data,
                                             clus.ctypes.data, ido.ctypes.data), "pxl_clusterize_digis")
        return {"module_start": ms, "clus_in_module": cim, "module_id": mid, "clus": clus, "id": ido}


class TrackExport:
    """Pinned host arrays for pxl_export_async: per track state (5), pt, eta, chi2, hit count,
    vertex and tuple slot (and the 15 covariance terms with cov=True), per vertex zv, wv, chi2,
    ptv2 and ndof, and the per-event index (first track, tracks, first vertex, vertices)."""

    def __init__(self, n_events: int, max_tracks: int, max_vertices: int, cov: bool = False):
        import torch
        pin = lambda n, dt: torch.empty(int(n), dtype=dt, pin_memory=True)
        self.n_events = n_events
        self.arrays = {"index": pin(4 * (n_events + 1), torch.int32), "state": pin(5 * max_tracks, torch.float32),
                       "pt": pin(max_tracks, torch.float32), "eta": pin(max_tracks, torch.float32),
                       "chi2": pin(max_tracks, torch.float32), "n_hits": pin(max_tracks, torch.uint8),
                       "vertex": pin(max_tracks, torch.int16), "tuple": pin(max_tracks, torch.int32),
                       "zv": pin(max_vertices, torch.float32), "wv": pin(max_vertices, torch.float32),
                       "vchi2": pin(max_vertices, torch.float32), "ptv2": pin(max_vertices, torch.float32),
                       "ndof": pin(max_vertices, torch.int32)}
        if cov:
            self.arrays["cov"] = pin(15 * max_tracks, torch.float32)
        self.desc = _native.PxlExport(max_tracks=max_tracks, max_vertices=max_vertices)
        for k, t in self.arrays.items():
            setattr(self.desc, k, t.data_ptr())

    def bytes(self) -> int:
        return int(_native.lib().pxl_export_bytes(ctypes.byref(self.desc), self.n_events))

    def index(self) -> np.ndarray:
        """(n_events + 1, 4) uint32: first track, tracks, first vertex, vertices; last row the totals."""
        return self.arrays["index"].numpy().view(np.uint32).reshape(-1, 4)

    def event(self, e: int) -> dict[str, np.ndarray]:
        """The tracks and vertices of event e (after the copies completed)."""
        ft, nt, fv, nv = (int(v) for v in self.index()[e])
        out = {}
        for k, t in self.arrays.items():
            if k == "index":
                continue
            a = t.numpy()
            if k in ("state", "cov"):
                w = 5 if k == "state" else 15
                out[k] = a[w * ft:w * (ft + nt)].reshape(nt, w)
            elif k in ("zv", "wv", "vchi2", "ptv2", "ndof"):
                out[k] = a[fv:fv + nv]
            else:
                out[k] = a[ft:ft + nt]
        return out
