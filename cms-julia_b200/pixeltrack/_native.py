"""ctypes bindings of the C ABI in include/pxl.h (libpxl_b200.so) and of the
synthetic generator (libpxlgen.so). Loading fails loudly when a library is
missing: there is no CPU fallback for the reconstruction."""
from __future__ import annotations

import ctypes
from pathlib import Path

LIBDIR = Path(__file__).resolve().parent.parent / "lib"

PXL_ERR = {-1: "bad argument", -2: "CUDA error", -3: "bad conditions", -4: "capacity", -5: "bad state"}

STAGE_DIGIS, STAGE_HITS, STAGE_TUPLES, STAGE_FIT, STAGE_CLASSIFY, STAGE_VERTICES = 1, 2, 4, 8, 16, 32
STAGE_ALL = 0x3F

INPUT_SLOTS = 2  # PXL_INPUT_SLOTS
TUNE_STAGES = ("doublets", "hit_lists", "connect", "cell_lists", "fishbone", "ntuplets", "cell_tracks",
               "early_dup", "classify", "hit_to_tuple", "fits")

WARN_BITS = {
    0x1: "modules", 0x2: "pixels_per_module", 0x4: "clusters_per_module", 0x8: "hits_clamped",
    0x10: "doublets", 0x20: "columns", 0x40: "tuples", 0x80: "fit_domain", 0x100: "fits_capped",
    0x200: "vertex", 0x400: "lists", 0x800: "buffer", 0x1000: "fed_format",
}


class PxlConditions(ctypes.Structure):
    _fields_ = [
        ("cabling_map", ctypes.c_void_p), ("cabling_map_bytes", ctypes.c_size_t),
        ("fed_ids", ctypes.c_void_p), ("fed_ids_bytes", ctypes.c_size_t),
        ("gain", ctypes.c_void_p), ("gain_bytes", ctypes.c_size_t),
        ("cpe", ctypes.c_void_p), ("cpe_bytes", ctypes.c_size_t),
        ("beamspot", ctypes.c_void_p), ("beamspot_bytes", ctypes.c_size_t),
    ]


class PxlParams(ctypes.Structure):
    _fields_ = [
        ("device", ctypes.c_int32), ("max_events", ctypes.c_int32),
        ("max_words", ctypes.c_int64), ("max_hits", ctypes.c_int64), ("max_doublets", ctypes.c_int64),
        ("max_tuples", ctypes.c_int64),
        ("hits_per_event", ctypes.c_int32), ("doublets_per_event", ctypes.c_int32),
        ("tuples_per_event", ctypes.c_int32), ("fits_per_multiplicity", ctypes.c_int32),
        ("include_errors", ctypes.c_int32), ("use_quality", ctypes.c_int32),
        ("blocks_per_event", ctypes.c_int32), ("threads_per_block", ctypes.c_int32),
        ("columns_per_event", ctypes.c_int32), ("fit_precision", ctypes.c_int32),
    ]


class PxlEventCounts(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint32) for n in (
        "n_words", "n_modules", "n_clusters", "n_hits", "n_doublets", "n_tuples", "n_tuple_hits",
        "n_vertices", "n_vertex_tracks", "warnings", "n_errors", "n_fits_fp64")]


class PxlExport(ctypes.Structure):
    _fields_ = [("max_tracks", ctypes.c_int64), ("max_vertices", ctypes.c_int64)] + [
        (n, ctypes.c_void_p) for n in ("index", "state", "cov", "pt", "eta", "chi2", "n_hits", "vertex", "tuple",
                                       "zv", "wv", "vchi2", "ptv2", "ndof")]


_lib = None
_gen = None

# exported entry points and their signatures
_SIGS = {
    "pxl_version": (ctypes.c_int32, []),
    "pxl_params_default": (ctypes.c_int32, [ctypes.POINTER(PxlParams)]),
    "pxl_params_extended": (ctypes.c_int32, [ctypes.POINTER(PxlParams)]),
    "pxl_ctx_create": (ctypes.c_int32, [ctypes.POINTER(PxlConditions), ctypes.POINTER(PxlParams),
                                        ctypes.POINTER(ctypes.c_void_p)]),
    "pxl_ctx_destroy": (ctypes.c_int32, [ctypes.c_void_p]),
    "pxl_event_run": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_uint32,
                                       ctypes.c_void_p]),
    "pxl_event_continue": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p]),
    "pxl_batch_run": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32,
                                       ctypes.c_int32, ctypes.c_uint32, ctypes.c_void_p]),
    "pxl_batch_stage": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32,
                                         ctypes.c_void_p]),
    "pxl_graph_capture": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_uint32]),
    "pxl_slot_stage": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p,
                                        ctypes.c_int32, ctypes.c_void_p]),
    "pxl_slot_launch": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p]),
    "pxl_graph_launch": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_void_p]),
    "pxl_sync": (ctypes.c_int32, [ctypes.c_void_p]),
    "pxl_autotune": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32,
                                      ctypes.c_void_p]),
    "pxl_graph_kernel_nodes": (ctypes.c_int32, [ctypes.c_void_p]),
    "pxl_export_async": (ctypes.c_int32, [ctypes.c_void_p, ctypes.POINTER(PxlExport), ctypes.c_void_p,
                                          ctypes.c_void_p]),
    "pxl_export_bytes": (ctypes.c_int64, [ctypes.POINTER(PxlExport), ctypes.c_int32]),
    "pxl_validate_counts": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p]),
    "pxl_results_async": (ctypes.c_int64, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p]),
    "pxl_profile_enable": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_int32]),
    "pxl_profile_read": (ctypes.c_int32, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_float),
                                          ctypes.POINTER(ctypes.c_char_p), ctypes.c_int32]),
    "pxl_event_counts": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_int32, ctypes.POINTER(PxlEventCounts)]),
    "pxl_copy_product": (ctypes.c_int64, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p,
                                          ctypes.c_int64]),
    "pxl_clusterize_digis": (ctypes.c_int32, [ctypes.c_void_p] + [ctypes.c_void_p] * 4 + [ctypes.c_int32,
                             ctypes.c_int32] + [ctypes.c_void_p] * 5),
    "pxl_clusterize_digis_noalloc": (ctypes.c_int32, [ctypes.c_void_p] * 4 + [ctypes.c_int32, ctypes.c_int32]
                                     + [ctypes.c_void_p] * 6),
    "pxl_fit_workspace_bytes": (ctypes.c_int64, [ctypes.c_int32]),
    "pxl_adjoint_workspace_bytes": (ctypes.c_int64, [ctypes.c_int32, ctypes.c_int32]),
    "pxl_riemann_fit": (ctypes.c_int32, [ctypes.c_void_p] * 3 + [ctypes.c_int32, ctypes.c_double, ctypes.c_int32] +
                        [ctypes.c_void_p] * 5 + [ctypes.c_int64, ctypes.c_void_p]),
    "pxl_bl_fit_adjoint": (ctypes.c_int32, [ctypes.c_void_p] * 3 + [ctypes.c_int32, ctypes.c_double] +
                           [ctypes.c_void_p] * 3 + [ctypes.c_int32] + [ctypes.c_void_p] * 5 +
                           [ctypes.c_int64, ctypes.c_void_p]),
    "pxl_bl_fit": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32,
                                    ctypes.c_double, ctypes.c_int32] + [ctypes.c_void_p] * 6 +
                   [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p]),
}


def exported_symbols() -> list[str]:
    return sorted(_SIGS)


def lib() -> ctypes.CDLL:
    """The CUDA library; raises if it was not built."""
    global _lib
    if _lib is None:
        path = LIBDIR / "libpxl_b200.so"
        if not path.exists():
            raise RuntimeError(f"{path} is missing: build it with cms-julia_b200/build.py (no CPU fallback)")
        _lib = ctypes.CDLL(str(path))
        for name, (res, args) in _SIGS.items():
            f = getattr(_lib, name)
            f.restype = res
            f.argtypes = args
    return _lib


def gen() -> ctypes.CDLL:
    global _gen
    if _gen is None:
        path = LIBDIR / "libpxlgen.so"
        if not path.exists():
            raise RuntimeError(f"{path} is missing: build it with cms-julia_b200/build.py")
        _gen = ctypes.CDLL(str(path))
        P = ctypes.POINTER(ctypes.c_void_p)
        S = ctypes.POINTER(ctypes.c_size_t)
        _gen.pxlgen_conditions.restype = ctypes.c_int
        _gen.pxlgen_conditions.argtypes = [P, S] * 5
        _gen.pxlgen_events.restype = ctypes.c_int
        _gen.pxlgen_events.argtypes = [ctypes.c_uint64, ctypes.c_int32, ctypes.c_int32, ctypes.c_double,
                                       ctypes.c_int32, ctypes.c_int32, P, S, ctypes.c_void_p]
        _gen.pxlgen_fit_tracks.restype = ctypes.c_int32
        _gen.pxlgen_fit_tracks.argtypes = [ctypes.c_uint64, ctypes.c_int32, ctypes.c_int32] + [ctypes.c_void_p] * 5
        _gen.pxlgen_module_positions.restype = ctypes.c_int32
        _gen.pxlgen_module_positions.argtypes = [ctypes.c_void_p]
        _gen.pxlgen_free.restype = None
        _gen.pxlgen_free.argtypes = [ctypes.c_void_p]
    return _gen


def check(rc: int, what: str) -> int:
    """Raises on a fatal status; returns the warning bits otherwise."""
    if rc < 0:
        raise RuntimeError(f"{what} failed: {PXL_ERR.get(rc, rc)}")
    return rc


def warn_names(bits: int) -> list[str]:
    return [n for b, n in WARN_BITS.items() if bits & b]
