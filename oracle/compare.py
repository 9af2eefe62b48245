"""Test infrastructure: comparison of the CUDA chain's products with the CPU oracle's.

Used by tests/ and by bench.py's parity check (outside any timed region) as the checker;
the product path never imports it."""
from __future__ import annotations

import numpy as np

DIGI_PRODUCTS = ("xx", "yy", "adc", "module_ind", "clus", "pdigi", "raw_id_arr")
HIT_FLOAT_PRODUCTS = ("xl", "yl", "xerr", "yerr", "xg", "yg", "zg", "rg")
HIT_INT_PRODUCTS = ("iphi", "charge", "xsize", "ysize", "det_ind")


def same_bits(a: np.ndarray, b: np.ndarray) -> bool:
    """Bit-exact equality (floats compared by their bit patterns)."""
    if a.shape != b.shape or a.dtype != b.dtype:
        return False
    if a.dtype.kind == "f":
        return bool(np.array_equal(a.view(np.uint32 if a.itemsize == 4 else np.uint64),
                                   b.view(np.uint32 if b.itemsize == 4 else np.uint64)))
    return bool(np.array_equal(a, b))


def first_diff(a: np.ndarray, b: np.ndarray) -> str:
    if a.shape != b.shape:
        return f"shape {a.shape} vs {b.shape}"
    idx = np.flatnonzero(a != b) if a.dtype.kind != "f" else np.flatnonzero(
        a.view(np.uint32 if a.itemsize == 4 else np.uint64) != b.view(np.uint32 if b.itemsize == 4 else np.uint64))
    if len(idx) == 0:
        return "equal"
    i = idx[0]
    return f"{len(idx)} differences, first at {i}: {a[i]} vs {b[i]}"


def compare_digis_clusters(gpu, orc, event: int = 0) -> list[str]:
    errs = []
    c = gpu.counts(event)
    oc = orc.counts()
    for k_g, k_o in (("n_words", "n_words"), ("n_modules", "n_modules"), ("n_clusters", "n_clusters")):
        if getattr(c, k_g) != oc[k_o]:
            errs.append(f"{k_g}: gpu {getattr(c, k_g)} oracle {oc[k_o]}")
    for name in DIGI_PRODUCTS:
        g, o = gpu.product(name, event), orc.get(name)
        if not same_bits(g, o):
            errs.append(f"{name}: {first_diff(g, o)}")
    nm = oc["n_modules"]
    for name, n in (("module_start", nm + 1), ("module_id", nm), ("clus_in_module", 2000), ("clus_module_start", 2001)):
        g, o = gpu.product(name, event)[:n], orc.get(name)[:n]
        if not same_bits(g, o):
            errs.append(f"{name}: {first_diff(g, o)}")
    return errs


def compare_ca(gpu, orc, event: int = 0, classified: bool = False) -> list[str]:
    """Doublets, per-hit / per-cell lists, tuples, duplicate flags and multiplicity
    (the last two only before classification changes the quality flags)."""
    errs = []
    c = gpu.counts(event)
    oc = orc.counts()
    if c.n_doublets != oc["n_cells"]:
        errs.append(f"n_doublets: gpu {c.n_doublets} oracle {oc['n_cells']}")
    if c.n_tuples != oc["n_tuples"]:
        errs.append(f"n_tuples: gpu {c.n_tuples} oracle {oc['n_tuples']}")
    if errs:
        return errs
    for name in ("cells", "outer_hit_of_cell", "cell_neighbors", "cell_tracks"):
        g, o = gpu.product(name, event), orc.get(name)
        if not same_bits(g, o):
            errs.append(f"{name}: {first_diff(g, o)}")
    nt, nth = oc["n_tuples"], oc["n_tuple_hits"]
    g, o = gpu.product("tuple_off", event), orc.get("tuple_off")
    if not same_bits(g, o):
        errs.append(f"tuple_off: {first_diff(g, o)}")
    for name in ("tuple_hits", "det_hits"):
        g, o = gpu.product(name, event), orc.get(name)[:nth]
        if not same_bits(g, o):
            errs.append(f"{name}: {first_diff(g, o)}")
    if classified:
        return errs
    g, o = gpu.product("quality", event)[:nt], orc.get("quality")[:nt]
    if not same_bits(g, o):
        errs.append(f"quality: {first_diff(g, o)}")
    tm_off = orc.get("tm_off")
    tm = np.concatenate([tm_off, orc.get("tm_bins")[:tm_off[-1]].astype(np.uint32)])
    g = gpu.product("tuple_multiplicity", event)
    if not same_bits(g, tm):
        errs.append(f"tuple_multiplicity: {first_diff(g, tm)}")
    return errs


# FP64 fits on the GPU and on the CPU use the same operation order; only the
# transcendentals (atan, log, sin, cos, asinh: CUDA vs the C library, each within
# 2 ulp in FP64) differ, and the results are stored as FP32.
FIT_RTOL = 1e-5
FIT_ATOL = {"state": 1e-6, "cov": 1e-12, "pt": 1e-6, "eta": 1e-6, "chi2": 1e-6}


def compare_fits(gpu, orc, event: int = 0) -> list[str]:
    errs = []
    nt = orc.counts()["n_tuples"]
    fg, fo = gpu.product("fitted", event)[:nt], orc.get("fitted")[:nt]
    if not same_bits(fg, fo):
        errs.append(f"fitted: {first_diff(fg, fo)}")
        return errs
    sel = fo.astype(bool)
    for name, w in (("state", 5), ("cov", 15), ("pt", 1), ("eta", 1), ("chi2", 1)):
        g = gpu.product(name, event)[:nt * w].reshape(nt, w)[sel]
        o = orc.get(name)[:nt * w].reshape(nt, w)[sel]
        if name == "pt":
            # pT = 1 / |q/pT|: compared as its reciprocal with the bounds of state[2], since a
            # nearly straight track's curvature is known to an absolute, not a relative, error
            with np.errstate(divide="ignore"):
                g, o = 1.0 / g.astype(np.float64), 1.0 / o.astype(np.float64)
        bad = ~np.isclose(g, o, rtol=FIT_RTOL, atol=FIT_ATOL[name], equal_nan=True)
        if bad.any():
            i = np.argwhere(bad)[0]
            errs.append(f"{name}: {int(bad.sum())} values off, first {tuple(i)}: {g[tuple(i)]} vs {o[tuple(i)]}")
    return errs


def compare_quality(gpu, orc, event: int = 0) -> list[str]:
    nt = orc.counts()["n_tuples"]
    g, o = gpu.product("quality", event)[:nt], orc.get("quality")[:nt]
    return [] if same_bits(g, o) else [f"quality: {first_diff(g, o)}"]


def compare_vertices(gpu, orc, event: int = 0) -> list[str]:
    errs = []
    c = gpu.counts(event)
    oc = orc.counts()
    if c.n_vertices != oc["nv_final"] or c.n_vertex_tracks != oc["n_vtx_tracks"]:
        return [f"vertices: gpu {c.n_vertices}/{c.n_vertex_tracks} oracle {oc['nv_final']}/{oc['n_vtx_tracks']}"]
    nv = oc["nv_final"]
    for name in ("idv", "sort_ind"):
        g, o = gpu.product(name, event), orc.get(name)
        if not same_bits(g, o):
            errs.append(f"{name}: {first_diff(g, o)}")
    n = max(nv, oc["n_vtx_tracks"])
    g, o = gpu.product("ndof", event)[:n], orc.get("ndof")[:n]
    if not same_bits(g, o):
        errs.append(f"ndof: {first_diff(g, o)}")
    for name in ("zv", "wv", "vchi2", "ptv2"):
        g, o = gpu.product(name, event)[:nv], orc.get(name)[:nv]
        if not np.allclose(g, o, rtol=1e-5, atol=1e-7):
            errs.append(f"{name}: {first_diff(g, o)}")
    return errs


def compare_hits(gpu, orc, event: int = 0) -> list[str]:
    errs = []
    c = gpu.counts(event)
    oc = orc.counts()
    if c.n_hits != oc["n_hits"]:
        errs.append(f"n_hits: gpu {c.n_hits} oracle {oc['n_hits']}")
        return errs
    for name in HIT_FLOAT_PRODUCTS + HIT_INT_PRODUCTS + ("hits_layer_start", "phi_off", "phi_bins", "agc"):
        g, o = gpu.product(name, event), orc.get(name)
        if not same_bits(g, o):
            errs.append(f"{name}: {first_diff(g, o)}")
    return errs


def compare_event(gpu, orc, event: int = 0) -> list[str]:
    """Every product of one event after the whole chain."""
    return (compare_digis_clusters(gpu, orc, event) + compare_hits(gpu, orc, event)
            + compare_ca(gpu, orc, event, classified=True) + compare_fits(gpu, orc, event)
            + compare_quality(gpu, orc, event) + compare_vertices(gpu, orc, event))


COUNT_PAIRS = (("n_words", "n_words"), ("n_modules", "n_modules"), ("n_clusters", "n_clusters"),
               ("n_hits", "n_hits"), ("n_doublets", "n_cells"), ("n_tuples", "n_tuples"),
               ("n_tuple_hits", "n_tuple_hits"), ("n_vertices", "nv_final"), ("n_vertex_tracks", "n_vtx_tracks"),
               ("n_errors", "n_errors"))


def compare_counts(gpu_counts, oracle_counts) -> list[int]:
    """Events whose per-event counts differ. gpu_counts: EventCounts per event; oracle_counts:
    the (n_events, 11) array of Oracle.run_batch(counts=True)."""
    from .oracle import COUNT_NAMES
    idx = {n: i for i, n in enumerate(COUNT_NAMES)}
    bad = []
    for e, c in enumerate(gpu_counts):
        if any(int(getattr(c, g)) != int(oracle_counts[e, idx[o]]) for g, o in COUNT_PAIRS):
            bad.append(e)
    return bad
