"""Comparison helpers: CUDA chain products against the CPU oracle's products."""
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


def compare_ca(gpu, orc, event: int = 0) -> list[str]:
    """Doublets, per-hit / per-cell lists, tuples, duplicate flags and multiplicity."""
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
    g, o = gpu.product("quality", event)[:nt], orc.get("quality")[:nt]
    if not same_bits(g, o):
        errs.append(f"quality: {first_diff(g, o)}")
    tm_off = orc.get("tm_off")
    tm = np.concatenate([tm_off, orc.get("tm_bins")[:tm_off[-1]].astype(np.uint32)])
    g = gpu.product("tuple_multiplicity", event)
    if not same_bits(g, tm):
        errs.append(f"tuple_multiplicity: {first_diff(g, tm)}")
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
