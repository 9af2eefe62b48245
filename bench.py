"""Benchmark of the pixel reconstruction chain on B200.

One step = the whole chain (raw FED words -> digis -> clusters -> rechits -> CA
ntuplets -> broken-line fits -> classification -> vertices) over one batch of
synthetic PU50 events (1000 by default), replayed as one CUDA graph with the input
already in HBM; two contexts on two streams take alternate steps, so that two batches are
in flight. Also measured: the same metric end to end through the public API
(host->device copy of the raw events from pinned memory and device->host copy of the
batch's track and vertex collections inside the timed region), the plain per-event launch sequence,
per-kernel times (live CUDA events) for the roofline of the dominant kernel, and the
CPU baseline (the serial restatement of the reference on the host cores).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
for p in (ROOT, ROOT / "cms-julia_b200"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))

METRIC = "PU50 events/s on 1 B200 batched vs plain; BL fits/s and err vs FP64"
WORKLOAD = ("synthetic PU50 events (50 vertices x Poisson(30) helix tracks, |eta|<2.5, pT 0.5-10 GeV, 1e-4 noise, "
            "1% inefficiency) on a seeded Phase-1-like geometry, batched by prefix offsets, one CUDA graph per step; "
            "two contexts on two streams take alternate steps, so that two batches are in flight")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--events", type=int, default=1000)
    ap.add_argument("--pu", type=float, default=50.0)
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--plain-events", type=int, default=200)
    ap.add_argument("--cpu-sample", type=int, default=160)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--profile-only", action="store_true")
    ap.add_argument("--fit-tracks", type=int, default=1 << 20)
    ap.add_argument("--fit-oracle-sample", type=int, default=4000)
    ap.add_argument("--no-fits", action="store_true")
    ap.add_argument("--fits-only", action="store_true", help="only the stand-alone fit and adjoint measurements")
    ap.add_argument("--uneven-events", type=int, default=4096)
    ap.add_argument("--uneven-steps", type=int, default=3)
    ap.add_argument("--no-uneven", action="store_true")
    ap.add_argument("--no-parity", action="store_true", help="skip the per-event comparison with the oracle")
    ap.add_argument("--adjoint-sample", type=int, default=500)
    ap.add_argument("--bpe", type=int, default=0, help="blocks per event for the per-event kernels (0: automatic)")
    ap.add_argument("--contexts", type=int, default=2, help="contexts (each on its own stream) taking turns")
    return ap.parse_args()


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines: list[str] = []
        self._t = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self) -> dict:
        sm, smax, reasons = [], 0.0, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = max(smax, float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax or None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------------ algorithmic bytes per kernel group
def segment_bytes(name: str, c: dict) -> float | None:
    """Compulsory traffic of one kernel group over the batch: inputs read once, outputs written
    once (conditions tables are L2-resident and not counted)."""
    D, H, C, T, TH, I = c["words"], c["hits"], c["cells"], c["tuples"], c["tuple_hits"], c["items"]
    table = {
        "unpack_calib": 4 * D + 22 * D,            # words in; xx,yy,adc,moduleInd,clus,pdigi,rawId out
        "module_starts": 4 * D,                    # moduleInd read by the count and fill passes
        "find_clus_tiny": 14 * D,                  # moduleInd,x,y,adc in; clus (and moduleInd) out (modules <= 16 digis;
                                                   # the larger ones only read their range bounds here)
        "get_hits_warp": 14 * D + 40 * H,          # digis in; per-cluster sums out
        "cpe": 40 * H + 60 * H,                    # sums in; hit SoA and packed coordinates out
        "phi_binner": 4 * H,                       # iphi in; bins out
        "doublets_count": 30 * H + 8 * I + 4 * C,  # inner-hit fields and binned hit records (once per hit) in,
                                                   # per-item counts and pool offsets, pooled outer hits out
        "doublets_fill": 8 * I + 4 * C + 22 * C,   # counts and pool in, cell SoA out
        "connect": 24 * C + 22 * H,                # cell hits and outer-hit records in, hit coordinates (once)
        "outer_hit_lists": 41 * C + 8 * H,         # outer hits in, lists sorted, candidate records out
        "neighbour_lists": 16 * C,                 # pair list in, lists filled and sorted
        "ntuplets_fill": 5 * T + 6 * TH,           # tuple offsets, hits, detector indices out
        "fast_duplicate_remover": 12 * T,          # qualities in and out, cell track lists in
        "broken_line_fit_4": 22 * TH + 4 * TH + 8 * T + 93 * T,
        "vertices": 4 * T + 80 * T,
    }
    return table.get(name)


# dram__bytes_read.sum + dram__bytes_write.sum per unit of work, from ncu captures of the
# 300-event case (profiles/), scaled to a launch by the units it processes
TRAFFIC_PER_UNIT = {
    "doublets_count": ("hits", (77.30e6 + 113.63e6) / 3_215_253),
    "connect": ("cells", (483.81e6 + 75.11e6) / 25_257_080),
}

FIT_B = 0.0114256972711507  # 1/(pT R) at 3.8 T, GeV^-1 cm^-1


def bench_uneven(args, local: int, rank: int, world: int, plain_value: float) -> dict:
    """Batched uneven events: 4096 events with pileup drawn uniformly from [0, 200] (about
    1k-130k digis per event), extended per-event capacities so that no event is truncated, as
    four resident 1024-event quarters on two contexts (each holding two quarters in its two
    input slots, each slot one captured CUDA graph over prefix-offset packed input) that run
    on two streams, so that two quarters are in flight; launch shapes from the autotuner. The
    parity check (outside the timed region) compares every event's counts with the oracle run
    with the same capacities, and every product of the ten largest events."""
    import torch
    from pixeltrack import dist as pdist
    from pixeltrack import PixelChain, batch_params, gen
    E = args.uneven_events
    NQ = 4
    H = E // NQ
    conds = gen.conditions()
    blob, offs = gen.events(E, gen.MODE_UNIFORM, pu=200.0, seed=args.seed + 31 + 7919 * rank)
    words = int(np.diff(offs).sum() // 4)
    params = batch_params(H, words_per_event=int(words / E * 1.4) + 4096, hits_per_event_avg=24_000,
                          doublets_per_event_avg=360_000, tuples_per_event_avg=36_000, device=local,
                          extended=True)
    chains = [PixelChain(conds, params) for _ in range(2)]
    streams = [torch.cuda.Stream(device=local) for _ in range(2)]
    shs = [s_.cuda_stream for s_ in streams]
    quarters = [(blob[int(offs[k * H]):int(offs[(k + 1) * H])], offs[k * H:(k + 1) * H + 1] - offs[k * H])
                for k in range(NQ)]
    # quarter k runs on context k % 2 from its input slot k // 2

    def timed_step(candidates):
        """Tunes the launch shapes among candidates on each context's first quarter, captures
        the quarters' graphs (resident in the contexts' input slots) and times the step."""
        tuned = {}
        for i, c in enumerate(chains):
            c.stage_batch(*quarters[i], shs[i])
            streams[i].synchronize()
            t = c.autotune(candidates=candidates)
            tuned = tuned or t
            c.stage_batch(*quarters[i], shs[i])
            streams[i].synchronize()
            c.capture_graph()
            c.stage_slot(1, *quarters[i + 2], shs[i])
            streams[i].synchronize()

        def step():
            for k in range(NQ):
                chains[k % 2].launch_slot(k // 2, shs[k % 2])

        for _ in range(args.warmup):
            step()
        warn = 0
        for c in chains:
            warn |= c.sync()
        torch.cuda.synchronize()
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0.record(streams[0])
        streams[1].wait_event(t0)
        for _ in range(args.uneven_steps):
            step()
        streams[0].wait_stream(streams[1])
        t1.record(streams[0])
        t1.synchronize()
        return pdist.max_over_ranks(t0.elapsed_time(t1), device=torch.device("cuda", local)) / args.uneven_steps, \
            tuned, warn

    # static grids only, then with the persistent work queues among the candidates (kept)
    ms_static, tuned_static, _ = timed_step((4, 8, 16, 32, 64, 128))
    ms, tuned, warn = timed_step((4, 8, 16, 32, 64, 128, -2, -8))
    # per-event counts of each half, and the full products of the largest events
    counts = []
    big = set(np.argsort(np.diff(offs))[-10:].tolist())
    parity = {"events": E, "caps": "extended"}
    prod_err = {}
    orc = None
    good = 0
    if not args.no_parity:
        from oracle import oracle
        from oracle.compare import compare_event
        orc = oracle.Oracle(conds, oracle.EXTENDED_CAPS)
        _, ocnt = orc.run_batch(blob, offs, os.cpu_count() or 1, counts=True)
        expected = validator_counts(ocnt)
    for k in range(NQ):
        chain = chains[k % 2]
        chain.launch_slot(k // 2, shs[k % 2])
        warn |= chain.sync()
        if orc is not None:
            good += chain.validate_counts(expected[k * H:(k + 1) * H])[0]
        for e in range(H):
            counts.append(chain.counts(e))
            if orc is not None and k * H + e in big:
                g = k * H + e
                orc.run_event(blob[int(offs[g]):int(offs[g + 1])], 63)
                errs = compare_event(chain, orc, e)
                if errs:
                    prod_err[g] = errs[:3]
    for c in chains:
        c.close()
    if orc is not None:
        from oracle.compare import compare_counts
        bad = compare_counts(counts, ocnt)
        parity.update({"count_mismatch_events": len(bad), "first_mismatch": bad[:5],
                       "product_sample": sorted(big), "product_mismatch_events": len(prod_err),
                       "product_errors": prod_err, "validator": {"validated_events": E, "good_events": good}})
    tot = {"digis_min": 10 ** 9, "digis_max": 0, "hits": 0, "cells": 0, "tuples": 0, "vertices": 0,
           "capped_events": 0, "buffer_overflow_events": 0}
    from pixeltrack._native import WARN_BITS
    for c in counts:
        tot["digis_min"] = min(tot["digis_min"], c.n_words)
        tot["digis_max"] = max(tot["digis_max"], c.n_words)
        tot["hits"] += c.n_hits
        tot["cells"] += c.n_doublets
        tot["tuples"] += c.n_tuples
        tot["vertices"] += c.n_vertices
        tot["capped_events"] += int(bool(c.warnings & 0x5D))
        tot["buffer_overflow_events"] += int(bool(c.warnings & 0x800))
    value = world * E / (ms / 1e3)
    return {"workload": f"{E} synthetic events, pileup uniform in [0, 200], extended per-event capacities, "
                        f"{NQ} resident {H}-event quarters per step on two contexts and two streams (two quarters "
                        "in flight), each one CUDA graph over prefix-offset packed input, autotuned launch shapes",
            "events_per_step": E, "value": value,
            "unit": "events/s", "ms_per_step": ms, "steps": args.uneven_steps, "raw_bytes_per_step": int(offs[-1]),
            "over_plain_per_event_pu50": value / world / plain_value if plain_value else None,
            "blocks_per_event": tuned, "totals": tot, "warnings": [n for b, n in WARN_BITS.items() if warn & b],
            "static_grid": {"value": world * E / (ms_static / 1e3), "ms_per_step": ms_static,
                            "blocks_per_event": tuned_static,
                            "note": "the same batch with every stage on a static grid (no work queue)"},
            "parity": parity}


def bench_fits(args, local: int, rank: int, world: int) -> dict:
    """Stand-alone broken-line fits of 2^20 synthetic tracks of 3..8 hits (mix 30/40/20/10 %
    for 3/4/5/6-8): fits/s in mixed precision and in FP64, per-parameter error of the mixed
    mode against the FP64 mode on every track, and of the FP64 mode against the CPU oracle on
    a sample. Inputs resident in HBM (about 210 MB, larger than L2)."""
    import torch
    from pixeltrack import dist as pdist
    from pixeltrack import gen
    from pixeltrack.fits import bl_fit, workspace
    n = args.fit_tracks
    w = gen.fit_tracks(n, seed=args.seed + 104729 * rank)
    dev = torch.device("cuda", local)
    hits = torch.as_tensor(w["hits"]).to(dev)
    ge = torch.as_tensor(w["ge"]).to(dev)
    offs = torch.as_tensor(w["offsets"]).to(dev)
    ws = workspace(n, dev)
    stream = torch.cuda.Stream(device=dev)
    out = {}
    res = {}
    with torch.cuda.stream(stream):
        for prec, name in ((1, "mixed"), (0, "fp64")):
            for _ in range(args.warmup):
                r = bl_fit(hits, ge, offs, FIT_B, precision=prec, stream=stream, ws=ws)
            stream.synchronize()
            t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            t0.record(stream)
            for _ in range(args.steps):
                r = bl_fit(hits, ge, offs, FIT_B, precision=prec, stream=stream, ws=ws)
            t1.record(stream)
            t1.synchronize()
            ms = pdist.max_over_ranks(t0.elapsed_time(t1), device=dev) / args.steps
            res[name] = {k: v.double().cpu().numpy() for k, v in r.items() if k in ("state", "pt", "status")}
            out[name] = {"fits_per_s": world * n / (ms / 1e3), "ms_per_step": ms}
    # Riemann fits of the same tracks
    from pixeltrack.fits import riemann_fit
    rres = {}
    with torch.cuda.stream(stream):
        for prec, name in ((1, "riemann_mixed"), (0, "riemann_fp64")):
            for _ in range(args.warmup):
                r = riemann_fit(hits, ge, offs, FIT_B, precision=prec, stream=stream, ws=ws)
            stream.synchronize()
            t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            t0.record(stream)
            for _ in range(args.steps):
                r = riemann_fit(hits, ge, offs, FIT_B, precision=prec, stream=stream, ws=ws)
            t1.record(stream)
            t1.synchronize()
            ms = pdist.max_over_ranks(t0.elapsed_time(t1), device=dev) / args.steps
            rres[name] = {k: v.double().cpu().numpy() for k, v in r.items() if k in ("state", "status")}
            out[name] = {"fits_per_s": world * n / (ms / 1e3), "ms_per_step": ms}
    nh = np.diff(w["offsets"]).astype(np.int64)
    bytes_per_step = 48 * int(nh.sum()) + 4 * (n + 1) + (5 + 15 + 3) * 4 * n + 4 * n
    peak, peak_kind = load_peaks()
    for name in out:
        gbs = bytes_per_step / (out[name]["ms_per_step"] / 1e3) / 1e9
        out[name]["hbm"] = {"achieved": gbs, "peak": peak, "peak_kind": peak_kind, "unit": "GB/s", "frac": gbs / peak,
                            "algorithmic_bytes_per_step": bytes_per_step}
    # per-parameter error of the mixed mode against the FP64 mode (all tracks)
    a, b = res["mixed"]["state"], res["fp64"]["state"]
    ok = np.all(np.isfinite(b), axis=1) & (res["fp64"]["status"] == 0)
    d = np.abs(a[ok] - b[ok])
    stats = lambda v: {"median": float(np.median(v)), "p99": float(np.percentile(v, 99)), "max": float(v.max())}
    def param_err(a, b, ok):
        bad = ok & ~np.all(np.isfinite(a), axis=1)  # finite in FP64, not in the mixed mode
        ok = ok & ~bad
        d = np.abs(a[ok] - b[ok])
        return {"q_over_pt_rel": stats(d[:, 2] / np.abs(b[ok, 2])), "phi_abs_rad": stats(d[:, 0]),
                "cot_theta_rel": stats(d[:, 3] / np.maximum(np.abs(b[ok, 3]), 1e-3)),
                "d0_abs_cm": stats(d[:, 1]), "z0_abs_cm": stats(d[:, 4]), "tracks": int(ok.sum()),
                "nonfinite_mixed": int(bad.sum())}
    err = param_err(a, b, ok)
    rb = rres["riemann_fp64"]["state"]
    rok = np.all(np.isfinite(rb), axis=1) & (rres["riemann_fp64"]["status"] == 0)
    err_riemann = param_err(rres["riemann_mixed"]["state"], rb, rok)
    # FP64 mode against the CPU oracle on a sample (the oracle stores FP64, the GPU FP32)
    m = min(args.fit_oracle_sample, n)
    st, _, _ = oracle_fit_sample(w, m)
    okm = np.all(np.isfinite(st), axis=1)
    rel = np.abs(res["fp64"]["state"][:m][okm] - st[okm]) / np.maximum(np.abs(st[okm]), 1e-6)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        from oracle import oracle
        k = min(n, 200_000)
        _, _, dt = oracle.bl_fit_batch(w["hits"][: w["offsets"][k]], w["ge"][: w["offsets"][k]], w["offsets"][: k + 1],
                                       FIT_B, 1)
        cpu = {"value": k / dt, "unit": "fits/s", "cores": 1, "kind": "port",
               "sample": f"{k} of the {n} tracks, FP64 oracle fit, one thread"}
    return {"workload": f"2^{int(np.log2(n))} synthetic tracks, 3-8 hits (30/40/20/10 % for 3/4/5/6-8), helices with "
                        "0.02 X0 scattering kinks, 10 um r-phi / 20 um z smearing",
            "tracks": n, "mixed": out["mixed"], "fp64": out["fp64"], "err_mixed_vs_fp64": err,
            "riemann_mixed": out["riemann_mixed"], "riemann_fp64": out["riemann_fp64"],
            "riemann_err_mixed_vs_fp64": err_riemann,
            "fp64_vs_oracle": {"max_rel": float(rel.max()), "tracks": int(okm.sum())},
            "cpu_baseline": cpu}


def bench_adjoint(args, local: int, rank: int, world: int) -> dict:
    """Differentiable fit: chi2 and d(chi2)/d(hits) and d(sum chi2)/d(6-DOF alignment of the
    1856 modules) for 2^20 tracks of the fit workload, alignment translations ~ N(0, 50 um)
    and rotations ~ N(0, 0.1 mrad). The fit is recomputed in the backward kernel (no stored
    intermediates); the gradient is checked against the oracle's forward-mode derivative and
    central finite differences (h = 1e-6 cm) on a sample."""
    import torch
    from pixeltrack import dist as pdist
    from pixeltrack import gen
    from pixeltrack.fits import bl_fit_adjoint
    n = args.fit_tracks
    w = gen.fit_tracks(n, seed=args.seed + 7 + 104729 * rank)
    pos = gen.module_positions()
    rng = np.random.default_rng(args.seed)
    align = np.zeros((pos.shape[0], 6), np.float32)
    align[:, :3] = rng.normal(0, 50e-4, (pos.shape[0], 3))
    align[:, 3:] = rng.normal(0, 1e-4, (pos.shape[0], 3))
    dev = torch.device("cuda", local)
    T = lambda a: torch.as_tensor(a).to(dev)
    hits, ge, offs, mod, mpos, al = T(w["hits"]), T(w["ge"]), T(w["offsets"]), T(w["module"]), T(pos), T(align)
    stream = torch.cuda.Stream(device=dev)
    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            out = bl_fit_adjoint(hits, ge, offs, FIT_B, mod, mpos, al, True, stream=stream)
        stream.synchronize()
        torch.cuda.reset_peak_memory_stats(dev)
        base_mem = torch.cuda.memory_allocated(dev)
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        for _ in range(args.steps):
            out = bl_fit_adjoint(hits, ge, offs, FIT_B, mod, mpos, al, True, stream=stream)
        t1.record(stream)
        t1.synchronize()
    ms = pdist.max_over_ranks(t0.elapsed_time(t1), device=dev) / args.steps
    peak_extra = torch.cuda.max_memory_allocated(dev) - base_mem
    g = out["grad_hits"].double().cpu().numpy()
    # moved hits (as the kernel sees them) for the oracle checks
    hh = w["hits"].copy()
    on = w["module"] >= 0
    r = hh[on] - pos[w["module"][on]]
    hh[on] += align[w["module"][on], :3].astype(np.float64) + np.cross(align[w["module"][on], 3:].astype(np.float64), r)
    from oracle import oracle
    m = min(args.adjoint_sample, n)
    worst_fwd = 0.0
    for t in range(m):
        a, b = w["offsets"][t], w["offsets"][t + 1]
        cf, gf = oracle.bl_chi2_grad_fwd(hh[a:b], w["ge"][a:b], FIT_B)
        if np.isfinite(cf):
            worst_fwd = max(worst_fwd, float(np.abs(g[a:b] - gf).max() / np.abs(gf).max()))
    worst_fd = 0.0
    chi = lambda x, e: (lambda rr: rr["chi2_line"] + rr["chi2_circle"])(oracle.bl_fit(x.T, e.T, FIT_B))
    for t in range(min(32, m)):
        a, b = w["offsets"][t], w["offsets"][t + 1]
        x, e = hh[a:b], w["ge"][a:b]
        fd = np.zeros_like(x)
        for i in range(b - a):
            for k in range(3):
                xp, xm = x.copy(), x.copy()
                xp[i, k] += 1e-6
                xm[i, k] -= 1e-6
                fd[i, k] = (chi(xp, e) - chi(xm, e)) / 2e-6
        worst_fd = max(worst_fd, float(np.abs(g[a:b] - fd).max() / np.abs(fd).max()))
    nh = int(np.diff(w["offsets"]).sum())
    return {"workload": "the fit workload plus per-module 6-DOF alignment (t ~ N(0, 50 um), w ~ N(0, 0.1 mrad)) "
                        "on the 1856 modules", "tracks": n, "tracks_per_s": world * n / (ms / 1e3), "ms_per_step": ms,
            "memory": {"workspace_and_outputs_bytes": int(peak_extra), "inputs_bytes": int(48 * nh + 2 * nh + 4 * n),
                       "stored_intermediates_bytes": 0},
            "check": {"vs_forward_mode_max_rel": worst_fwd, "forward_mode_tracks": m,
                      "vs_central_fd_max_rel": worst_fd, "fd_tracks": min(32, m), "fd_step_cm": 1e-6},
            "dtype": "f64 arithmetic, f32 outputs, f64 alignment accumulation"}


def validator_counts(ocnt: np.ndarray) -> np.ndarray:
    """The oracle's counts written to the reference's count files and read back: (n, 5)
    modules, digis, clusters, tracks, vertices per event, the CountValidator's expectation."""
    import tempfile
    from oracle import oracle
    from pixeltrack.formats import read_counts, write_counts
    ix = [oracle.COUNT_NAMES.index(k) for k in ("n_modules", "n_words", "n_clusters", "n_tracks", "nv_final")]
    with tempfile.TemporaryDirectory() as d:
        write_counts(d, ocnt[:, ix])
        return read_counts(d)


def pu50_parity(chain, conds, blob, offs, E: int) -> dict:
    """Every event's counts against the oracle (all host threads), and every product of a few
    events (first, middle, last and the three largest), on the chain's last run; the
    CountValidator over the batch with the oracle's counts as its count files."""
    from oracle import oracle
    from oracle.compare import compare_counts, compare_event
    orc = oracle.Oracle(conds)
    _, ocnt = orc.run_batch(blob, offs, os.cpu_count() or 1, counts=True)
    bad = compare_counts([chain.counts(e) for e in range(E)], ocnt)
    good, _ = chain.validate_counts(validator_counts(ocnt))
    sample = sorted({0, E // 2, E - 1, *np.argsort(np.diff(offs))[-3:].tolist()})
    prod_err = {}
    for e in sample:
        orc.run_event(blob[int(offs[e]):int(offs[e + 1])], 63)
        errs = compare_event(chain, orc, e)
        if errs:
            prod_err[e] = errs[:3]
    return {"events": E, "caps": "reference", "count_mismatch_events": len(bad), "first_mismatch": bad[:5],
            "product_sample": sample, "product_mismatch_events": len(prod_err), "product_errors": prod_err,
            "validator": {"validated_events": E, "good_events": good}}


def chain_fit_precision(chain, conds, blob, offs, E: int, params, n_check: int = 200) -> dict:
    """The chain run again with its fits in mixed precision (fit_precision = 1): per-parameter
    error of the fitted tuples of n_check events against the FP64 chain's (the same tuples), and
    the live time of the fit segments in both modes (non-graph runs)."""
    import ctypes
    from pixeltrack import PixelChain
    p = type(params)()
    ctypes.memmove(ctypes.byref(p), ctypes.byref(params), ctypes.sizeof(params))
    p.fit_precision = 1
    mixed = PixelChain(conds, p)
    fit_ms = {}
    for name, ch in (("fp64", chain), ("mixed", mixed)):
        ch.profile(True)
        for _ in range(2):
            ch.run_batch(blob, offs)
            segs = dict(ch.profile_read())
        ch.profile(False)
        fit_ms[name] = (segs.get("broken_line_fit_3", 0.0) + segs.get("broken_line_fit_4", 0.0) +
                        segs.get("broken_line_refit_fp64", 0.0))
    n_refit = sum(mixed.counts(e).n_fits_fp64 for e in range(E))
    n_fits = sum(int(mixed.product("fitted", e)[:mixed.counts(e).n_tuples].sum()) for e in range(E))
    chain.run_batch(blob, offs)
    rows = {"q_over_pt_rel": [], "phi_abs_rad": [], "cot_theta_rel": [], "d0_abs_cm": [], "z0_abs_cm": []}
    for e in np.linspace(0, E - 1, min(n_check, E)).astype(int):
        nt = chain.counts(e).n_tuples
        sel = chain.product("fitted", e)[:nt].astype(bool)
        a = mixed.product("state", e).reshape(-1, 5)[:nt][sel].astype(np.float64)
        b = chain.product("state", e).reshape(-1, 5)[:nt][sel].astype(np.float64)
        ok = np.all(np.isfinite(b), axis=1)
        a, b = a[ok], b[ok]
        rows["q_over_pt_rel"].append(np.abs(a[:, 2] - b[:, 2]) / np.abs(b[:, 2]))
        rows["phi_abs_rad"].append(np.abs(a[:, 0] - b[:, 0]))
        rows["cot_theta_rel"].append(np.abs(a[:, 3] - b[:, 3]) / np.maximum(np.abs(b[:, 3]), 1e-3))
        rows["d0_abs_cm"].append(np.abs(a[:, 1] - b[:, 1]))
        rows["z0_abs_cm"].append(np.abs(a[:, 4] - b[:, 4]))
    mixed.close()
    out = {k: {"median": float(np.median(np.concatenate(v))), "p99": float(np.percentile(np.concatenate(v), 99)),
               "max": float(np.concatenate(v).max())} for k, v in rows.items()}
    out["tracks"] = int(sum(len(v) for v in rows["q_over_pt_rel"]))
    out["events"] = int(min(n_check, E))
    out["fit_segments_ms"] = fit_ms
    out["refits_fp64"] = {"tuples": int(n_refit), "of_fitted": int(n_fits), "rule": "mixed fit pT >= 50 GeV"}
    return out


def oracle_fit_sample(w: dict, m: int):
    from oracle import oracle
    return oracle.bl_fit_batch(w["hits"][: w["offsets"][m]], w["ge"][: w["offsets"][m]], w["offsets"][: m + 1], FIT_B, 1)


def load_peaks() -> tuple[float, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ------------------------------------------------------------------ reference arm (CPU)
def run_reference(args, rank: int, world: int) -> None:
    if rank != 0:
        return
    from oracle import oracle
    from pixeltrack import gen
    conds = gen.conditions()
    # the same events as our arm's step (rank 0's batch)
    n = args.events
    blob, offs = gen.events(n, gen.MODE_PU, pu=args.pu, seed=args.seed)
    orc = oracle.Oracle(conds)
    threads = os.cpu_count() or 1
    for _ in range(max(1, args.warmup)):
        orc.run_batch(blob, offs, threads)
    t = 0.0
    for _ in range(args.steps):
        t += orc.run_batch(blob, offs, threads)
    value = n * args.steps / t
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "events/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int32/f32/f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "events_per_step": n, "pileup": args.pu},
        "cpu_baseline": {"value": value, "unit": "events/s", "cores": threads, "kind": "port",
                         "sample": f"{n} PU{int(args.pu)} events per step, full chain, event-parallel threads"},
        "e2e": {"value": value, "unit": "events/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "the reference is a Julia program; julia is not installed here, so its CPU path is timed as the "
                "oracle's serial C++ restatement",
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ our arm
def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", str(args.gpus)))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    import torch
    from pixeltrack import dist as pdist
    dist = None
    torch.cuda.set_device(local)
    if pdist.init("nccl"):
        import torch.distributed as dist
    from pixeltrack import PixelChain, batch_params, default_params, gen
    if args.fits_only:
        fits = bench_fits(args, local, rank, world)
        adjoint = bench_adjoint(args, local, rank, world)
        if rank == 0:
            print(json.dumps({"fits": fits, "adjoint": adjoint}), flush=True)
        return
    conds = gen.conditions()
    E = args.events
    blob, offs = gen.events(E, gen.MODE_PU, pu=args.pu, seed=pdist.rank_seed(args.seed, rank))
    words = np.diff(offs).sum() // 4
    params = batch_params(E, words_per_event=int(words / E * 1.3) + 4096, hits_per_event_avg=16_000,
                          doublets_per_event_avg=140_000, tuples_per_event_avg=11_000, device=local,
                          blocks_per_event=args.bpe)
    chain = PixelChain(conds, params)
    stream = torch.cuda.Stream(device=local)
    sh = stream.cuda_stream

    # launch shapes chosen by the autotuner on this batch (outside the timed region)
    chain.stage_batch(blob, offs, sh)
    stream.synchronize()
    tuned = chain.autotune() if args.bpe == 0 else {}

    # correctness guard and per-kernel profile (non-graph run, tuned shapes)
    chain.stage_batch(blob, offs, sh)
    stream.synchronize()
    chain.profile(True)
    prof_runs = []
    for _ in range(3):
        torch.cuda.nvtx.range_push("chain")  # profiler filter: --nvtx --nvtx-include "chain/"
        chain.run_batch(blob, offs, sync=False)
        torch.cuda.nvtx.range_pop()
        warn = chain.sync()
        prof_runs.append(chain.profile_read())
    chain.profile(False)
    seg_ms: dict[str, float] = {}
    for run in prof_runs[1:]:
        for name, ms in run:
            seg_ms[name] = seg_ms.get(name, 0.0) + ms / (len(prof_runs) - 1)
    totals = {"words": 0, "hits": 0, "cells": 0, "tuples": 0, "tuple_hits": 0, "vertices": 0, "items": 0}
    for e in range(E):
        c = chain.counts(e)
        totals["words"] += c.n_words
        totals["hits"] += c.n_hits
        totals["cells"] += c.n_doublets
        totals["tuples"] += c.n_tuples
        totals["tuple_hits"] += c.n_tuple_hits
        totals["vertices"] += c.n_vertices
        # doublet work items: inner hits over the 19 layer pairs (layer 0 is the inner layer
        # of 6 pairs, layer 1 of 4, layer 2 of 3, layers 4 and 7 of 2, layers 5 and 8 of 1)
        if c.n_hits:
            hls = chain.product("hits_layer_start", e).astype(np.int64)
            nl = np.diff(hls[:11])
            totals["items"] += int(6 * nl[0] + 4 * nl[1] + 3 * nl[2] + 2 * nl[4] + nl[5] + 2 * nl[7] + nl[8])
    if args.profile_only:
        print(json.dumps({"segments_ms": seg_ms, "totals": totals, "warnings": warn}), flush=True)
        return
    # parity of the batch with the oracle (outside every timed region)
    parity = None if args.no_parity else pu50_parity(chain, conds, blob, offs, E)
    # the chain's fits in mixed precision against its FP64 fits
    chain_mixed = chain_fit_precision(chain, conds, blob, offs, E, params)

    # batched graph: input in HBM, one replay per step. A second context on its own stream
    # takes every other step, so that two batches are in flight: one batch's kernels fill the
    # SMs that the other's last waves and per-event stages leave idle (the reference's
    # analogue is its several stream threads, each with its own producers).
    nctx = max(1, args.contexts)
    chains, streams, shs = [chain], [stream], [sh]
    for _ in range(nctx - 1):
        c = PixelChain(conds, params)
        s_ = torch.cuda.Stream(device=local)
        c.stage_batch(blob, offs, s_.cuda_stream)
        s_.synchronize()
        if args.bpe == 0:
            c.autotune()
        chains.append(c)
        streams.append(s_)
        shs.append(s_.cuda_stream)
    for c, s_, h_ in zip(chains, streams, shs):
        c.stage_batch(blob, offs, h_)
        s_.synchronize()
        c.capture_graph()
    kernels_per_step = chain.graph_kernel_nodes()
    for k in range(max(args.warmup, nctx)):
        chains[k % nctx].launch_graph(shs[k % nctx])
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        t0.record(stream)
        for s_ in streams[1:]:
            s_.wait_event(t0)
        for k in range(args.steps):
            chains[k % nctx].launch_graph(shs[k % nctx])
        for s_ in streams[1:]:
            stream.wait_stream(s_)
        t1.record(stream)
        t1.synchronize()
    ms = pdist.max_over_ranks(t0.elapsed_time(t1), device="cuda")
    ms_per_step = ms / args.steps
    value = world * E * args.steps / (ms / 1e3)

    # end to end through the public API: pinned host raw events in; the batch's track and vertex
    # collections out (pxl_export_async: the loose tracks' parameters, hit counts and vertex
    # ids, the vertices, and the per-event index, one copy per array). The two contexts take
    # alternate steps on their own streams; batch i+1 is copied into its context's next input
    # slot on a copy stream while batch i runs, and batch i's collections go to host memory on
    # a third stream.
    from pixeltrack import TrackExport
    pinned = torch.empty(len(blob), dtype=torch.uint8, pin_memory=True)
    pinned.numpy()[:] = blob
    pinned_np = pinned.numpy()
    probe = TrackExport(E, max_tracks=0, max_vertices=0)  # totals of this batch, to size the host arrays
    chain.export_async(probe)
    chain.sync()
    torch.cuda.synchronize()
    n_loose, n_vtx = int(probe.index()[E, 1]), int(probe.index()[E, 3])
    outs = [TrackExport(E, max_tracks=n_loose + n_loose // 8 + 1024, max_vertices=n_vtx + n_vtx // 8 + 64)
            for _ in range(2)]
    h2d = int(offs[-1] - offs[0]) + 8 * (E + 1)
    d2h = outs[0].bytes()
    copy = torch.cuda.Stream(device=local)
    d2h_stream = torch.cuda.Stream(device=local)

    def e2e_steps(n):
        chains[0].stage_slot(0, pinned_np, offs, copy.cuda_stream)
        for k in range(n):
            i, slot = k % nctx, (k // nctx) % 2
            chains[i].launch_slot(slot, shs[i])
            chains[i].export_async(outs[k % 2], shs[i], d2h_stream.cuda_stream)
            if k + 1 < n:
                chains[(k + 1) % nctx].stage_slot(((k + 1) // nctx) % 2, pinned_np, offs, copy.cuda_stream)

    e2e_steps(max(args.warmup, nctx))
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for s_ in [copy, d2h_stream] + streams[1:]:
        s_.wait_event(e0)
    e2e_steps(args.steps)
    for s_ in streams[1:] + [d2h_stream]:
        stream.wait_stream(s_)
    e1.record(stream)
    e1.synchronize()
    ems = pdist.max_over_ranks(e0.elapsed_time(e1), device="cuda")
    e2e_value = world * E * args.steps / (ems / 1e3)
    last = outs[(args.steps - 1) % 2].index()
    nv_check = int(last[E, 3])
    assert int(last[E, 1]) == n_loose and nv_check == n_vtx, "exported collections differ between steps"

    # plain per-event launch sequence (one event per launch sequence, input already in HBM)
    plain = PixelChain(conds, default_params(device=local))
    dev_blob = torch.as_tensor(blob).cuda()
    dev_offs = torch.as_tensor(offs.astype(np.int64)).cuda()
    npl = min(args.plain_events, E)
    for e in range(min(5, npl)):
        plain.run_batch_device(dev_blob.data_ptr(), dev_offs.data_ptr() + 8 * e, 1, stream=sh)
    stream.synchronize()
    p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    p0.record(stream)
    for e in range(npl):
        plain.run_batch_device(dev_blob.data_ptr(), dev_offs.data_ptr() + 8 * e, 1, stream=sh)
    p1.record(stream)
    p1.synchronize()
    plain_value = npl / (p0.elapsed_time(p1) / 1e3)
    plain.close()

    # roofline of the dominant kernel group (live CUDA-event times of the profiled runs)
    peak, peak_kind = load_peaks()
    dom = max(seg_ms, key=seg_ms.get) if seg_ms else None
    dom_bytes = segment_bytes(dom, totals) if dom else None
    roofline = None
    if dom:
        achieved = (dom_bytes / (seg_ms[dom] / 1e3) / 1e9) if dom_bytes else None
        tu = TRAFFIC_PER_UNIT.get(dom)
        traffic = tu[1] * totals[tu[0]] if tu else None
        roofline = {"kernel": dom, "bound": "hbm", "achieved": achieved, "peak": peak, "peak_kind": peak_kind,
                    "unit": "GB/s", "frac": (achieved / peak) if achieved else None, "traffic": traffic,
                    "ms_per_launch": seg_ms[dom], "algorithmic_bytes_per_launch": dom_bytes}

    # CPU baseline: the oracle (serial restatement of the reference) on the host cores
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        from oracle import oracle
        n = min(args.cpu_sample, E)
        sub = blob[: int(offs[n])]
        orc = oracle.Oracle(conds)
        threads = os.cpu_count() or 1
        orc.run_batch(sub, offs[: n + 1], threads)
        t = orc.run_batch(sub, offs[: n + 1], threads)
        cpu = {"value": n / t, "unit": "events/s", "cores": threads, "kind": "port",
               "sample": f"{n} of the {E} PU{int(args.pu)} events, full chain, {threads} event-parallel threads"}

    chain.close()
    uneven = None if args.no_uneven else bench_uneven(args, local, rank, world, plain_value)
    fits = None if args.no_fits else bench_fits(args, local, rank, world)
    adjoint = None if args.no_fits else bench_adjoint(args, local, rank, world)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "events/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int32/f32/f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "events_per_step": E, "pileup": args.pu, "contexts_in_flight": nctx,
                       "raw_bytes_per_step": int(offs[-1]), "l2": "inputs and intermediates larger than L2",
                       "parallelism": f"events sharded over {world} GPU(s), no data-path collective",
                       "blocks_per_event": tuned or args.bpe},
            "e2e": {"value": e2e_value, "unit": "events/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "plain": {"value": plain_value, "unit": "events/s", "events": npl,
                      "note": "one launch sequence per event, input in HBM"},
            "batched_over_plain": value / world / plain_value,
            "roofline": roofline, "cpu_baseline": cpu, "gpu_launches": kernels_per_step * args.steps,
            "clocks": clk.summary(), "segments_ms": seg_ms, "totals": totals, "warnings": warn, "fits": fits,
            "adjoint": adjoint, "uneven_pu0_200": uneven, "parity": parity,
            "chain_fit_mixed_vs_fp64": chain_mixed,
            "vertices_per_event": nv_check / E,
        }
        print(json.dumps(line), flush=True)
    for c in chains:
        c.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
