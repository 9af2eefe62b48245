"""Parity of the CUDA fits, track classification and vertexing with the CPU oracle.
Tolerance for FP64 fit outputs stored as FP32: relative 1e-5 (parity.FIT_RTOL)."""
import json
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle
from parity import compare_ca, compare_fits, compare_quality, compare_vertices

GOLDEN = Path(__file__).resolve().parent / "golden"
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def chain(conditions):
    from pixeltrack import PixelChain, default_params
    c = PixelChain(conditions, default_params())
    yield c
    c.close()


@pytest.fixture(scope="module")
def orc(conditions):
    return oracle.Oracle(conditions)


def _check_event(chain, orc, ev):
    chain.run_event(ev, 63)
    orc.run_event(ev, 63)
    errs = compare_ca(chain, orc, classified=True) + compare_fits(chain, orc) + compare_quality(chain, orc) + \
        compare_vertices(chain, orc)
    return errs


def test_single_event_full_chain(chain, orc, event_single):
    blob, offs = event_single
    errs = _check_event(chain, orc, blob[offs[0]:offs[1]])
    assert not errs, errs
    assert chain.counts().n_vertices == 1


def test_pu50_full_chain(chain, orc, events_pu50):
    blob, offs = events_pu50
    for e in range(len(offs) - 1):
        errs = _check_event(chain, orc, blob[offs[e]:offs[e + 1]])
        assert not errs, (e, errs)


def test_batch_full_chain(conditions, orc, events_pu50):
    from pixeltrack import PixelChain, batch_params
    blob, offs = events_pu50
    n = len(offs) - 1
    with PixelChain(conditions, batch_params(n)) as bc:
        bc.run_batch(blob, offs, stages=63)
        for e in range(n):
            orc.run_event(blob[offs[e]:offs[e + 1]], 63)
            errs = compare_fits(bc, orc, e) + compare_quality(bc, orc, e) + compare_vertices(bc, orc, e)
            assert not errs, (e, errs)


def test_producer_path_matches_batch(conditions, events_pu50):
    """The five producers called in turn (stage by stage) give the products of one run."""
    from pixeltrack import framework, producers
    from pixeltrack.formats import FedRawDataCollection
    blob, offs = events_pu50
    ev_bytes = bytes(blob[offs[0]:offs[1]])
    reg = framework.ProductRegistry()
    src = producers.Source(reg)
    path = producers.make_path(reg)
    es = producers.eventsetup_from_blobs(conditions)
    event = framework.Event(0, 1, reg)
    event.emplace(src.raw_put, FedRawDataCollection.from_bytes(ev_bytes))
    for p in path:
        p.produce(event, es)
    vtx = event.get(reg.consumes(producers.ZVertexSoA))
    orc = oracle.Oracle(conditions)
    orc.run_event(ev_bytes, 63)
    assert vtx.nv_final == orc.counts()["nv_final"]
    assert np.array_equal(vtx.idv, orc.get("idv"))
    es.get(producers.GPUContext).chain.close()


def _fixture_tracks():
    data = json.loads((GOLDEN / "brokenline_fixtures.json").read_text())
    hits, ge, offs = [], [], [0]
    for n in ("3", "4", "5"):
        fx = data["fits"][n]
        hits += fx["hits"]
        ge += fx["ge"]
        offs.append(offs[-1] + len(fx["hits"]))
    return data, np.array(hits, np.float64), np.array(ge, np.float32), np.array(offs, np.int32)


@pytest.mark.parametrize("precision", [0, 1])
def test_standalone_fit_fixtures(precision):
    import torch
    from pixeltrack.fits import bl_fit
    data, hits, ge, offs = _fixture_tracks()
    out = bl_fit(torch.as_tensor(hits).cuda(), torch.as_tensor(ge).cuda(), torch.as_tensor(offs).cuda(), data["B"],
                 precision=precision)
    # FP64 fit: outputs stored as FP32; mixed precision: within 1e-5 of FP64
    tol = 1e-6 if precision == 0 else 1e-5
    for k, n in enumerate(("3", "4", "5")):
        ref = data["fits"][n]["oracle"]
        np.testing.assert_allclose(out["state"][k].cpu().numpy(), ref["state"], rtol=tol, atol=tol)
        np.testing.assert_allclose(out["pt"][k].item(), ref["pt"], rtol=max(tol, 1e-6))


def test_autotuned_shapes_keep_results(conditions, events_pu50):
    """After pxl_autotune picks per-stage launch shapes, a graph replay of the batch still
    reproduces the oracle's tracks and vertices (launch shape never changes results)."""
    from pixeltrack import PixelChain, batch_params
    blob, offs = events_pu50
    n = len(offs) - 1
    with PixelChain(conditions, batch_params(n)) as bc:
        bc.stage_batch(blob, offs)
        chosen = bc.autotune(candidates=(2, 16, 64), reps=1)
        assert set(chosen.values()) <= {2, 16, 64}
        bc.stage_batch(blob, offs)
        bc.capture_graph()
        bc.launch_graph()
        bc.sync()
        orc = oracle.Oracle(conditions)
        for e in range(n):
            orc.run_event(blob[offs[e]:offs[e + 1]], 63)
            errs = compare_ca(bc, orc, e, classified=True) + compare_fits(bc, orc, e) + compare_quality(bc, orc, e) \
                + compare_vertices(bc, orc, e)
            assert not errs, (e, errs)


def _fit_workload(n, seed):
    from pixeltrack import gen
    return gen.fit_tracks(n, seed=seed)


def test_standalone_fits_all_hit_counts_match_oracle():
    """Tracks of 3..8 hits in mixed order (the fit workload generator) through the bucketed
    FP64 fit: state, pt and chi2 equal the oracle's within FP32 storage precision."""
    import torch
    from pixeltrack.fits import bl_fit
    B = 0.0114256972711507
    w = _fit_workload(600, seed=21)
    out = bl_fit(torch.as_tensor(w["hits"]).cuda(), torch.as_tensor(w["ge"]).cuda(),
                 torch.as_tensor(w["offsets"]).cuda(), B, precision=0)
    st = out["state"].cpu().numpy()
    pt = out["pt"].cpu().numpy()
    status = out["status"].cpu().numpy()
    seen = set()
    for t in range(600):
        a, b = w["offsets"][t], w["offsets"][t + 1]
        ref = oracle.bl_fit(w["hits"][a:b].T, w["ge"][a:b].T, B)
        assert status[t] == ref["rc"]
        if ref["rc"]:
            continue
        seen.add(b - a)
        np.testing.assert_allclose(st[t], ref["state"], rtol=2e-6, atol=1e-7)
        np.testing.assert_allclose(pt[t], ref["pt"], rtol=2e-6)
    assert seen == {3, 4, 5, 6, 7, 8}


def test_mixed_precision_fit_error_bounds():
    """FP32 mode against the FP64 mode on the 2^20 tracks of the fit workload: relative error
    below 1e-5 for q/pT and cot(theta) on every track, and absolute bounds for phi, d0 and z0
    (the last at the FP32 storage of values up to 20 cm)."""
    import torch
    from pixeltrack.fits import bl_fit
    B = 0.0114256972711507
    w = _fit_workload(1 << 20, seed=22)
    args = (torch.as_tensor(w["hits"]).cuda(), torch.as_tensor(w["ge"]).cuda(), torch.as_tensor(w["offsets"]).cuda(), B)
    f64 = bl_fit(*args, precision=0)["state"].double().cpu().numpy()
    f32 = bl_fit(*args, precision=1)["state"].double().cpu().numpy()
    ok = np.all(np.isfinite(f64), axis=1)
    d = np.abs(f32[ok] - f64[ok])
    qpt = d[:, 2] / np.abs(f64[ok, 2])
    cot = d[:, 3] / np.maximum(np.abs(f64[ok, 3]), 1e-3)
    assert qpt.max() < 1e-5
    assert cot.max() < 1e-5
    assert d[:, 0].max() < 1e-6       # phi, rad
    assert d[:, 1].max() < 1e-6       # d0, cm
    assert d[:, 4].max() < 5e-6       # z0, cm


def test_chain_mixed_precision_fit(conditions, events_pu50):
    """The chain with fit_precision = 1 (the FP32 fit): the same tuples and fitted set as the
    FP64 chain, and parameters within 1e-5 relative (q/pT, cot(theta)) of the FP64 chain's.
    The tuples whose FP32 fit gives pT >= 50 GeV are fitted again in FP64 (n_fits_fp64): a
    small share, and bit-equal to the FP64 chain's fits."""
    from pixeltrack import PixelChain, batch_params
    blob, offs = events_pu50
    res = {}
    for prec in (0, 1):
        with PixelChain(conditions, batch_params(4, words_per_event=90_000, fit_precision=prec)) as c:
            c.run_batch(blob, offs)
            res[prec] = [(c.product("fitted", e), c.product("state", e).reshape(-1, 5), c.counts(e).n_tuples,
                          c.product("pt", e), c.counts(e).n_fits_fp64) for e in range(4)]
    for e in range(4):
        (f0, s0, n0, p0, r0), (f1, s1, n1, p1, r1) = res[0][e], res[1][e]
        assert n0 == n1 and np.array_equal(f0, f1)
        assert r0 == 0 and 0 < r1 < 0.05 * f0[:n0].sum()
        stiff = f0[:n0].astype(bool) & (p0[:n0] >= 60.0)  # clear of the 50 GeV rule's edge
        assert stiff.any() and np.array_equal(s1[:n0][stiff], s0[:n0][stiff])
        sel = f0[:n0].astype(bool)
        a, b = s1[:n0][sel].astype(np.float64), s0[:n0][sel].astype(np.float64)
        ok = np.all(np.isfinite(b), axis=1)
        assert ok.sum() > 1000
        assert (np.abs(a[ok, 2] - b[ok, 2]) / np.abs(b[ok, 2])).max() < 1e-5
        assert (np.abs(a[ok, 3] - b[ok, 3]) / np.maximum(np.abs(b[ok, 3]), 1e-3)).max() < 1e-5


@pytest.mark.parametrize("strides", [-1, -8])
def test_work_queue_launches_keep_results(conditions, events_pu50, strides):
    """The doublet, connect, fishbone and ntuplet stages launched as persistent work queues
    (virtual blocks pulled from a device counter, events with the most hits first) give the
    oracle's results, as the static grids do."""
    from pixeltrack import PixelChain, batch_params
    blob, offs = events_pu50
    n = len(offs) - 1
    with PixelChain(conditions, batch_params(n)) as bc:
        bc.stage_batch(blob, offs)
        chosen = bc.autotune(candidates=(strides,), reps=1)
        assert chosen["doublets"] == strides and chosen["ntuplets"] == strides
        bc.stage_batch(blob, offs)
        bc.capture_graph()
        bc.launch_graph()
        assert bc.sync() == 0
        orc = oracle.Oracle(conditions)
        for e in range(n):
            orc.run_event(blob[offs[e]:offs[e + 1]], 63)
            errs = compare_ca(bc, orc, e, classified=True) + compare_fits(bc, orc, e) + compare_quality(bc, orc, e) \
                + compare_vertices(bc, orc, e)
            assert not errs, (e, errs)
