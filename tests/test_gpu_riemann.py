"""Stand-alone Riemann fits (pxl_riemann_fit) against the CPU oracle's FP64 restatement of
riemann_fit.jl: FP64 mode within FP32 storage precision, mixed mode within the stated
bounds, and exact recovery of a noise-free helix."""
import numpy as np
import pytest

from oracle import oracle

pytestmark = pytest.mark.gpu
B = 0.0114256972711507


def _run(w, precision):
    import torch
    from pixeltrack.fits import riemann_fit
    t = lambda a: torch.as_tensor(a).cuda()
    out = riemann_fit(t(w["hits"]), t(w["ge"]), t(w["offsets"]), B, precision=precision)
    return {k: v.cpu().numpy() for k, v in out.items()}


def test_riemann_fp64_matches_oracle():
    from pixeltrack import gen
    w = gen.fit_tracks(800, seed=51)
    out = _run(w, 0)
    seen = set()
    for t in range(800):
        a, b = w["offsets"][t], w["offsets"][t + 1]
        r = oracle.riemann_fit(w["hits"][a:b], w["ge"][a:b], B)
        assert out["status"][t] == r["rc"]
        if r["rc"]:
            continue
        seen.add(b - a)
        np.testing.assert_allclose(out["state"][t], r["state"], rtol=2e-6, atol=1e-7)
        np.testing.assert_allclose(out["pt"][t], r["pt"], rtol=2e-6)
        np.testing.assert_allclose(out["chi2"][t], [r["chi2_circle"], r["chi2_line"]], rtol=1e-4, atol=1e-6)
    assert seen == {3, 4, 5, 6, 7, 8}


def test_riemann_mixed_precision_bounds():
    """FP32 mode against FP64 on the 2^20 workload tracks: q/pT and cot(theta) within 1e-5
    relative on every track."""
    from pixeltrack import gen
    w = gen.fit_tracks(1 << 20, seed=52)
    f64 = _run(w, 0)["state"].astype(np.float64)
    f32 = _run(w, 1)["state"].astype(np.float64)
    ok = np.all(np.isfinite(f64), axis=1)
    d = np.abs(f32[ok] - f64[ok])
    qpt = d[:, 2] / np.abs(f64[ok, 2])
    assert qpt.max() < 1e-5
    assert (d[:, 3] / np.maximum(np.abs(f64[ok, 3]), 1e-3)).max() < 1e-5
    assert d[:, 0].max() < 1e-6 and d[:, 1].max() < 1e-6 and d[:, 4].max() < 1e-5


def test_riemann_exact_helix():
    R, phis = 300.0, np.array([0.01, 0.025, 0.04, 0.055, 0.07])
    hits = np.stack([R * np.sin(phis), R - R * np.cos(phis), 0.3 + 0.7 * R * phis], 1)
    ge = np.zeros((5, 6), np.float32)
    ge[:, 0] = ge[:, 2] = 1e-6
    ge[:, 5] = 4e-6
    out = _run({"hits": hits, "ge": ge, "offsets": np.array([0, 5], np.int32)}, 0)
    np.testing.assert_allclose(out["pt"][0], R * B, rtol=1e-6)
    np.testing.assert_allclose(out["state"][0, 3:], [0.7, 0.3], rtol=1e-6)
    assert abs(out["state"][0, 1]) < 1e-6
