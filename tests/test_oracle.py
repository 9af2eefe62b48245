"""The CPU oracle against the reference's own known-answer tests and fixtures."""
import json
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle

GOLDEN = Path(__file__).resolve().parent / "golden"


@pytest.mark.parametrize("kn", range(5))
def test_clustering_known_answer(kn):
    """test/gpu_clustering_t.jl:245-280: ncl == sum(nClustersInModule), then the charge cut
    leaves no noise module and numbers clusters 1..n without holes."""
    z = np.load(GOLDEN / f"clustering_kn{kn}.npz")
    r = oracle.clusterize_digis(z["id"], z["x"], z["y"], z["adc"], charge_cut=False)
    assert int(r["clus_in_module"].sum()) == int(z["ncl"])
    r = oracle.clusterize_digis(z["id"], z["x"], z["y"], z["adc"], charge_cut=True)
    ids, clus, nclus = r["id"], r["clus"], r["clus_in_module"]
    assert not np.any(ids == 666)
    valid = ids != 9999
    assert np.all(clus[valid] >= 1)
    assert np.all(clus[valid] <= nclus[ids[valid]])
    keys = np.unique(ids[valid].astype(np.int64) * 1000 + clus[valid])
    for mod in np.unique(ids[valid]):
        got = np.sort(keys[keys // 1000 == mod] % 1000)
        assert np.array_equal(got, np.arange(1, nclus[mod] + 1))


def test_clustering_diagonal():
    """plugin-SiPixelClusterizer/testClustering.jl:13-35: 6 clusters."""
    z = np.load(GOLDEN / "clustering_diag8.npz")
    r = oracle.clusterize_digis(z["id"], z["x"], z["y"], z["adc"], charge_cut=False)
    assert int(r["clus_in_module"].sum()) == 6


def test_brokenline_fixtures_regression():
    """test/testBrokenLine.jl fixtures through the FP64 oracle fit (goldens generated once)."""
    data = json.loads((GOLDEN / "brokenline_fixtures.json").read_text())
    for n, fx in data["fits"].items():
        hits = np.array(fx["hits"], np.float64).T
        ge = np.array(fx["ge"], np.float32).T
        r = oracle.bl_fit(hits, ge, data["B"])
        np.testing.assert_allclose(r["state"], fx["oracle"]["state"], rtol=1e-12, atol=1e-14)
        np.testing.assert_allclose(r["cov"], fx["oracle"]["cov"], rtol=1e-10, atol=1e-20)


def test_brokenline_recovers_helix():
    """Hits on an exact circle and line: the fit returns the generating parameters."""
    B = 0.0114256972711507
    R = 50.0  # cm
    xc, yc = 0.0, R
    phis = np.array([-np.pi / 2 + a for a in (0.06, 0.14, 0.22, 0.32)])
    x = xc + R * np.cos(phis)
    y = yc + R * np.sin(phis)
    s = R * (phis + np.pi / 2)
    cot = 0.7
    z = 0.1 + cot * s
    hits = np.vstack([x, y, z])
    ge = np.zeros((6, 4), np.float32)
    ge[0] = ge[2] = 1e-6
    ge[5] = 4e-6
    r = oracle.bl_fit(hits, ge, B)
    assert r["rc"] == 0
    np.testing.assert_allclose(r["pt"], B * R, rtol=5e-3)
    np.testing.assert_allclose(r["state"][3], cot, rtol=5e-3)


def test_phi_binner_invariants(conditions, events_pu50):
    """his_to_container_cpu.jl invariants on the event's phi histogram: every hit once,
    in the bin of its iphi, bins holding hit ids in decreasing order."""
    blob, offs = events_pu50
    orc = oracle.Oracle(conditions)
    orc.run_event(blob[offs[0]:offs[1]], stages=3)
    c = orc.counts()
    off = orc.get("phi_off")
    bins = orc.get("phi_bins")
    iphi = orc.get("iphi")
    hls = orc.get("hits_layer_start")
    assert off[-1] == c["n_hits"] == hls[-1]
    assert np.array_equal(np.sort(bins), np.arange(1, c["n_hits"] + 1))
    for b in range(1280):
        seg = bins[off[b]:off[b + 1]]
        assert np.all(np.diff(seg.astype(np.int64)) < 0)
        if len(seg):
            phib = ((iphi[seg.astype(np.int64) - 1].astype(np.int32) >> 9) & 127)
            assert np.all(phib == b % 128)


def test_chain_counts_plausible(conditions, event_single, events_pu50):
    """The whole oracle chain on the generator's events reconstructs the vertices."""
    orc = oracle.Oracle(conditions)
    blob, offs = event_single
    orc.run_event(blob[offs[0]:offs[1]])
    c = orc.counts()
    assert c["flags"] == 0
    assert c["nv_final"] == 1 and c["n_vtx_tracks"] > 50
    blob, offs = events_pu50
    orc.run_event(blob[offs[0]:offs[1]])
    c = orc.counts()
    assert c["flags"] == 0
    assert 35 <= c["nv_final"] <= 60


def test_forward_mode_gradient_matches_central_differences():
    """The oracle's dual-number gradient of chi2_line + chi2_circle agrees with central
    finite differences (h = 1e-6 cm) of the oracle's own FP64 fit."""
    import sys
    sys.path.insert(0, str(Path(__file__).resolve().parents[1] / "cms-julia_b200"))
    from pixeltrack import gen
    B = 0.0114256972711507
    w = gen.fit_tracks(40, seed=41)
    chi = lambda hh, ge: (lambda r: r["chi2_line"] + r["chi2_circle"])(oracle.bl_fit(hh.T, ge.T, B))
    for t in range(40):
        a, b = w["offsets"][t], w["offsets"][t + 1]
        hits, ge = w["hits"][a:b], w["ge"][a:b]
        c, g = oracle.bl_chi2_grad_fwd(hits, ge, B)
        assert abs(c - chi(hits, ge)) <= 1e-12 * abs(c)
        fd = np.zeros_like(hits)
        for i in range(b - a):
            for k in range(3):
                hp, hm = hits.copy(), hits.copy()
                hp[i, k] += 1e-6
                hm[i, k] -= 1e-6
                fd[i, k] = (chi(hp, ge) - chi(hm, ge)) / 2e-6
        assert np.abs(g - fd).max() <= 1e-6 * np.abs(fd).max()


def test_extended_capacities_keep_whole_events(conditions):
    """Pileup-200 events pass the reference's per-event doublet and tuple capacities
    (ca_hit_ntuplet_generator.jl:40, PixelTrackHeterogeneous.jl:55), which truncate them; the
    extended mode keeps them whole and agrees with the reference mode wherever no capacity is
    reached (a PU50 event is identical in both)."""
    from pixeltrack import gen
    blob, offs = gen.events(2, gen.MODE_PU, pu=200, seed=77)
    ref, ext = oracle.Oracle(conditions), oracle.Oracle(conditions, oracle.EXTENDED_CAPS)
    for e in range(2):
        ev = blob[offs[e]:offs[e + 1]]
        ref.run_event(ev)
        ext.run_event(ev)
        cr, cx = ref.counts(), ext.counts()
        assert cr["n_cells"] == 458752 and cr["flags"] & 0x10  # doublets capped
        assert cr["n_tuples"] == 32768 and cr["flags"] & 0x40   # tuples capped at the TrackSOA stride
        assert cx["flags"] == 0 and cx["n_cells"] > 458752 and cx["n_tuples"] > cr["n_tuples"]
        assert cx["n_hits"] == cr["n_hits"]
        # the kept doublets are the first ones (inner, outer hit and layer pair; the used flag
        # and the fishbone's kills depend on the doublets past the cap)
        n = cr["n_cells"]
        assert np.array_equal(ext.get("cells").reshape(-1, 5)[:n, :3], ref.get("cells").reshape(-1, 5)[:, :3])
    blob, offs = gen.events(1, gen.MODE_PU, pu=50, seed=11)
    ref.run_event(blob[offs[0]:offs[1]])
    ext.run_event(blob[offs[0]:offs[1]])
    assert ref.counts() == ext.counts()
    nt = ref.counts()["n_tuples"]
    for name in ("cells", "phi_bins", "tuple_hits", "cell_neighbors", "cell_tracks"):
        assert np.array_equal(ref.get(name), ext.get(name)[:len(ref.get(name))]), name
    for name in ("quality", "pt", "chi2"):
        assert np.array_equal(ref.get(name)[:nt], ext.get(name)[:nt]), name
    assert ref.get("zv").tolist() == ext.get("zv").tolist()
