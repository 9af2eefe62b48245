"""The hand-written broken-line adjoint (pxl_bl_fit_adjoint) against the CPU oracle:
forward-mode dual-number derivatives through the reference formulation, central finite
differences (h = 1e-6 cm) of the oracle's FP64 chi2, and alignment gradients against
finite differences over the alignment parameters. Tolerance: 1e-6 relative (norm-wise
per track, gradients stored as float32)."""
import numpy as np
import pytest

from oracle import oracle

pytestmark = pytest.mark.gpu
B = 0.0114256972711507


@pytest.fixture(scope="module")
def workload():
    from pixeltrack import gen
    return gen.fit_tracks(400, seed=31)


def _gpu_adjoint(w, **kw):
    import torch
    from pixeltrack.fits import bl_fit_adjoint
    t = lambda a: torch.as_tensor(a).cuda()
    return bl_fit_adjoint(t(w["hits"]), t(w["ge"]), t(w["offsets"]), B, **{k: (t(v) if isinstance(v, np.ndarray) else v)
                                                                           for k, v in kw.items()})


def test_adjoint_matches_forward_mode(workload):
    w = workload
    out = _gpu_adjoint(w)
    g = out["grad_hits"].double().cpu().numpy()
    c = out["chi2"].double().cpu().numpy()
    seen = set()
    for t in range(len(w["offsets"]) - 1):
        a, b = w["offsets"][t], w["offsets"][t + 1]
        cf, gf = oracle.bl_chi2_grad_fwd(w["hits"][a:b], w["ge"][a:b], B)
        if not np.isfinite(cf):
            continue
        seen.add(b - a)
        assert abs(c[t] - cf) <= 1e-6 * abs(cf) + 1e-12
        assert np.abs(g[a:b] - gf).max() <= 1e-6 * np.abs(gf).max()
    assert seen == {3, 4, 5, 6, 7, 8}


def test_adjoint_matches_central_differences(workload):
    w = workload
    out = _gpu_adjoint(w)
    g = out["grad_hits"].double().cpu().numpy()
    h = 1e-6
    chi = lambda hh, ge: (lambda r: r["chi2_line"] + r["chi2_circle"])(oracle.bl_fit(hh.T, ge.T, B))
    for t in range(0, 60):
        a, b = w["offsets"][t], w["offsets"][t + 1]
        hits, ge = w["hits"][a:b].copy(), w["ge"][a:b]
        fd = np.zeros_like(hits)
        for i in range(b - a):
            for k in range(3):
                hp, hm = hits.copy(), hits.copy()
                hp[i, k] += h
                hm[i, k] -= h
                fd[i, k] = (chi(hp, ge) - chi(hm, ge)) / (2 * h)
        assert np.abs(g[a:b] - fd).max() <= 1e-6 * np.abs(fd).max(), t


def test_adjoint_translation_invariance(workload):
    """chi2 does not change under a common shift of a track's hits: gradients sum to zero."""
    w = workload
    g = _gpu_adjoint(w)["grad_hits"].double().cpu().numpy()
    for t in range(len(w["offsets"]) - 1):
        a, b = w["offsets"][t], w["offsets"][t + 1]
        s = g[a:b].sum(axis=0)
        assert np.abs(s).max() <= 1e-5 * np.abs(g[a:b]).max()


def test_alignment_gradient_matches_finite_differences():
    from pixeltrack import gen
    w = gen.fit_tracks(3000, seed=32)
    pos = gen.module_positions()
    rng = np.random.default_rng(5)
    align = np.zeros((pos.shape[0], 6), np.float32)
    align[:, :3] = rng.normal(0, 50e-4, (pos.shape[0], 3))
    align[:, 3:] = rng.normal(0, 1e-4, (pos.shape[0], 3))
    out = _gpu_adjoint(w, module=w["module"], module_pos=pos, align=align, want_align_grad=True)
    ga = out["grad_align64"].cpu().numpy()
    ga32 = out["grad_align"].double().cpu().numpy()
    assert np.abs(ga32 - ga).max() <= 1e-6 * np.abs(ga).max()
    # translation gradients equal the sums of the hit gradients on each module
    gh = out["grad_hits"].double().cpu().numpy()
    mods = w["module"]
    busiest = np.argsort(-np.bincount(mods[mods >= 0], minlength=pos.shape[0]))[:3]
    for m in busiest:
        np.testing.assert_allclose(ga[m, :3], gh[mods == m].sum(axis=0), rtol=1e-5, atol=1e-6 * np.abs(ga[m, :3]).max())
    # finite differences of the oracle's total chi2 over the tracks that touch module m

    def moved(al):
        hh = w["hits"].copy()
        on = mods >= 0
        c = pos[mods[on]]
        r = hh[on] - c
        t, om = al[mods[on], :3].astype(np.float64), al[mods[on], 3:].astype(np.float64)
        hh[on] += t + np.cross(om, r)
        return hh

    offs = w["offsets"]
    track_of_hit = np.repeat(np.arange(len(offs) - 1), np.diff(offs))
    for m in busiest[:2]:
        tracks = np.unique(track_of_hit[mods == m])

        def total(al):
            hh = moved(al)
            s = 0.0
            for t in tracks:
                r = oracle.bl_fit(hh[offs[t]:offs[t + 1]].T, w["ge"][offs[t]:offs[t + 1]].T, B)
                s += r["chi2_line"] + r["chi2_circle"]
            return s

        base = align.astype(np.float64)
        for k, h in ((0, 1e-6), (2, 1e-6), (5, 1e-7)):
            ap, am = base.copy(), base.copy()
            ap[m, k] += h
            am[m, k] -= h
            fd = (total(ap) - total(am)) / (2 * h)
            assert abs(ga[m, k] - fd) <= 1e-5 * np.abs(ga[m]).max() + 1e-6 * abs(fd), (m, k, ga[m, k], fd)
