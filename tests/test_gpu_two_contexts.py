"""Two contexts in flight on two streams, as the throughput benchmark runs them: each
context's graph replays, alternating with the other's and overlapping it, give the same
products as one context run alone (no state is shared between contexts), including the
batched export of tracks and vertices."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

E = 8
PRODUCTS = ("tuple_off", "tuple_hits", "quality", "state", "pt", "idv", "zv")


@pytest.fixture(scope="module")
def batch():
    from pixeltrack import gen
    return gen.events(E, gen.MODE_PU, pu=50, seed=919)


def _snapshot(chain):
    snap = []
    for e in range(E):
        c = chain.counts(e)
        snap.append((c.n_hits, c.n_doublets, c.n_tuples, c.n_vertices,
                     [chain.product(p, e).copy() for p in PRODUCTS]))
    return snap


def test_alternating_contexts_match_one_context(conditions, batch):
    import torch
    from pixeltrack import PixelChain, TrackExport, batch_params
    blob, offs = batch
    params = batch_params(E, words_per_event=90_000)
    with PixelChain(conditions, params) as ref:
        ref.run_batch(blob, offs)
        want = _snapshot(ref)
    chains = [PixelChain(conditions, params) for _ in range(2)]
    streams = [torch.cuda.Stream() for _ in range(2)]
    try:
        for c, s in zip(chains, streams):
            c.stage_batch(blob, offs, s.cuda_stream)
            s.synchronize()
            c.capture_graph()
        outs = [TrackExport(E, max_tracks=60_000, max_vertices=E * 1024) for _ in range(2)]
        copy = torch.cuda.Stream()
        for k in range(6):  # alternate steps, both contexts in flight
            i = k % 2
            chains[i].launch_graph(streams[i].cuda_stream)
            chains[i].export_async(outs[i], streams[i].cuda_stream, copy.cuda_stream)
        torch.cuda.synchronize()
        for c in chains:
            assert c.sync() == 0
            got = _snapshot(c)
            for e in range(E):
                assert got[e][:4] == want[e][:4], e
                for name, g, w in zip(PRODUCTS, got[e][4], want[e][4]):
                    assert np.array_equal(g, w, equal_nan=True), (e, name)
        a, b = (o.index() for o in outs)
        assert np.array_equal(a, b)
        assert np.array_equal(outs[0].arrays["state"].numpy()[:a[E, 1]], outs[1].arrays["state"].numpy()[:a[E, 1]])
    finally:
        for c in chains:
            c.close()
