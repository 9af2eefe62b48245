"""Batched, stream-ordered copy-out (pxl_export_async) and per-context synchronisation.

The export must hold, event after event, exactly the loose tracks of each event's TrackSOA in
tuple order and its vertices, as the per-event product copies give them; and pxl_sync on one
context must not wait for another context's work on another stream."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

E = 8


@pytest.fixture(scope="module")
def batch(conditions):
    from pixeltrack import PixelChain, batch_params, gen
    blob, offs = gen.events(E, gen.MODE_PU, pu=50, seed=515)
    chain = PixelChain(conditions, batch_params(E, words_per_event=90_000))
    chain.stage_batch(blob, offs)
    chain.capture_graph()
    chain.launch_graph()
    assert chain.sync() == 0
    yield chain
    chain.close()


def test_export_equals_per_event_products(batch):
    import torch
    from pixeltrack import TrackExport
    out = TrackExport(E, max_tracks=60_000, max_vertices=E * 1024, cov=True)
    copy = torch.cuda.Stream()
    for _ in range(2):  # two calls: the second uses the other device export set
        batch.export_async(out, copy_stream=copy.cuda_stream)
        copy.synchronize()
        idx = out.index()
        assert idx[E, 1] == idx[:E, 1].sum() and idx[E, 3] == idx[:E, 3].sum()
        for e in range(E):
            ev = out.event(e)
            q = batch.product("quality", e)
            nt = batch.counts(e).n_tuples
            loose = np.flatnonzero(q[:nt] == 2)
            assert np.array_equal(ev["tuple"], loose + 1)
            st = batch.product("state", e).reshape(-1, 5)
            cv = batch.product("cov", e).reshape(-1, 15)
            assert np.array_equal(ev["state"], st[loose]) and np.array_equal(ev["cov"], cv[loose])
            for k in ("pt", "eta", "chi2"):
                assert np.array_equal(ev[k], batch.product(k, e)[loose]), k
            assert np.array_equal(ev["vertex"], batch.product("idv", e)[loose])
            off = batch.product("tuple_off", e).astype(np.int64)
            assert np.array_equal(ev["n_hits"], (off[loose + 1] - off[loose]).astype(np.uint8))
            nv = batch.counts(e).n_vertices
            assert len(ev["zv"]) == nv
            for k, p in (("zv", "zv"), ("wv", "wv"), ("vchi2", "vchi2"), ("ptv2", "ptv2"), ("ndof", "ndof")):
                assert np.array_equal(ev[k], batch.product(p, e)[:nv]), k


def test_export_bytes_and_truncation(batch):
    import torch
    from pixeltrack import TrackExport
    small = TrackExport(E, max_tracks=100, max_vertices=10)
    assert small.bytes() == 16 * (E + 1) + 100 * (20 + 4 + 4 + 4 + 1 + 2 + 4) + 10 * 20
    batch.export_async(small)
    torch.cuda.synchronize()
    idx = small.index()
    assert idx[E, 1] > 100  # more tracks than the host arrays hold: only the first 100 came over
    full = TrackExport(E, max_tracks=60_000, max_vertices=E * 1024)
    batch.export_async(full)
    torch.cuda.synchronize()
    assert np.array_equal(small.arrays["state"].numpy(), full.arrays["state"].numpy()[:500])


def test_sync_waits_for_its_own_context_only(conditions, batch):
    """Context A's pxl_sync returns while context B's stream is still busy: B's stream holds a
    half-second device sleep ahead of B's chain, and A ran on another stream."""
    import torch
    from pixeltrack import PixelChain, default_params, gen
    blob, offs = gen.events(1, gen.MODE_PU, pu=20, seed=3)
    sb = torch.cuda.Stream()
    with PixelChain(conditions, default_params()) as a:
        a.run_event(blob[offs[0]:offs[1]])  # warm
        with torch.cuda.stream(sb):
            torch.cuda._sleep(int(1e9))  # about half a second at B200 clocks
        batch.launch_graph(sb.cuda_stream)
        a.run_event(blob[offs[0]:offs[1]])  # pxl_event_run + pxl_sync on A's own stream
        busy = not sb.query()
        sb.synchronize()
        assert busy, "A's sync waited for B's stream"
        assert batch.sync() == 0
