"""Parity of the CUDA chain (through the C ABI) with the CPU oracle on the same inputs.
Integer products and the FP32 rechit arithmetic are compared bit for bit."""
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle
from parity import compare_ca, compare_digis_clusters, compare_hits

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


@pytest.mark.parametrize("kn", range(5))
@pytest.mark.parametrize("cut", [False, True])
def test_clustering_known_answer_gpu(chain, kn, cut):
    z = np.load(GOLDEN / f"clustering_kn{kn}.npz")
    g = chain.clusterize_digis(z["id"], z["x"], z["y"], z["adc"], charge_cut=cut)
    o = oracle.clusterize_digis(z["id"], z["x"], z["y"], z["adc"], charge_cut=cut)
    if not cut:
        assert int(g["clus_in_module"].sum()) == int(z["ncl"])
    nm = int(o["module_start"][0])
    assert np.array_equal(g["module_start"][:nm + 1], o["module_start"][:nm + 1])
    assert np.array_equal(g["module_id"][:nm], o["module_id"][:nm])
    assert np.array_equal(g["clus_in_module"], o["clus_in_module"])
    assert np.array_equal(g["clus"], o["clus"])
    assert np.array_equal(g["id"], o["id"])


def test_clustering_diagonal_gpu(chain):
    z = np.load(GOLDEN / "clustering_diag8.npz")
    g = chain.clusterize_digis(z["id"], z["x"], z["y"], z["adc"], charge_cut=False)
    assert int(g["clus_in_module"].sum()) == 6


def _run_both(chain, orc, ev, stages):
    chain.run_event(ev, stages)
    orc.run_event(ev, stages)


def test_single_event_digis_hits(chain, orc, event_single):
    blob, offs = event_single
    ev = blob[offs[0]:offs[1]]
    _run_both(chain, orc, ev, 3)
    errs = compare_digis_clusters(chain, orc) + compare_hits(chain, orc)
    assert not errs, errs


def test_pu50_events_digis_hits(chain, orc, events_pu50):
    blob, offs = events_pu50
    for e in range(len(offs) - 1):
        ev = blob[offs[e]:offs[e + 1]]
        _run_both(chain, orc, ev, 3)
        errs = compare_digis_clusters(chain, orc) + compare_hits(chain, orc)
        assert not errs, (e, errs)


def test_single_event_ca(chain, orc, event_single):
    blob, offs = event_single
    ev = blob[offs[0]:offs[1]]
    _run_both(chain, orc, ev, 7)
    errs = compare_ca(chain, orc)
    assert not errs, errs


def test_pu50_events_ca(chain, orc, events_pu50):
    blob, offs = events_pu50
    for e in range(len(offs) - 1):
        ev = blob[offs[e]:offs[e + 1]]
        _run_both(chain, orc, ev, 7)
        errs = compare_ca(chain, orc)
        assert not errs, (e, errs)


def test_batch_ca_matches_oracle(conditions, orc, events_pu50):
    from pixeltrack import PixelChain, batch_params
    blob, offs = events_pu50
    n = len(offs) - 1
    with PixelChain(conditions, batch_params(n)) as bc:
        bc.run_batch(blob, offs, stages=7)
        for e in range(n):
            orc.run_event(blob[offs[e]:offs[e + 1]], 7)
            errs = compare_ca(bc, orc, e)
            assert not errs, (e, errs)


def test_batch_ca_with_overflowing_tuple_pool(conditions, orc, events_pu50, monkeypatch):
    """The count pass keeps each tuple's record in a pool of 4096 parts, from which the fill
    moves the tuples into place. With one record per part (PXL_TUPLE_POOL_PART, read when the
    context is created) a PU50 batch overflows the pool, and the fill walks the tuples again:
    the products must be the same."""
    from pixeltrack import PixelChain, batch_params
    blob, offs = events_pu50
    n = len(offs) - 1
    monkeypatch.setenv("PXL_TUPLE_POOL_PART", "1")
    with PixelChain(conditions, batch_params(n)) as bc:
        monkeypatch.delenv("PXL_TUPLE_POOL_PART")
        bc.run_batch(blob, offs, stages=7)
        for e in range(n):
            orc.run_event(blob[offs[e]:offs[e + 1]], 7)
            errs = compare_ca(bc, orc, e)
            assert not errs, (e, errs)


def test_batch_matches_oracle(conditions, orc, events_pu50):
    from pixeltrack import PixelChain, batch_params
    blob, offs = events_pu50
    n = len(offs) - 1
    with PixelChain(conditions, batch_params(n)) as bc:
        bc.run_batch(blob, offs, stages=3)
        for e in range(n):
            orc.run_event(blob[offs[e]:offs[e + 1]], 3)
            errs = compare_digis_clusters(bc, orc, e) + compare_hits(bc, orc, e)
            assert not errs, (e, errs)


def test_graph_replay_is_deterministic(conditions, events_pu50):
    from pixeltrack import PixelChain, batch_params
    blob, offs = events_pu50
    n = len(offs) - 1
    with PixelChain(conditions, batch_params(n)) as bc:
        bc.stage_batch(blob, offs)
        bc.capture_graph(3)
        bc.launch_graph()
        bc.sync()
        first = {k: bc.product(k, n - 1) for k in ("clus", "xg", "phi_bins")}
        bc.launch_graph()
        bc.sync()
        for k, v in first.items():
            assert np.array_equal(v, bc.product(k, n - 1))


def test_input_slots_overlap_copy_and_chain(conditions, events_pu50):
    """Two batches alternate through the two input slots, each copied on a copy stream
    while the other slot's graph runs: every launch gives the products of a plain run of
    its own batch."""
    import torch
    from pixeltrack import PixelChain, batch_params, gen
    blob_a, offs_a = events_pu50
    n = len(offs_a) - 1
    blob_b, offs_b = gen.events(n, gen.MODE_PU, pu=50, seed=12)
    batches = [(blob_a, offs_a), (blob_b, offs_b)]
    want = []
    with PixelChain(conditions, batch_params(n)) as bc:
        for blob, offs in batches:
            bc.run_batch(blob, offs)
            bc.sync()
            want.append(([bc.counts(e).n_vertices for e in range(n)], bc.product("xg", n - 1)))
        pinned = []
        for blob, _ in batches:
            t = torch.empty(len(blob), dtype=torch.uint8, pin_memory=True)
            t.numpy()[:] = blob
            pinned.append(t.numpy())
        res = torch.empty(n, dtype=torch.int32, pin_memory=True)
        stream, copy = torch.cuda.Stream(), torch.cuda.Stream()
        bc.stage_batch(blob_a, offs_a, stream.cuda_stream)
        stream.synchronize()
        bc.capture_graph()
        bc.stage_slot(0, pinned[0], offs_a, copy.cuda_stream)
        for i in range(6):
            k = i % 2
            bc.launch_slot(k, stream.cuda_stream)
            bc.results_async(res.data_ptr(), n, stream.cuda_stream)
            bc.stage_slot(1 - k, pinned[1 - k], batches[1 - k][1], copy.cuda_stream)
            stream.synchronize()
            assert res.numpy().tolist() == want[k][0], i
            assert np.array_equal(bc.product("xg", n - 1), want[k][1]), i
        copy.synchronize()


def test_slot_launch_needs_captured_event_count(conditions, events_pu50):
    from pixeltrack import PixelChain, batch_params
    blob, offs = events_pu50
    n = len(offs) - 1
    with PixelChain(conditions, batch_params(n)) as bc:
        with pytest.raises(RuntimeError, match="bad state"):
            bc.launch_slot(1)
        bc.stage_batch(blob, offs)
        bc.capture_graph()
        bc.stage_slot(1, blob[: int(offs[n - 1])], offs[:n])
        with pytest.raises(RuntimeError, match="bad state"):
            bc.launch_slot(1)
        bc.stage_slot(1, blob, offs)
        bc.launch_slot(1)
        bc.sync()
