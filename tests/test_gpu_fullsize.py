"""The benchmark's batch at full size (1000 synthetic PU50 events in one launch sequence,
one captured graph) checked through properties that hold at any size: sample events equal
the oracle, every per-key list is sorted as the reference fills it, list offsets are
consistent with the counts, the batch raises no warning and graph replays repeat."""
import numpy as np
import pytest

from oracle import oracle
from parity import compare_ca, compare_digis_clusters, compare_fits, compare_hits, compare_quality, compare_vertices

pytestmark = pytest.mark.gpu

E = 1000


@pytest.fixture(scope="module")
def full_batch(conditions):
    from pixeltrack import PixelChain, batch_params, gen
    blob, offs = gen.events(E, gen.MODE_PU, pu=50, seed=2024)
    words = int(np.diff(offs).sum() // 4)
    params = batch_params(E, words_per_event=words // E * 13 // 10 + 4096, hits_per_event_avg=16_000,
                          doublets_per_event_avg=140_000, tuples_per_event_avg=11_000)
    chain = PixelChain(conditions, params)
    chain.stage_batch(blob, offs)
    chain.capture_graph()
    chain.launch_graph()
    warn = chain.sync()
    yield chain, blob, offs, warn
    chain.close()


def test_no_warnings(full_batch):
    assert full_batch[3] == 0


@pytest.mark.parametrize("e", [0, 517, E - 1])
def test_sample_events_match_oracle(conditions, full_batch, e):
    chain, blob, offs, _ = full_batch
    orc = oracle.Oracle(conditions)
    orc.run_event(blob[offs[e]:offs[e + 1]], 63)
    errs = (compare_digis_clusters(chain, orc, e) + compare_hits(chain, orc, e) + compare_ca(chain, orc, e, classified=True)
            + compare_fits(chain, orc, e) + compare_quality(chain, orc, e) + compare_vertices(chain, orc, e))
    assert not errs, errs


def _csr(a: np.ndarray, nkeys: int):
    off = a[:nkeys + 1].astype(np.int64)
    return off, a[nkeys + 1:]


@pytest.mark.parametrize("e", [3, 250, 761])
def test_lists_sorted_and_consistent(full_batch, e):
    chain = full_batch[0]
    c = chain.counts(e)
    for name, nkeys, ascending in (("outer_hit_of_cell", c.n_hits, True), ("cell_neighbors", c.n_doublets, True),
                                   ("cell_tracks", c.n_doublets, True)):
        off, lst = _csr(chain.product(name, e), nkeys)
        assert off[0] == 0 and np.all(np.diff(off) >= 0), name
        assert off[-1] == len(lst), name
        for k in np.flatnonzero(np.diff(off) > 1):
            seg = lst[off[k]:off[k + 1]].astype(np.int64)
            assert np.all(np.diff(seg) > 0) if ascending else np.all(np.diff(seg) < 0), (name, k)
    # every doublet ends on exactly one hit: the outer-hit lists hold each cell once
    off, lst = _csr(chain.product("outer_hit_of_cell", e), c.n_hits)
    assert np.array_equal(np.sort(lst), np.arange(1, c.n_doublets + 1))


def test_graph_replays_repeat(full_batch):
    import torch
    chain = full_batch[0]
    res = [torch.empty(E, dtype=torch.int32, pin_memory=True) for _ in range(2)]
    for r in res:
        chain.launch_graph()
        chain.results_async(r.data_ptr(), E)
        chain.sync()
    assert np.array_equal(res[0].numpy(), res[1].numpy())
    assert res[0].numpy().sum() == sum(chain.counts(e).n_vertices for e in range(E))
