"""Failure injection on the host (no device fault is ever provoked): corrupted FED
payload words, a FED directory that announces more FEDs than the event holds, and batch
buffers too small for the batch. The chain must flag what the reference flags, keep the
results of everything that fits identical to the oracle's, and never fault."""
import numpy as np
import pytest

from oracle import oracle
from parity import compare_digis_clusters, compare_hits

pytestmark = pytest.mark.gpu


def _corrupt_words(ev: bytes, rng, frac: float) -> bytes:
    from pixeltrack.formats import FedRawData, FedRawDataCollection
    c = FedRawDataCollection.from_bytes(ev)
    for fid, fd in list(c.feds.items()):
        if len(fd.data) < 24:
            continue
        w = np.frombuffer(fd.data, dtype=np.uint32).copy()
        payload = np.arange(2, len(w) - 2)  # 8-byte header and trailer kept
        # pixel address and ADC bits (invalid rows/columns give code 37), and a few words
        # moved to ROC 25 (code 25); link and ROC stay otherwise, so module runs stay whole
        pick = payload[rng.random(len(payload)) < frac]
        w[pick] ^= (rng.integers(1, 1 << 21, len(pick), dtype=np.uint64)).astype(np.uint32)
        roc25 = payload[rng.random(len(payload)) < frac / 4]
        w[roc25] = (w[roc25] & ~np.uint32(0x1F << 21)) | np.uint32(25 << 21)
        c.feds[fid] = FedRawData(fid, w.tobytes())
    return c.to_bytes()


def _errors(chain, e):
    g = chain.product("errors", e)
    return g.reshape(-1, 4) if g.size else g.reshape(0, 4)


def test_corrupted_words_match_oracle(conditions, events_pu50):
    from pixeltrack import PixelChain, default_params
    blob, offs = events_pu50
    rng = np.random.default_rng(3)
    orc = oracle.Oracle(conditions)
    with PixelChain(conditions, default_params()) as chain:
        for e in range(2):
            ev = _corrupt_words(bytes(blob[offs[e]:offs[e + 1]]), rng, 0.02)
            chain.run_event(ev, 3)
            orc.run_event(ev, 3)
            errs = compare_digis_clusters(chain, orc, 0) + compare_hits(chain, orc, 0)
            assert not errs, errs
            ge, oe = _errors(chain, 0), orc.get("errors").reshape(-1, 4)
            assert len(ge) == len(oe) > 0
            # records are appended in parallel: compare as sets of (rawId, word, type, fed)
            assert sorted(map(tuple, ge.tolist())) == sorted(map(tuple, oe.tolist()))


def test_directory_announcing_missing_feds(conditions, events_pu50):
    from pixeltrack import PixelChain, default_params
    blob, offs = events_pu50
    ev = bytearray(blob[offs[0]:offs[1]])
    n = int.from_bytes(ev[:4], "little")
    ev[:4] = (n + 3).to_bytes(4, "little")  # three FEDs more than the event holds
    orc = oracle.Oracle(conditions)
    with PixelChain(conditions, default_params()) as chain:
        chain.run_event(bytes(ev), 3)
        orc.run_event(bytes(ev), 3)
        errs = compare_digis_clusters(chain, orc, 0) + compare_hits(chain, orc, 0)
        assert not errs, errs
        assert chain.counts(0).warnings & 0x800  # the truncated directory is flagged


def test_batch_buffers_too_small(conditions, events_pu50):
    """Hit buffer for about two of the four events: the events that fit are exact through
    the whole chain, the others are emptied with the buffer warning, and the run completes."""
    from pixeltrack import PixelChain, batch_params
    from parity import compare_ca
    blob, offs = events_pu50
    orc = oracle.Oracle(conditions)
    nh = []
    for e in range(4):
        orc.run_event(blob[offs[e]:offs[e + 1]], 3)
        nh.append(orc.counts()["n_hits"])
    cap = nh[0] + nh[1] + nh[2] // 2
    params = batch_params(4, hits_per_event_avg=cap // 4 + 1)
    with PixelChain(conditions, params) as bc:
        bc.run_batch(blob, offs, stages=7)
        warn = bc.sync()
        assert warn & 0x800
        for e in range(2):
            orc.run_event(blob[offs[e]:offs[e + 1]], 7)
            errs = compare_digis_clusters(bc, orc, e) + compare_hits(bc, orc, e) + compare_ca(bc, orc, e)
            assert not errs, (e, errs)
        for e in (2, 3):
            c = bc.counts(e)
            assert c.warnings & 0x800 and c.n_hits == 0 and c.n_doublets == 0 and c.n_tuples == 0


def _edit_fed(ev: bytes, k: int, edit) -> bytes:
    """The event with edit(bytearray of FED data) applied to its k-th non-empty FED."""
    from pixeltrack.formats import FedRawData, FedRawDataCollection
    c = FedRawDataCollection.from_bytes(ev)
    fid = [f for f, fd in c.feds.items() if len(fd.data) >= 24][k]
    data = bytearray(c.feds[fid].data)
    c.feds[fid] = FedRawData(fid, bytes(edit(data)))
    return c.to_bytes()


def _set_word(data: bytearray, off: int, fn):
    w = int.from_bytes(data[off:off + 4], "little")
    data[off:off + 4] = (fn(w) & 0xFFFFFFFF).to_bytes(4, "little")
    return data


# FED header / trailer conditions (SiPixelRawToClusterCUDA.jl:90-128, ErrorChecker.jl:82-137):
# (edit, whether the reference raises on it)
FED_CASES = {
    "header_check_fails": (lambda d: _set_word(d, 4, lambda w: (w & 0x0FFFFFFF) | (0x3 << 28)), False),
    "foreign_source_id": (lambda d: _set_word(d, 0, lambda w: (w & ~(0xFFF << 8)) | (1234 << 8)), False),
    "more_headers": (lambda d: _set_word(d, 0, lambda w: w | 0x8), True),
    "trailer_check_fails": (lambda d: _set_word(d, len(d) - 4, lambda w: (w & 0x0FFFFFFF) | (0x7 << 28)), True),
    "wrong_fragment_length": (lambda d: _set_word(d, len(d) - 4, lambda w: (w & ~0xFFFFFF) | ((w + 5) & 0xFFFFFF)),
                              True),
    "more_trailers": (lambda d: _set_word(d, len(d) - 8, lambda w: w | 0x8), True),
    "size_not_64bit_words": (lambda d: d + bytearray(4), True),
}


@pytest.mark.parametrize("case", sorted(FED_CASES))
def test_fed_header_trailer_conditions(conditions, events_pu50, case):
    """Each condition as the reference meets it: no error record (its checker has
    _includeErrors = false), the raise conditions flagged (PXL_WARN_FED_FORMAT, 0x1000), and the
    digis and clusters of the event equal to the oracle's."""
    from pixeltrack import PixelChain, default_params
    blob, offs = events_pu50
    edit, raises = FED_CASES[case]
    ev = _edit_fed(bytes(blob[offs[1]:offs[2]]), 5, edit)
    orc = oracle.Oracle(conditions)
    with PixelChain(conditions, default_params()) as chain:
        warn = chain.run_event(ev, 3)
        flags = orc.run_event(ev, 3)
        assert bool(warn & 0x1000) == raises and bool(flags & 0x1000) == raises, (warn, flags)
        errs = compare_digis_clusters(chain, orc, 0) + compare_hits(chain, orc, 0)
        assert not errs, errs
        assert len(_errors(chain, 0)) == len(orc.get("errors").reshape(-1, 4))


def _split_module_runs(conditions, ev: bytes, n_splits: int, seed: int) -> bytes:
    """The event with, in n_splits FEDs, one word in the middle of a module's run replaced by
    a word of another module of the same FED: the module id then starts two runs (data only
    corruption gives), which the reference's charge cut handles in its serial order."""
    from pixeltrack.formats import FedRawData, FedRawDataCollection
    rng = np.random.default_rng(seed)
    c = FedRawDataCollection.from_bytes(ev)
    orc = oracle.Oracle(conditions)
    done = 0
    for fid in sorted(c.feds):
        if done == n_splits:
            break
        fd = c.feds[fid]
        if len(fd.data) < 64:
            continue
        one = FedRawDataCollection({fid: fd}).to_bytes()
        orc.run_event(one, 1)
        mid = orc.get("module_ind")
        w = np.frombuffer(fd.data, dtype=np.uint32).copy()
        # runs of equal valid ids among the payload words (word 2 + k is digi k)
        runs = []
        k = 0
        while k < len(mid):
            j = k
            while j + 1 < len(mid) and mid[j + 1] == mid[k]:
                j += 1
            if mid[k] != 9999 and j - k >= 5:
                runs.append((k, j))
            k = j + 1
        if len(runs) < 2:
            continue
        a = runs[int(rng.integers(len(runs)))]
        others = [r for r in runs if mid[r[0]] != mid[a[0]]]
        b = others[int(rng.integers(len(others)))]
        w[2 + (a[0] + a[1]) // 2] = w[2 + b[0]]
        c.feds[fid] = FedRawData(fid, w.tobytes())
        done += 1
    assert done == n_splits
    return c.to_bytes()


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_repeated_module_runs_match_oracle(conditions, events_pu50, seed):
    from pixeltrack import PixelChain, default_params
    blob, offs = events_pu50
    ev = _split_module_runs(conditions, bytes(blob[offs[2]:offs[3]]), 6, seed)
    orc = oracle.Oracle(conditions)
    with PixelChain(conditions, default_params()) as chain:
        chain.run_event(ev, 3)
        orc.run_event(ev, 3)
        nm = orc.counts()["n_modules"]
        ids = orc.get("module_id")[:nm]
        assert len(np.unique(ids)) < nm  # some module id starts two runs
        errs = compare_digis_clusters(chain, orc, 0) + compare_hits(chain, orc, 0)
        assert not errs, errs
