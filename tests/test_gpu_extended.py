"""Extended-capacity mode on high-pileup events (PU up to 260) above the reference's per-event
capacities: the CUDA chain with pxl_params_extended must equal the oracle run with the same
enlarged capacities on every product, and with the reference's capacities both must
truncate the same way (ca_hit_ntuplet_generator.jl:40 doublets, PixelTrackHeterogeneous.jl:55
tuples)."""
import numpy as np
import pytest

from oracle import oracle
from parity import compare_event

pytestmark = pytest.mark.gpu

E = 4


@pytest.fixture(scope="module")
def high_pu():
    from pixeltrack import gen
    blob, offs = gen.events(E, gen.MODE_UNIFORM, pu=260, seed=4242)
    return blob, offs


def _batch(conditions, blob, offs, extended):
    from pixeltrack import PixelChain, batch_params
    params = batch_params(E, words_per_event=160_000, hits_per_event_avg=48_000,
                          doublets_per_event_avg=1_000_000, tuples_per_event_avg=100_000, extended=extended)
    chain = PixelChain(conditions, params)
    chain.stage_batch(blob, offs)
    chain.capture_graph()
    chain.launch_graph()
    return chain, chain.sync()


def test_events_exceed_reference_capacities(conditions, high_pu):
    """The sample really is above the caps: the reference-capacity oracle truncates it."""
    blob, offs = high_pu
    orc = oracle.Oracle(conditions)
    _, cnt = orc.run_batch(blob, offs, 4, counts=True)
    flags = cnt[:, oracle.COUNT_NAMES.index("flags")]
    assert np.count_nonzero(flags & 0x50) >= 2, flags


def test_extended_mode_matches_extended_oracle(conditions, high_pu):
    blob, offs = high_pu
    chain, warn = _batch(conditions, blob, offs, extended=True)
    try:
        assert warn == 0, warn
        orc = oracle.Oracle(conditions, oracle.EXTENDED_CAPS)
        for e in range(E):
            orc.run_event(blob[offs[e]:offs[e + 1]], 63)
            assert orc.counts()["flags"] == 0
            errs = compare_event(chain, orc, e)
            assert not errs, (e, errs)
        # the 16-bit reference-layout hit ids equal the 32-bit ones while ids fit
        for name in ("phi_bins", "tuple_hits"):
            assert np.array_equal(chain.product(name + "16", 0), chain.product(name, 0))
    finally:
        chain.close()


def test_reference_capacities_truncate_like_the_oracle(conditions, high_pu):
    blob, offs = high_pu
    chain, warn = _batch(conditions, blob, offs, extended=False)
    try:
        assert warn & 0x50
        orc = oracle.Oracle(conditions)
        for e in range(E):
            orc.run_event(blob[offs[e]:offs[e + 1]], 63)
            errs = compare_event(chain, orc, e)
            assert not errs, (e, errs)
    finally:
        chain.close()
