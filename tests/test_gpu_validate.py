"""The CountValidator (count_to_validator.jl:18-84) on the device over a batch: counts taken
from the oracle and written to the reference's count files validate every event; counts off by
more than the reference's tolerances fail with the check that failed, and a track count within
the 1.2 % tolerance passes."""
import numpy as np
import pytest

from oracle import oracle

pytestmark = pytest.mark.gpu

E = 4


def test_validator_on_batch(tmp_path, conditions, events_pu50):
    from pixeltrack import PixelChain, batch_params
    from pixeltrack.formats import read_counts, write_counts
    blob, offs = events_pu50
    _, cnt = oracle.Oracle(conditions).run_batch(blob, offs, 4, counts=True)
    ix = [oracle.COUNT_NAMES.index(k) for k in ("n_modules", "n_words", "n_clusters", "n_tracks", "nv_final")]
    write_counts(tmp_path, cnt[:, ix])
    expected = read_counts(tmp_path)
    with PixelChain(conditions, batch_params(E, words_per_event=90_000)) as chain:
        chain.run_batch(blob, offs)
        good, st = chain.validate_counts(expected)
        assert good == E and np.all(st & 0xFF == 0)
        assert np.array_equal(st >> 8, expected[:, 3])
        bad = expected.copy()
        bad[0, 1] += 1                                        # digis
        bad[1, 3] = int(bad[1, 3] * 1.05)                     # tracks 5 % off
        bad[2, 4] += 1                                        # vertices
        bad[3, 3] = int(bad[3, 3] * 1.005)                    # tracks 0.5 % off: within tolerance
        good, st = chain.validate_counts(bad)
        assert good == 1
        assert (st[0] & 0xFF) == 2 and (st[1] & 0xFF) == 8 and (st[2] & 0xFF) == 16 and (st[3] & 0xFF) == 0
