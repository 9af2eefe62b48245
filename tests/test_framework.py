"""Host-side producer boundary and formats (no GPU)."""
import numpy as np
import pytest

from pixeltrack import framework, producers
from pixeltrack.formats import FedRawDataCollection, split_events


def test_registry_rules():
    reg = framework.ProductRegistry()
    t1 = reg.produces(FedRawDataCollection)
    with pytest.raises(ValueError):
        reg.produces(FedRawDataCollection)
    with pytest.raises(ValueError):
        reg.consumes(producers.TrackSOA)
    g = reg.consumes(FedRawDataCollection)
    assert g.index == t1.index


def test_plugin_names_match_reference():
    ed, es = framework.plugin_names()
    for n in ("BeamSpotToPOD", "SiPixelRawToClusterCUDA", "SiPixelRecHitCUDA", "CAHitNtupletCUDA",
              "PixelVertexProducerCUDA"):
        assert n in ed
    for n in ("BeamSpotESProducer", "SiPixelFedCablingMapGPUWrapperESProducer",
              "SiPixelGainCalibrationForHLTGPUESProducer", "PixelCPEFastESProducer"):
        assert n in es


def test_path_tokens_chain():
    reg = framework.ProductRegistry()
    producers.Source(reg)
    path = producers.make_path(reg)
    assert [type(p).__name__ for p in path] == list(producers.PATH)


def test_raw_roundtrip(events_pu50):
    blob, offs = events_pu50
    b = bytes(blob)
    assert np.array_equal(split_events(b), offs)
    ev = b[offs[0]:offs[1]]
    c = FedRawDataCollection.from_bytes(ev)
    assert c.to_bytes() == ev
    assert all(1200 <= f < 1350 for f in c.feds)


def test_conditions_roundtrip(tmp_path, conditions):
    from pixeltrack.formats import read_conditions, write_conditions
    write_conditions(tmp_path, conditions)
    assert read_conditions(tmp_path) == conditions
    es = framework.EventSetup()
    for cls in (producers.BeamSpotESProducer, producers.SiPixelFedCablingMapGPUWrapperESProducer,
                producers.SiPixelGainCalibrationForHLTGPUESProducer, producers.PixelCPEFastESProducer):
        cls(str(tmp_path)).produce(es)
    assert es.get(producers.SiPixelFedIds).fed_ids[0] == 1200
    assert abs(es.get(producers.BeamSpotPOD).z - 0.3) < 1e-6


def test_count_files_roundtrip(tmp_path, conditions, events_pu50):
    """The count files (digicluster.bin, tracks.bin, vertices.bin, read as ReadRAW.jl:47-59 reads
    them) written from the oracle's counts of the events read back record by record."""
    import pytest
    from oracle import oracle
    from pixeltrack.formats import read_counts, write_counts
    blob, offs = events_pu50
    _, cnt = oracle.Oracle(conditions).run_batch(blob, offs, 2, counts=True)
    ix = [oracle.COUNT_NAMES.index(k) for k in ("n_modules", "n_words", "n_clusters", "n_tracks", "nv_final")]
    counts = cnt[:, ix]
    write_counts(tmp_path, counts)
    assert (tmp_path / "digicluster.bin").stat().st_size == 12 * len(counts)
    assert (tmp_path / "tracks.bin").stat().st_size == 4 * len(counts)
    assert np.array_equal(read_counts(tmp_path), counts)
    assert np.all(counts[:, 3] > 0) and np.all(counts[:, 4] > 0)
    (tmp_path / "vertices.bin").write_bytes(b"\0" * 4)
    with pytest.raises(ValueError):
        read_counts(tmp_path)
