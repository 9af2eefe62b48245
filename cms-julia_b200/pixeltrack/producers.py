"""The five event producers and the conditions producers of the reference's
pixel chain, with the same plugin names, tokens and product types, backed by
the CUDA library. Products live on the GPU and are copied out on access.

  BeamSpotToPOD            plugin-BeamSpotProducer/BeamSpotToPOD.jl:4-16
  SiPixelRawToClusterCUDA  plugin-SiPixelClusterizer/SiPixelRawToClusterCUDA.jl:27-152
  SiPixelRecHitCUDA        plugin-SiPixelRecHits/SiPixelRecHitCUDA.jl:8-45
  CAHitNtupletCUDA         plugin-PixelTriplets/ca_hit_ntuplet.jl:1-19
  PixelVertexProducerCUDA  plugin-PixelVertexFinding/pixel_vertex_producer_cuda.jl:3-30
ES producers: BeamSpotESProducer, SiPixelFedCablingMapGPUWrapperESProducer,
SiPixelGainCalibrationForHLTGPUESProducer, PixelCPEFastESProducer.
"""
from __future__ import annotations

import struct
from pathlib import Path

import numpy as np

from . import _native
from .chain import PixelChain, default_params
from .formats import FedRawDataCollection
from .framework import (EDProducer, ESProducer, Event, EventSetup, ProductRegistry, add_plugin,
                        add_plugin_module)

# ----------------------------------------------------------------- conditions products


class _Blob:
    def __init__(self, **blobs: bytes):
        self.blobs = blobs


class SiPixelFedCablingMapGPUWrapper(_Blob):
    pass


class SiPixelFedIds(_Blob):
    @property
    def fed_ids(self) -> np.ndarray:
        b = self.blobs["fedIds.bin"]
        n = struct.unpack_from("<I", b, 0)[0]
        return np.frombuffer(b, dtype=np.uint32, count=n, offset=4)


class SiPixelGainCalibrationForHLTGPU(_Blob):
    pass


class PixelCPEFast(_Blob):
    pass


class BeamSpotPOD:
    FIELDS = ("x", "y", "z", "sigmaZ", "beamWidthX", "beamWidthY", "dxdz", "dydz", "emittanceX", "emittanceY",
              "betaStar")

    def __init__(self, blob: bytes):
        self.blob = blob
        for name, v in zip(self.FIELDS, struct.unpack_from("<11f", blob, 0)):
            setattr(self, name, v)


class GPUContext:
    """One reconstruction context shared by the producers of a stream (the device side of
    all ES products). Created on first use from the ES products."""

    def __init__(self, es: EventSetup, params=None):
        conds = {
            "cablingMap.bin": es.get(SiPixelFedCablingMapGPUWrapper).blobs["cablingMap.bin"],
            "fedIds.bin": es.get(SiPixelFedIds).blobs["fedIds.bin"],
            "gain.bin": es.get(SiPixelGainCalibrationForHLTGPU).blobs["gain.bin"],
            "cpefast.bin": es.get(PixelCPEFast).blobs["cpefast.bin"],
            "beamspot.bin": es.get(BeamSpotPOD).blob,
        }
        self.chain = PixelChain(conds, params if params is not None else default_params())


def gpu_context(es: EventSetup) -> GPUContext:
    if not es.has(GPUContext):
        es.put(GPUContext(es))
    return es.get(GPUContext)


class BeamSpotESProducer(ESProducer):
    def __init__(self, data_dir: str):
        self.data = Path(data_dir)

    def produce(self, es: EventSetup) -> None:
        es.put(BeamSpotPOD((self.data / "beamspot.bin").read_bytes()))


class SiPixelFedCablingMapGPUWrapperESProducer(ESProducer):
    def __init__(self, data_dir: str):
        self.data = Path(data_dir)

    def produce(self, es: EventSetup) -> None:
        es.put(SiPixelFedIds(**{"fedIds.bin": (self.data / "fedIds.bin").read_bytes()}))
        es.put(SiPixelFedCablingMapGPUWrapper(**{"cablingMap.bin": (self.data / "cablingMap.bin").read_bytes()}))


class SiPixelGainCalibrationForHLTGPUESProducer(ESProducer):
    def __init__(self, data_dir: str):
        self.data = Path(data_dir)

    def produce(self, es: EventSetup) -> None:
        es.put(SiPixelGainCalibrationForHLTGPU(**{"gain.bin": (self.data / "gain.bin").read_bytes()}))


class PixelCPEFastESProducer(ESProducer):
    def __init__(self, data_dir: str):
        self.data = Path(data_dir)

    def produce(self, es: EventSetup) -> None:
        es.put(PixelCPEFast(**{"cpefast.bin": (self.data / "cpefast.bin").read_bytes()}))


def eventsetup_from_blobs(conds: dict[str, bytes]) -> EventSetup:
    """An EventSetup holding the conditions products built from in-memory blobs."""
    es = EventSetup()
    es.put(BeamSpotPOD(conds["beamspot.bin"]))
    es.put(SiPixelFedIds(**{"fedIds.bin": conds["fedIds.bin"]}))
    es.put(SiPixelFedCablingMapGPUWrapper(**{"cablingMap.bin": conds["cablingMap.bin"]}))
    es.put(SiPixelGainCalibrationForHLTGPU(**{"gain.bin": conds["gain.bin"]}))
    es.put(PixelCPEFast(**{"cpefast.bin": conds["cpefast.bin"]}))
    return es


# ----------------------------------------------------------------- event products


class _DeviceProduct:
    """Product whose arrays stay on the GPU; attribute access copies them out."""
    ARRAYS: tuple[str, ...] = ()

    def __init__(self, chain: PixelChain, event: int = 0):
        self._chain = chain
        self._event = event
        self._cache: dict[str, np.ndarray] = {}

    def array(self, name: str) -> np.ndarray:
        if name not in self._cache:
            self._cache[name] = self._chain.product(name, self._event)
        return self._cache[name]

    def __getattr__(self, name: str):
        if name in type(self).ARRAYS:
            return self.array(name)
        raise AttributeError(name)


class SiPixelDigisSoA(_DeviceProduct):
    ARRAYS = ("xx", "yy", "adc", "module_ind", "clus", "pdigi", "raw_id_arr")

    @property
    def n_digis(self) -> int:
        return self._chain.counts(self._event).n_words

    @property
    def n_modules(self) -> int:
        return self._chain.counts(self._event).n_modules


class SiPixelDigiErrorsSoA(_DeviceProduct):
    ARRAYS = ("errors",)


class SiPixelClustersSoA(_DeviceProduct):
    ARRAYS = ("module_start", "clus_in_module", "module_id", "clus_module_start")

    @property
    def n_clusters(self) -> int:
        return self._chain.counts(self._event).n_clusters


class TrackingRecHit2DHeterogeneous(_DeviceProduct):
    ARRAYS = ("xl", "yl", "xerr", "yerr", "xg", "yg", "zg", "rg", "iphi", "charge", "xsize", "ysize", "det_ind",
              "hits_layer_start", "phi_off", "phi_bins", "agc")

    @property
    def n_hits(self) -> int:
        return self._chain.counts(self._event).n_hits


class TrackSOA(_DeviceProduct):
    ARRAYS = ("tuple_off", "tuple_hits", "det_hits", "quality", "chi2", "eta", "pt", "state", "cov", "fitted")

    @property
    def n_tuples(self) -> int:
        return self._chain.counts(self._event).n_tuples


class ZVertexSoA(_DeviceProduct):
    ARRAYS = ("idv", "zv", "wv", "vchi2", "ptv2", "ndof", "sort_ind")

    @property
    def nv_final(self) -> int:
        return self._chain.counts(self._event).n_vertices


# ----------------------------------------------------------------- event producers


class BeamSpotToPOD(EDProducer):
    def __init__(self, reg: ProductRegistry):
        self.bs_put = reg.produces(BeamSpotPOD)

    def produce(self, event: Event, es: EventSetup) -> None:
        event.emplace(self.bs_put, es.get(BeamSpotPOD))


class SiPixelRawToClusterCUDA(EDProducer):
    def __init__(self, reg: ProductRegistry):
        self.is_run2 = True
        self.include_errors = True
        self.use_quality = True
        self.raw_get = reg.consumes(FedRawDataCollection)
        self.digi_put = reg.produces(SiPixelDigisSoA)
        self.digi_error_put = reg.produces(SiPixelDigiErrorsSoA)
        self.cluster_put = reg.produces(SiPixelClustersSoA)

    def produce(self, event: Event, es: EventSetup) -> None:
        ctx = gpu_context(es)
        raw = event.get(self.raw_get)
        buf = raw.to_bytes() if isinstance(raw, FedRawDataCollection) else bytes(raw)
        ctx.chain.run_event(buf, _native.STAGE_DIGIS)
        event.emplace(self.digi_put, SiPixelDigisSoA(ctx.chain))
        event.emplace(self.cluster_put, SiPixelClustersSoA(ctx.chain))


class SiPixelRecHitCUDA(EDProducer):
    def __init__(self, reg: ProductRegistry):
        self.bs_get = reg.consumes(BeamSpotPOD)
        self.cluster_get = reg.consumes(SiPixelClustersSoA)
        self.digi_get = reg.consumes(SiPixelDigisSoA)
        self.hit_put = reg.produces(TrackingRecHit2DHeterogeneous)

    def produce(self, event: Event, es: EventSetup) -> None:
        ctx = gpu_context(es)
        event.get(self.cluster_get)
        event.get(self.digi_get)
        ctx.chain.continue_stages(_native.STAGE_HITS)
        event.emplace(self.hit_put, TrackingRecHit2DHeterogeneous(ctx.chain))


class CAHitNtupletCUDA(EDProducer):
    B_FIELD = 0.0114256972711507  # 1/fieldInGeV, ca_hit_ntuplet.jl:11

    def __init__(self, reg: ProductRegistry):
        self.hit_get = reg.consumes(TrackingRecHit2DHeterogeneous)
        self.track_put = reg.produces(TrackSOA)

    def produce(self, event: Event, es: EventSetup) -> None:
        ctx = gpu_context(es)
        event.get(self.hit_get)
        ctx.chain.continue_stages(_native.STAGE_TUPLES | _native.STAGE_FIT | _native.STAGE_CLASSIFY)
        event.emplace(self.track_put, TrackSOA(ctx.chain))


class PixelVertexProducerCUDA(EDProducer):
    def __init__(self, reg: ProductRegistry):
        self.track_get = reg.consumes(TrackSOA)
        self.vertex_put = reg.produces(ZVertexSoA)
        self.pt_min = 0.5

    def produce(self, event: Event, es: EventSetup) -> None:
        ctx = gpu_context(es)
        event.get(self.track_get)
        ctx.chain.continue_stages(_native.STAGE_VERTICES)
        event.emplace(self.vertex_put, ZVertexSoA(ctx.chain))


for _name, _cls in (("BeamSpotToPOD", BeamSpotToPOD), ("SiPixelRawToClusterCUDA", SiPixelRawToClusterCUDA),
                    ("SiPixelRecHitCUDA", SiPixelRecHitCUDA), ("CAHitNtupletCUDA", CAHitNtupletCUDA),
                    ("PixelVertexProducerCUDA", PixelVertexProducerCUDA)):
    add_plugin_module(_name, _cls)
for _name, _cls in (("BeamSpotESProducer", BeamSpotESProducer),
                    ("SiPixelFedCablingMapGPUWrapperESProducer", SiPixelFedCablingMapGPUWrapperESProducer),
                    ("SiPixelGainCalibrationForHLTGPUESProducer", SiPixelGainCalibrationForHLTGPUESProducer),
                    ("PixelCPEFastESProducer", PixelCPEFastESProducer)):
    add_plugin(_name, _cls)

# the reference's path (main.jl:101-117), minus the validator
PATH = ("BeamSpotToPOD", "SiPixelRawToClusterCUDA", "SiPixelRecHitCUDA", "CAHitNtupletCUDA", "PixelVertexProducerCUDA")


class Source(EDProducer):
    """Emplaces the raw FED collection of each event (Framework/Source.jl:52-82)."""

    def __init__(self, reg: ProductRegistry):
        self.raw_put = reg.produces(FedRawDataCollection)


def make_path(reg: ProductRegistry):
    from .framework import create_plugin_module
    return [create_plugin_module(n, reg) for n in PATH]
