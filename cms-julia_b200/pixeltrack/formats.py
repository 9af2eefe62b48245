"""The reference's on-disk formats and the raw event container.

raw.bin    per event: int32 nFeds, then per FED int32 fedId, int32 size, size bytes
           (bin/ReadRAW.jl:9-31)
Conditions: cablingMap.bin, fedIds.bin, gain.bin, cpefast.bin, beamspot.bin, read
           as opaque blobs (their layouts are parsed by the native library).
Counts:    digicluster.bin (3 x u32 per event), tracks.bin, vertices.bin (u32 per event)
           (ReadRAW.jl:47-59)
"""
from __future__ import annotations

import struct
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

CONDITION_FILES = ("cablingMap.bin", "fedIds.bin", "gain.bin", "cpefast.bin", "beamspot.bin")


@dataclass
class FedRawData:
    """FedRawData (DataFormats/data_formats.jl:41-60): one FED's bytes."""
    fedid: int
    data: bytes


@dataclass
class FedRawDataCollection:
    """FedRawDataCollection (DataFormats/data_formats.jl:62-121), indexed by FED id."""
    feds: dict[int, FedRawData] = field(default_factory=dict)

    def fed_data(self, fedid: int) -> FedRawData:
        return self.feds.get(fedid, FedRawData(fedid, b""))

    def to_bytes(self) -> bytes:
        out = [struct.pack("<i", len(self.feds))]
        for fid, fd in self.feds.items():
            out.append(struct.pack("<ii", fid, len(fd.data)))
            out.append(fd.data)
        return b"".join(out)

    @staticmethod
    def from_bytes(buf: bytes) -> "FedRawDataCollection":
        n = struct.unpack_from("<i", buf, 0)[0]
        p = 4
        c = FedRawDataCollection()
        for _ in range(n):
            fid, size = struct.unpack_from("<ii", buf, p)
            p += 8
            c.feds[fid] = FedRawData(fid, bytes(buf[p:p + size]))  # a repeated id keeps the last (ReadRAW.jl:28)
            p += size
        return c


def split_events(blob: bytes | np.ndarray) -> np.ndarray:
    """Event byte offsets (n_events + 1) of a raw.bin stream, walking the FED records
    as readevent does (ReadRAW.jl:23-31)."""
    b = memoryview(bytes(blob) if isinstance(blob, np.ndarray) else blob)
    offs = [0]
    p = 0
    n = len(b)
    while p < n:
        nfeds = struct.unpack_from("<i", b, p)[0]
        p += 4
        for _ in range(nfeds):
            _fid, size = struct.unpack_from("<ii", b, p)
            p += 8 + size
        offs.append(p)
    return np.asarray(offs, dtype=np.uint64)


def read_raw(path: str | Path) -> tuple[bytes, np.ndarray]:
    blob = Path(path).read_bytes()
    return blob, split_events(blob)


def write_raw(path: str | Path, blob: bytes) -> None:
    Path(path).write_bytes(blob)


def read_conditions(data_dir: str | Path) -> dict[str, bytes]:
    d = Path(data_dir)
    return {name: (d / name).read_bytes() for name in CONDITION_FILES}


def write_conditions(data_dir: str | Path, conds: dict[str, bytes]) -> None:
    d = Path(data_dir)
    d.mkdir(parents=True, exist_ok=True)
    for name in CONDITION_FILES:
        (d / name).write_bytes(conds[name])


COUNT_FILES = ("digicluster.bin", "tracks.bin", "vertices.bin")


def read_counts(data_dir: str | Path) -> np.ndarray:
    """Validation counts (the CountValidator's inputs, read as ReadRAW.jl:47-59 reads them, one
    record per event in event order): (n_events, 5) uint32 = nModules, nDigis, nClusters (from
    digicluster.bin), nTracks (tracks.bin), nVertices (vertices.bin)."""
    d = Path(data_dir)
    dc = np.fromfile(d / "digicluster.bin", dtype="<u4").reshape(-1, 3)
    tr = np.fromfile(d / "tracks.bin", dtype="<u4")
    vx = np.fromfile(d / "vertices.bin", dtype="<u4")
    if not (len(dc) == len(tr) == len(vx)):
        raise ValueError(f"count files disagree on the event count: {len(dc)}, {len(tr)}, {len(vx)}")
    return np.column_stack([dc, tr, vx]).astype(np.uint32)


def write_counts(data_dir: str | Path, counts: np.ndarray) -> None:
    """Writes the three count files for (n_events, 5) counts (the read_counts layout)."""
    d = Path(data_dir)
    d.mkdir(parents=True, exist_ok=True)
    c = np.ascontiguousarray(counts, dtype="<u4").reshape(-1, 5)
    np.ascontiguousarray(c[:, :3]).tofile(d / "digicluster.bin")
    np.ascontiguousarray(c[:, 3]).tofile(d / "tracks.bin")
    np.ascontiguousarray(c[:, 4]).tofile(d / "vertices.bin")
