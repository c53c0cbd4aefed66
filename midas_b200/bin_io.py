"""Map.bin / nMap.bin I/O (the MIDAS v3 pixel-split map format).

Layout (fixed by FF_HEDM/src/MapHeader.h and FF_HEDM/src/MapperCore.h:19-25, mirrored by
packages/midas_integrate/midas_integrate/bin_io.py):

* optional 64-byte header: u32 magic 0x3050414D ("MAP0"), u32 version 3,
  32-byte SHA-256 parameter hash, u8 q_mode, u8 gradient_mode, 6 pad bytes,
  f64 wavelength, 8 reserved bytes;
* Map.bin: 24-byte records {f32 y, f32 z, f64 frac, f32 deltaR, f32 areaWeight};
* nMap.bin: one {i32 count, i32 offset} pair per (R, eta) bin, offset in records.

The header is auto-detected by its magic; its hash is not validated (the GPU
stream reader prints it and moves on, IntegratorFitPeaksGPUStream.cu:757-766).
"""
from __future__ import annotations

import hashlib
import struct
from dataclasses import dataclass
from pathlib import Path
from typing import Optional, Sequence

import numpy as np

MAP_HEADER_MAGIC = 0x3050414D
MAP_HEADER_VERSION = 3
MAP_HEADER_SIZE = 64

PXLIST_DTYPE = np.dtype([("y", "<f4"), ("z", "<f4"), ("frac", "<f8"),
                         ("deltaR", "<f4"), ("areaWeight", "<f4")])
NMAP_DTYPE = np.dtype([("count", "<i4"), ("offset", "<i4")])
assert PXLIST_DTYPE.itemsize == 24 and NMAP_DTYPE.itemsize == 8


@dataclass
class MapHeader:
    magic: int = MAP_HEADER_MAGIC
    version: int = MAP_HEADER_VERSION
    param_hash: bytes = b"\x00" * 32
    q_mode: int = 0
    gradient_mode: int = 0
    wavelength: float = 0.0

    def to_bytes(self) -> bytes:
        if len(self.param_hash) != 32:
            raise ValueError("param_hash must be 32 bytes")
        b = bytearray(MAP_HEADER_SIZE)
        struct.pack_into("<II", b, 0, self.magic, self.version)
        b[8:40] = self.param_hash
        b[40] = self.q_mode & 0xFF
        b[41] = self.gradient_mode & 0xFF
        struct.pack_into("<d", b, 48, self.wavelength)
        return bytes(b)

    @classmethod
    def from_bytes(cls, raw: bytes) -> Optional["MapHeader"]:
        if len(raw) < MAP_HEADER_SIZE:
            return None
        magic, version = struct.unpack_from("<II", raw, 0)
        if magic != MAP_HEADER_MAGIC:
            return None
        return cls(magic, version, bytes(raw[8:40]), raw[40], raw[41],
                   struct.unpack_from("<d", raw, 48)[0])


def compute_param_hash(**kw) -> bytes:
    """SHA-256 over an alphabetised ``key=value`` string of the geometry/binning keys
    (the cache-invalidation hash of bin_io.compute_param_hash: all 15 distortion
    terms, Parallax and Wavelength included)."""
    keys_float6 = ["EtaBinSize", "EtaMax", "EtaMin", "Lsd", "Parallax", "RBinSize", "RMax",
                   "RMin", "RhoD"]
    trans = list(kw.get("TransOpt", ()))
    parts = [f"BC={kw['Ycen']:.6f},{kw['Zcen']:.6f}"]
    for k in ["EtaBinSize", "EtaMax", "EtaMin", "Lsd"]:
        parts.append(f"{k}={float(kw.get(k, 0.0)):.6f}")
    parts.append(f"NrPixelsY={int(kw['NrPixelsY'])}")
    parts.append(f"NrPixelsZ={int(kw['NrPixelsZ'])}")
    for k in ["Parallax", "RBinSize", "RMax", "RMin", "RhoD"]:
        parts.append(f"{k}={float(kw.get(k, 0.0)):.6f}")
    parts.append(f"TransOpt={len(trans)}")
    parts.append(f"Wavelength={float(kw.get('Wavelength', 0.0)):.8f}")
    head = "|".join(parts) + "".join(f",{int(t)}" for t in trans[:10])
    tail = [f"p{i}={float(kw.get(f'p{i}', 0.0)):.6f}" for i in range(15)]
    tail += [f"pxY={float(kw['pxY']):.6f}", f"pxZ={float(kw.get('pxZ', kw['pxY'])):.6f}",
             f"tx={float(kw.get('tx', 0.0)):.6f}", f"ty={float(kw.get('ty', 0.0)):.6f}",
             f"tz={float(kw.get('tz', 0.0)):.6f}"]
    full = head + "|" + "|".join(tail)
    if kw.get("qMode", 0):
        full += "|qMode=1"
    del keys_float6
    return hashlib.sha256(full.encode("ascii")).digest()


@dataclass
class PixelMap:
    """A Map.bin / nMap.bin pair held in memory."""
    pxList: np.ndarray          # PXLIST_DTYPE records
    counts: np.ndarray          # int32 per bin
    offsets: np.ndarray         # int32 per bin
    map_header: Optional[MapHeader] = None
    nmap_header: Optional[MapHeader] = None

    @property
    def n_bins(self) -> int:
        return int(self.counts.shape[0])

    @property
    def n_entries(self) -> int:
        return int(self.pxList.shape[0])

    def nmap_pairs(self) -> np.ndarray:
        """Contiguous int32 [n_bins, 2] array of (count, offset)."""
        out = np.empty((self.n_bins, 2), dtype=np.int32)
        out[:, 0] = self.counts
        out[:, 1] = self.offsets
        return out


def _split(raw: np.ndarray):
    hdr = MapHeader.from_bytes(bytes(raw[:MAP_HEADER_SIZE]))
    return hdr, raw[MAP_HEADER_SIZE:] if hdr is not None else raw


def load_map(map_path, nmap_path) -> PixelMap:
    """Read Map.bin and nMap.bin (memory-mapped), auto-detecting the header."""
    m = np.memmap(map_path, mode="r", dtype=np.uint8)
    mh, mbody = _split(m)
    if mbody.nbytes % PXLIST_DTYPE.itemsize:
        raise ValueError(f"Map.bin payload of {mbody.nbytes} bytes is not a whole number of "
                         f"24-byte records (legacy 16-byte map?)")
    px = mbody.view(PXLIST_DTYPE)
    n = np.memmap(nmap_path, mode="r", dtype=np.uint8)
    nh, nbody = _split(n)
    if nbody.nbytes % NMAP_DTYPE.itemsize:
        raise ValueError("nMap.bin payload is not a whole number of (count, offset) pairs")
    pairs = nbody.view(NMAP_DTYPE)
    return PixelMap(px, np.array(pairs["count"], dtype=np.int32),
                    np.array(pairs["offset"], dtype=np.int32), mh, nh)


def write_map(map_path, nmap_path, *, pxList, counts, offsets,
              header: Optional[MapHeader] = None) -> None:
    """Write Map.bin / nMap.bin; with a header, the same 64 bytes go before both files."""
    px = np.ascontiguousarray(pxList, dtype=PXLIST_DTYPE)
    counts = np.asarray(counts, dtype=np.int32)
    offsets = np.asarray(offsets, dtype=np.int32)
    if counts.shape != offsets.shape or counts.ndim != 1:
        raise ValueError("counts and offsets must be 1-D arrays of equal length")
    pairs = np.empty(counts.shape[0], dtype=NMAP_DTYPE)
    pairs["count"] = counts
    pairs["offset"] = offsets
    hb = header.to_bytes() if header is not None else b""
    with open(map_path, "wb") as f:
        f.write(hb)
        f.write(px.tobytes())
    with open(nmap_path, "wb") as f:
        f.write(hb)
        f.write(pairs.tobytes())


def pack_records(records: Sequence[tuple], bin_lists: Sequence[Sequence[int]]) -> PixelMap:
    """Build a PixelMap from (y, z, frac, deltaR, areaWeight) tuples and per-bin index lists
    (each bin's records become one contiguous slab)."""
    counts = np.array([len(b) for b in bin_lists], dtype=np.int32)
    offsets = np.zeros_like(counts)
    if len(counts) > 1:
        offsets[1:] = np.cumsum(counts[:-1])
    flat = [records[i] for b in bin_lists for i in b]
    px = np.array(flat, dtype=PXLIST_DTYPE) if flat else np.empty(0, dtype=PXLIST_DTYPE)
    return PixelMap(px, counts, offsets)


def from_arrays(records: np.ndarray, nmap: np.ndarray) -> PixelMap:
    """PixelMap from a record array and an int32 [n_bins, 2] (count, offset) array."""
    nmap = np.asarray(nmap, dtype=np.int32).reshape(-1, 2)
    return PixelMap(np.ascontiguousarray(records, dtype=PXLIST_DTYPE),
                    np.ascontiguousarray(nmap[:, 0]), np.ascontiguousarray(nmap[:, 1]))
