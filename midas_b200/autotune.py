"""Autotuner of the batched caking plan: picks the encoding, tile shape and register-run
length for a map by timing candidate plans on the device.

The knobs (all plan options of ``CakePlan``):
  encoding     'mmad' (tensor cores, frames read in place), 'mma' (tensor cores, frames
               transposed into byte planes first), 'runs' (CUDA cores); the tensor-core
               encodings are candidates for 8/16-bit frames only, and their tiles (12 R rows x
               4 eta columns, 128 frames a pass) are fixed by the kernels (24 x 2 tiles, which
               stage fewer pixels twice, measured slower);
  pipeline     'mma' only: the kernel's stage slots and producer warps (CakePlan.MMA_PIPELINES),
               timed on the one plan without rebuilding it;
  tile_rows    R rows per strip (8 or 16): the register block of a consumer warp (bins per
               warp along R) and, with the pixel cap, the tile shape;
  run_len      rows per run record (2, 4, 8; 0 = the plan's own choice from the map's run
               statistics): bins one staged value feeds;
  tile_pixels  staged pixels per tile at most (0 = as many as shared memory holds): the
               tile's footprint on the detector, hence its number of eta columns.
Frames per lane (two u16 frames per 32-bit word, 64 per group) are fixed by the kernel.

``tune`` builds each candidate plan, cakes the given sample batch ``reps`` times after a
warm-up, and keeps the fastest; results are cached per (map, detector, binning, mode,
semantics, batch size) in memory and, when ``cache_path`` is given, in a JSON file.
"""
from __future__ import annotations

import hashlib
import json
from dataclasses import asdict, dataclass, field
from pathlib import Path
from typing import Dict, List, Optional, Sequence

import numpy as np
import torch

from . import _lib as L
from .kernels import CakePlan

TENSOR_CANDIDATES = [
    {"encoding": "mmad", "tile_rows": 0, "run_len": 0, "tile_pixels": 0},
    {"encoding": "mma", "tile_rows": 0, "run_len": 0, "tile_pixels": 0},
]
DEFAULT_CANDIDATES = [
    {"tile_rows": 16, "run_len": 0, "tile_pixels": 0},
    {"tile_rows": 16, "run_len": 4, "tile_pixels": 0},
    {"tile_rows": 16, "run_len": 8, "tile_pixels": 320},
    {"tile_rows": 8, "run_len": 0, "tile_pixels": 0},
    {"tile_rows": 8, "run_len": 4, "tile_pixels": 0},
]


@dataclass
class TuneResult:
    best: Dict[str, int]
    best_ms: float
    table: List[dict] = field(default_factory=list)
    key: str = ""


_CACHE: Dict[str, TuneResult] = {}


def map_key(pixmap, *, n_r, n_eta, n_pixels_y, n_pixels_z, mode, semantics, batch) -> str:
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(pixmap.counts).tobytes())
    h.update(np.ascontiguousarray(pixmap.pxList[:: max(1, pixmap.n_entries // 4096)]).tobytes())
    h.update(json.dumps([n_r, n_eta, n_pixels_y, n_pixels_z, mode, semantics, batch]).encode())
    return h.hexdigest()[:24]


def tune(pixmap, frames: torch.Tensor, *, n_r: int, n_eta: int, n_pixels_y: int, n_pixels_z: int,
         mode: str = "floor", semantics: str = "py", bc_y: float = 0.0, bc_z: float = 0.0, dark=None,
         candidates: Optional[Sequence[dict]] = None, reps: int = 3, device="cuda",
         cache_path: Optional[str] = None) -> TuneResult:
    """Time the candidate plans on ``frames`` (a device batch like the ones to be caked) and
    return the fastest configuration with the whole table."""
    F = frames.shape[0]
    key = map_key(pixmap, n_r=n_r, n_eta=n_eta, n_pixels_y=n_pixels_y, n_pixels_z=n_pixels_z, mode=mode,
                  semantics=semantics, batch=F)
    if key in _CACHE:
        return _CACHE[key]
    if cache_path and Path(cache_path).exists():
        saved = json.loads(Path(cache_path).read_text()).get(key)
        if saved:
            _CACHE[key] = TuneResult(**saved)
            return _CACHE[key]
    table = []
    stream = torch.cuda.current_stream()
    if candidates is None:
        candidates = list(DEFAULT_CANDIDATES)
        if frames.dtype in (torch.uint8, torch.uint16):
            candidates = TENSOR_CANDIDATES + candidates
    for cand in candidates:
        row = dict(cand)
        try:
            plan = CakePlan(pixmap, n_r=n_r, n_eta=n_eta, n_pixels_y=n_pixels_y, n_pixels_z=n_pixels_z, mode=mode,
                            semantics=semantics, bc_y=bc_y, bc_z=bc_z, device=device, **cand)
        except L.MidasError as e:
            row["error"] = str(e)
            table.append(row)
            continue
        if dark is not None:
            plan.set_dark(dark)
        ck, aw, sm = plan.integrate(frames)           # warm-up, buffers
        bufs = {"cake": ck, "lineout_aw": aw, "lineout_sm": sm}
        info = plan.info
        pipes = CakePlan.MMA_PIPELINES if cand.get("encoding") == "mma" and "pipeline" not in cand else [None]
        for pipe in pipes:
            r2 = dict(row)
            if pipe is not None:
                plan.set_mma_pipeline(*pipe)
                plan.integrate(frames, out=bufs)       # the variant's first launch
                r2["pipeline"] = list(pipe)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(reps):
                plan.integrate(frames, out=bufs)
            e1.record(stream)
            torch.cuda.synchronize()
            r2.update(ms=round(e0.elapsed_time(e1) / reps, 4), tiles=info["n_tiles"], run_len_used=info["run_len"],
                      tile_pixels_used=info["tile_pixels"], map_bytes=info["map_bytes"])
            table.append(r2)
        plan.close()
        del ck, aw, sm, bufs
    ok = [r for r in table if "ms" in r]
    if not ok:
        raise RuntimeError(f"no candidate plan could be built: {table}")
    best = min(ok, key=lambda r: r["ms"])
    res = TuneResult({k: best.get(k, "runs" if k == "encoding" else 0)
                      for k in ("encoding", "tile_rows", "run_len", "tile_pixels", "pipeline")}, best["ms"], table, key)
    _CACHE[key] = res
    if cache_path:
        p = Path(cache_path)
        data = json.loads(p.read_text()) if p.exists() else {}
        data[key] = asdict(res)
        p.write_text(json.dumps(data, indent=1))
    return res
