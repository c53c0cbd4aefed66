"""Fused multi-shift caking: build_fused_geometry of the reference
(packages/midas_integrate/midas_integrate/fused_csr.py:139-296) as one device plan.

The reference's Family II aliasing mitigation averages the cakes of ``n_shifts`` maps
whose R edges are shifted by k / n_shifts of a bin, each normalised by its own bin areas
and interpolated linearly in R onto the unshifted axis, and folds that average into one
sparse matrix (M = 1/N sum_k P_k D_k M_k) so that a frame costs one pass.  Here the
same matrix is built on the host by ``mi_plan_create_fused`` / ``mi_fused_csr`` and
tiled like any other map: ``FusedPlan`` cakes F frames per launch on any encoding, with
the dark subtracted and both lineouts reduced in the same launch.  The fused plan's bin
areas are all 1 (the normalisation is in the weights), so ``normalize`` changes nothing
-- as for the reference's fused geometry, whose ``area_per_bin`` is ones.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import replace
from typing import List, Optional, Sequence, Tuple

import numpy as np
import torch

from . import _lib as L
from .bin_io import PixelMap
from .kernels import CakePlan, _device_index, r_axis
from .mapper import MapperParams, build_map


def shifted_params(p: MapperParams, k: int, n_shifts: int) -> MapperParams:
    """Shift k of n: RMin + k / n x RBinSize (fused_csr.py:199-201; R binning only)."""
    if p.q_mode:
        raise ValueError("fused maps shift R bin edges; Q binning is not shifted by the reference")
    return replace(p, RMin=p.RMin + p.RBinSize * k / n_shifts)


def shift_maps(p: MapperParams, n_shifts: int, *, device: int = 0, mask: Optional[np.ndarray] = None
               ) -> Tuple[List[PixelMap], List[np.ndarray]]:
    """The n shifted maps (DetectorMapper, on ``device``; -1 = host) and their R axes."""
    if n_shifts < 1:
        raise ValueError(f"n_shifts must be >= 1; got {n_shifts}")
    if p.RBinSize <= 0:
        raise ValueError(f"RBinSize must be > 0; got {p.RBinSize}")
    maps, axes = [], []
    for k in range(n_shifts):
        pk = shifted_params(p, k, n_shifts)
        pm, _ = build_map(pk, device=device, mask=mask)
        maps.append(pm)
        axes.append(r_axis(n_r=pk.n_r, RMin=pk.RMin, RBinSize=pk.RBinSize))
    return maps, axes


def _descs(pixmaps: Sequence[PixelMap], r_axes, n_eta: int, ny: int, nz: int, bc_y: float, bc_z: float):
    n = len(pixmaps)
    if n == 0 or len(r_axes) != n:
        raise ValueError("one R axis per shifted map is needed")
    descs = (L.MiMapDesc * n)()
    axes = (C.c_void_p * n)()
    keep = []
    for k, (pm, ax) in enumerate(zip(pixmaps, r_axes)):
        a = np.ascontiguousarray(ax, dtype=np.float64)
        if pm.n_bins != a.size * n_eta:
            raise ValueError(f"shift {k}: PixelMap has {pm.n_bins} bins; R axis {a.size} x n_eta {n_eta}")
        recs = np.ascontiguousarray(pm.pxList)
        nmap = np.ascontiguousarray(pm.nmap_pairs())
        keep += [recs, nmap, a]
        descs[k] = L.MiMapDesc(recs.ctypes.data if recs.size else None, recs.shape[0], nmap.ctypes.data,
                               a.size, n_eta, ny, nz, float(bc_y), float(bc_z))
        axes[k] = a.ctypes.data
    return descs, axes, keep


def fused_csr(pixmaps: Sequence[PixelMap], r_axes, *, n_eta: int, n_pixels_y: int, n_pixels_z: int,
              mode: str = "gradient", bc_y: float = 0.0, bc_z: float = 0.0):
    """The fused weights on the host (no device): (row_ptr int64 [n_bins + 1], col int32,
    w float64), bins on shift 0's R axis, flat pixel = z * NY + y."""
    if mode not in ("bilinear", "gradient"):
        raise ValueError(f"mode must be 'bilinear' or 'gradient'; got {mode!r}")
    descs, axes, keep = _descs(pixmaps, r_axes, n_eta, n_pixels_y, n_pixels_z, bc_y, bc_z)
    n = len(pixmaps)
    nnz = C.c_int64(0)
    lib = L.lib()
    L.check(lib.mi_fused_csr(descs, n, axes, L.MODE[mode], None, None, None, 0, C.byref(nnz)), "mi_fused_csr")
    n_bins = np.asarray(r_axes[0]).size * n_eta
    row_ptr = np.zeros(n_bins + 1, np.int64)
    col = np.zeros(max(nnz.value, 1), np.int32)
    w = np.zeros(max(nnz.value, 1), np.float64)
    L.check(lib.mi_fused_csr(descs, n, axes, L.MODE[mode], row_ptr.ctypes.data, col.ctypes.data, w.ctypes.data,
                             col.size, C.byref(nnz)), "mi_fused_csr")
    del keep
    return row_ptr, col[:nnz.value], w[:nnz.value]


class FusedPlan(CakePlan):
    """A device plan of the fused multi-shift map (py semantics; bilinear or gradient).

    Args:
        pixmaps: the shifted maps (shift 0 first), r_axes: their R bin centres.
        n_eta, n_pixels_y, n_pixels_z, bc_y, bc_z, device, encoding, tile_rows, tile_pixels,
            run_len, host_threads: as for ``CakePlan``.
    The cake is on shift 0's R axis (n_r = len(r_axes[0])).
    """

    def __init__(self, pixmaps: Sequence[PixelMap], r_axes, *, n_eta: int, n_pixels_y: int, n_pixels_z: int,
                 mode: str = "gradient", bc_y: float = 0.0, bc_z: float = 0.0, device="cuda",
                 encoding: str = "auto", tile_rows: int = 0, tile_pixels: int = 0, run_len: int = 0,
                 host_threads: int = 0):
        if mode not in ("bilinear", "gradient"):
            raise ValueError(f"mode must be 'bilinear' or 'gradient'; got {mode!r}")
        if encoding not in L.ENC:
            raise ValueError(f"unknown encoding {encoding!r}")
        self.device = torch.device("cuda", _device_index(device))
        self.n_r, self.n_eta = int(np.asarray(r_axes[0]).size), int(n_eta)
        self.ny, self.nz = int(n_pixels_y), int(n_pixels_z)
        self.mode, self.normalize, self.semantics = mode, True, "py"
        self.bc_y, self.bc_z = float(bc_y), float(bc_z)
        self.variance = False
        self.n_shifts = len(pixmaps)
        self.r_axis = np.ascontiguousarray(r_axes[0], dtype=np.float64)
        descs, axes, keep = _descs(pixmaps, r_axes, self.n_eta, self.ny, self.nz, self.bc_y, self.bc_z)
        opts = L.MiPlanOpts(L.MODE[mode], 1, L.SEM["py"], int(tile_rows), int(tile_pixels), 0, L.ENC[encoding],
                            int(run_len), 0, int(host_threads))
        h = C.c_void_p()
        L.check(L.lib().mi_plan_create_fused(descs, len(pixmaps), axes, C.byref(opts), self.device.index,
                                             C.byref(h)), "mi_plan_create_fused")
        del keep
        self._h = h
        self._dark = None


def build_fused_plan(params: MapperParams, *, n_shifts: int = 4, mode: str = "gradient", device=0,
                     mask: Optional[np.ndarray] = None, **plan_kw) -> FusedPlan:
    """build_fused_geometry(params, n_shifts, mode) as a device plan: the shifted maps are
    built by the device DetectorMapper, folded on the host, tiled for ``device``."""
    dev = _device_index(device if not isinstance(device, int) else f"cuda:{device}")
    maps, axes = shift_maps(params, n_shifts, device=dev, mask=mask)
    return FusedPlan(maps, axes, n_eta=params.n_eta, n_pixels_y=params.NrPixelsY, n_pixels_z=params.NrPixelsZ,
                     mode=mode, bc_y=params.BC_y, bc_z=params.BC_z, device=f"cuda:{dev}", **plan_kw)
