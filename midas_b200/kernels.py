"""Caking on the B200 through libmidas_b200 -- the midas_integrate kernels API.

Mirrors packages/midas_integrate/midas_integrate/kernels.py (``build_csr``,
``integrate``, ``profile_1d``, ``AREA_THRESHOLD``, ``r_axis``, ``eta_axis``) so
a caller of the reference can switch imports; ``CakePlan`` is the native,
batched interface underneath (F frames per launch, dark subtraction fused,
lineouts reduced in the same launch).

Every computation runs in the CUDA library; torch tensors are only buffers
(device pointers and the current stream).  There is no CPU path: a plan needs a
CUDA device and raises otherwise.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Dict, Optional, Tuple

import numpy as np
import torch

from . import _lib as L
from .bin_io import PixelMap

AREA_THRESHOLD = 1e-9

_TORCH_DT = {
    torch.uint8: L.DT_U8, torch.uint16: L.DT_U16, torch.uint32: L.DT_U32,
    torch.int64: L.DT_I64, torch.float32: L.DT_F32, torch.float64: L.DT_F64,
    torch.int32: L.DT_I32,
}


def dtype_code(t: torch.dtype) -> int:
    if t not in _TORCH_DT:
        raise TypeError(f"unsupported frame dtype {t}")
    return _TORCH_DT[t]


def _device_index(device) -> int:
    d = torch.device(device)
    if d.type != "cuda":
        raise RuntimeError("midas_b200 runs on CUDA devices only (got device %r)" % (device,))
    if not torch.cuda.is_available():
        raise RuntimeError("midas_b200 needs a CUDA device; none is available")
    return d.index if d.index is not None else torch.cuda.current_device()


class CakePlan:
    """Device-resident caking plan for one (map, binning, mode, normalisation).

    Args:
        pixmap: the Map.bin / nMap.bin pair (``bin_io.PixelMap``).
        n_r, n_eta: bin grid; bins are R-major.
        n_pixels_y, n_pixels_z: detector shape; flat pixel = z * NY + y.
        mode: 'floor' | 'bilinear' | 'gradient'.
        normalize: divide by the bin area (Normalize key).
        semantics: 'py' (midas_integrate kernels.py), 'gpustream'
            (IntegratorFitPeaksGPUStream normaliser and fp32 resampling), 'ic'
            (IntegrationCore.c integration_apply_map: bilinear/gradient only) or 'omp'
            (IntegratorZarrOMP.c: the 'ic' sums, a nonzero sum divided by the bin's whole
            area, masked bins NaN (``set_bin_mask``), the lineouts computed from the cake:
            lineout_sm = mean of the row's nonzero, non-NaN bins).
        bc_y, bc_z: beam centre (px), used by gradient mode.
        device: CUDA device.
        tile_rows, tile_pixels, frames_per_lane: tiling knobs (0 = default).
        encoding: 'auto' (= 'runs') | 'runs' (register-blocked radial runs) | 'csr'
            (per-bin term lists) | 'mma' (tensor cores, exact int8 products; 8/16-bit
            frames only) | 'mmad' (tensor cores reading the frames in place, 8/16-bit
            frames); run_len: rows per run record (2, 4, 8; 0 = auto).
        variance: a variance plan (integrate_with_variance, kernels.py:474-536): frames
            are per-pixel variance maps, caked with the squared coalesced weights and
            divided by the squared bin area; its lineouts are the propagated variances of
            profile_1d_with_variance (kernels.py:604-645).
        host_threads: host threads that build the plan (0 = all cores).
    """

    def __init__(self, pixmap: PixelMap, *, n_r: int, n_eta: int, n_pixels_y: int,
                 n_pixels_z: int, mode: str = "floor", normalize: bool = True,
                 semantics: str = "py", bc_y: float = 0.0, bc_z: float = 0.0,
                 device="cuda", tile_rows: int = 0, tile_pixels: int = 0,
                 frames_per_lane: int = 0, encoding: str = "auto", run_len: int = 0,
                 variance: bool = False, host_threads: int = 0):
        if pixmap.n_bins != n_r * n_eta:
            raise ValueError(f"PixelMap has {pixmap.n_bins} bins; n_r * n_eta = {n_r * n_eta}")
        if mode not in L.MODE:
            raise ValueError(f"unknown integration mode {mode!r}; expected 'floor' | 'bilinear' | 'gradient'")
        if semantics not in L.SEM:
            raise ValueError(f"unknown semantics {semantics!r}")
        self.device = torch.device("cuda", _device_index(device))
        self.n_r, self.n_eta = int(n_r), int(n_eta)
        self.ny, self.nz = int(n_pixels_y), int(n_pixels_z)
        self.mode, self.normalize, self.semantics = mode, bool(normalize), semantics
        self.bc_y, self.bc_z = float(bc_y), float(bc_z)
        self.variance = bool(variance)
        recs = np.ascontiguousarray(pixmap.pxList)
        nmap = np.ascontiguousarray(pixmap.nmap_pairs())
        desc = L.MiMapDesc(recs.ctypes.data if recs.size else None, recs.shape[0],
                           nmap.ctypes.data, self.n_r, self.n_eta, self.ny, self.nz,
                           self.bc_y, self.bc_z)
        if encoding not in L.ENC:
            raise ValueError(f"unknown encoding {encoding!r}; expected 'auto' | 'csr' | 'runs' | 'mma' | 'mmad'")
        opts = L.MiPlanOpts(L.MODE[mode], int(self.normalize), L.SEM[semantics],
                            int(tile_rows), int(tile_pixels), int(frames_per_lane),
                            L.ENC[encoding], int(run_len), int(self.variance), int(host_threads))
        h = C.c_void_p()
        L.check(L.lib().mi_plan_create(C.byref(desc), C.byref(opts), self.device.index,
                                       C.byref(h)), "mi_plan_create")
        self._h = h
        self._dark = None

    # -- lifecycle --------------------------------------------------------
    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            L.lib().mi_plan_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def n_bins(self) -> int:
        return self.n_r * self.n_eta

    @property
    def info(self) -> Dict[str, int]:
        inf = L.MiPlanInfo()
        L.check(L.lib().mi_plan_get_info(self._h, C.byref(inf)), "mi_plan_get_info")
        return {k: getattr(inf, k) for k, _ in L.MiPlanInfo._fields_}

    def status(self) -> int:
        """Device status word of the plan's launches (0, or MI_E_TIMEOUT when a bounded
        in-kernel wait expired); reading it synchronises the device and clears it."""
        st = C.c_int(0)
        L.check(L.lib().mi_plan_status(self._h, C.byref(st)), "mi_plan_status")
        return st.value

    def set_dark(self, dark) -> None:
        """Per-pixel dark (ny*nz floats; frames are cast and have it subtracted)."""
        if dark is None:
            L.check(L.lib().mi_plan_set_dark(self._h, None), "mi_plan_set_dark")
            self._dark = None
            return
        d = np.ascontiguousarray(np.asarray(dark, dtype=np.float32).reshape(-1))
        if d.size != self.ny * self.nz:
            raise ValueError(f"dark has {d.size} pixels, expected {self.ny * self.nz}")
        L.check(L.lib().mi_plan_set_dark(self._h, d.ctypes.data), "mi_plan_set_dark")
        self._dark = d

    def set_bin_mask(self, bin_mask) -> None:
        """Semantics 'omp' only: bins flagged in ``bin_mask`` (n_bins, nonzero = the bin holds
        a masked pixel; DetectorMapper's bin mask) are NaN in every cake, as the OpenMP
        integrator writes them (IntegratorZarrOMP.c:1766-1767).  None clears it."""
        if bin_mask is None:
            L.check(L.lib().mi_plan_set_bin_mask(self._h, None), "mi_plan_set_bin_mask")
            return
        m = np.ascontiguousarray(np.asarray(bin_mask).reshape(-1) != 0, dtype=np.uint8)
        if m.size != self.n_r * self.n_eta:
            raise ValueError(f"bin mask has {m.size} entries, expected {self.n_r * self.n_eta}")
        L.check(L.lib().mi_plan_set_bin_mask(self._h, m.ctypes.data), "mi_plan_set_bin_mask")

    MMA_PIPELINES = ((8, 6), (7, 6), (6, 6), (5, 5), (7, 7), (4, 4))

    def set_mma_pipeline(self, stages: int, producers: int) -> None:
        """MMA encoding only: the tensor-core kernel's stage slots and producer warps, one of
        ``MMA_PIPELINES`` (default 8 / 6).  Results are identical; only the time differs."""
        L.check(L.lib().mi_plan_set_mma_pipeline(self._h, int(stages), int(producers)), "mi_plan_set_mma_pipeline")

    # -- work ---------------------------------------------------------------
    def _frames(self, frames: torch.Tensor) -> Tuple[torch.Tensor, int, int]:
        if frames.device != self.device:
            raise ValueError(f"frames on {frames.device}, plan on {self.device}")
        if frames.dim() == 2:
            frames = frames.unsqueeze(0)
        if frames.dim() != 3 and frames.dim() != 2:
            raise ValueError("frames must be (F, NZ, NY), (NZ, NY) or (F, NZ*NY)")
        F = frames.shape[0]
        per = frames[0].numel() if F else self.ny * self.nz
        if per != self.ny * self.nz:
            raise ValueError(f"frame has {per} pixels, expected {self.ny * self.nz}")
        flat = frames.reshape(F, per)
        if F and flat.stride(1) != 1:
            flat = flat.contiguous()
        return flat, F, flat.stride(0) if F else per

    def integrate(self, frames: torch.Tensor, *, cake: bool = True, lineouts: bool = True,
                  out: Optional[Dict[str, torch.Tensor]] = None, stream=None,
                  sum_into: Optional[torch.Tensor] = None):
        """Cake a batch of frames (device tensor, any supported dtype).

        sum_into: a float64 [n_r, n_eta] device tensor that the batch's cakes are added to
        (the SumImages running sum, IntegratorFitPeaksGPUStream.cu:1043-1046; needs cake).

        Returns (cake [F, n_r, n_eta] float32 or None, lineout_aw [F, n_r] float64 or None,
        lineout_sm [F, n_r] float64 or None)."""
        if sum_into is not None:
            if not cake:
                raise ValueError("sum_into adds the cakes: cake must be on")
            if (sum_into.dtype != torch.float64 or sum_into.device != self.device or not sum_into.is_contiguous()
                    or sum_into.numel() != self.n_bins):
                raise ValueError("sum_into is a contiguous float64 tensor of n_r x n_eta on the plan's device")
        flat, F, stride = self._frames(frames)
        out = out or {}
        ck = out.get("cake") if cake else None
        if cake and ck is None:
            ck = torch.empty((F, self.n_r, self.n_eta), dtype=torch.float32, device=self.device)
        aw = sm = None
        if lineouts:
            aw = out.get("lineout_aw")
            sm = out.get("lineout_sm")
            if aw is None:
                aw = torch.empty((F, self.n_r), dtype=torch.float64, device=self.device)
            if sm is None:
                sm = torch.empty((F, self.n_r), dtype=torch.float64, device=self.device)
        if F:
            L.check(L.lib().mi_integrate_batch(self._h, flat.data_ptr(), dtype_code(flat.dtype), F,
                                               stride, L.ptr(ck), L.ptr(aw), L.ptr(sm),
                                               L.stream_ptr(stream)), "mi_integrate_batch")
            if sum_into is not None:
                L.check(L.lib().mi_sum_cake(self._h, ck.data_ptr(), F, sum_into.data_ptr(), L.stream_ptr(stream)),
                        "mi_sum_cake")
        return ck, aw, sm

    def capture(self, frames: torch.Tensor, out: Dict[str, torch.Tensor], *, cake: bool = True,
                lineouts: bool = True) -> "torch.cuda.CUDAGraph":
        """Record ``integrate(frames, out=out)`` (every launch of the batch: pixel-major
        staging, caking, lineouts) as a CUDA graph; ``graph.replay()`` then re-runs it on
        whatever the same buffers hold.  A first ``integrate`` on the buffers warms up the
        kernels before the capture."""
        self.integrate(frames, cake=cake, lineouts=lineouts, out=out)
        torch.cuda.synchronize(self.device)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self.integrate(frames, cake=cake, lineouts=lineouts, out=out)
        return g

    def upload(self, host_frames: torch.Tensor, device_frames: torch.Tensor, stream=None) -> None:
        """Copy host frames (CPU tensor (F, NZ, NY), page-locked for an asynchronous copy) to
        device frames of the same shape and dtype: only the pixels the map can read cross
        PCIe -- per group of 16 rows of the referenced band, the columns the group references
        (``info["upload_pixels"]`` per frame), one 3-D copy per group; the device frames'
        other pixels are left as they are."""
        if host_frames.device.type != "cpu" or device_frames.device != self.device:
            raise ValueError("upload copies a CPU tensor into a tensor on the plan's device")
        if host_frames.dtype != device_frames.dtype or host_frames.shape[0] > device_frames.shape[0]:
            raise ValueError("host and device frames must have one dtype and room for the frames")
        hf, F, hs = self._frames_host(host_frames)
        df = device_frames.reshape(device_frames.shape[0], -1)
        if df.shape[1] != self.ny * self.nz or (F and df.stride(1) != 1):
            raise ValueError("device frames must be contiguous frames of ny*nz pixels")
        L.check(L.lib().mi_upload_frames(self._h, hf.data_ptr(), dtype_code(hf.dtype), F, hs, df.data_ptr(),
                                         df.stride(0), L.stream_ptr(stream)), "mi_upload_frames")

    def stage_host(self, src: np.ndarray, dst: torch.Tensor) -> None:
        """Copy host frames ``src`` (numpy (F, NZ, NY) or (NZ, NY), C-contiguous) into the
        host tensor ``dst`` of the same dtype (e.g. page-locked staging for ``upload``): only
        the pixels ``upload`` sends (``info["upload_pixels"]`` per frame), in C with the
        interpreter lock released."""
        a = np.ascontiguousarray(src)
        F = a.shape[0] if a.ndim == 3 else 1
        if a.size != F * self.ny * self.nz or dst.device.type != "cpu":
            raise ValueError("stage_host copies host frames of ny*nz pixels into a CPU tensor")
        df = dst.reshape(dst.shape[0] if dst.dim() == 3 else 1, -1)
        if df.shape[0] < F or df.stride(1) != 1 or str(a.dtype) != str(dst.dtype).replace("torch.", ""):
            raise ValueError("stage_host needs a contiguous destination of the same dtype with room for the frames")
        L.check(L.lib().mi_stage_host_frames(self._h, a.ctypes.data, dtype_code(dst.dtype), F, self.ny * self.nz,
                                             df.data_ptr(), df.stride(0)), "mi_stage_host_frames")

    def _frames_host(self, frames: torch.Tensor):
        F = frames.shape[0]
        flat = frames.reshape(F, -1)
        if flat.shape[1] != self.ny * self.nz:
            raise ValueError(f"frame has {flat.shape[1]} pixels, expected {self.ny * self.nz}")
        if F and flat.stride(1) != 1:
            raise ValueError("host frames must be contiguous along the pixels")
        return flat, F, flat.stride(0) if F else self.ny * self.nz

    def integrate_plain(self, frame: torch.Tensor, stream=None):
        """The reference algorithm, one frame per launch: (cake float64 [n_r, n_eta], aw, sm)."""
        flat, F, _ = self._frames(frame)
        if F != 1:
            raise ValueError("integrate_plain takes exactly one frame")
        ck = torch.empty((self.n_r, self.n_eta), dtype=torch.float64, device=self.device)
        aw = torch.empty(self.n_r, dtype=torch.float64, device=self.device)
        sm = torch.empty(self.n_r, dtype=torch.float64, device=self.device)
        L.check(L.lib().mi_integrate_plain(self._h, flat.data_ptr(), dtype_code(flat.dtype),
                                           ck.data_ptr(), aw.data_ptr(), sm.data_ptr(),
                                           L.stream_ptr(stream)), "mi_integrate_plain")
        return ck, aw, sm

    def bin_table(self, r_lo, r_hi, eta_lo, eta_hi, *, px: float, lsd: float,
                  wavelength: float = 0.0) -> np.ndarray:
        """Per-bin axes [n_r * n_eta, 5]: R mean (px), 2-theta (deg), eta mean (deg), bin
        area (areaWeight of the records on the detector), Q (1/A; 0 without a wavelength),
        as the GPU stream's static output header (IntegratorFitPeaksGPUStream.cu:817-899).
        px and lsd in one unit (um)."""
        edges = [np.ascontiguousarray(np.asarray(a, dtype=np.float64).reshape(-1)) for a in (r_lo, r_hi)]
        edges += [np.ascontiguousarray(np.asarray(a, dtype=np.float64).reshape(-1)) for a in (eta_lo, eta_hi)]
        if edges[0].size != self.n_r or edges[1].size != self.n_r:
            raise ValueError(f"R edges need {self.n_r} values")
        if edges[2].size != self.n_eta or edges[3].size != self.n_eta:
            raise ValueError(f"eta edges need {self.n_eta} values")
        out = np.empty((self.n_bins, 5), dtype=np.float64)
        L.check(L.lib().mi_plan_bin_table(self._h, *[e.ctypes.data for e in edges], float(px), float(lsd),
                                          float(wavelength), out.ctypes.data), "mi_plan_bin_table")
        return out

    def profile(self, cake: torch.Tensor, stream=None):
        """Kernel (c) on a given cake [F, n_r, n_eta] (float32/float64) -> (aw, sm) [F, n_r]."""
        if cake.dim() == 2:
            cake = cake.unsqueeze(0)
        if cake.dtype not in (torch.float32, torch.float64):
            cake = cake.to(torch.float64)
        cake = cake.contiguous()
        F = cake.shape[0]
        aw = torch.empty((F, self.n_r), dtype=torch.float64, device=self.device)
        sm = torch.empty((F, self.n_r), dtype=torch.float64, device=self.device)
        L.check(L.lib().mi_profile_batch(self._h, cake.data_ptr(), dtype_code(cake.dtype), F,
                                         aw.data_ptr(), sm.data_ptr(), L.stream_ptr(stream)),
                "mi_profile_batch")
        return aw, sm


class PanelPlan:
    """Device-resident plan over several detector panels that share one binning.

    A bin of the merged cake is the sum of every panel's weighted pixels over the sum of
    their areas (one weight list over all panels); each panel keeps its own map, shape,
    beam centre, dark and frame type.  ``integrate`` takes one frame tensor per panel and
    runs kernel (a) once per panel and kernel (b) once for all of them.

    Args:
        pixmaps: one ``bin_io.PixelMap`` per panel, all with n_r * n_eta bins.
        shapes: (n_pixels_y, n_pixels_z) of each panel.
        beam_centres: (bc_y, bc_z) of each panel (used by gradient mode).
        n_r, n_eta, mode, normalize, semantics, device, tile_rows, tile_pixels, run_len:
            as for ``CakePlan`` (run encoding, tile_rows <= 16).
        encoding: 'runs' or 'mma' (tensor cores; every panel's frames 8/16-bit).
    """

    def __init__(self, pixmaps, *, shapes, n_r: int, n_eta: int, beam_centres=None, mode: str = "floor",
                 normalize: bool = True, semantics: str = "py", device="cuda", tile_rows: int = 0,
                 tile_pixels: int = 0, run_len: int = 0, encoding: str = "runs"):
        n = len(pixmaps)
        if encoding not in ("runs", "mma"):
            raise ValueError(f"panel plans use the 'runs' or 'mma' encoding, not {encoding!r}")
        if n == 0 or len(shapes) != n or (beam_centres is not None and len(beam_centres) != n):
            raise ValueError("one shape (and beam centre) per panel map is needed")
        if mode not in L.MODE or semantics not in L.SEM:
            raise ValueError(f"unknown mode {mode!r} or semantics {semantics!r}")
        self.device = torch.device("cuda", _device_index(device))
        self.n_r, self.n_eta, self.shapes = int(n_r), int(n_eta), [(int(a), int(b)) for a, b in shapes]
        bcs = beam_centres or [(0.0, 0.0)] * n
        descs = (L.MiMapDesc * n)()
        self._keep = []
        for i, pm in enumerate(pixmaps):
            if pm.n_bins != self.n_r * self.n_eta:
                raise ValueError(f"panel {i}: PixelMap has {pm.n_bins} bins; n_r * n_eta = {self.n_r * self.n_eta}")
            recs = np.ascontiguousarray(pm.pxList)
            nmap = np.ascontiguousarray(pm.nmap_pairs())
            self._keep += [recs, nmap]
            ny, nz = self.shapes[i]
            descs[i] = L.MiMapDesc(recs.ctypes.data if recs.size else None, recs.shape[0], nmap.ctypes.data,
                                   self.n_r, self.n_eta, ny, nz, float(bcs[i][0]), float(bcs[i][1]))
        opts = L.MiPlanOpts(L.MODE[mode], int(normalize), L.SEM[semantics], int(tile_rows), int(tile_pixels), 0,
                            L.ENC[encoding], int(run_len))
        h = C.c_void_p()
        L.check(L.lib().mi_plan_create_panels(descs, n, C.byref(opts), self.device.index, C.byref(h)),
                "mi_plan_create_panels")
        self._keep = []
        self._h = h

    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            L.lib().mi_plan_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def info(self) -> Dict[str, int]:
        inf = L.MiPlanInfo()
        L.check(L.lib().mi_plan_get_info(self._h, C.byref(inf)), "mi_plan_get_info")
        return {k: getattr(inf, k) for k, _ in L.MiPlanInfo._fields_}

    def status(self) -> int:
        st = C.c_int(0)
        L.check(L.lib().mi_plan_status(self._h, C.byref(st)), "mi_plan_status")
        return st.value

    def set_dark(self, darks) -> None:
        """One dark per panel ((nz, ny) floats each, or None)."""
        arrs = []
        ptrs = (C.c_void_p * len(self.shapes))()
        for i, d in enumerate(darks):
            if d is None:
                continue
            ny, nz = self.shapes[i]
            a = np.ascontiguousarray(np.asarray(d, dtype=np.float32).reshape(-1))
            if a.size != ny * nz:
                raise ValueError(f"panel {i}: dark has {a.size} pixels, expected {ny * nz}")
            arrs.append(a)
            ptrs[i] = a.ctypes.data
        L.check(L.lib().mi_plan_set_dark_panels(self._h, ptrs), "mi_plan_set_dark_panels")

    def integrate(self, frames, *, cake: bool = True, lineouts: bool = True, out=None, stream=None):
        """Frames of every panel (one device tensor (F, nz_i, ny_i) per panel, same F) ->
        (merged cake [F, n_r, n_eta] float32, lineout_aw [F, n_r], lineout_sm [F, n_r])."""
        n = len(self.shapes)
        if len(frames) != n:
            raise ValueError(f"{len(frames)} frame tensors for {n} panels")
        F = frames[0].shape[0]
        ptrs, dts, strides = (C.c_void_p * n)(), (C.c_int * n)(), (C.c_int64 * n)()
        flats = []
        for i, fr in enumerate(frames):
            if fr.device != self.device:
                raise ValueError(f"panel {i}: frames on {fr.device}, plan on {self.device}")
            ny, nz = self.shapes[i]
            if fr.shape[0] != F or fr[0].numel() != ny * nz:
                raise ValueError(f"panel {i}: frames must be ({F}, {nz}, {ny})")
            flat = fr.reshape(F, ny * nz)
            if F and flat.stride(1) != 1:
                flat = flat.contiguous()
            flats.append(flat)
            ptrs[i] = flat.data_ptr() if F else None
            dts[i] = dtype_code(flat.dtype)
            strides[i] = flat.stride(0) if F else ny * nz
        out = out or {}
        ck = out.get("cake") if cake else None
        if cake and ck is None:
            ck = torch.empty((F, self.n_r, self.n_eta), dtype=torch.float32, device=self.device)
        aw = sm = None
        if lineouts:
            aw = out.get("lineout_aw")
            sm = out.get("lineout_sm")
            if aw is None:
                aw = torch.empty((F, self.n_r), dtype=torch.float64, device=self.device)
            if sm is None:
                sm = torch.empty((F, self.n_r), dtype=torch.float64, device=self.device)
        L.check(L.lib().mi_integrate_panels(self._h, ptrs, dts, strides, F, L.ptr(ck), L.ptr(aw), L.ptr(sm),
                                            L.stream_ptr(stream)), "mi_integrate_panels")
        return ck, aw, sm


# ---------------------------------------------------------------------------
# midas_integrate-compatible surface
# ---------------------------------------------------------------------------
@dataclass
class CSRGeometry:
    """Geometry for a fixed detector + bin layout (kernels.py:CSRGeometry).

    Holds one device plan per (mode, normalize) pair, created on first use."""
    pixmap: PixelMap
    area_per_bin: torch.Tensor
    n_r: int
    n_eta: int
    n_pixels_y: int
    n_pixels_z: int
    bc_y: float = 0.0
    bc_z: float = 0.0
    semantics: str = "py"
    build_modes: Tuple[str, ...] = ("floor", "bilinear", "gradient")
    dtype: torch.dtype = torch.float32
    compute_variance: bool = False
    plans: Dict[Tuple[str, bool, bool], CakePlan] = field(default_factory=dict)

    @property
    def n_bins(self) -> int:
        return self.n_r * self.n_eta

    @property
    def device(self) -> torch.device:
        return self.area_per_bin.device

    def plan(self, mode: str, normalize: bool = True, variance: bool = False) -> CakePlan:
        if mode not in L.MODE:
            raise ValueError(f"unknown integration mode {mode!r}; expected 'floor' | 'bilinear' | 'gradient'")
        if mode not in self.build_modes:
            raise RuntimeError(f"build_csr was called without {mode!r} in build_modes; "
                               "rebuild with build_modes including this mode.")
        if variance and not self.compute_variance:
            raise RuntimeError(
                f"build_csr was called without compute_variance=True (mode={mode!r}); "
                "rebuild with compute_variance=True to use integrate_with_variance.")
        key = (mode, bool(normalize), bool(variance))
        if key not in self.plans:
            self.plans[key] = CakePlan(self.pixmap, n_r=self.n_r, n_eta=self.n_eta,
                                       n_pixels_y=self.n_pixels_y, n_pixels_z=self.n_pixels_z,
                                       mode=mode, normalize=normalize, semantics=self.semantics,
                                       bc_y=self.bc_y, bc_z=self.bc_z, device=self.device,
                                       variance=variance)
        return self.plans[key]

    def any_plan(self, variance: bool = False) -> CakePlan:
        """A plan of this geometry for the eta reductions (all plans share the bin areas)."""
        for (_, _, v), p in self.plans.items():
            if v == variance:
                return p
        return self.plan(self.build_modes[0], True, variance)


def _area_in(pixmap: PixelMap, ny: int, nz: int) -> np.ndarray:
    """In-bounds areaWeight per bin (the bounds-checked area of kernels.py:306-311)."""
    px = pixmap.pxList
    counts = pixmap.counts.astype(np.int64)
    if (counts < 0).any():
        raise ValueError("nMap.bin contains negative pixel counts")
    end = pixmap.offsets.astype(np.int64) + counts
    if ((end > pixmap.n_entries) & (counts > 0)).any():
        raise ValueError("bin(s) reference past end of pxList")
    area = np.zeros(pixmap.n_bins, dtype=np.float64)
    if counts.sum() == 0:
        return area
    idx = np.concatenate([np.arange(o, o + c) for o, c in zip(pixmap.offsets, counts) if c])
    b = np.repeat(np.arange(pixmap.n_bins), counts)
    rec = px[idx]
    iy = rec["y"].astype(np.float64).astype(np.int64)
    iz = rec["z"].astype(np.float64).astype(np.int64)
    ok = (iy >= 0) & (iy < ny) & (iz >= 0) & (iz < nz)
    np.add.at(area, b, np.where(ok, rec["areaWeight"].astype(np.float64), 0.0))
    return area


def build_csr(pixmap: PixelMap, *, n_r: int, n_eta: int, n_pixels_y: int, n_pixels_z: int,
              device="cuda", dtype: torch.dtype = torch.float32, bc_y: float = 0.0,
              bc_z: float = 0.0, build_modes: Tuple[str, ...] = ("floor", "bilinear", "gradient"),
              compute_variance: bool = False, semantics: str = "py") -> CSRGeometry:
    """Prepare a map for integration (kernels.py:build_csr).  The per-mode device plans
    are built lazily by the first ``integrate`` call of that mode; ``compute_variance``
    allows the variance plans of ``integrate_with_variance``."""
    if pixmap.n_bins != n_r * n_eta:
        raise ValueError(f"PixelMap has {pixmap.n_bins} bins; n_r * n_eta = {n_r * n_eta}")
    dev = torch.device("cuda", _device_index(device))
    area = _area_in(pixmap, n_pixels_y, n_pixels_z)
    return CSRGeometry(pixmap=pixmap, area_per_bin=torch.from_numpy(area).to(dev, dtype),
                       n_r=n_r, n_eta=n_eta, n_pixels_y=n_pixels_y, n_pixels_z=n_pixels_z,
                       bc_y=bc_y, bc_z=bc_z, semantics=semantics,
                       build_modes=tuple(build_modes), dtype=dtype,
                       compute_variance=bool(compute_variance))


def integrate(image: torch.Tensor, geom: CSRGeometry, *, mode: str = "floor",
              normalize: bool = True) -> torch.Tensor:
    """Integrate one (dark-subtracted) image to the (n_r, n_eta) grid (kernels.py:integrate)."""
    plan = geom.plan(mode, normalize)
    flat = _flat_image(image, geom, "image")
    ck, _, _ = plan.integrate(flat.reshape(1, -1), cake=True, lineouts=False)
    return ck[0].to(geom.dtype)


def _flat_image(image: torch.Tensor, geom: CSRGeometry, what: str) -> torch.Tensor:
    flat = image.reshape(-1)
    if flat.numel() != geom.n_pixels_y * geom.n_pixels_z:
        raise ValueError(f"{what} numel {flat.numel()} != n_pixels {geom.n_pixels_y * geom.n_pixels_z}")
    flat = flat.to(geom.device)
    if flat.dtype not in _TORCH_DT:
        flat = flat.to(torch.float32)
    return flat


def integrate_with_variance(image: torch.Tensor, geom: CSRGeometry, *, mode: str = "floor",
                            normalize: bool = True, variance_image: Optional[torch.Tensor] = None):
    """Integrate one frame and propagate per-pixel variance (kernels.py:474-536):
    (intensity, variance), both (n_r, n_eta).  ``variance_image`` None = Poisson (the
    image is its own variance).  The variance is the cake of the variance image under
    the squared coalesced weights, over the squared bin area when normalising."""
    flat = _flat_image(image, geom, "image")
    vflat = flat if variance_image is None else _flat_image(variance_image, geom, "variance_image")
    vplan = geom.plan(mode, normalize, variance=True)
    iplan = geom.plan(mode, normalize)
    ck, _, _ = iplan.integrate(flat.reshape(1, -1), cake=True, lineouts=False)
    vk, _, _ = vplan.integrate(vflat.reshape(1, -1), cake=True, lineouts=False)
    return ck[0].to(geom.dtype), vk[0].to(geom.dtype)


def profile_1d(int2d: torch.Tensor, geom: CSRGeometry, *, mode: str = "area_weighted") -> torch.Tensor:
    """Reduce (n_r, n_eta) -> (n_r,) over eta (kernels.py:profile_1d)."""
    if mode not in ("area_weighted", "simple_mean"):
        raise ValueError(f"unknown profile_1d mode {mode!r}")
    aw, sm = geom.any_plan().profile(int2d.to(geom.device).reshape(1, geom.n_r, geom.n_eta))
    return (aw[0] if mode == "area_weighted" else sm[0]).to(geom.dtype)


def profile_1d_with_variance(int2d: torch.Tensor, var2d: torch.Tensor, geom: CSRGeometry, *,
                             mode: str = "area_weighted"):
    """(I_1d, Var_1d) over eta (kernels.py:604-645): Var_1d = sum(A^2 Var) / (sum A)^2
    (area_weighted) or sum(Var) / N^2 (simple_mean)."""
    if mode not in ("area_weighted", "simple_mean"):
        raise ValueError(f"unknown profile_1d_with_variance mode {mode!r}")
    shape = (1, geom.n_r, geom.n_eta)
    aw, sm = geom.any_plan().profile(int2d.to(geom.device).reshape(shape))
    vaw, vsm = geom.any_plan(variance=True).profile(var2d.to(geom.device).reshape(shape))
    if mode == "area_weighted":
        return aw[0].to(geom.dtype), vaw[0].to(geom.dtype)
    return sm[0].to(geom.dtype), vsm[0].to(geom.dtype)


def r_axis(*, n_r: int, RMin: float, RBinSize: float) -> np.ndarray:
    """R at bin centres."""
    return RMin + RBinSize * (np.arange(n_r, dtype=np.float64) + 0.5)


def eta_axis(*, n_eta: int, EtaMin: float, EtaBinSize: float) -> np.ndarray:
    """Eta at bin centres."""
    return EtaMin + EtaBinSize * (np.arange(n_eta, dtype=np.float64) + 0.5)
