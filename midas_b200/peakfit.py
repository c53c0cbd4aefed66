"""Batched pseudo-Voigt peak fits on the device (kernel (d) of libmidas_b200).

``fit_batch`` fits every (frame, peak) window of a batch of lineouts in one launch,
one warp per window; ``fit_peaks`` mirrors the single-lineout API of
packages/midas_integrate/midas_integrate/peakfit.py:334 (output rows in the
PF_PARAMS_PER_PEAK = 7 layout of FF_HEDM/src/PeakFit.h).

Output columns per window (MI_FIT_NOUT = 11):
    0 area, 1 center, 2 sig, 3 gam, 4 FWHM, 5 eta, 6 chi2/dof,
    7 peak height, 8 bg0, 9 bg1, 10 two-theta (deg, from center * px / Lsd)
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib as L

MODELS = {"pv": L.FIT_PV, "tch": L.FIT_TCH, 0: L.FIT_PV, 1: L.FIT_TCH}


@dataclass
class FitResult:
    params: torch.Tensor   # [F, n_peaks, 11] float64
    iters: torch.Tensor    # [F, n_peaks] int32; -1 = peak not within 2 bins of the grid


def fit_batch(x: torch.Tensor, lineouts: torch.Tensor, peaks: torch.Tensor, *, model="pv",
              half_window: int = 20, x_bin: float = 1.0, max_iter: int = 100, px_um: float = 0.0,
              lsd_um: float = 0.0, stream=None) -> FitResult:
    """Fit all peaks of all lineouts.  x [n_x], lineouts [F, n_x], peaks [n_peaks]: device
    float64 tensors on one device."""
    dev = lineouts.device
    if dev.type != "cuda":
        raise RuntimeError("fit_batch runs on a CUDA device")
    x = x.to(dev, torch.float64).contiguous()
    lo = lineouts.to(torch.float64).contiguous()
    if lo.dim() == 1:
        lo = lo.unsqueeze(0)
    pk = peaks.to(dev, torch.float64).contiguous()
    F, n_x = lo.shape
    if x.numel() != n_x:
        raise ValueError("x and lineouts disagree in length")
    out = torch.zeros((F, pk.numel(), L.FIT_NOUT), dtype=torch.float64, device=dev)
    it = torch.zeros((F, pk.numel()), dtype=torch.int32, device=dev)
    opts = L.MiFitOpts(MODELS[model], int(half_window), int(max_iter), float(x_bin), float(px_um),
                       float(lsd_um))
    with torch.cuda.device(dev):
        L.check(L.lib().mi_fit_batch(x.data_ptr(), lo.data_ptr(), F, n_x, pk.data_ptr(), pk.numel(),
                                     C.byref(opts), out.data_ptr(), it.data_ptr(), L.stream_ptr(stream)),
                "mi_fit_batch")
    return FitResult(out, it)


class FitPlan:
    """The reference's fit jobs for one (x axis, peak list, options), fit on the device.

    kind "peaks": fitPeaks / fit_peaks (FF_HEDM/src/PeakFit.c:275-545;
    packages/midas_integrate/midas_integrate/peakfit.py:334) -- nearest bin per peak, ROI
    +- half_window bins, overlapping ROIs merged into one joint TCH fit.
    kind "eta": the per-eta-bin fits of FF_HEDM/src/IntegratorZarrOMP.c:1902-2030 -- height-
    normalised pseudo-Voigt singlets, doublets for adjacent peaks closer than doublet_sep,
    on every eta column of a cake with at least 5 nonzero samples.
    device="cpu" builds the job table only (``jobs``, ``info``); it cannot run.
    """

    def __init__(self, x, peaks, *, kind: str = "peaks", half_window: int = 20, x_bin: float = 1.0,
                 max_iter: int = 200, doublet_sep: float = 0.0, px_um: float = 0.0, lsd_um: float = 0.0,
                 device="cuda"):
        self.device = torch.device(device)
        xs = np.ascontiguousarray(np.asarray(x, np.float64))
        pk = np.ascontiguousarray(np.asarray(peaks, np.float64).reshape(-1))
        self.n_x, self.n_peaks = xs.size, pk.size
        k = {"peaks": L.FIT_KIND_PEAKS, "eta": L.FIT_KIND_ETA}[kind]
        self.kind = kind
        opts = L.MiFitJobOpts(k, int(half_window), int(max_iter), 0, float(x_bin), float(doublet_sep),
                              float(px_um), float(lsd_um))
        h = C.c_void_p()
        dev = -1 if self.device.type == "cpu" else (self.device.index or 0)
        L.check(L.lib().mi_fit_plan_create(xs.ctypes.data, xs.size, pk.ctypes.data, pk.size, C.byref(opts),
                                           dev, C.byref(h)), "mi_fit_plan_create")
        self._h = h

    def jobs(self):
        """The job table: (jobs [n_jobs, 4] = first sample, last sample, peaks, first entry;
        peak ids [n_valid] = the caller's index of each entry)."""
        inf = self.info()
        jb = np.zeros((inf["n_jobs"], 4), np.int32)
        ids = np.zeros(inf["n_valid"], np.int32)
        L.check(L.lib().mi_fit_plan_jobs(self._h, jb.ctypes.data, ids.ctypes.data), "mi_fit_plan_jobs")
        return jb, ids

    def info(self):
        nj, nv, mx = C.c_int(), C.c_int(), C.c_int()
        L.check(L.lib().mi_fit_plan_info(self._h, C.byref(nj), C.byref(nv), C.byref(mx)), "mi_fit_plan_info")
        return {"n_jobs": nj.value, "n_valid": nv.value, "max_job_peaks": mx.value}

    def run(self, series: torch.Tensor, *, n_sub: int = 1, ld_series=None, ld_sub: int = 0, ld_x: int = 1,
            stream=None) -> FitResult:
        """Fit the series of a device tensor (float32 or float64).  A [F, n_x] tensor is F
        lineouts; see ``fit_cake_eta`` for the eta columns of a cake."""
        if series.device.type != "cuda":
            raise RuntimeError("FitPlan.run takes a CUDA tensor")
        if series.dtype not in (torch.float32, torch.float64):
            series = series.to(torch.float64)
        series = series.contiguous()
        n_series = series.shape[0] if series.dim() > 1 else 1
        if ld_series is None:
            ld_series = series.stride(0) if series.dim() > 1 else 0
        dt = L.DT_F64 if series.dtype == torch.float64 else L.DT_F32
        tot = n_series * n_sub
        out = torch.zeros((tot, self.n_peaks, L.FIT_NOUT), dtype=torch.float64, device=series.device)
        it = torch.zeros((tot, self.n_peaks), dtype=torch.int32, device=series.device)
        with torch.cuda.device(series.device):
            L.check(L.lib().mi_fit_plan_run(self._h, series.data_ptr(), dt, n_series, n_sub, int(ld_series),
                                            int(ld_sub), int(ld_x), out.data_ptr(), it.data_ptr(),
                                            L.stream_ptr(stream)), "mi_fit_plan_run")
        return FitResult(out, it)

    def fit_cake_eta(self, cake: torch.Tensor, stream=None) -> FitResult:
        """Per-eta fits of a [F, n_r, n_eta] cake: params [F * n_eta, n_peaks, 11] (series
        f * n_eta + e)."""
        F, n_r, n_eta = cake.shape
        if n_r != self.n_x:
            raise ValueError("cake rows and the plan's x axis disagree")
        cake = cake.contiguous()
        return self.run(cake.reshape(F, -1), n_sub=n_eta, ld_series=n_r * n_eta, ld_sub=1, ld_x=n_eta,
                        stream=stream)

    def close(self):
        if getattr(self, "_h", None):
            L.lib().mi_fit_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def fit_peaks(x, intensity, peak_locations, *, x_bin_size: float, fit_roi_padding: int = 20,
              device="cuda") -> np.ndarray:
    """Single-lineout API of peakfit.py:fit_peaks (the reference's fitPeaks): rows
    [area, center, sig, gam, FWHM, eta, chi2/dof] of the peaks within 2 bins of the grid, in
    ascending bin order (overlapping windows fit jointly); (n_peaks, 7) zeros when none is."""
    xs = np.asarray(x, np.float64)
    locs = np.asarray(peak_locations, np.float64).reshape(-1)
    if locs.size == 0 or xs.size == 0:
        return np.zeros((0, 7), np.float64)
    plan = FitPlan(xs, locs, kind="peaks", half_window=fit_roi_padding, x_bin=x_bin_size, device=device)
    try:
        y = torch.as_tensor(np.asarray(intensity, np.float64), device=device).reshape(1, -1)
        r = plan.run(y)
        p, it = r.params[0].cpu().numpy(), r.iters[0].cpu().numpy()
    finally:
        plan.close()
    idx = np.array([int(np.argmin(np.abs(xs - c))) for c in locs])
    valid = np.abs(xs[idx] - locs) < 2.0 * x_bin_size
    if not valid.any():
        return np.zeros((locs.size, 7), np.float64)
    order = [k for k in np.argsort(idx, kind="stable") if valid[k]]
    rows = p[order, :7].copy()
    rows[it[order] < 0] = 0.0
    return rows


@dataclass
class AutoResult:
    params: torch.Tensor   # [F, max_peaks, 11] float64, first n_found[f] rows filled
    n_found: torch.Tensor  # [F] int32


def fit_autodetect(x: torch.Tensor, lineouts: torch.Tensor, *, max_peaks: int, x_bin: float,
                   roi_padding: int = 20, snip_iter: int = 50, px_um: float = 0.0, lsd_um: float = 0.0,
                   stream=None) -> AutoResult:
    """fitPeaksAutoDetect (FF_HEDM/src/PeakFit.c:720-877) of every lineout on the device:
    SNIP background, peak detection, joint TCH fits on the background-subtracted profile,
    the reference's quality filter; rows in position order."""
    dev = lineouts.device
    if dev.type != "cuda":
        raise RuntimeError("fit_autodetect runs on a CUDA device")
    lo = lineouts.to(torch.float64).contiguous()
    if lo.dim() == 1:
        lo = lo.unsqueeze(0)
    xs = x.to(dev, torch.float64).contiguous()
    F, n_x = lo.shape
    if xs.numel() != n_x:
        raise ValueError("x and lineouts disagree in length")
    out = torch.zeros((F, max(max_peaks, 0), L.FIT_NOUT), dtype=torch.float64, device=dev)
    found = torch.zeros(F, dtype=torch.int32, device=dev)
    with torch.cuda.device(dev):
        L.check(L.lib().mi_fit_autodetect(xs.data_ptr(), lo.data_ptr(), F, n_x, int(max_peaks), float(x_bin),
                                          int(roi_padding), int(snip_iter), float(px_um), float(lsd_um),
                                          out.data_ptr(), found.data_ptr(), L.stream_ptr(stream)),
                "mi_fit_autodetect")
    return AutoResult(out, found)


PEAK_ROW_DTYPE = np.dtype([("frame_idx", "<i4"), ("eta_idx", "<i4"), ("peak_nr", "<i4"), ("eta_deg", "<f8"),
                           ("area", "<f8"), ("sig", "<f8"), ("gam", "<f8"), ("FWHM_deg", "<f8"),
                           ("eta_mix", "<f8"), ("chi_sq", "<f8"), ("center_2theta", "<f8"),
                           ("d_spacing_A", "<f8")])


def peak_rows(params, *, px_um: float, lsd_um: float, wavelength_a: float, eta_deg=None,
              first_frame: int = 0, eta_idx: int = -1) -> np.ndarray:
    """Output rows of the fitted peaks, one per (frame, peak), as pfio_make_row builds them
    (FF_HEDM/src/PeakFitIO.c:52-82): the first seven fit outputs, the centre converted to
    2-theta = atan(center * px / Lsd) (deg) and the d-spacing lambda / (2 sin theta)
    (0 when theta <= 1e-10 rad).  params: [F, n_peaks, >= 7] fit outputs (``FitResult.params``)."""
    p = params.detach().cpu().numpy() if hasattr(params, "detach") else np.asarray(params)
    p = p.reshape(-1, p.shape[-2], p.shape[-1]) if p.ndim >= 2 else p.reshape(1, 1, -1)
    F, n_peaks = p.shape[0], p.shape[1]
    rows = np.zeros(F * n_peaks, dtype=PEAK_ROW_DTYPE)
    flat = p.reshape(F * n_peaks, -1)
    rows["frame_idx"] = np.repeat(np.arange(F, dtype=np.int32) + first_frame, n_peaks)
    rows["eta_idx"] = eta_idx
    rows["peak_nr"] = np.tile(np.arange(n_peaks, dtype=np.int32), F)
    rows["eta_deg"] = 0.0 if eta_deg is None else eta_deg
    for k, name in enumerate(("area", None, "sig", "gam", "FWHM_deg", "eta_mix", "chi_sq")):
        if name:
            rows[name] = flat[:, k]
    tth = np.arctan(flat[:, 1] * px_um / lsd_um) * 180.0 / np.pi
    theta = tth * np.pi / 360.0
    rows["center_2theta"] = tth
    with np.errstate(divide="ignore"):
        rows["d_spacing_A"] = np.where(theta > 1e-10, wavelength_a / (2.0 * np.sin(theta)), 0.0)
    return rows
