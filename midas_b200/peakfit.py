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


def fit_peaks(x, intensity, peak_locations, *, x_bin_size: float, fit_roi_padding: int = 20,
              model="tch", device="cuda") -> np.ndarray:
    """Single-lineout API (peakfit.py:fit_peaks): returns (n_peaks, 7) rows
    [area, center, sig, gam, FWHM, eta, chi2/dof]; rejected peaks are zero rows."""
    xt = torch.as_tensor(np.asarray(x, np.float64), device=device)
    yt = torch.as_tensor(np.asarray(intensity, np.float64), device=device).reshape(1, -1)
    pt = torch.as_tensor(np.asarray(peak_locations, np.float64), device=device)
    r = fit_batch(xt, yt, pt, model=model, half_window=fit_roi_padding, x_bin=x_bin_size)
    return r.params[0, :, :7].cpu().numpy()


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
