"""Fit plans on the device against the reference's own fits and an FP64 least-squares check.

* fit_peaks on the lineouts of tests/golden/peakfit.npz against the reference's
  midas_integrate peakfit.fit_peaks output recorded there (scipy TRF; one isolated peak and
  one overlapping pair fit jointly).  The reference quotes about 1e-5 relative agreement
  between its two optimisers (packages/midas_integrate/README.md:70-73).
* per-eta fits (IntegratorZarrOMP.c:1902-2030, height-normalised pseudo-Voigt singlets and
  doublets) against scipy's bounded least squares on the same objective, bounds and start
  in FP64 (the reference's NLopt build is not available to run)."""
from pathlib import Path

import numpy as np
import pytest
import torch
from scipy.optimize import least_squares

from midas_b200 import peakfit
from midas_b200.peakfit import FitPlan

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"


def test_fit_peaks_matches_reference_fits(cuda):
    g = np.load(GOLDEN / "peakfit.npz")
    x, Y, centers, ref = g["x"], g["lineouts"], g["centers"], g["ref_fits"]
    for f in range(Y.shape[0]):
        got = peakfit.fit_peaks(x, Y[f], centers, x_bin_size=0.25, fit_roi_padding=40, device=cuda)
        assert got.shape == ref[f].shape
        for k in range(ref.shape[1]):
            r, o = ref[f, k], got[k]
            assert abs(o[1] - r[1]) <= 1e-4, (f, k, o[1], r[1])                 # centre (x units)
            assert abs(o[4] - r[4]) <= 1e-4 * r[4], (f, k, o[4], r[4])           # FWHM
            assert abs(o[0] - r[0]) <= 1e-4 * r[0], (f, k, o[0], r[0])           # area
            assert abs(o[5] - r[5]) <= 1e-3, (f, k, o[5], r[5])                 # mixing
            assert abs(o[6] - r[6]) <= 1e-3 * r[6], (f, k, o[6], r[6])           # chi2 / dof


def test_batched_lineouts_match_single_calls(cuda):
    g = np.load(GOLDEN / "peakfit.npz")
    x, Y, centers = g["x"], g["lineouts"], g["centers"]
    fp = FitPlan(x, centers, kind="peaks", half_window=40, x_bin=0.25, device=cuda)
    r = fp.run(torch.from_numpy(Y).to(cuda))
    assert (r.iters >= 0).all()
    for f in range(Y.shape[0]):
        one = fp.run(torch.from_numpy(Y[f:f + 1]).to(cuda))
        assert torch.equal(one.params[0], r.params[f])       # a series' fit does not depend on the batch
    fp.close()


def _pv(x, p, n_p):
    mu, bg = p[3 * n_p], p[3 * n_p + 1]
    out = np.full_like(x, bg)
    for k in range(n_p):
        c, G, I = p[3 * k: 3 * k + 3]
        dr2 = (x - c) ** 2
        out += I * (mu / (1 + 4 * dr2 / G ** 2) + (1 - mu) * np.exp(-4 * np.log(2) * dr2 / G ** 2))
    return out


def _lsq_eta(R, I, locs, step):
    """pf_fit_singlet_pv / pf_fit_doublet_pv start and bounds (PeakFit.c:922-1110), FP64 bounded
    least squares; returns centres and SNR."""
    n = R.size
    bg0 = max(0.0, 0.5 * (I[0] + I[-1]))
    mx = I.max()
    if len(locs) == 1:
        p0 = [locs[0], 3 * step, mx - bg0, 0.5, bg0]
        lb = [R[0], step / 2, (mx - bg0) / 100, 0, 0]
        ub = [R[-1], step * n / 2, mx * 1.5, 1, bg0 * 1.5 if bg0 > 0 else mx * 0.5]
    else:
        ig = max(mx - bg0, 1e-6)
        cm = 0.5 * (locs[0] + locs[1])
        p0 = [locs[0], 3 * step, ig / 2, locs[1], 3 * step, ig / 2, 0.5, bg0]
        lb = [R[0], step / 2, ig / 100, cm, step / 2, ig / 100, 0, 0]
        ub = [cm, step * n / 2, mx * 1.5, R[-1], step * n / 2, mx * 1.5, 1, bg0 * 1.5 if bg0 > 0 else mx * 0.5]
    n_p = len(locs)
    res = least_squares(lambda p: _pv(R, p, n_p) - I, np.clip(p0, lb, ub), bounds=(lb, ub), method="trf",
                        x_scale="jac", xtol=1e-14, ftol=1e-14, gtol=1e-14, max_nfev=20000)
    rms = np.sqrt((res.fun ** 2).sum() / n)
    return [(res.x[3 * k], res.x[3 * k + 2] / rms) for k in range(n_p)]


def test_eta_fits_match_bounded_least_squares(cuda):
    rng = np.random.default_rng(5)
    F, n_r, n_eta, step = 2, 240, 6, 0.25
    R = 100.0 + step * (np.arange(n_r) + 0.5)
    locs = np.array([115.0, 131.0, 132.2, 150.0])       # 131.0 / 132.2 form a doublet at sep 2
    cake = np.zeros((F, n_r, n_eta), np.float64)
    for f in range(F):
        for e in range(n_eta):
            p = []
            for c in locs:
                p += [c + 0.05 * np.sin(e + f) + 0.02 * rng.standard_normal(), 1.1 + 0.1 * rng.random(),
                      800 + 300 * rng.random()]
            p += [0.4 + 0.2 * rng.random(), 90.0]
            cake[f, :, e] = _pv(R, np.array(p), len(locs)) + rng.normal(0, 1.0, n_r)
    cake[1, :, 3] = 0.0                                   # an empty eta column is skipped
    cake = cake.astype(np.float32)
    fp = FitPlan(R, locs, kind="eta", half_window=20, x_bin=step, doublet_sep=2.0, px_um=200.0, lsd_um=1e6,
                 device=cuda)
    assert fp.info() == {"n_jobs": 3, "n_valid": 4, "max_job_peaks": 2}
    r = fp.fit_cake_eta(torch.from_numpy(cake).to(cuda))
    out, it = r.params.cpu().numpy(), r.iters.cpu().numpy()
    jobs = [[0], [1, 2], [3]]
    for f in range(F):
        for e in range(n_eta):
            s = f * n_eta + e
            if f == 1 and e == 3:
                assert (it[s] == -3).all() and not out[s].any()
                continue
            prof = cake[f, :, e].astype(np.float64)
            for jb in jobs:
                lo_p, hi_p = locs[jb].min(), locs[jb].max()
                sel = (R >= lo_p - 20 * step) & (R <= hi_p + 20 * step)
                ref = _lsq_eta(R[sel], prof[sel], list(locs[jb]), step)
                for k, (c, snr) in zip(jb, ref):
                    assert it[s, k] > 0
                    assert abs(out[s, k, 1] - c) <= 1e-4, (f, e, k, out[s, k, 1], c)
                    assert abs(out[s, k, 6] - snr) <= 1e-4 * snr, (f, e, k, out[s, k, 6], snr)
                    assert abs(out[s, k, 10] - np.degrees(np.arctan(c * 200.0 / 1e6))) <= 1e-7
    fp.close()


def test_autodetect_matches_oracle_detection_and_fit_plan(cuda):
    """fitPeaksAutoDetect on the device: the peaks it keeps are the oracle's detected bins
    (SNIP + detection restated in FP64 on the CPU), fit jointly on the background-
    subtracted profile exactly as a fit plan fits them, after the reference's filter."""
    import oracle
    rng = np.random.default_rng(9)
    n, F, max_peaks = 800, 5, 4
    x = 20.0 + 0.25 * (np.arange(n) + 0.5)
    Y = []
    for f in range(F):
        y = 300.0 + 40.0 * np.sin(x / 60.0) + 0.1 * (x - x[0])
        for k, c in enumerate((40.2, 75.9, 78.4, 110.3, 180.6)):
            w = 0.8 + 0.2 * k
            y = y + (400.0 + 150 * k + 30 * f) * np.exp(-0.5 * ((x - c - 0.05 * f) / w) ** 2)
        Y.append(y + rng.normal(0, 0.5, n))
    Y = np.array(Y)
    r = peakfit.fit_autodetect(torch.from_numpy(x).to(cuda), torch.from_numpy(Y).to(cuda), max_peaks=max_peaks,
                               x_bin=0.25, roi_padding=20, snip_iter=50)
    out, found = r.params.cpu().numpy(), r.n_found.cpu().numpy()
    for f in range(F):
        corr, sel = oracle.snip_detect(x, Y[f], n_iter=50, x_bin=0.25, max_sel=min(3 * max_peaks, n // 2))
        fp = FitPlan(x, x[sel], kind="peaks", half_window=20, x_bin=0.25, device=cuda)
        ref = fp.run(torch.from_numpy(corr[None]).to(cuda)).params[0].cpu().numpy()
        fp.close()
        # the reference's filter, restated: |area| > 0 and FWHM > 0, FWHM <= max(5 median, 2 bins),
        # the largest areas, position order
        keep = [i for i in range(len(sel)) if abs(ref[i, 0]) > 0 and ref[i, 4] > 0]
        if len(keep) > 2:
            med = np.sort(ref[keep, 4])[len(keep) // 2]
            keep = [i for i in keep if ref[i, 4] <= max(5 * med, 0.5)]
        if len(keep) > max_peaks:
            keep = sorted(keep, key=lambda i: -abs(ref[i, 0]))[:max_peaks]
        keep = sorted(keep)
        assert found[f] == len(keep), (f, found[f], keep)
        for j, i in enumerate(keep):
            assert abs(out[f, j, 1] - ref[i, 1]) <= 1e-4, (f, j, out[f, j, 1], ref[i, 1])
            assert abs(out[f, j, 4] - ref[i, 4]) <= 1e-4 * ref[i, 4]
        assert not out[f, found[f]:].any()
