"""Fit-job construction of the fit plans (host logic, no GPU): the jobs fitPeaks forms
(FF_HEDM/src/PeakFit.c:292-350; _partition_into_jobs, packages/midas_integrate/midas_integrate/
peakfit.py:198-240) and the per-eta singlet/doublet jobs of IntegratorZarrOMP.c:1906-1984,
checked against plain-Python restatements of those rules."""
from pathlib import Path

import numpy as np
import pytest

from midas_b200.peakfit import FitPlan

GOLDEN = Path(__file__).resolve().parent / "golden"


def _jobs_peaks(x, locs, pad, x_bin, max_peaks=8):
    """fitPeaks' job rule restated: nearest bins within 2 bins, sorted, merged on overlap."""
    valid = []
    for p, loc in enumerate(locs):
        b = int(np.argmin(np.abs(x - loc)))
        if abs(x[b] - loc) < 2 * x_bin:
            valid.append((b, p))
    valid.sort(key=lambda t: t[0])
    jobs, ids = [], []
    for b, p in valid:
        s, e = max(0, b - pad), min(x.size - 1, b + pad)
        if jobs and s <= jobs[-1][1] and jobs[-1][2] < max_peaks:
            jobs[-1][1] = e
            jobs[-1][2] += 1
        else:
            jobs.append([s, e, 1, len(ids)])
        ids.append(p)
    return np.array(jobs, np.int32).reshape(-1, 4), np.array(ids, np.int32)


def _jobs_eta(x, locs, pad, x_bin, sep):
    n = len(locs)
    flag, pair = [0] * n, [-1] * n
    if sep > 0:
        for p in range(n - 1):
            if flag[p]:
                continue
            if abs(locs[p + 1] - locs[p]) < sep:
                flag[p], flag[p + 1], pair[p], pair[p + 1] = 1, 2, p + 1, p
    jobs, ids = [], []
    for p in range(n):
        if flag[p] == 2:
            continue
        q = pair[p] if flag[p] == 1 else -1
        lo_p = min(locs[p], locs[q]) if q >= 0 else locs[p]
        hi_p = max(locs[p], locs[q]) if q >= 0 else locs[p]
        inside = np.nonzero((x >= lo_p - pad * x_bin))[0]
        below = np.nonzero(x <= hi_p + pad * x_bin)[0]
        if inside.size == 0 or below.size == 0:
            continue
        lo, hi = int(inside[0]), int(below[-1])
        if hi - lo < 5:
            continue
        jobs.append([lo, hi, 2 if q >= 0 else 1, len(ids)])
        ids.extend(sorted([p, q], key=lambda k: locs[k]) if q >= 0 else [p])
    return np.array(jobs, np.int32).reshape(-1, 4), np.array(ids, np.int32)


def test_reference_fixture_forms_one_joint_job():
    g = np.load(GOLDEN / "peakfit.npz")
    fp = FitPlan(g["x"], g["centers"], kind="peaks", half_window=40, x_bin=0.25, device="cpu")
    jobs, ids = fp.jobs()
    assert jobs.tolist() == [[81, 161, 1, 0], [203, 324, 2, 1]]
    assert ids.tolist() == [0, 1, 2]
    assert fp.info() == {"n_jobs": 2, "n_valid": 3, "max_job_peaks": 2}
    fp.close()


@pytest.mark.parametrize("seed", range(8))
def test_peak_jobs_match_restated_rule(seed):
    rng = np.random.default_rng(seed)
    n = int(rng.integers(50, 400))
    x = 10.0 + 0.5 * (np.arange(n) + 0.5)
    locs = rng.uniform(x[0] - 3, x[-1] + 3, size=int(rng.integers(1, 14)))
    pad = int(rng.integers(2, 30))
    fp = FitPlan(x, locs, kind="peaks", half_window=pad, x_bin=0.5, device="cpu")
    jobs, ids = fp.jobs()
    rj, ri = _jobs_peaks(x, locs, pad, 0.5)
    assert np.array_equal(jobs, rj)
    assert np.array_equal(ids, ri)
    fp.close()


@pytest.mark.parametrize("seed", range(8))
def test_eta_jobs_match_restated_rule(seed):
    rng = np.random.default_rng(100 + seed)
    n = int(rng.integers(30, 300))
    x = 5.0 + 0.25 * (np.arange(n) + 0.5)
    locs = np.sort(rng.uniform(x[0] - 2, x[-1] + 2, size=int(rng.integers(1, 10))))
    if seed % 2:
        locs = locs[::-1].copy()       # the doublet rule pairs neighbours in the given order
    pad = int(rng.integers(2, 20))
    sep = float(rng.uniform(0, 4))
    fp = FitPlan(x, locs, kind="eta", half_window=pad, x_bin=0.25, doublet_sep=sep, device="cpu")
    jobs, ids = fp.jobs()
    rj, ri = _jobs_eta(x, locs, pad, 0.25, sep)
    assert np.array_equal(jobs[:, :3], rj[:, :3])
    assert np.array_equal(ids, ri)
    fp.close()


def test_host_only_plan_refuses_to_run():
    fp = FitPlan(np.arange(10.0), [5.0], kind="peaks", half_window=3, x_bin=1.0, device="cpu")
    import torch
    with pytest.raises(RuntimeError):
        fp.run(torch.zeros((1, 10), dtype=torch.float64))
    fp.close()
