"""The oracle's restatement of fitPeaksAutoDetect's background subtraction and detection
(FF_HEDM/src/PeakFit.c:549-755), on the CPU: SNIP leaves a smooth background near zero,
the detected bins sit on the synthetic peaks, and candidates closer than min_sep merge."""
import numpy as np

import oracle


def _profile(rng, n=800, centres=(40.2, 75.9, 110.3, 180.6), noise=0.5):
    x = 20.0 + 0.25 * (np.arange(n) + 0.5)
    y = 300.0 + 40.0 * np.sin(x / 60.0) + 0.1 * (x - x[0])
    for k, c in enumerate(centres):
        w = 0.8 + 0.2 * k
        y += (400.0 + 150 * k) * np.exp(-0.5 * ((x - c) / w) ** 2)
    return x, y + rng.normal(0, noise, n)


def test_snip_and_detection_find_the_peaks():
    rng = np.random.default_rng(0)
    x, y = _profile(rng)
    corr, sel = oracle.snip_detect(x, y, n_iter=50, x_bin=0.25, max_sel=12)
    assert corr.shape == y.shape and (corr >= 0).all()
    for c in (40.2, 75.9, 110.3, 180.6):
        assert np.min(np.abs(x[sel] - c)) < 0.5, (c, x[sel])
    assert np.all(np.diff(sel) >= 3)
    # away from the peaks the corrected profile is small against the peak heights
    far = np.all([np.abs(x - c) > 8 for c in (40.2, 75.9, 110.3, 180.6)], axis=0)
    assert np.median(corr[far]) < 20.0


def test_no_background_and_short_profiles():
    x = np.arange(8.0)
    corr, sel = oracle.snip_detect(x, np.ones(8), n_iter=0, x_bin=1.0, max_sel=3)
    assert sel.size == 0 and np.array_equal(corr, np.ones(8))
