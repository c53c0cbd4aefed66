"""Device map builder vs the reference DetectorMapper core, the batched LM fitter vs the
FP64 oracle fit, and the synthetic frame source."""
import numpy as np
import pytest
import torch

import oracle
from conftest import GOLDEN, MAPPER_CASES, load_mapper_case, rel_err
from midas_b200 import peakfit, synth
from midas_b200.kernels import CakePlan
from midas_b200.mapper import build_map

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("tag", MAPPER_CASES)
def test_device_mapper_matches_reference(cuda, tag):
    from test_mapper_host import build_with_edges
    g = load_mapper_case(tag)
    recs, nmap, mask = build_with_edges(g, 0)
    # Same source as the host build, which is bit-identical to the reference.  The device
    # build's sin/cos/atan2 round differently from the host libm, and the segment/circle
    # intersection quadratic is ill-conditioned near tangency, so a few overlap areas move
    # by ~1e-8 relative: same records, weights within 1e-6.
    np.testing.assert_array_equal(nmap, g["nmap"])
    np.testing.assert_array_equal(mask, g["bin_mask"])
    ref = g["records"]
    np.testing.assert_array_equal(recs["y"], ref["y"])
    np.testing.assert_array_equal(recs["z"], ref["z"])
    np.testing.assert_allclose(recs["frac"], ref["frac"], rtol=1e-6)
    np.testing.assert_allclose(recs["areaWeight"], ref["areaWeight"], rtol=1e-6)
    np.testing.assert_allclose(recs["deltaR"], ref["deltaR"], rtol=1e-6, atol=1e-6)


def test_device_mapper_equals_host_mapper_on_synthetic_workload(cuda):
    w = synth.scaled(synth.sweep_2880(), 8)
    pm_d, _ = build_map(w.mapper, device=0)
    pm_h, _ = build_map(w.mapper, device=-1)
    np.testing.assert_array_equal(pm_d.counts, pm_h.counts)
    np.testing.assert_array_equal(pm_d.pxList["y"], pm_h.pxList["y"])
    np.testing.assert_allclose(pm_d.pxList["frac"], pm_h.pxList["frac"], rtol=1e-6)


def _lineouts(kind, F, rng):
    x = 200.0 + 0.25 * (np.arange(1200) + 0.5)
    peaks = np.array([260.3, 331.77, 402.1, 480.55])
    Y = []
    for f in range(F):
        y = 90.0 + 0.01 * (x - x[0])
        for k, c in enumerate(peaks):
            cc = c + 0.05 * rng.standard_normal()
            if kind == 0:
                h, w, e = 3000.0 * (1 + 0.2 * k), 1.5 + 0.2 * rng.random(), 0.3 + 0.4 * rng.random()
                u = (x - cc) / (w / 2)
                y = y + h * (e / (1 + u * u) + (1 - e) * np.exp(-np.log(2) * u * u))
            else:
                A = 6000.0 * (1 + 0.1 * k)
                fwhm = 1.6 + 0.2 * rng.random()
                sg = fwhm / (2 * np.sqrt(2 * np.log(2)))
                e = 0.5
                G = np.exp(-0.5 * ((x - cc) / sg) ** 2) / (sg * np.sqrt(2 * np.pi))
                L = (fwhm / 2 / np.pi) / ((x - cc) ** 2 + (fwhm / 2) ** 2)
                y = y + A * (e * L + (1 - e) * G)
        Y.append(y + rng.normal(0, 2.0, size=x.size))
    return x, np.array(Y), peaks


@pytest.mark.parametrize("kind", [0, 1])
def test_fitter_matches_fp64_oracle(cuda, kind):
    rng = np.random.default_rng(21 + kind)
    x, Y, peaks = _lineouts(kind, 24, rng)
    res = peakfit.fit_batch(torch.from_numpy(x).to(cuda), torch.from_numpy(Y).to(cuda),
                            torch.from_numpy(peaks).to(cuda), model=kind, half_window=60, x_bin=0.25,
                            max_iter=200, px_um=200.0, lsd_um=1e6)
    out, iters = res.params.cpu().numpy(), res.iters.cpu().numpy()
    assert (iters > 0).all()
    for f in range(Y.shape[0]):
        for k, c in enumerate(peaks):
            ref, it = oracle.fit(x, Y[f], c, half_window=60, model=kind, max_iter=500, x_bin=0.25,
                                 px_um=200.0, lsd_um=1e6)
            assert it > 0
            assert abs(out[f, k, 1] - ref[1]) <= 1e-4, (f, k, out[f, k, 1], ref[1])   # centre, px
            assert abs(out[f, k, 4] - ref[4]) <= 1e-4 * max(1.0, ref[4])              # FWHM
            assert abs(out[f, k, 10] - ref[10]) <= 1e-6                                # 2-theta deg


def test_fitter_rejects_far_peaks(cuda):
    x = torch.linspace(0, 10, 41, dtype=torch.float64, device=cuda)
    y = torch.ones((2, 41), dtype=torch.float64, device=cuda)
    res = peakfit.fit_batch(x, y, torch.tensor([50.0, 5.0], dtype=torch.float64, device=cuda), model=0,
                            half_window=10, x_bin=0.25)
    assert res.iters[0, 0].item() == -1


def test_synthetic_frames(cuda):
    w = synth.scaled(synth.sweep_2880(), 8)
    fr = w.frames(0, 3)
    fr2 = w.frames(1, 1)
    assert fr.dtype == torch.uint16 and fr.shape == (3, *w.shape)
    assert torch.equal(fr[1], fr2[0])                     # counter-based: frame 1 is frame 1
    dark = w.dark()
    m = (fr[0].float() - dark).mean().item()
    assert 80 < m < 5000
    assert not torch.equal(fr[0], fr[2])


def test_synthetic_workload_end_to_end(cuda):
    """Map on the GPU -> frames on the GPU -> batched caking -> FP64 oracle on the same frames."""
    w = synth.scaled(synth.sweep_2880(), 8)
    pm, _ = build_map(w.mapper, device=0)
    plan = CakePlan(pm, n_r=w.n_r, n_eta=w.n_eta, n_pixels_y=w.mapper.NrPixelsY,
                    n_pixels_z=w.mapper.NrPixelsZ, mode=w.mode, bc_y=w.mapper.BC_y, bc_z=w.mapper.BC_z,
                    device=cuda)
    dark = w.dark()
    plan.set_dark(dark.cpu().numpy())
    fr = w.frames(0, 5)
    ck, aw, sm = plan.integrate(fr)
    sub = fr.cpu().numpy().astype(np.float32) - dark.cpu().numpy()[None]
    recs = pm.pxList
    nmap = pm.nmap_pairs()
    area = oracle.area_in(recs, nmap, pm.n_bins, w.mapper.NrPixelsY, w.mapper.NrPixelsZ)
    for f in range(5):
        rc, _ = oracle.integrate(recs, nmap, pm.n_bins, w.mapper.NrPixelsY, w.mapper.NrPixelsZ,
                                 sub[f].astype(np.float64), mode=w.mode, bc_y=w.mapper.BC_y, bc_z=w.mapper.BC_z)
        assert rel_err(ck[f].cpu().numpy(), rc)[0] <= 1e-6
        raw_, _ = oracle.profile(rc, area, w.n_r, w.n_eta)
        assert rel_err(aw[f].cpu().numpy(), raw_)[0] <= 1e-6
