"""The synthetic workloads the bench and the GPU tests run are the benchmark configurations:
frame shapes and types, geometry, bin grids, integration modes, corrections and the signal
model (rings, drift, spots).  A change to a workload that moves it off its configuration fails
here, on CPU."""
import numpy as np
import pytest

from midas_b200 import synth


def test_single_frame_config_2048_floor():
    w = synth.powder_2048()
    m = w.mapper
    assert (m.NrPixelsZ, m.NrPixelsY) == (2048, 2048) and w.frame_dtype == "uint16"
    assert w.wavelength_A == pytest.approx(0.172979) and m.Lsd == 1_000_000.0 and m.px == 200.0
    assert (m.BC_y, m.BC_z) == (1024.3, 1022.7) and (m.ty, m.tz) == (0.1, -0.05)
    assert (w.n_r, w.n_eta, w.mode) == (990, 72, "floor")
    assert w.lattice_A == pytest.approx(5.4116) and len(w.ring_radii()) == 10
    assert (w.fwhm_px, w.mix_eta) == (1.5, 0.5)


def test_sweep_config_2880_gradient():
    w = synth.sweep_2880()
    m = w.mapper
    assert (m.NrPixelsZ, m.NrPixelsY) == (2880, 2880) and w.frame_dtype == "uint16"
    assert w.n_frames == 1440 and w.amp_drift == pytest.approx(0.2)
    assert (w.n_spots, w.spot_sigma, w.spot_amp) == (50, 2.0, 5e4)
    assert (m.RBinSize, m.EtaBinSize) == (0.25, 1.0)
    assert (w.n_r, w.n_eta, w.mode) == (3960, 360, "gradient")
    assert m.SolidAngleCorrection and m.PolarizationCorrection and m.PolarizationFraction == pytest.approx(0.99)
    assert m.Parallax > 0
    assert w.name == "sweep_2880x2880_u16_3960x360_gradient"


def test_pixel_array_panel_config_int32_with_module_gaps():
    w = synth.pilatus_1679()
    m = w.mapper
    assert (m.NrPixelsY, m.NrPixelsZ) == (1475, 1679) and w.frame_dtype == "int32" and m.px == 172.0
    mask = np.asarray(w.mask()).reshape(m.NrPixelsZ, m.NrPixelsY)
    # the gaps between modules are masked, whole rows and columns of them
    assert mask.any() and not mask.all()
    assert w.module_gaps == (487, 7, 195, 17)


def test_serving_mix_spans_the_configured_sizes_and_rates():
    mix = synth.serving_mix()
    assert len(mix) == 6
    shapes = {(w.mapper.NrPixelsZ, w.mapper.NrPixelsY) for w, _ in mix}
    assert {(1024, 1024), (2048, 2048), (2880, 2880), (1679, 1475)} <= shapes
    rates = [r for _, r in mix]
    assert min(rates) >= 10 and max(rates) <= 500
    bins = [w.n_r * w.n_eta for w, _ in mix]
    assert min(bins) >= 2e4 and max(bins) <= 1.5e6
