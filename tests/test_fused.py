"""Fused multi-shift maps (build_fused_geometry, packages/midas_integrate/midas_integrate/
fused_csr.py:139-296) on the host: the oracle's naive multi-map averaging and the fused
weights of mi_fused_csr both reproduce the reference's fused cakes (tests/golden/fused.npz,
made by the reference itself from its own shifted maps)."""
import numpy as np
import pytest

import oracle
from conftest import load_fused_case, rel_err
from midas_b200 import fused


def _apply(row_ptr, col, w, image):
    img = np.asarray(image, np.float64).reshape(-1)
    out = np.zeros(row_ptr.size - 1)
    for b in range(out.size):
        s = slice(row_ptr[b], row_ptr[b + 1])
        out[b] = np.dot(w[s], img[col[s]])
    return out


@pytest.mark.parametrize("mode", ["bilinear", "gradient"])
def test_oracle_naive_average_matches_reference_fused_cake(mode):
    g = load_fused_case()
    got = oracle.fused_average(g["nmaps"], g["r_axes"], g["n_eta"], g["ny"], g["nz"], g["image"], mode=mode,
                               bc_y=g["bc_y"], bc_z=g["bc_z"])
    assert rel_err(got, g[f"cake_{mode}"])[0] <= 1e-12


@pytest.mark.parametrize("mode", ["bilinear", "gradient"])
def test_fused_csr_matches_reference_fused_cake(mode):
    g = load_fused_case()
    row_ptr, col, w = fused.fused_csr(g["maps"], g["r_axes"], n_eta=g["n_eta"], n_pixels_y=g["ny"],
                                      n_pixels_z=g["nz"], mode=mode, bc_y=g["bc_y"], bc_z=g["bc_z"])
    assert row_ptr.size == g["r_axes"][0].size * g["n_eta"] + 1 and row_ptr[-1] == col.size
    assert np.all(np.diff(row_ptr) >= 0) and np.all(w != 0)
    assert rel_err(_apply(row_ptr, col, w, g["image"]), g[f"cake_{mode}"])[0] <= 1e-12


def test_one_shift_is_the_normalised_map():
    """n_shifts = 1: the fused weights are the shift's own weights over its bin areas."""
    g = load_fused_case()
    rec, nm = g["nmaps"][0]
    n_bins = g["r_axes"][0].size * g["n_eta"]
    row_ptr, col, w = fused.fused_csr(g["maps"][:1], g["r_axes"][:1], n_eta=g["n_eta"], n_pixels_y=g["ny"],
                                      n_pixels_z=g["nz"], mode="bilinear", bc_y=g["bc_y"], bc_z=g["bc_z"])
    want, _ = oracle.integrate(rec, nm, n_bins, g["ny"], g["nz"], g["image"], mode="bilinear", semantics="py",
                               normalize=True, bc_y=g["bc_y"], bc_z=g["bc_z"])
    assert rel_err(_apply(row_ptr, col, w, g["image"]), want)[0] <= 1e-12


def test_fused_host_maps_from_the_mapper():
    """Shifted maps from this library's host DetectorMapper: R axes shifted by k / n of a
    bin, and the fused weights equal the oracle's naive average on a random image."""
    from midas_b200.mapper import MapperParams
    p = MapperParams(NrPixelsY=40, NrPixelsZ=36, px=200.0, Lsd=250000.0, BC_y=19.4, BC_z=17.7, ty=0.1,
                     RMin=2.0, RMax=18.0, RBinSize=1.0, EtaBinSize=20.0)
    maps, axes = fused.shift_maps(p, 3, device=-1)
    assert np.allclose(axes[1] - axes[0], 1.0 / 3) and np.allclose(axes[2] - axes[0], 2.0 / 3)
    img = np.random.default_rng(3).uniform(0, 100, size=(36, 40))
    row_ptr, col, w = fused.fused_csr(maps, axes, n_eta=p.n_eta, n_pixels_y=40, n_pixels_z=36, mode="gradient",
                                      bc_y=p.BC_y, bc_z=p.BC_z)
    want = oracle.fused_average([(m.pxList, m.nmap_pairs()) for m in maps], axes, p.n_eta, 40, 36, img,
                                mode="gradient", bc_y=p.BC_y, bc_z=p.BC_z)
    assert rel_err(_apply(row_ptr, col, w, img), want)[0] <= 1e-12


def test_fused_rejects_bad_input():
    g = load_fused_case()
    with pytest.raises(ValueError):
        fused.fused_csr(g["maps"], g["r_axes"], n_eta=g["n_eta"], n_pixels_y=g["ny"], n_pixels_z=g["nz"],
                        mode="floor")
    with pytest.raises(ValueError):
        fused.fused_csr(g["maps"], g["r_axes"][:2], n_eta=g["n_eta"], n_pixels_y=g["ny"], n_pixels_z=g["nz"])
    with pytest.raises(RuntimeError):   # a detector without rows
        fused.fused_csr(g["maps"], g["r_axes"], n_eta=g["n_eta"], n_pixels_y=g["ny"], n_pixels_z=0)
