"""The FP64 oracle is pinned to the reference: golden vectors from the reference's own
midas_integrate kernels (build_csr/integrate/profile_1d in FP64) and from its compiled
IntegrationCore.c (integration_apply_map); variance propagation (integrate_with_variance,
profile_1d_with_variance), hybrid payload decoding and dark averaging (image.py)."""
import numpy as np
import pytest

import oracle
from conftest import (KERNEL_CASES, MAPPER_CASES, VARIANCE_CASES, load_image_case, load_kernels_case,
                      load_mapper_case, load_variance_case)


@pytest.mark.parametrize("tag", KERNEL_CASES)
@pytest.mark.parametrize("mode", ["floor", "bilinear", "gradient"])
@pytest.mark.parametrize("norm", [True, False])
def test_oracle_matches_reference_python(tag, mode, norm):
    g = load_kernels_case(tag)
    nb = g["n_r"] * g["n_eta"]
    ck, _ = oracle.integrate(g["records"], g["nmap"], nb, g["ny"], g["nz"], g["image"], mode=mode,
                             normalize=norm, bc_y=g["bc_y"], bc_z=g["bc_z"])
    key = f"{mode}_{'n' if norm else 'r'}"
    np.testing.assert_allclose(ck, g["cake_" + key], rtol=1e-12, atol=1e-9)
    area = oracle.area_in(g["records"], g["nmap"], nb, g["ny"], g["nz"])
    np.testing.assert_allclose(area, g["area_per_bin"], rtol=1e-12, atol=0)
    aw, sm = oracle.profile(ck, area, g["n_r"], g["n_eta"])
    np.testing.assert_allclose(aw, g["aw_" + key], rtol=1e-12, atol=1e-9)
    np.testing.assert_allclose(sm, g["sm_" + key], rtol=1e-12, atol=1e-9)


@pytest.mark.parametrize("tag", MAPPER_CASES)
@pytest.mark.parametrize("mode", ["bilinear", "gradient"])
def test_oracle_matches_reference_integration_core(tag, mode):
    """integration_apply_map (IntegrationCore.c) sums vs oracle raw sums of (image - dark).
    IntegrationCore normalises by every record's areaWeight: identical to the in-bounds
    area for DetectorMapper maps, whose records are all on the detector."""
    g = load_mapper_case(tag)
    nb = g["nmap"].shape[0]
    img = g["image"] - g["dark"]
    ck, area = oracle.integrate(g["records"], g["nmap"], nb, g["ny"], g["nz"], img, mode=mode,
                                normalize=False, bc_y=g["bc_y"], bc_z=g["bc_z"])
    # IntegrationCore floors the FP64 sample position through floorf(): a position a few
    # 1e-8 px below an integer rounds up in float, giving a negative fraction.  The Python
    # reference (np.floor) and the oracle do not, so a handful of bins differ at ~1e-8.
    np.testing.assert_allclose(ck, g[f"ic_sums_{mode}"], rtol=1e-7, atol=1e-9)
    exact = np.isclose(ck, g[f"ic_sums_{mode}"], rtol=1e-12, atol=1e-12)
    assert exact.mean() > 0.999
    np.testing.assert_allclose(area, g[f"ic_norms_{mode}"], rtol=1e-6, atol=1e-9)


def test_oracle_gpustream_semantics_area_covers_all_records():
    g = load_kernels_case("a")
    nb = g["n_r"] * g["n_eta"]
    _, a_py = oracle.integrate(g["records"], g["nmap"], nb, g["ny"], g["nz"], g["image"], semantics="py")
    _, a_gs = oracle.integrate(g["records"], g["nmap"], nb, g["ny"], g["nz"], g["image"],
                               semantics="gpustream")
    assert np.all(a_gs >= a_py - 1e-12)
    assert np.any(a_gs > a_py + 1e-6)          # the case has off-detector records


@pytest.mark.skipif(not oracle.ref_available(), reason="reference C sources not compiled here")
@pytest.mark.parametrize("tag", MAPPER_CASES)
def test_reference_integrator_reproduces_fixture(tag):
    g = load_mapper_case(tag)
    n_r, n_eta = g["r_lo"].size, g["eta_lo"].size
    sums, norms = oracle.ref_integrate(g["records"], g["nmap"], n_r, n_eta, g["image"], g["ny"], g["nz"],
                                       dark=g["dark"], bc_y=g["bc_y"], bc_z=g["bc_z"], gradient=1, n_threads=2)
    np.testing.assert_allclose(sums, g["ic_sums_gradient"], rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("tag", MAPPER_CASES)
@pytest.mark.parametrize("mode", ["bilinear", "gradient"])
def test_oracle_ic_semantics_reproduces_integration_core(tag, mode):
    """Semantics 'ic' restates integration_apply_map itself (float-rounded floorf base
    pixel included): the fixture's IntegrationCore sums and norms to 1e-12."""
    g = load_mapper_case(tag)
    nb = g["nmap"].shape[0]
    ck, area = oracle.integrate(g["records"], g["nmap"], nb, g["ny"], g["nz"], g["image"] - g["dark"],
                                mode=mode, semantics="ic", normalize=False, bc_y=g["bc_y"], bc_z=g["bc_z"])
    np.testing.assert_allclose(ck, g[f"ic_sums_{mode}"], rtol=1e-12, atol=1e-9)
    np.testing.assert_allclose(area, g[f"ic_norms_{mode}"], rtol=1e-12, atol=1e-12)


@pytest.mark.skipif(not oracle.ref_available(), reason="reference C sources not compiled here")
def test_oracle_ic_semantics_matches_integration_core_at_detector_scale():
    """On a 1440x1440 detector positions reach ~1440 px, where a float holds them to
    ~1e-4 px: IntegrationCore's floorf() then picks the upper pixel for positions just
    below an integer and extrapolates, moving some bins by ~1e-5 relative from the
    midas_integrate result.  Semantics 'ic' reproduces that; 'py' does not."""
    from midas_b200 import synth
    from midas_b200.mapper import build_map
    w = synth.scaled(synth.sweep_2880(), 2)
    pm, _ = build_map(w.mapper, device=-1)
    ny, nz = w.mapper.NrPixelsY, w.mapper.NrPixelsZ
    rng = np.random.default_rng(5)
    img = rng.poisson(300.0, size=(nz, ny)).astype(np.float64)
    dark = np.round(100 + 5 * rng.standard_normal((nz, ny)), 3)
    sums, norms = oracle.ref_integrate(pm.pxList, pm.nmap_pairs(), w.n_r, w.n_eta, img, ny, nz, dark=dark,
                                       bc_y=w.mapper.BC_y, bc_z=w.mapper.BC_z, gradient=1, n_threads=8)
    ck, area = oracle.integrate(pm.pxList, pm.nmap_pairs(), pm.n_bins, ny, nz, img - dark, mode="gradient",
                                semantics="ic", normalize=False, bc_y=w.mapper.BC_y, bc_z=w.mapper.BC_z)
    np.testing.assert_allclose(ck, sums, rtol=1e-10, atol=1e-8)
    np.testing.assert_allclose(area, norms, rtol=1e-12, atol=1e-12)
    py, _ = oracle.integrate(pm.pxList, pm.nmap_pairs(), pm.n_bins, ny, nz, img - dark, mode="gradient",
                             semantics="py", normalize=False, bc_y=w.mapper.BC_y, bc_z=w.mapper.BC_z)
    assert np.max(np.abs(py - sums) / np.maximum(np.abs(sums), 1.0)) > 1e-7


# ---- variance propagation, hybrid payloads, dark averaging ---------------------------


@pytest.mark.parametrize("tag", VARIANCE_CASES)
@pytest.mark.parametrize("mode", ["floor", "bilinear", "gradient"])
@pytest.mark.parametrize("norm", [True, False])
def test_oracle_variance_matches_reference_python(tag, mode, norm):
    """integrate_with_variance / profile_1d_with_variance of the reference (FP64 CSR with
    squared coalesced weights) against the oracle's per-bin coalescing."""
    g = load_variance_case(tag)
    nb = g["n_r"] * g["n_eta"]
    key = f"{mode}_{'n' if norm else 'r'}"
    kw = dict(mode=mode, normalize=norm, bc_y=g["bc_y"], bc_z=g["bc_z"])
    ck, _ = oracle.integrate(g["records"], g["nmap"], nb, g["ny"], g["nz"], g["image"], **kw)
    np.testing.assert_allclose(ck, g["int_" + key], rtol=1e-12, atol=1e-9)
    var = oracle.integrate_var(g["records"], g["nmap"], nb, g["ny"], g["nz"], g["var_image"], **kw)
    np.testing.assert_allclose(var, g["var_" + key], rtol=1e-12, atol=1e-9)
    area = g["area_per_bin"]
    aw, sm = oracle.profile(ck, area, g["n_r"], g["n_eta"])
    vaw, vsm = oracle.profile_var(var, area, g["n_r"], g["n_eta"])
    np.testing.assert_allclose(aw, g["i1_area_weighted_" + key], rtol=1e-12, atol=1e-9)
    np.testing.assert_allclose(sm, g["i1_simple_mean_" + key], rtol=1e-12, atol=1e-9)
    np.testing.assert_allclose(vaw, g["v1_area_weighted_" + key], rtol=1e-12, atol=1e-9)
    np.testing.assert_allclose(vsm, g["v1_simple_mean_" + key], rtol=1e-12, atol=1e-9)


def test_oracle_variance_poisson_default_and_coalescing():
    g = load_variance_case("a")
    nb = g["n_r"] * g["n_eta"]
    kw = dict(mode="bilinear", normalize=True, bc_y=g["bc_y"], bc_z=g["bc_z"])
    var = oracle.integrate_var(g["records"], g["nmap"], nb, g["ny"], g["nz"], g["image"], **kw)
    np.testing.assert_allclose(var, g["var_poisson_bilinear_n"], rtol=1e-12, atol=1e-9)
    # coalescing matters: squaring the per-record terms instead gives a different answer
    # wherever two records of a bin share a pixel
    assert var.sum() > 0


@pytest.mark.parametrize("k", [0, 1, 2])
def test_oracle_hybrid_decode_matches_reference(k):
    g = load_image_case()
    out = oracle.decode_hybrid(g[f"payload_{k}"].tobytes(), int(g["ny"]), int(g["nz"]))
    np.testing.assert_array_equal(out, g[f"decoded_{k}"])


def test_oracle_dark_average_matches_reference():
    g = load_image_case()
    mean = oracle.average_frames(g["dark_frames"])
    # the reference returns the FP64 mean; the stream server stores it as float
    np.testing.assert_array_equal(mean, g["dark_mean"].astype(np.float32))


def test_oracle_bin_table_columns():
    """R/eta centres, 2-theta = atan(R px / Lsd), Q = 4 pi / lambda sin(theta); the area column
    is the in-bounds area wherever no record sits in (-1, 0) (case a has integer positions)."""
    g = load_kernels_case("a")
    n_r, n_eta = g["n_r"], g["n_eta"]
    r_lo = 10.0 + np.arange(n_r)
    e_lo = -180.0 + 30.0 * np.arange(n_eta)
    t = oracle.bin_table(g["records"], g["nmap"], n_r, n_eta, g["ny"], g["nz"], r_lo, r_lo + 1, e_lo, e_lo + 30,
                         200.0, 1e6, 0.172979)
    rm = np.repeat(r_lo + 0.5, n_eta)
    np.testing.assert_allclose(t[:, 0], rm)
    np.testing.assert_allclose(t[:, 1], np.degrees(np.arctan(rm * 200.0 / 1e6)), rtol=1e-14)
    np.testing.assert_allclose(t[:, 2], np.tile(e_lo + 15.0, n_r))
    np.testing.assert_allclose(t[:, 3], g["area_per_bin"], rtol=1e-12)
    q = 4 * np.pi / 0.172979 * np.sin(np.arctan(rm * 200.0 / 1e6) / 2)
    np.testing.assert_allclose(t[:, 4], q, rtol=1e-14)


@pytest.mark.parametrize("tag", MAPPER_CASES)
@pytest.mark.parametrize("mode", ["bilinear", "gradient"])
def test_oracle_omp_semantics_from_integration_core_sums(tag, mode):
    """Semantics 'omp' (IntegratorZarrOMP.c:1709-1778) applies the OpenMP loop's rules to the
    IntegrationCore sums: a nonzero sum divided by the whole area.  Pinned on the compiled
    reference integrator's sums and norms recorded in the fixture; the lineout is the mean
    of the nonzero, non-NaN bins of each row (:1829-1843) after the bin mask's NaNs."""
    g = load_mapper_case(tag)
    nb = g["nmap"].shape[0]
    n_r, n_eta = g["r_lo"].size, g["eta_lo"].size
    ck, area = oracle.integrate(g["records"], g["nmap"], nb, g["ny"], g["nz"], g["image"] - g["dark"],
                                mode=mode, semantics="omp", normalize=True, bc_y=g["bc_y"], bc_z=g["bc_z"])
    sums, norms = g[f"ic_sums_{mode}"], g[f"ic_norms_{mode}"]
    want = np.where(sums != 0, sums / np.where(norms != 0, norms, 1.0), 0.0)
    np.testing.assert_allclose(ck, want, rtol=1e-10, atol=1e-12)
    mask = np.random.default_rng(3).random(nb) < 0.05      # bins holding a masked pixel
    ck = np.where(mask, np.nan, ck)
    a_in = oracle.area_in(g["records"], g["nmap"], nb, g["ny"], g["nz"])
    aw, sm = oracle.profile_omp(ck, a_in, n_r, n_eta)
    v = ck.reshape(n_r, n_eta)
    ok = (v != 0) & ~np.isnan(v)
    want_sm = np.where(ok.sum(1) > 0, np.where(ok, v, 0).sum(1) / np.maximum(ok.sum(1), 1), 0.0)
    np.testing.assert_allclose(sm, want_sm, rtol=1e-12, atol=1e-12)
