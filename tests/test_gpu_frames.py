"""Parity of the device-side variance propagation, hybrid (dtype 6) payload decoding, dark
averaging and per-bin axis table with the reference's golden outputs and the oracle,
called through the C ABI."""
import numpy as np
import pytest
import torch

import oracle
from conftest import (MAPPER_CASES, VARIANCE_CASES, load_image_case, load_mapper_case, load_variance_case,
                      rel_err)
from midas_b200 import _lib as L
from midas_b200.bin_io import from_arrays
from midas_b200.image import HybridDecoder, average_dark_frames, average_frames, decode_hybrid_payload
from midas_b200.kernels import CakePlan, build_csr, integrate_with_variance, profile_1d_with_variance

pytestmark = pytest.mark.gpu

# cake bins and lineouts: <= 1e-6 relative to FP64 (tau-guarded, as the caking tests)
TOL = 1e-6


@pytest.mark.parametrize("tag", VARIANCE_CASES)
@pytest.mark.parametrize("mode", ["floor", "bilinear", "gradient"])
@pytest.mark.parametrize("norm", [True, False])
def test_variance_api_matches_reference_golden(cuda, tag, mode, norm):
    """integrate_with_variance + profile_1d_with_variance against the reference package's
    FP64 output on the same map, image and variance image."""
    g = load_variance_case(tag)
    pm = from_arrays(g["records"], g["nmap"])
    geom = build_csr(pm, n_r=g["n_r"], n_eta=g["n_eta"], n_pixels_y=g["ny"], n_pixels_z=g["nz"], device=cuda,
                     dtype=torch.float64, bc_y=g["bc_y"], bc_z=g["bc_z"], compute_variance=True)
    key = f"{mode}_{'n' if norm else 'r'}"
    img = torch.from_numpy(g["image"].astype(np.float32)).to(cuda)
    var = torch.from_numpy(g["var_image"].astype(np.float32)).to(cuda)
    I, V = integrate_with_variance(img, geom, mode=mode, normalize=norm, variance_image=var)
    assert I.shape == V.shape == (g["n_r"], g["n_eta"])
    assert rel_err(I.cpu().numpy(), g["int_" + key])[0] <= TOL
    assert rel_err(V.cpu().numpy(), g["var_" + key])[0] <= TOL
    for pm_ in ("area_weighted", "simple_mean"):
        i1, v1 = profile_1d_with_variance(I, V, geom, mode=pm_)
        assert rel_err(i1.cpu().numpy(), g[f"i1_{pm_}_{key}"])[0] <= TOL
        assert rel_err(v1.cpu().numpy(), g[f"v1_{pm_}_{key}"])[0] <= TOL


def test_variance_poisson_default(cuda):
    g = load_variance_case("a")
    pm = from_arrays(g["records"], g["nmap"])
    geom = build_csr(pm, n_r=g["n_r"], n_eta=g["n_eta"], n_pixels_y=g["ny"], n_pixels_z=g["nz"], device=cuda,
                     dtype=torch.float64, bc_y=g["bc_y"], bc_z=g["bc_z"], compute_variance=True)
    img = torch.from_numpy(g["image"].astype(np.float32)).to(cuda)
    _, V = integrate_with_variance(img, geom, mode="bilinear")
    assert rel_err(V.cpu().numpy(), g["var_poisson_bilinear_n"])[0] <= TOL


def test_variance_needs_compute_variance(cuda):
    g = load_variance_case("a")
    pm = from_arrays(g["records"], g["nmap"])
    geom = build_csr(pm, n_r=g["n_r"], n_eta=g["n_eta"], n_pixels_y=g["ny"], n_pixels_z=g["nz"], device=cuda)
    with pytest.raises(RuntimeError, match="compute_variance=True"):
        integrate_with_variance(torch.zeros(g["nz"], g["ny"], device=cuda), geom)


@pytest.mark.parametrize("tag", VARIANCE_CASES)
@pytest.mark.parametrize("mode", ["floor", "bilinear", "gradient"])
@pytest.mark.parametrize("sem", ["py", "gpustream"])
@pytest.mark.parametrize("enc", ["runs", "csr"])
def test_variance_plan_batch_matches_oracle(cuda, tag, mode, sem, enc):
    """A batch of variance maps through one variance plan: every frame's bin variances and
    both propagated lineout variances against the oracle (coalesced squared weights)."""
    g = load_variance_case(tag)
    pm = from_arrays(g["records"], g["nmap"])
    plan = CakePlan(pm, n_r=g["n_r"], n_eta=g["n_eta"], n_pixels_y=g["ny"], n_pixels_z=g["nz"], mode=mode,
                    semantics=sem, bc_y=g["bc_y"], bc_z=g["bc_z"], device=cuda, encoding=enc, variance=True)
    rng = np.random.default_rng(3)
    frames = np.stack([g["var_image"] * s for s in rng.uniform(0.5, 2.0, 5)]).astype(np.float32)
    ck, aw, sm = plan.integrate(torch.from_numpy(frames).to(cuda))
    nb = g["n_r"] * g["n_eta"]
    area = oracle.area_in(g["records"], g["nmap"], nb, g["ny"], g["nz"])
    for f in range(frames.shape[0]):
        rv = oracle.integrate_var(g["records"], g["nmap"], nb, g["ny"], g["nz"], frames[f].astype(np.float64),
                                  mode=mode, semantics=sem, bc_y=g["bc_y"], bc_z=g["bc_z"])
        vaw, vsm = oracle.profile_var(rv, area, g["n_r"], g["n_eta"])
        assert rel_err(ck[f].cpu().numpy(), rv)[0] <= TOL
        assert rel_err(aw[f].cpu().numpy(), vaw)[0] <= TOL
        assert rel_err(sm[f].cpu().numpy(), vsm)[0] <= TOL
    # kernel (c) on the variance cake gives the same propagated lineouts
    paw, psm = plan.profile(ck)
    assert rel_err(paw.cpu().numpy(), aw.cpu().numpy())[0] <= TOL
    assert rel_err(psm.cpu().numpy(), sm.cpu().numpy())[0] <= TOL


def test_variance_plan_has_no_plain_path(cuda):
    g = load_variance_case("a")
    pm = from_arrays(g["records"], g["nmap"])
    plan = CakePlan(pm, n_r=g["n_r"], n_eta=g["n_eta"], n_pixels_y=g["ny"], n_pixels_z=g["nz"], device=cuda,
                    variance=True)
    with pytest.raises(L.MidasError, match="variance"):
        plan.integrate_plain(torch.zeros(g["nz"], g["ny"], device=cuda))


# ---- hybrid payloads ------------------------------------------------------------------
@pytest.mark.parametrize("k", [0, 1, 2])
def test_hybrid_decode_matches_reference(cuda, k):
    g = load_image_case()
    ny, nz = int(g["ny"]), int(g["nz"])
    payload = g[f"payload_{k}"].tobytes()
    out = decode_hybrid_payload(payload, n_pixels_y=ny, n_pixels_z=nz, device=cuda)
    np.testing.assert_array_equal(out.cpu().numpy(), g[f"decoded_{k}"])
    np.testing.assert_array_equal(out.cpu().numpy(), oracle.decode_hybrid(payload, ny, nz))


def test_hybrid_decoder_reuse_and_dark(cuda):
    """A decoder reused across payloads of different overflow counts; the decoded frame with
    the dark subtracted by kernel (a) equals the reference's fused expand/overlay kernels,
    (float)raw - dark, bit for bit."""
    g = load_image_case()
    ny, nz = int(g["ny"]), int(g["nz"])
    dec = HybridDecoder(ny, nz, max_overflow=1, device=cuda)
    dark = np.random.default_rng(5).uniform(80, 120, size=(nz, ny)).astype(np.float32)
    dark_d = torch.from_numpy(dark).to(cuda)
    for k in (1, 0, 2, 1):
        fr = dec.decode(g[f"payload_{k}"].tobytes())
        sub = torch.empty_like(fr)
        L.check(L.lib().mi_cast_dark(fr.data_ptr(), L.DT_F32, ny * nz, 1, dark_d.data_ptr(), sub.data_ptr(),
                                     L.stream_ptr()), "mi_cast_dark")
        np.testing.assert_array_equal(sub.cpu().numpy(), g[f"decoded_{k}"] - dark)
    dec.check()


def test_hybrid_rejects_bad_payloads(cuda):
    g = load_image_case()
    ny, nz = int(g["ny"]), int(g["nz"])
    payload = g["payload_1"].tobytes()
    with pytest.raises(ValueError, match="hybrid payload size"):
        decode_hybrid_payload(payload[:-1], n_pixels_y=ny, n_pixels_z=nz, device=cuda)
    with pytest.raises(ValueError, match="too small"):
        decode_hybrid_payload(payload[:10], n_pixels_y=ny, n_pixels_z=nz, device=cuda)
    # an overflow index outside the frame: skipped by the kernel, reported in the status word
    n = ny * nz
    bad = (np.array([1], np.uint32).tobytes() + np.zeros(n, np.uint16).tobytes()
           + np.array([n + 3], np.int32).tobytes() + np.array([7], np.int64).tobytes())
    dec = HybridDecoder(ny, nz, device=cuda)
    fr = dec.decode(bad)
    with pytest.raises(L.MidasError) as e:
        dec.check()
    assert e.value.code == L.MI_E_RANGE
    assert float(fr.abs().max()) == 0.0
    dec.check()                                   # cleared


# ---- dark averaging -------------------------------------------------------------------
def test_average_dark_frames_matches_reference(cuda, tmp_path):
    g = load_image_case()
    ny, nz = int(g["ny"]), int(g["nz"])
    f = tmp_path / "dark.bin"
    g["dark_frames"].tofile(f)
    mean = average_dark_frames(f, n_pixels_y=ny, n_pixels_z=nz, dtype="int64", device=cuda)
    assert mean.dtype == torch.float32 and mean.shape == (nz, ny)
    np.testing.assert_array_equal(mean.cpu().numpy(), g["dark_mean"].astype(np.float32))
    with pytest.raises(ValueError, match="too small"):
        f2 = tmp_path / "short.bin"
        g["dark_frames"][0].reshape(-1)[:10].tofile(f2)
        average_dark_frames(f2, n_pixels_y=ny, n_pixels_z=nz, device=cuda)


@pytest.mark.parametrize("dt", [torch.uint16, torch.int32, torch.float32, torch.uint8])
def test_average_frames_strided(cuda, dt):
    rng = np.random.default_rng(9)
    k, nz, ny = 9, 31, 45
    big = rng.integers(0, 250, size=(k, nz + 3, ny)).astype(np.float64)
    if dt == torch.float32:
        big = big + rng.uniform(0, 1, size=big.shape)
    host = torch.from_numpy(big).to(dt)
    dev = host.to(cuda)
    sub = dev.reshape(k, -1)[:, : nz * ny]          # frame_stride > pixels
    mean = average_frames(sub)
    np.testing.assert_array_equal(mean.cpu().numpy(),
                                  oracle.average_frames(host.reshape(k, -1)[:, : nz * ny].numpy()))


# ---- per-bin axis table ---------------------------------------------------------------
@pytest.mark.parametrize("tag", MAPPER_CASES)
def test_bin_table_matches_oracle(cuda, tag):
    g = load_mapper_case(tag)
    n_r, n_eta = g["r_lo"].size, g["eta_lo"].size
    pm = from_arrays(g["records"], g["nmap"])
    plan = CakePlan(pm, n_r=n_r, n_eta=n_eta, n_pixels_y=g["ny"], n_pixels_z=g["nz"], mode="bilinear",
                    device=cuda)
    t = plan.bin_table(g["r_lo"], g["r_hi"], g["eta_lo"], g["eta_hi"], px=g["px"], lsd=g["lsd"],
                       wavelength=0.172979)
    ref = oracle.bin_table(g["records"], g["nmap"], n_r, n_eta, g["ny"], g["nz"], g["r_lo"], g["r_hi"],
                           g["eta_lo"], g["eta_hi"], g["px"], g["lsd"], 0.172979)
    np.testing.assert_array_equal(t[:, [0, 2]], ref[:, [0, 2]])
    np.testing.assert_allclose(t[:, [1, 4]], ref[:, [1, 4]], rtol=1e-14, atol=0)
    np.testing.assert_allclose(t[:, 3], ref[:, 3], rtol=1e-12, atol=1e-12)
    t0 = plan.bin_table(g["r_lo"], g["r_hi"], g["eta_lo"], g["eta_hi"], px=g["px"], lsd=g["lsd"])
    assert np.all(t0[:, 4] == 0.0)
