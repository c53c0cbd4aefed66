"""Parity of the direct tensor-core caking path (MI_ENC_MMAD: frames read in place into
tensor memory as byte planes, signed fixed-point weights in four digit planes, exact int8 tcgen05 products, FP64
recombination) with the FP64 oracle, through the C ABI: every mode x semantics x
normalisation on random maps (rows of 8k and of other widths: vector and pixel-by-pixel
granule loads), DetectorMapper maps with a dark over batches crossing the 128-frame launch,
u8 frames, batch independence, variance plans, strided frames and a detector-scale sweep."""
import numpy as np
import pytest
import torch

from conftest import KERNEL_CASES, MAPPER_CASES, load_kernels_case, load_mapper_case, rel_err
from midas_b200 import _lib as L
from midas_b200.bin_io import from_arrays
from midas_b200.kernels import CakePlan
from test_gpu_mma import TOL, _check, _oracle

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("tag", KERNEL_CASES)
@pytest.mark.parametrize("mode", ["floor", "bilinear", "gradient"])
@pytest.mark.parametrize("norm", [True, False])
@pytest.mark.parametrize("sem", ["py", "gpustream", "ic"])
def test_mmad_matches_oracle_u16(cuda, tag, mode, norm, sem):
    g = load_kernels_case(tag)
    if sem == "ic" and mode == "floor":
        pytest.skip("IntegrationCore has no floor mode")
    pm = from_arrays(g["records"], g["nmap"])
    plan = CakePlan(pm, n_r=g["n_r"], n_eta=g["n_eta"], n_pixels_y=g["ny"], n_pixels_z=g["nz"], mode=mode,
                    normalize=norm, semantics=sem, bc_y=g["bc_y"], bc_z=g["bc_z"], device=cuda, encoding="mmad")
    rng = np.random.default_rng(11)
    frames = np.clip(np.rint(g["image"][None] * rng.uniform(20, 65, size=(9, 1, 1))), 0, 65535).astype(np.uint16)
    frames[0, 0, :3] = 65535
    res = plan.integrate(torch.from_numpy(frames).to(cuda))
    assert plan.status() == 0
    _check(res, _oracle(g, frames, mode, norm, sem, g["n_r"]))


@pytest.mark.parametrize("tag", MAPPER_CASES)
@pytest.mark.parametrize("mode", ["floor", "bilinear", "gradient"])
def test_mmad_detector_maps_with_dark(cuda, tag, mode):
    g = load_mapper_case(tag)
    n_r, n_eta = g["r_lo"].size, g["eta_lo"].size
    pm = from_arrays(g["records"], g["nmap"])
    plan = CakePlan(pm, n_r=n_r, n_eta=n_eta, n_pixels_y=g["ny"], n_pixels_z=g["nz"], mode=mode,
                    bc_y=g["bc_y"], bc_z=g["bc_z"], device=cuda, encoding="mmad")
    rng = np.random.default_rng(5)
    F = 200
    raw = rng.integers(90, 60000, size=(F, g["nz"], g["ny"])).astype(np.uint16)
    dark = (100.0 + 5.0 * rng.standard_normal((g["nz"], g["ny"]))).astype(np.float32)
    plan.set_dark(dark)
    res = plan.integrate(torch.from_numpy(raw).to(cuda))
    gg = dict(g, n_r=n_r)
    sub = raw.astype(np.float64) - dark[None].astype(np.float64)
    _check(res, _oracle(gg, sub, mode, True, "py", n_r))
    plan.set_dark(None)
    res = plan.integrate(torch.from_numpy(raw[:5]).to(cuda))
    _check(res, _oracle(gg, raw[:5], mode, True, "py", n_r))
    assert plan.status() == 0


def test_mmad_u8_frames_and_batch_independence(cuda):
    g = load_kernels_case("a")
    pm = from_arrays(g["records"], g["nmap"])
    plan = CakePlan(pm, n_r=g["n_r"], n_eta=g["n_eta"], n_pixels_y=g["ny"], n_pixels_z=g["nz"], mode="bilinear",
                    device=cuda, encoding="mmad")
    rng = np.random.default_rng(2)
    frames = rng.integers(0, 256, size=(130, g["nz"], g["ny"])).astype(np.uint8)
    ck, aw, sm = plan.integrate(torch.from_numpy(frames).to(cuda))
    _check((ck[:4], aw[:4], sm[:4]), _oracle(g, frames[:4], "bilinear", True, "py", g["n_r"]))
    _check((ck[126:], aw[126:], sm[126:]), _oracle(g, frames[126:], "bilinear", True, "py", g["n_r"]))
    for f in (0, 63, 64, 127, 129):
        c1, a1, s1 = plan.integrate(torch.from_numpy(frames[f:f + 1]).to(cuda))
        assert torch.equal(c1[0], ck[f]) and torch.equal(a1[0], aw[f]) and torch.equal(s1[0], sm[f])


def test_mmad_strided_and_unaligned_frames(cuda):
    """Frames inside a larger buffer (stride of the row-padded layout) and frames starting at
    an address that is not 16-byte aligned take the pixel-by-pixel granule loads."""
    g = load_mapper_case("m1")
    n_r, n_eta = g["r_lo"].size, g["eta_lo"].size
    pm = from_arrays(g["records"], g["nmap"])
    plan = CakePlan(pm, n_r=n_r, n_eta=n_eta, n_pixels_y=g["ny"], n_pixels_z=g["nz"], mode="gradient",
                    bc_y=g["bc_y"], bc_z=g["bc_z"], device=cuda, encoding="mmad")
    rng = np.random.default_rng(8)
    raw = rng.integers(0, 60000, size=(7, g["nz"], g["ny"])).astype(np.uint16)
    ref = plan.integrate(torch.from_numpy(raw).to(cuda))
    npx = g["ny"] * g["nz"]
    buf = torch.zeros(7 * (npx + 3) + 1, dtype=torch.uint16, device=cuda)
    for f in range(7):
        buf[1 + f * (npx + 3):1 + f * (npx + 3) + npx] = torch.from_numpy(raw[f].reshape(-1)).to(cuda)
    ck = torch.empty((7, n_r, n_eta), dtype=torch.float32, device=cuda)
    aw = torch.empty((7, n_r), dtype=torch.float64, device=cuda)
    sm = torch.empty((7, n_r), dtype=torch.float64, device=cuda)
    L.check(L.lib().mi_integrate_batch(plan._h, buf.data_ptr() + 2, L.DT_U16, 7, npx + 3, ck.data_ptr(),
                                       aw.data_ptr(), sm.data_ptr(), L.stream_ptr()), "mi_integrate_batch")
    torch.cuda.synchronize()
    for x, y in zip((ck, aw, sm), ref):
        assert torch.equal(x, y)


@pytest.mark.parametrize("mode", ["floor", "gradient"])
def test_mmad_variance_plan(cuda, mode):
    g = load_kernels_case("d")
    pm = from_arrays(g["records"], g["nmap"])
    plan = CakePlan(pm, n_r=g["n_r"], n_eta=g["n_eta"], n_pixels_y=g["ny"], n_pixels_z=g["nz"], mode=mode,
                    bc_y=g["bc_y"], bc_z=g["bc_z"], device=cuda, encoding="mmad", variance=True)
    rng = np.random.default_rng(4)
    var = rng.integers(1, 60000, size=(6, g["nz"], g["ny"])).astype(np.uint16)
    res = plan.integrate(torch.from_numpy(var).to(cuda))
    _check(res, _oracle(g, var, mode, True, "py", g["n_r"], var=True))


def test_mmad_matches_oracle_at_detector_scale(cuda):
    """A 1440x1440 detector with the sweep geometry (gradient, RBin 0.25 px, eta 1 deg), 130
    frames with a dark: sampled frames of both launches against the oracle, and the whole
    batch against the byte-plane MMA encoding."""
    from midas_b200 import synth
    from midas_b200.mapper import build_map
    w = synth.scaled(synth.sweep_2880(), 2)
    m = w.mapper
    pm, _ = build_map(m, device=0)
    kw = dict(n_r=w.n_r, n_eta=w.n_eta, n_pixels_y=m.NrPixelsY, n_pixels_z=m.NrPixelsZ, mode="gradient",
              bc_y=m.BC_y, bc_z=m.BC_z, device=cuda)
    direct = CakePlan(pm, encoding="mmad", **kw)
    mma = CakePlan(pm, encoding="mma", **kw)
    dark = w.dark().cpu().numpy()
    direct.set_dark(dark)
    mma.set_dark(dark)
    frames = w.frames(0, 130)
    cd, ad, sd = direct.integrate(frames)
    cm, am, sm_ = mma.integrate(frames)
    assert direct.status() == 0
    assert rel_err(cd.cpu().numpy(), cm.cpu().numpy())[0] <= 2 * TOL
    assert rel_err(ad.cpu().numpy(), am.cpu().numpy())[0] <= 2 * TOL
    g = dict(records=pm.pxList, nmap=pm.nmap_pairs(), ny=m.NrPixelsY, nz=m.NrPixelsZ, bc_y=m.BC_y, bc_z=m.BC_z)
    pick = [0, 63, 127, 129]
    sub = frames.cpu().numpy()[pick].astype(np.float64) - dark[None].astype(np.float64)
    ref = _oracle(g, sub, "gradient", True, "py", w.n_r)
    _check((cd[pick], ad[pick], sd[pick]), ref)
