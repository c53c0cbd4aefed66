"""Parity of the tensor-core caking path (MI_ENC_MMA: exact int8 tcgen05 products, FP64
recombination) with the FP64 oracle, through the C ABI: every mode x semantics x
normalisation on random and DetectorMapper maps, u16 and u8 frames, darks, batches crossing
the 128-frame launch, variance plans, panels, and the refusal of other frame types."""
import numpy as np
import pytest
import torch

import oracle
from conftest import KERNEL_CASES, MAPPER_CASES, load_kernels_case, load_mapper_case, rel_err
from midas_b200 import _lib as L
from midas_b200.bin_io import from_arrays
from midas_b200.kernels import CakePlan, PanelPlan

pytestmark = pytest.mark.gpu

TOL = 1e-6


def _oracle(g, frames, mode, norm, sem, n_r, records=None, nmap=None, var=False):
    rec = g["records"] if records is None else records
    nm = g["nmap"] if nmap is None else nmap
    nb = nm.shape[0]
    area = oracle.area_in(rec, nm, nb, g["ny"], g["nz"])
    out = []
    for f in frames:
        f64 = np.asarray(f, np.float64)
        if var:
            ck = oracle.integrate_var(rec, nm, nb, g["ny"], g["nz"], f64, mode=mode, semantics=sem, normalize=norm,
                                      bc_y=g["bc_y"], bc_z=g["bc_z"])
            aw, sm = oracle.profile_var(ck, area, n_r, nb // n_r)
        else:
            ck, _ = oracle.integrate(rec, nm, nb, g["ny"], g["nz"], f64, mode=mode, semantics=sem, normalize=norm,
                                     bc_y=g["bc_y"], bc_z=g["bc_z"])
            aw, sm = oracle.profile(ck, area, n_r, nb // n_r)
        out.append((ck, aw, sm))
    return [np.array(x) for x in zip(*out)]


def _check(res, ref):
    for got, want in zip(res, ref):
        e = rel_err(got.cpu().numpy(), want)[0]
        assert e <= TOL, e


@pytest.mark.parametrize("tag", KERNEL_CASES)
@pytest.mark.parametrize("mode", ["floor", "bilinear", "gradient"])
@pytest.mark.parametrize("norm", [True, False])
@pytest.mark.parametrize("sem", ["py", "gpustream", "ic"])
def test_mma_matches_oracle_u16(cuda, tag, mode, norm, sem):
    g = load_kernels_case(tag)
    if sem == "ic" and mode == "floor":
        pytest.skip("IntegrationCore has no floor mode")
    pm = from_arrays(g["records"], g["nmap"])
    plan = CakePlan(pm, n_r=g["n_r"], n_eta=g["n_eta"], n_pixels_y=g["ny"], n_pixels_z=g["nz"], mode=mode,
                    normalize=norm, semantics=sem, bc_y=g["bc_y"], bc_z=g["bc_z"], device=cuda, encoding="mma")
    rng = np.random.default_rng(11)
    frames = np.clip(np.rint(g["image"][None] * rng.uniform(20, 65, size=(9, 1, 1))), 0, 65535).astype(np.uint16)
    frames[0, 0, :3] = 65535                      # saturated pixels: the high byte plane at its top
    res = plan.integrate(torch.from_numpy(frames).to(cuda))
    assert plan.status() == 0
    _check(res, _oracle(g, frames, mode, norm, sem, g["n_r"]))


@pytest.mark.parametrize("tag", MAPPER_CASES)
@pytest.mark.parametrize("mode", ["floor", "bilinear", "gradient"])
def test_mma_detector_maps_with_dark(cuda, tag, mode):
    """DetectorMapper maps, raw u16 frames, a float dark; 200 frames (two launches of the
    128-frame kernel); then the dark is cleared."""
    g = load_mapper_case(tag)
    n_r, n_eta = g["r_lo"].size, g["eta_lo"].size
    pm = from_arrays(g["records"], g["nmap"])
    plan = CakePlan(pm, n_r=n_r, n_eta=n_eta, n_pixels_y=g["ny"], n_pixels_z=g["nz"], mode=mode,
                    bc_y=g["bc_y"], bc_z=g["bc_z"], device=cuda, encoding="mma")
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


def test_mma_u8_frames_and_batch_independence(cuda):
    g = load_kernels_case("a")
    pm = from_arrays(g["records"], g["nmap"])
    plan = CakePlan(pm, n_r=g["n_r"], n_eta=g["n_eta"], n_pixels_y=g["ny"], n_pixels_z=g["nz"], mode="bilinear",
                    device=cuda, encoding="mma")
    rng = np.random.default_rng(2)
    frames = rng.integers(0, 256, size=(130, g["nz"], g["ny"])).astype(np.uint8)
    ck, aw, sm = plan.integrate(torch.from_numpy(frames).to(cuda))
    _check((ck[:4], aw[:4], sm[:4]), _oracle(g, frames[:4], "bilinear", True, "py", g["n_r"]))
    # a frame's result does not depend on its batch: bit-identical alone
    for f in (0, 77, 129):
        c1, a1, s1 = plan.integrate(torch.from_numpy(frames[f:f + 1]).to(cuda))
        assert torch.equal(c1[0], ck[f]) and torch.equal(a1[0], aw[f]) and torch.equal(s1[0], sm[f])


@pytest.mark.parametrize("mode", ["floor", "gradient"])
def test_mma_variance_plan(cuda, mode):
    g = load_kernels_case("d")
    pm = from_arrays(g["records"], g["nmap"])
    plan = CakePlan(pm, n_r=g["n_r"], n_eta=g["n_eta"], n_pixels_y=g["ny"], n_pixels_z=g["nz"], mode=mode,
                    bc_y=g["bc_y"], bc_z=g["bc_z"], device=cuda, encoding="mma", variance=True)
    rng = np.random.default_rng(4)
    var = rng.integers(1, 60000, size=(6, g["nz"], g["ny"])).astype(np.uint16)
    res = plan.integrate(torch.from_numpy(var).to(cuda))
    _check(res, _oracle(g, var, mode, True, "py", g["n_r"], var=True))


def test_mma_rejects_other_frame_types(cuda):
    g = load_kernels_case("c")
    pm = from_arrays(g["records"], g["nmap"])
    plan = CakePlan(pm, n_r=g["n_r"], n_eta=g["n_eta"], n_pixels_y=g["ny"], n_pixels_z=g["nz"], device=cuda,
                    encoding="mma")
    with pytest.raises(L.MidasError, match="8/16-bit"):
        plan.integrate(torch.zeros(2, g["nz"], g["ny"], dtype=torch.float32, device=cuda))


def test_mma_matches_run_encoding_at_detector_scale(cuda):
    """A 1440x1440 detector with the sweep geometry (gradient mode, fine binning): the MMA
    plan and the run plan agree with each other and with the oracle on sampled frames."""
    from midas_b200 import synth
    from midas_b200.mapper import build_map
    w = synth.scaled(synth.sweep_2880(), 2)
    m = w.mapper
    pm, _ = build_map(m, device=0)
    kw = dict(n_r=w.n_r, n_eta=w.n_eta, n_pixels_y=m.NrPixelsY, n_pixels_z=m.NrPixelsZ, mode="gradient",
              bc_y=m.BC_y, bc_z=m.BC_z, device=cuda)
    mma = CakePlan(pm, encoding="mma", **kw)
    runs = CakePlan(pm, encoding="runs", **kw)
    dark = w.dark().cpu().numpy()
    mma.set_dark(dark)
    runs.set_dark(dark)
    frames = w.frames(0, 20)
    cm, am, sm_ = mma.integrate(frames)
    cr, ar, sr = runs.integrate(frames)
    assert mma.status() == 0
    assert rel_err(cm.cpu().numpy(), cr.cpu().numpy())[0] <= 2 * TOL
    g = dict(records=pm.pxList, nmap=pm.nmap_pairs(), ny=m.NrPixelsY, nz=m.NrPixelsZ, bc_y=m.BC_y, bc_z=m.BC_z)
    sub = frames.cpu().numpy()[[0, 19]].astype(np.float64) - dark[None].astype(np.float64)
    ref = _oracle(g, sub, "gradient", True, "py", w.n_r)
    _check((cm[[0, 19]], am[[0, 19]], sm_[[0, 19]]), ref)


@pytest.mark.parametrize("encoding", ["mma", "mmad"])
def test_tensor_core_ic_semantics_at_detector_scale(cuda, encoding):
    """IntegrationCore semantics on a 1440x1440 detector (gradient mode): its bilinear bin
    weights include negative ones, which the signed weight digits carry; the cake matches
    the oracle to the same bar as the other semantics."""
    from midas_b200 import synth
    from midas_b200.mapper import build_map
    w = synth.scaled(synth.sweep_2880(), 2)
    m = w.mapper
    pm, _ = build_map(m, device=0)
    plan = CakePlan(pm, n_r=w.n_r, n_eta=w.n_eta, n_pixels_y=m.NrPixelsY, n_pixels_z=m.NrPixelsZ, mode="gradient",
                    semantics="ic", bc_y=m.BC_y, bc_z=m.BC_z, device=cuda, encoding=encoding)
    frames = w.frames(0, 3)
    res = plan.integrate(frames)
    assert plan.status() == 0
    g = dict(records=pm.pxList, nmap=pm.nmap_pairs(), ny=m.NrPixelsY, nz=m.NrPixelsZ, bc_y=m.BC_y, bc_z=m.BC_z)
    ref = _oracle(g, frames.cpu().numpy().astype(np.float64), "gradient", True, "ic", w.n_r)
    _check(res, ref)


def test_mma_panels(cuda):
    """Four u16 panels of a scaled panel set, one merged cake through the MMA plan, against
    the run-encoded panel plan."""
    from midas_b200 import synth
    from midas_b200.mapper import build_map
    ws = synth.scaled_panels(synth.panel_set(q_bin=0.02, eta_bin=10.0, mode="floor"), 8)[:4]
    maps = [build_map(w.mapper, device=0, mask=w.mask())[0] for w in ws]
    shapes = [(w.mapper.NrPixelsY, w.mapper.NrPixelsZ) for w in ws]
    bcs = [(w.mapper.BC_y, w.mapper.BC_z) for w in ws]
    kw = dict(shapes=shapes, beam_centres=bcs, n_r=ws[0].n_r, n_eta=ws[0].n_eta, mode="floor", device=cuda)
    pm = PanelPlan(maps, encoding="mma", **kw)
    pr = PanelPlan(maps, **kw)
    darks = [w.dark().cpu().numpy() for w in ws]
    pm.set_dark(darks)
    pr.set_dark(darks)
    frames = [w.frames(0, 9) for w in ws]
    a = pm.integrate(frames)
    b = pr.integrate(frames)
    for x, y in zip(a, b):
        assert rel_err(x.cpu().numpy(), y.cpu().numpy())[0] <= 2 * TOL


def test_host_threads_option_builds_the_same_plan(cuda):
    """A plan built on two host threads (the serving loop's admission setting) cakes
    bit-identically to one built on all cores, for both encodings."""
    g = load_kernels_case("b")
    pm = from_arrays(g["records"], g["nmap"])
    rng = np.random.default_rng(12)
    frames = torch.from_numpy(rng.integers(0, 60000, size=(5, g["nz"], g["ny"])).astype(np.uint16)).to(cuda)
    for enc in ("mma", "runs"):
        kw = dict(n_r=g["n_r"], n_eta=g["n_eta"], n_pixels_y=g["ny"], n_pixels_z=g["nz"], mode="gradient",
                  bc_y=g["bc_y"], bc_z=g["bc_z"], device=cuda, encoding=enc)
        a = CakePlan(pm, host_threads=2, **kw).integrate(frames)
        b = CakePlan(pm, **kw).integrate(frames)
        for x, y in zip(a, b):
            assert torch.equal(x, y)


def test_mma_coarse_bins_split_bands(cuda):
    """A 2048^2 powder map with coarse bins (990 x 72: 1 px in R, 5 deg in eta): tile blobs
    of whole 12-row bands exceed the kernel's blob slots, so bands are cut into 6-, 3- or
    1-row sub-bands with their own cake store boxes. Agrees with the run encoding."""
    from midas_b200 import synth
    from midas_b200.mapper import build_map
    w = synth.powder_2048()
    m = w.mapper
    pm, _ = build_map(m, device=0)
    kw = dict(n_r=w.n_r, n_eta=w.n_eta, n_pixels_y=m.NrPixelsY, n_pixels_z=m.NrPixelsZ, mode=w.mode,
              bc_y=m.BC_y, bc_z=m.BC_z, device=cuda)
    mma = CakePlan(pm, encoding="mma", **kw)
    runs = CakePlan(pm, encoding="runs", **kw)
    # unsplit: one item per band of 12 rows and slot of 8 columns (9 slots of 72 columns)
    assert mma.info["n_items"] > (w.n_r + 11) // 12 * 9
    dark = w.dark().cpu().numpy()
    mma.set_dark(dark)
    runs.set_dark(dark)
    frames = w.frames(0, 130)
    a = mma.integrate(frames)
    b = runs.integrate(frames)
    assert mma.status() == 0
    for x, y in zip(a, b):
        assert rel_err(x.cpu().numpy(), y.cpu().numpy())[0] <= 2 * TOL
