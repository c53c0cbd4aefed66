"""Fused multi-shift plans (mi_plan_create_fused; build_fused_geometry of
packages/midas_integrate/midas_integrate/fused_csr.py:139-296) on the device: the
reference's fused cakes (tests/golden/fused.npz) on every encoding, lineouts, a frame
batch, and a detector-scale plan from the device mapper against the oracle's naive
multi-map averaging."""
import numpy as np
import pytest
import torch

import oracle
from conftest import load_fused_case, rel_err
from midas_b200 import fused

pytestmark = pytest.mark.gpu
TOL = 1e-6


def _apply(row_ptr, col, w, image):
    img = np.asarray(image, np.float64).reshape(-1)
    n_bins = row_ptr.size - 1
    return np.bincount(np.repeat(np.arange(n_bins), np.diff(row_ptr)), weights=w * img[col], minlength=n_bins)


@pytest.mark.parametrize("mode", ["bilinear", "gradient"])
@pytest.mark.parametrize("encoding", ["runs", "csr"])
def test_fused_plan_matches_reference_cake(cuda, mode, encoding):
    g = load_fused_case()
    plan = fused.FusedPlan(g["maps"], g["r_axes"], n_eta=g["n_eta"], n_pixels_y=g["ny"], n_pixels_z=g["nz"],
                           mode=mode, bc_y=g["bc_y"], bc_z=g["bc_z"], device=cuda, encoding=encoding)
    img = torch.from_numpy(g["image"].astype(np.float32)).to(cuda)[None]
    cake, aw, sm = plan.integrate(img)
    assert plan.status() == 0
    want = g[f"cake_{mode}"]
    assert rel_err(cake.cpu().numpy().reshape(-1), want)[0] <= TOL
    n_r = g["r_axes"][0].size
    ref_aw, ref_sm = oracle.profile(want, np.ones(want.size), n_r, g["n_eta"])
    assert rel_err(aw.cpu().numpy()[0], ref_aw)[0] <= TOL
    assert rel_err(sm.cpu().numpy()[0], ref_sm)[0] <= TOL


@pytest.mark.parametrize("encoding", ["mma", "mmad", "runs"])
def test_fused_plan_u16_batch(cuda, encoding):
    """A batch of u16 frames (the tensor-core encodings take 8/16-bit frames only) against
    the host fused weights (pinned to the reference by the CPU tests) applied in FP64."""
    g = load_fused_case()
    row_ptr, col, w = fused.fused_csr(g["maps"], g["r_axes"], n_eta=g["n_eta"], n_pixels_y=g["ny"],
                                      n_pixels_z=g["nz"], mode="gradient", bc_y=g["bc_y"], bc_z=g["bc_z"])
    plan = fused.FusedPlan(g["maps"], g["r_axes"], n_eta=g["n_eta"], n_pixels_y=g["ny"], n_pixels_z=g["nz"],
                           mode="gradient", bc_y=g["bc_y"], bc_z=g["bc_z"], device=cuda, encoding=encoding)
    rng = np.random.default_rng(5)
    frames = np.clip(np.rint(g["image"][None] * rng.uniform(1, 70, size=(5, 1, 1))), 0, 65535).astype(np.uint16)
    cake, _, _ = plan.integrate(torch.from_numpy(frames).to(cuda))
    assert plan.status() == 0
    got = cake.cpu().numpy().reshape(5, -1)
    for f in range(5):
        assert rel_err(got[f], _apply(row_ptr, col, w, frames[f]))[0] <= TOL


def test_fused_plan_from_device_mapper(cuda):
    """build_fused_plan on a 720x720 detector (four shifts built by the device mapper),
    against the oracle's naive average of the same shifted maps."""
    from midas_b200 import synth
    w = synth.scaled(synth.sweep_2880(), 4)
    p = w.mapper
    plan = fused.build_fused_plan(p, n_shifts=4, mode="gradient", device=cuda.index or 0)
    maps, axes = fused.shift_maps(p, 4, device=cuda.index or 0)
    frames = w.frames(0, 2)
    cake, aw, _ = plan.integrate(frames)
    assert plan.status() == 0
    img = frames[1].cpu().numpy().astype(np.float64)
    want = oracle.fused_average([(m.pxList, m.nmap_pairs()) for m in maps], axes, p.n_eta, p.NrPixelsY,
                                p.NrPixelsZ, img, mode="gradient", bc_y=p.BC_y, bc_z=p.BC_z)
    assert rel_err(cake[1].cpu().numpy().reshape(-1), want)[0] <= TOL


def test_fused_plan_rejects_other_semantics(cuda):
    g = load_fused_case()
    with pytest.raises(ValueError):
        fused.FusedPlan(g["maps"], g["r_axes"], n_eta=g["n_eta"], n_pixels_y=g["ny"], n_pixels_z=g["nz"],
                        mode="floor", device=cuda)
