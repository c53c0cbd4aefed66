"""SumImages (IntegratorFitPeaksGPUStream.cu:1043-1046): the running FP64 sum of the
cakes over every batch, through CakePlan.integrate(sum_into=...) / mi_sum_cake, against
the sum of the oracle's cakes; NaN bins of the OpenMP semantics add nothing."""
import numpy as np
import pytest
import torch

import oracle
from conftest import load_mapper_case, rel_err
from midas_b200.bin_io import from_arrays
from midas_b200.kernels import CakePlan

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("encoding", ["runs", "mma"])
def test_running_sum_over_batches(cuda, encoding):
    g = load_mapper_case("m2")
    n_r, n_eta = g["r_lo"].size, g["eta_lo"].size
    pm = from_arrays(g["records"], g["nmap"])
    plan = CakePlan(pm, n_r=n_r, n_eta=n_eta, n_pixels_y=g["ny"], n_pixels_z=g["nz"], mode="gradient",
                    bc_y=g["bc_y"], bc_z=g["bc_z"], device=cuda, encoding=encoding)
    rng = np.random.default_rng(2)
    frames = np.clip(np.rint(g["image"][None] * rng.uniform(1, 60, size=(11, 1, 1))), 0, 65535).astype(np.uint16)
    acc = torch.zeros((n_r, n_eta), dtype=torch.float64, device=cuda)
    for a, b in ((0, 3), (3, 3), (3, 11)):          # an empty batch in the middle
        plan.integrate(torch.from_numpy(frames[a:b]).to(cuda), sum_into=acc)
    assert plan.status() == 0
    want = np.zeros(n_r * n_eta)
    for f in frames:
        ck, _ = oracle.integrate(g["records"], g["nmap"], n_r * n_eta, g["ny"], g["nz"], f.astype(np.float64),
                                 mode="gradient", semantics="py", bc_y=g["bc_y"], bc_z=g["bc_z"])
        want += ck
    assert rel_err(acc.cpu().numpy().reshape(-1), want)[0] <= 1e-6


def test_sum_skips_nan_bins_and_checks_arguments(cuda):
    g = load_mapper_case("m1")
    n_r, n_eta = g["r_lo"].size, g["eta_lo"].size
    pm = from_arrays(g["records"], g["nmap"])
    plan = CakePlan(pm, n_r=n_r, n_eta=n_eta, n_pixels_y=g["ny"], n_pixels_z=g["nz"], mode="bilinear",
                    semantics="omp", bc_y=g["bc_y"], bc_z=g["bc_z"], device=cuda)
    mask = np.zeros(n_r * n_eta, np.uint8)
    mask[::7] = 1
    plan.set_bin_mask(mask)
    img = torch.from_numpy(g["image"].astype(np.float32)).to(cuda)[None].repeat(2, 1, 1)
    acc = torch.zeros(n_r * n_eta, dtype=torch.float64, device=cuda)
    ck, _, _ = plan.integrate(img, sum_into=acc)
    c = ck.cpu().numpy().reshape(2, -1).astype(np.float64)
    assert np.isnan(c[:, ::7]).all()
    s = acc.cpu().numpy()
    assert np.all(s[::7] == 0.0) and np.isfinite(s).all()
    assert np.allclose(s, np.nansum(c, axis=0), rtol=1e-12, atol=0)
    with pytest.raises(ValueError):
        plan.integrate(img, sum_into=acc.float())
    with pytest.raises(ValueError):
        plan.integrate(img, cake=False, sum_into=acc)


def test_sweep_sum_over_batches_matches_one_launch(cuda):
    """SweepSum over batches of a sweep equals the sum of one launch's cakes (FP64), and its
    reduce is a no-op without a process group."""
    from midas_b200.sweep import SweepSum
    g = load_mapper_case("m1")
    n_r, n_eta = g["r_lo"].size, g["eta_lo"].size
    pm = from_arrays(g["records"], g["nmap"])
    plan = CakePlan(pm, n_r=n_r, n_eta=n_eta, n_pixels_y=g["ny"], n_pixels_z=g["nz"], mode="bilinear",
                    bc_y=g["bc_y"], bc_z=g["bc_z"], device=cuda, encoding="mma")
    rng = np.random.default_rng(8)
    frames = torch.from_numpy(np.clip(np.rint(g["image"][None] * rng.uniform(1, 50, size=(9, 1, 1))), 0,
                                      65535).astype(np.uint16)).to(cuda)
    s = SweepSum(plan)
    for a, b in ((0, 4), (4, 9)):
        s.add(plan, frames[a:b])
    ck, _, _ = plan.integrate(frames)
    want = ck.double().sum(0).reshape(-1)
    got = s.reduce()
    assert s.frames == 9
    torch.testing.assert_close(got, want, rtol=1e-12, atol=1e-9)
