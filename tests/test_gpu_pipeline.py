"""The tensor-core kernel's pipeline variants (stage slots x producer warps) give the same
cake bit for bit; unsupported pairs and other encodings are refused."""
import numpy as np
import pytest
import torch

from conftest import load_mapper_case
from midas_b200 import _lib as L
from midas_b200.bin_io import from_arrays
from midas_b200.kernels import CakePlan

pytestmark = pytest.mark.gpu


def test_pipeline_variants_agree_bitwise(cuda):
    g = load_mapper_case("m2")
    n_r, n_eta = g["r_lo"].size, g["eta_lo"].size
    pm = from_arrays(g["records"], g["nmap"])
    plan = CakePlan(pm, n_r=n_r, n_eta=n_eta, n_pixels_y=g["ny"], n_pixels_z=g["nz"], mode="gradient",
                    bc_y=g["bc_y"], bc_z=g["bc_z"], device=cuda, encoding="mma")
    plan.set_dark(g["dark"].astype(np.float32))
    rng = np.random.default_rng(4)
    frames = torch.from_numpy(np.clip(np.rint(g["image"][None] * rng.uniform(1, 90, size=(70, 1, 1))), 0,
                                      65535).astype(np.uint16)).to(cuda)
    ref = [t.cpu().numpy() for t in plan.integrate(frames)]
    for pipe in CakePlan.MMA_PIPELINES:
        plan.set_mma_pipeline(*pipe)
        got = [t.cpu().numpy() for t in plan.integrate(frames)]
        assert plan.status() == 0
        for a, b in zip(got, ref):
            np.testing.assert_array_equal(a, b)
    with pytest.raises(L.MidasError):
        plan.set_mma_pipeline(3, 6)
    runs = CakePlan(pm, n_r=n_r, n_eta=n_eta, n_pixels_y=g["ny"], n_pixels_z=g["nz"], device=cuda)
    with pytest.raises(L.MidasError):
        runs.set_mma_pipeline(7, 6)
