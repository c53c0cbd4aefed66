"""mi_integrate_batch_static: the batched integration for callers that cannot have device
memory allocated for them once running (a detector front-end that reserves the device's
whole memory budget at start-up and hands the library only its own buffers).  It keeps its
lineout scratch in a fixed array in the library; its results must equal those of
mi_integrate_batch, call after call.

Collected last (file name) so a run that stops at the first failure has run everything
else first; it also passes alone in a fresh process."""
import ctypes as C

import numpy as np
import pytest
import torch

from conftest import load_mapper_case, rel_err
from midas_b200 import _lib as L
from midas_b200 import synth
from midas_b200.bin_io import from_arrays
from midas_b200.kernels import CakePlan
from midas_b200.mapper import build_map

pytestmark = pytest.mark.gpu


def _static_call(plan, frames, ck, aw, sm):
    flat = frames.reshape(frames.shape[0], -1)
    return L.lib().mi_integrate_batch_static(plan._h, flat.data_ptr(), L.DT_U16, flat.shape[0], flat.stride(0),
                                             ck.data_ptr(), aw.data_ptr(), sm.data_ptr(), L.stream_ptr())


@pytest.mark.parametrize("enc", ["runs", "csr"])
def test_static_scratch_entry_point_matches_batched(cuda, enc):
    g = load_mapper_case("m2")
    n_r, n_eta = g["r_lo"].size, g["eta_lo"].size
    plan = CakePlan(from_arrays(g["records"], g["nmap"]), n_r=n_r, n_eta=n_eta, n_pixels_y=g["ny"],
                    n_pixels_z=g["nz"], mode="gradient", bc_y=g["bc_y"], bc_z=g["bc_z"], device=cuda, encoding=enc)
    rng = np.random.default_rng(17)
    dark = (100 + 3 * rng.standard_normal((g["nz"], g["ny"]))).astype(np.float32)
    plan.set_dark(dark)
    frames = torch.from_numpy(rng.integers(80, 9000, size=(70, g["nz"], g["ny"])).astype(np.uint16)).to(cuda)
    ref_ck, ref_aw, ref_sm = plan.integrate(frames)
    for call in range(2):                    # the array keeps the previous call's contents
        ck = torch.full_like(ref_ck, float("nan"))
        aw = torch.full_like(ref_aw, float("nan"))
        sm = torch.full_like(ref_sm, float("nan"))
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        L.check(_static_call(plan, frames, ck, aw, sm), "mi_integrate_batch_static")
        torch.cuda.synchronize()
        if call == 1:                        # after the first call's set-up: no device memory taken
            assert torch.cuda.mem_get_info()[0] == free0
        assert rel_err(ck.cpu().numpy(), ref_ck.cpu().numpy())[0] <= 1e-6
        assert rel_err(aw.cpu().numpy(), ref_aw.cpu().numpy())[0] <= 1e-6
        assert rel_err(sm.cpu().numpy(), ref_sm.cpu().numpy())[0] <= 1e-6
    assert plan.status() == 0


def test_static_scratch_tensor_core_plan_in_chunks(cuda):
    """The tensor-core (MMA) encoding through the fixed array: 990 x 360 bins need
    990 x 12 x 2 doubles of scratch per frame, so 100 frames run as chunks of 44, 44 and 12
    launches, against one 100-frame launch of mi_integrate_batch."""
    w = synth.scaled(synth.sweep_2880(), 4)
    pm, _ = build_map(w.mapper, device=0)
    plan = CakePlan(pm, n_r=w.n_r, n_eta=w.n_eta, n_pixels_y=w.mapper.NrPixelsY, n_pixels_z=w.mapper.NrPixelsZ,
                    mode=w.mode, bc_y=w.mapper.BC_y, bc_z=w.mapper.BC_z, device=cuda, encoding="mma")
    assert (1 << 20) // (w.n_r * 12 * 2) < 100
    plan.set_dark(w.dark(device=cuda).cpu().numpy())
    frames = w.frames(0, 100, device=cuda)
    ref_ck, ref_aw, ref_sm = plan.integrate(frames)
    for call in range(2):
        ck = torch.full_like(ref_ck, float("nan"))
        aw = torch.full_like(ref_aw, float("nan"))
        sm = torch.full_like(ref_sm, float("nan"))
        L.check(_static_call(plan, frames, ck, aw, sm), "mi_integrate_batch_static")
        torch.cuda.synchronize()
        assert rel_err(ck.cpu().numpy(), ref_ck.cpu().numpy())[0] <= 1e-6
        assert rel_err(aw.cpu().numpy(), ref_aw.cpu().numpy())[0] <= 1e-6
        assert rel_err(sm.cpu().numpy(), ref_sm.cpu().numpy())[0] <= 1e-6
    assert plan.status() == 0
    plan.close()


def test_static_scratch_rejects_plans_beyond_the_array(cuda):
    n_r, n_eta = 44000, 12              # 44000 rows x 12 items x 2 doubles > 2^20 per frame
    nmap = np.zeros((n_r * n_eta, 2), np.int32)
    recs = np.zeros(0, dtype=np.dtype([("y", "<f4"), ("z", "<f4"), ("frac", "<f8"), ("deltaR", "<f4"),
                                       ("areaWeight", "<f4")]))
    plan = CakePlan(from_arrays(recs, nmap), n_r=n_r, n_eta=n_eta, n_pixels_y=8, n_pixels_z=8, device=cuda)
    frames = torch.zeros((1, 8, 8), dtype=torch.uint16, device=cuda)
    ck = torch.empty((1, n_r, n_eta), dtype=torch.float32, device=cuda)
    aw = torch.empty((1, n_r), dtype=torch.float64, device=cuda)
    sm = torch.empty((1, n_r), dtype=torch.float64, device=cuda)
    assert _static_call(plan, frames, ck, aw, sm) == L.MI_E_RANGE
    assert b"fixed array" in L.lib().mi_last_error()
