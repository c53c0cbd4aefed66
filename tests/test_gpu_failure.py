"""Failure detection without a GPU fault: a bounded device wait that nothing completes ends
with MI_E_TIMEOUT read by the host, and the context keeps working (the caking kernels use
the same bounded mbarrier waits and report through the plan's status word)."""
import ctypes as C

import numpy as np
import pytest
import torch

from conftest import load_kernels_case
from midas_b200 import _lib as L
from midas_b200.bin_io import from_arrays
from midas_b200.kernels import CakePlan

pytestmark = pytest.mark.gpu


def _selftest(polls, arrive):
    st = C.c_int(12345)
    L.check(L.lib().mi_selftest_wait(polls, arrive, 0, C.byref(st)), "mi_selftest_wait")
    return st.value


def test_lost_wait_times_out_and_the_context_survives(cuda):
    assert _selftest(2000, 0) == L.MI_E_TIMEOUT
    assert _selftest(2000, 1) == L.MI_OK
    g = load_kernels_case("a")
    plan = CakePlan(from_arrays(g["records"], g["nmap"]), n_r=g["n_r"], n_eta=g["n_eta"], n_pixels_y=g["ny"],
                    n_pixels_z=g["nz"], device=cuda, encoding="mma")
    frames = torch.from_numpy(np.ones((3, g["nz"], g["ny"]), np.uint16)).to(cuda)
    ck, aw, sm = plan.integrate(frames)
    torch.cuda.synchronize()
    assert plan.status() == 0 and torch.isfinite(ck).all()
    assert _selftest(1, 0) == L.MI_E_TIMEOUT
