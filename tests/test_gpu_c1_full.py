"""The plain-method configuration at full size: one 2048 x 2048 u16 detector (wavelength
0.172979 A, Lsd 1 m, 200 um pixels, beam centre (1024.3, 1022.7), tilts 0.1 / -0.05 deg),
ten Debye-Scherrer rings, RMin 10 .. RMax 1000 px at 1 px and eta -180 .. 180 at 5 deg
(990 x 72 bins), floor mode, ten frames of the seeded generator with a dark of 100 + N(0, 5).
The map is built on the device; every bin of the cake and both lineouts of every frame are
compared with the FP64 oracle, for the tensor-core and the run encoding and for the
midas_integrate and GPU-stream semantics, at <= 1e-6 relative."""
import numpy as np
import pytest
import torch

import oracle
from conftest import rel_err
from midas_b200 import synth
from midas_b200.kernels import CakePlan
from midas_b200.mapper import build_map

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def c1(cuda):
    w = synth.powder_2048()
    pm, _ = build_map(w.mapper, device=0)
    dark = w.dark(device=cuda)
    frames = w.frames(0, 10, device=cuda)
    sub = frames.cpu().numpy().astype(np.float32) - dark.cpu().numpy()[None]
    return w, pm, dark, frames, sub


@pytest.mark.parametrize("enc", ["mma", "runs"])
@pytest.mark.parametrize("sem", ["py", "gpustream"])
def test_c1_full_size_bin_by_bin(cuda, c1, enc, sem):
    w, pm, dark, frames, sub = c1
    m = w.mapper
    ny, nz = m.NrPixelsY, m.NrPixelsZ
    assert (w.n_r, w.n_eta) == (990, 72)
    plan = CakePlan(pm, n_r=w.n_r, n_eta=w.n_eta, n_pixels_y=ny, n_pixels_z=nz, mode="floor", semantics=sem,
                    bc_y=m.BC_y, bc_z=m.BC_z, device=cuda, encoding=enc)
    plan.set_dark(dark.cpu().numpy())
    cake, aw, sm = plan.integrate(frames)
    assert plan.status() == 0
    recs, nmap = pm.pxList, pm.nmap_pairs()
    area = oracle.area_in(recs, nmap, pm.n_bins, ny, nz)
    for f in range(frames.shape[0]):
        ref, _ = oracle.integrate(recs, nmap, pm.n_bins, ny, nz, sub[f].astype(np.float64), mode="floor",
                                  semantics=sem, bc_y=m.BC_y, bc_z=m.BC_z)
        assert rel_err(cake[f].cpu().numpy(), ref)[0] <= 1e-6, (enc, sem, f)
        aw_ref, sm_ref = oracle.profile(ref, area, w.n_r, w.n_eta)
        assert rel_err(aw[f].cpu().numpy(), aw_ref)[0] <= 1e-6
        assert rel_err(sm[f].cpu().numpy(), sm_ref)[0] <= 1e-6
    plan.close()
