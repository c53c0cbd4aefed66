"""Panel plans: several detectors with their own geometry, beam centre, mask and frame type
caked into one merged Q x eta result.  A merged bin is the sum of all panels' weighted
pixels over the sum of their areas (one concatenated weight list); the FP64 oracle
computes it from each panel's raw sums and areas."""
import numpy as np
import pytest
import torch

import oracle
from conftest import rel_err
from midas_b200 import synth
from midas_b200.kernels import CakePlan, PanelPlan
from midas_b200.mapper import build_map

pytestmark = pytest.mark.gpu

TOL = 1e-6
TORCH_DT = {"uint16": torch.uint16, "int32": torch.int32}


def _panels(ws):
    maps = [build_map(w.mapper, device=0, mask=w.mask())[0] for w in ws]
    shapes = [(w.mapper.NrPixelsY, w.mapper.NrPixelsZ) for w in ws]
    bcs = [(w.mapper.BC_y, w.mapper.BC_z) for w in ws]
    return maps, shapes, bcs


def _oracle_merged(ws, maps, frames, darks, mode, semantics="py"):
    """FP64 merged cake and lineouts of frame 0 of every panel."""
    n_r, n_eta = ws[0].n_r, ws[0].n_eta
    nb = n_r * n_eta
    raw = np.zeros(nb)
    area = np.zeros(nb)
    area_in = np.zeros(nb)
    for w, pm, fr, dk in zip(ws, maps, frames, darks):
        m = w.mapper
        sub = (fr.astype(np.float32) - dk).astype(np.float64)
        s, a = oracle.integrate(pm.pxList, pm.nmap_pairs(), nb, m.NrPixelsY, m.NrPixelsZ, sub, mode=mode,
                                semantics=semantics, normalize=False, bc_y=m.BC_y, bc_z=m.BC_z)
        raw += s
        area += a
        area_in += oracle.area_in(pm.pxList, pm.nmap_pairs(), nb, m.NrPixelsY, m.NrPixelsZ)
    cake = np.where(area > 1e-9, raw / np.where(area > 1e-9, area, 1.0), 0.0)
    aw, sm = oracle.profile(cake, area_in, n_r, n_eta)
    return cake, aw, sm


@pytest.mark.parametrize("mode,which", [("gradient", [0, 1, 2, 3]), ("floor", [0, 1, 2, 3, 4])])
def test_panel_plan_matches_merged_oracle(cuda, mode, which):
    """Four u16 panels (u16 pixel-major staging) in gradient mode; all five panels, the int32
    one included (fp32 staging), in floor mode."""
    ws = [synth.scaled_panels(synth.panel_set(q_bin=0.02, eta_bin=10.0, mode=mode), 8)[i] for i in which]
    maps, shapes, bcs = _panels(ws)
    plan = PanelPlan(maps, shapes=shapes, beam_centres=bcs, n_r=ws[0].n_r, n_eta=ws[0].n_eta, mode=mode,
                     device=cuda)
    darks = [w.dark().cpu().numpy() for w in ws]
    plan.set_dark(darks)
    F = 70
    frames = [w.frames(0, F, dtype=TORCH_DT[w.frame_dtype]) for w in ws]
    ck, aw, sm = plan.integrate(frames)
    assert plan.status() == 0
    host = [f.cpu().numpy() for f in frames]
    for f in (0, 37, F - 1):
        rc, raw_, rsm = _oracle_merged(ws, maps, [h[f] for h in host], darks, mode)
        assert rel_err(ck[f].cpu().numpy(), rc)[0] <= TOL
        assert rel_err(aw[f].cpu().numpy(), raw_)[0] <= TOL
        assert rel_err(sm[f].cpu().numpy(), rsm)[0] <= TOL
    # the four square panels tile the azimuth around the beam; the int32 panel sees the
    # same azimuths as two of them, so with it the merged cake really merges bins
    if 4 in which:
        nb = ws[0].n_r * ws[0].n_eta
        reach = sum((pm.counts > 0).astype(int) for pm in maps)
        assert (reach >= 2).sum() > 0.02 * nb


def test_single_panel_plan_equals_cake_plan(cuda):
    w = synth.scaled(synth.sweep_2880(), 8)
    pm, _ = build_map(w.mapper, device=0)
    m = w.mapper
    kw = dict(n_r=w.n_r, n_eta=w.n_eta, mode=w.mode, device=cuda)
    pp = PanelPlan([pm], shapes=[(m.NrPixelsY, m.NrPixelsZ)], beam_centres=[(m.BC_y, m.BC_z)], **kw)
    cp = CakePlan(pm, n_pixels_y=m.NrPixelsY, n_pixels_z=m.NrPixelsZ, bc_y=m.BC_y, bc_z=m.BC_z, **kw)
    dark = w.dark().cpu().numpy()
    pp.set_dark([dark])
    cp.set_dark(dark)
    fr = w.frames(0, 9)
    a = pp.integrate([fr])
    b = cp.integrate(fr)
    for x, y in zip(a, b):
        assert torch.equal(x, y)


def test_panel_plan_rejects_single_frame_entry_points(cuda):
    ws = synth.scaled_panels(synth.panel_set(q_bin=0.05, eta_bin=20.0), 16)[:2]
    maps, shapes, bcs = _panels(ws)
    plan = PanelPlan(maps, shapes=shapes, beam_centres=bcs, n_r=ws[0].n_r, n_eta=ws[0].n_eta, device=cuda)
    fr = ws[0].frames(0, 2).reshape(2, -1)
    from midas_b200 import _lib as L
    aw = torch.empty((2, ws[0].n_r), dtype=torch.float64, device=cuda)
    rc = L.lib().mi_integrate_batch(plan._h, fr.data_ptr(), L.DT_U16, 2, fr.stride(0), None, aw.data_ptr(),
                                    aw.data_ptr(), L.stream_ptr())
    assert rc == L.MI_E_ARG and b"mi_integrate_panels" in L.lib().mi_last_error()
    ck = torch.empty((ws[0].n_r, ws[0].n_eta), dtype=torch.float64, device=cuda)
    rc = L.lib().mi_integrate_plain(plan._h, fr.data_ptr(), L.DT_U16, ck.data_ptr(), None, None, L.stream_ptr())
    assert rc == L.MI_E_UNSUPPORTED
