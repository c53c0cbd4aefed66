"""The continuous-batching server on the device: streams with different maps, detector
shapes and frame types served concurrently must give every frame the result it gets
alone through the same path (the one-frame kernel for a batch of one frame, a one-frame
launch of the stream's batched encoding otherwise), and that result must match the FP64
oracle."""
import threading
import time

import numpy as np
import pytest
import torch

import oracle
from conftest import rel_err
from midas_b200 import peakfit, synth
from midas_b200.kernels import CakePlan
from midas_b200.server import CakeServer, DeviceBackend

pytestmark = pytest.mark.gpu

N_FRAMES = 12


def _mix():
    return [synth.scaled(synth.sweep_2880(), 8), synth.scaled(synth.powder_2048(), 8),
            synth.scaled(synth.pilatus_1679(), 5), synth.scaled(synth.detector_1024(1), 4)]


def _alone(cfg, frame, batch_size, small_batch=1):
    """One frame, one launch, on a plan of its own, through the path the server takes for
    a batch of ``batch_size`` frames; fits on that frame's lineout alone."""
    enc = DeviceBackend.encoding_for(cfg)
    plan = CakePlan(cfg.pixmap, n_r=cfg.n_r, n_eta=cfg.n_eta, n_pixels_y=cfg.n_pixels_y,
                    n_pixels_z=cfg.n_pixels_z, mode=cfg.mode, bc_y=cfg.bc_y, bc_z=cfg.bc_z,
                    tile_rows=cfg.tile_rows if enc == "runs" else 0, encoding=enc, device="cuda")
    plan.set_dark(cfg.dark)
    if batch_size <= small_batch:
        _, aw, sm = plan.integrate_plain(torch.from_numpy(frame).cuda())
        aw, sm = aw[None], sm[None]
    else:
        _, aw, sm = plan.integrate(torch.from_numpy(frame[None]).cuda(), cake=False)
    fit = peakfit.fit_batch(torch.from_numpy(cfg.r_axis).cuda(), aw, torch.from_numpy(cfg.peaks).cuda(),
                            model=cfg.fit_model, half_window=cfg.fit_half_window, x_bin=cfg.x_bin)
    out = aw[0].cpu().numpy(), sm[0].cpu().numpy(), fit.params[0].cpu().numpy()
    plan.close()
    return out


@pytest.mark.parametrize("graphs", [8, 0])
def test_results_are_the_same_alone_and_in_the_mix(cuda, graphs):
    """graphs: batches up to this size replay a recorded CUDA graph (0: direct calls)."""
    work = _mix()
    cfgs = [synth.serving_stream(w) for w in work]
    frames = [synth.host_frames(w, 0, N_FRAMES) for w in work]
    assert frames[2].dtype == np.int32
    srv = CakeServer(backend=DeviceBackend(max_batch=5, max_inflight=2, graph_batches=graphs)).start()
    try:
        ids = [srv.admit(c) for c in cfgs]
        results = {}

        def producer(k):
            rng = np.random.default_rng(k)
            futs = []
            for i, f in enumerate(frames[k]):
                futs.append(srv.submit(ids[k], f))
                if i % 4 == 3:                          # bursts of four: one-frame and batched paths
                    time.sleep(rng.exponential(2e-3))
            results[k] = [fu.result(timeout=120) for fu in futs]

        th = [threading.Thread(target=producer, args=(k,)) for k in range(len(work))]
        for t in th:
            t.start()
        for t in th:
            t.join()
    finally:
        srv.stop()
    assert srv.completed == N_FRAMES * len(work)
    assert srv.batches < srv.completed                  # some launches carried several frames
    sizes = {r.batch_size for res in results.values() for r in res}
    assert 1 in sizes and max(sizes) > 1                # both the one-frame and the batched path
    for k, cfg in enumerate(cfgs):
        res = results[k]
        assert [r.seq for r in res] == list(range(N_FRAMES))
        for i, r in enumerate(res):
            aw, sm, fit = _alone(cfg, frames[k][i], r.batch_size)
            np.testing.assert_array_equal(r.lineout_aw, aw)     # bitwise: batch composition is invisible
            np.testing.assert_array_equal(r.lineout_sm, sm)
            np.testing.assert_array_equal(r.fits, fit)
        # and the served lineout is the FP64 oracle's
        pm = cfg.pixmap
        recs, nmap = pm.pxList, pm.nmap_pairs()
        ck, _ = oracle.integrate(recs, nmap, pm.n_bins, cfg.n_pixels_y, cfg.n_pixels_z,
                                 (frames[k][0].astype(np.float32) - cfg.dark).astype(np.float64),
                                 mode=cfg.mode, bc_y=cfg.bc_y, bc_z=cfg.bc_z)
        area = oracle.area_in(recs, nmap, pm.n_bins, cfg.n_pixels_y, cfg.n_pixels_z)
        ref_aw, ref_sm = oracle.profile(ck, area, cfg.n_r, cfg.n_eta)
        assert rel_err(res[0].lineout_aw, ref_aw)[0] <= 1e-6, cfg.name
        assert rel_err(res[0].lineout_sm, ref_sm)[0] <= 1e-6, cfg.name
    lat = srv.latency_ms()
    assert lat["n"] == N_FRAMES * len(work) and lat["p99"] >= lat["p50"] > 0


def test_stream_admitted_and_removed_while_others_run(cuda):
    a, b = synth.scaled(synth.powder_2048(), 8), synth.scaled(synth.detector_1024(0), 4)
    ca, cb = synth.serving_stream(a), synth.serving_stream(b)
    fa, fb = synth.host_frames(a, 0, 6), synth.host_frames(b, 3, 6)
    with CakeServer(backend=DeviceBackend(max_batch=4)) as srv:
        sa = srv.admit(ca)
        futs_a = [srv.submit(sa, f) for f in fa[:3]]
        sb = srv.admit(cb)                               # admitted while stream a has work queued
        futs_b = [srv.submit(sb, f) for f in fb]
        futs_a += [srv.submit(sa, f) for f in fa[3:]]
        srv.remove(sb, drain=True)
        assert all(f.done() for f in futs_b)
        ra = [f.result(timeout=60) for f in futs_a]
        rb = [f.result(timeout=60) for f in futs_b]
    for i in range(6):
        np.testing.assert_array_equal(ra[i].lineout_aw, _alone(ca, fa[i], ra[i].batch_size)[0])
        np.testing.assert_array_equal(rb[i].lineout_aw, _alone(cb, fb[i], rb[i].batch_size)[0])
