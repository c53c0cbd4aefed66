"""Parity of the CUDA caking path (kernels (a)-(c), batched and plain) with the FP64 oracle
and with the reference's golden outputs, called through the C ABI."""
import numpy as np
import pytest
import torch

import oracle
from conftest import KERNEL_CASES, MAPPER_CASES, load_kernels_case, load_mapper_case, rel_err
from midas_b200 import _lib as L
from midas_b200.bin_io import from_arrays
from midas_b200.kernels import CakePlan, build_csr, integrate, profile_1d

pytestmark = pytest.mark.gpu

# cake bins: <= 1e-6 relative to the FP64 oracle (tau-guarded: |ref| floored at 1e-3 * median)
TOL = 1e-6


def _frames_like(img, F, seed=0):
    rng = np.random.default_rng(seed)
    scale = 1.0 + 0.2 * rng.standard_normal(F)
    return np.stack([img * s for s in scale]).astype(np.float32)


def _oracle_batch(g, frames, mode, norm, sem, records=None, nmap=None):
    rec = g["records"] if records is None else records
    nm = g["nmap"] if nmap is None else nmap
    nb = nm.shape[0]
    cakes, aws, sms = [], [], []
    area = oracle.area_in(rec, nm, nb, g["ny"], g["nz"])
    n_r = g["n_r"] if "n_r" in g else g["r_lo"].size
    n_eta = nb // n_r
    for f in frames:
        ck, _ = oracle.integrate(rec, nm, nb, g["ny"], g["nz"], f.astype(np.float64), mode=mode,
                                 semantics=sem, normalize=norm, bc_y=g["bc_y"], bc_z=g["bc_z"])
        aw, sm = oracle.profile(ck, area, n_r, n_eta)
        cakes.append(ck)
        aws.append(aw)
        sms.append(sm)
    return np.array(cakes), np.array(aws), np.array(sms)


@pytest.mark.parametrize("tag", KERNEL_CASES)
@pytest.mark.parametrize("mode", ["floor", "bilinear", "gradient"])
@pytest.mark.parametrize("norm", [True, False])
@pytest.mark.parametrize("sem", ["py", "gpustream", "ic"])
@pytest.mark.parametrize("enc", ["runs", "csr"])
def test_batched_matches_oracle(cuda, tag, mode, norm, sem, enc):
    g = load_kernels_case(tag)
    pm = from_arrays(g["records"], g["nmap"])
    if sem == "ic" and mode == "floor":
        with pytest.raises(L.MidasError, match="no floor mode"):
            CakePlan(pm, n_r=g["n_r"], n_eta=g["n_eta"], n_pixels_y=g["ny"], n_pixels_z=g["nz"], mode=mode,
                     semantics=sem, device=cuda)
        return
    plan = CakePlan(pm, n_r=g["n_r"], n_eta=g["n_eta"], n_pixels_y=g["ny"], n_pixels_z=g["nz"], mode=mode,
                    normalize=norm, semantics=sem, bc_y=g["bc_y"], bc_z=g["bc_z"], device=cuda, encoding=enc)
    frames = _frames_like(g["image"], 7, seed=1)
    ck, aw, sm = plan.integrate(torch.from_numpy(frames).to(cuda))
    rc, raw, rsm = _oracle_batch(g, frames, mode, norm, sem)
    assert rel_err(ck.cpu().numpy(), rc)[0] <= TOL
    assert rel_err(aw.cpu().numpy(), raw)[0] <= TOL
    assert rel_err(sm.cpu().numpy(), rsm)[0] <= TOL


@pytest.mark.parametrize("tag", KERNEL_CASES)
@pytest.mark.parametrize("mode", ["floor", "bilinear", "gradient"])
def test_midas_integrate_api_matches_reference_golden(cuda, tag, mode):
    """build_csr / integrate / profile_1d against the reference package's own FP64 output."""
    g = load_kernels_case(tag)
    pm = from_arrays(g["records"], g["nmap"])
    geom = build_csr(pm, n_r=g["n_r"], n_eta=g["n_eta"], n_pixels_y=g["ny"], n_pixels_z=g["nz"],
                     device=cuda, dtype=torch.float64, bc_y=g["bc_y"], bc_z=g["bc_z"])
    np.testing.assert_allclose(geom.area_per_bin.cpu().numpy(), g["area_per_bin"], rtol=1e-12)
    for norm in (True, False):
        key = f"{mode}_{'n' if norm else 'r'}"
        img = torch.from_numpy(g["image"].astype(np.float32)).to(cuda)
        ck = integrate(img, geom, mode=mode, normalize=norm)
        assert ck.shape == (g["n_r"], g["n_eta"])
        # the image is given to the device as float32: compare against the reference on that image
        ref, _ = oracle.integrate(g["records"], g["nmap"], g["n_r"] * g["n_eta"], g["ny"], g["nz"],
                                  g["image"].astype(np.float32).astype(np.float64), mode=mode, normalize=norm,
                                  bc_y=g["bc_y"], bc_z=g["bc_z"])
        assert rel_err(ck.cpu().numpy(), ref)[0] <= TOL
        assert rel_err(ck.cpu().numpy(), g["cake_" + key])[0] <= 1e-6
        for pmode, gk in (("area_weighted", "aw_"), ("simple_mean", "sm_")):
            prof = profile_1d(ck, geom, mode=pmode)
            assert rel_err(prof.cpu().numpy(), g[gk + key])[0] <= 1e-6


ENCODINGS = [("csr", 1, 0, 8), ("csr", 2, 0, 8), ("csr", 4, 0, 8), ("runs", 0, 2, 8), ("runs", 0, 4, 8),
             ("runs", 0, 4, 16), ("runs", 0, 8, 16), ("runs", 0, 4, 32), ("runs", 0, 8, 32), ("runs", 0, 0, 12)]


@pytest.mark.parametrize("tag", MAPPER_CASES)
@pytest.mark.parametrize("mode", ["floor", "gradient"])
@pytest.mark.parametrize("enc,fpl,rl,rows", ENCODINGS)
def test_detector_maps_u16_with_dark(cuda, tag, mode, enc, fpl, rl, rows):
    """DetectorMapper maps, raw u16 frames and a float dark (cast + dark fused into staging),
    every tile encoding and register-run shape."""
    g = load_mapper_case(tag)
    n_r, n_eta = g["r_lo"].size, g["eta_lo"].size
    pm = from_arrays(g["records"], g["nmap"])
    plan = CakePlan(pm, n_r=n_r, n_eta=n_eta, n_pixels_y=g["ny"], n_pixels_z=g["nz"], mode=mode,
                    bc_y=g["bc_y"], bc_z=g["bc_z"], device=cuda, frames_per_lane=fpl, tile_rows=rows,
                    encoding=enc, run_len=rl)
    fpl = max(fpl, 1)
    rng = np.random.default_rng(5)
    F = 33 * fpl + 3                      # crosses frame-group boundaries
    raw = rng.integers(90, 60000, size=(F, g["nz"], g["ny"])).astype(np.uint16)
    dark = (100.0 + 5.0 * rng.standard_normal((g["nz"], g["ny"]))).astype(np.float32)
    plan.set_dark(dark)
    ck, aw, sm = plan.integrate(torch.from_numpy(raw).to(cuda))
    sub = raw.astype(np.float32) - dark[None]          # what the reference subtracts, in float
    gg = dict(g, n_r=n_r)
    rc, raw_, rsm = _oracle_batch(gg, sub, mode, True, "py")
    assert rel_err(ck.cpu().numpy(), rc)[0] <= TOL
    assert rel_err(aw.cpu().numpy(), raw_)[0] <= TOL
    assert rel_err(sm.cpu().numpy(), rsm)[0] <= TOL


@pytest.mark.skipif(not oracle.ref_available(), reason="reference integrator not compiled")
def test_ic_semantics_matches_reference_integrator_at_detector_scale(cuda):
    """The batched path with IntegrationCore semantics against integration_apply_map itself
    (compiled from the reference sources), on a 1440x1440 u16 detector with a dark,
    gradient mode: cake within 1e-6 relative of the reference's own integrator."""
    from midas_b200 import synth
    from midas_b200.mapper import build_map
    w = synth.scaled(synth.sweep_2880(), 2)
    m = w.mapper
    pm, _ = build_map(m, device=0)
    plan = CakePlan(pm, n_r=w.n_r, n_eta=w.n_eta, n_pixels_y=m.NrPixelsY, n_pixels_z=m.NrPixelsZ,
                    mode="gradient", semantics="ic", bc_y=m.BC_y, bc_z=m.BC_z, device=cuda)
    dark = w.dark().cpu().numpy()
    plan.set_dark(dark)
    frames = w.frames(0, 3)
    ck, _, _ = plan.integrate(frames)
    ck = ck.cpu().numpy()
    for f in range(3):
        sums, norms = oracle.ref_integrate(pm.pxList, pm.nmap_pairs(), w.n_r, w.n_eta,
                                           frames[f].cpu().numpy().astype(np.float64), m.NrPixelsY, m.NrPixelsZ,
                                           dark=dark.astype(np.float64), bc_y=m.BC_y, bc_z=m.BC_z, gradient=1,
                                           n_threads=8)
        ref = np.where(norms > 1e-9, sums / np.where(norms > 1e-9, norms, 1.0), 0.0)
        assert rel_err(ck[f].reshape(-1), ref)[0] <= TOL


def test_frame_result_independent_of_batch(cuda):
    g = load_mapper_case("m2")
    n_r, n_eta = g["r_lo"].size, g["eta_lo"].size
    plan = CakePlan(from_arrays(g["records"], g["nmap"]), n_r=n_r, n_eta=n_eta, n_pixels_y=g["ny"],
                    n_pixels_z=g["nz"], mode="gradient", bc_y=g["bc_y"], bc_z=g["bc_z"], device=cuda)
    rng = np.random.default_rng(9)
    raw = torch.from_numpy(rng.integers(0, 4000, size=(70, g["nz"], g["ny"])).astype(np.uint16)).to(cuda)
    ck_all, aw_all, _ = plan.integrate(raw)
    for k in (0, 31, 32, 69):
        ck1, aw1, _ = plan.integrate(raw[k:k + 1])
        assert torch.equal(ck1[0], ck_all[k])
        assert torch.equal(aw1[0], aw_all[k])
    ck2, _, _ = plan.integrate(raw[10:45])
    assert torch.equal(ck2, ck_all[10:45])
    assert plan.status() == 0


@pytest.mark.parametrize("dt", [torch.uint8, torch.uint16, torch.int32, torch.int64, torch.float32,
                                torch.float64])
@pytest.mark.parametrize("enc", ["runs", "csr"])
def test_dtypes_agree(cuda, dt, enc):
    g = load_mapper_case("m1")
    n_r, n_eta = g["r_lo"].size, g["eta_lo"].size
    plan = CakePlan(from_arrays(g["records"], g["nmap"]), n_r=n_r, n_eta=n_eta, n_pixels_y=g["ny"],
                    n_pixels_z=g["nz"], mode="floor", device=cuda, encoding=enc)
    rng = np.random.default_rng(3)
    raw = torch.from_numpy(rng.integers(0, 250, size=(4, g["nz"], g["ny"])).astype(np.uint8)).to(cuda)
    ref, _, _ = plan.integrate(raw)
    out, _, _ = plan.integrate(raw.to(dt))
    assert torch.equal(out, ref)


def test_plain_reference_algorithm_matches_oracle(cuda):
    g = load_mapper_case("m2")
    n_r, n_eta = g["r_lo"].size, g["eta_lo"].size
    pm = from_arrays(g["records"], g["nmap"])
    rng = np.random.default_rng(2)
    raw = rng.integers(100, 3000, size=(g["nz"], g["ny"])).astype(np.uint16)
    dark = (100 + rng.standard_normal((g["nz"], g["ny"]))).astype(np.float32)
    for mode in ("floor", "bilinear", "gradient"):
        plan = CakePlan(pm, n_r=n_r, n_eta=n_eta, n_pixels_y=g["ny"], n_pixels_z=g["nz"], mode=mode,
                        bc_y=g["bc_y"], bc_z=g["bc_z"], device=cuda)
        plan.set_dark(dark)
        ck, aw, sm = plan.integrate_plain(torch.from_numpy(raw).to(cuda))
        gg = dict(g, n_r=n_r)
        sub = (raw.astype(np.float32) - dark)[None]
        # the plain kernel is the reference GPU algorithm: sample positions resampled in
        # FP32 (integrate_noMapMask), i.e. the oracle's gpustream positions; DetectorMapper
        # records are all on the detector, so both normalisers agree here
        rc, raw_, rsm = _oracle_batch(gg, sub, mode, True, "gpustream")
        # plain FP32 accumulation without compensation, as in the reference GPU kernel
        assert rel_err(ck.cpu().numpy(), rc[0])[0] <= 2e-6
        assert rel_err(aw.cpu().numpy(), raw_[0])[0] <= 2e-6
        bk, _, _ = plan.integrate(torch.from_numpy(raw).to(cuda))
        rp, _, _ = _oracle_batch(gg, sub, mode, True, "py")
        assert rel_err(bk[0].cpu().numpy(), rp[0])[0] <= TOL


def test_profile_kernel_on_given_cake(cuda):
    g = load_kernels_case("d")
    plan = CakePlan(from_arrays(g["records"], g["nmap"]), n_r=g["n_r"], n_eta=g["n_eta"], n_pixels_y=g["ny"],
                    n_pixels_z=g["nz"], device=cuda)
    rng = np.random.default_rng(4)
    cake = rng.uniform(-5, 500, size=(3, g["n_r"], g["n_eta"]))
    aw, sm = plan.profile(torch.from_numpy(cake).to(cuda))
    area = g["area_per_bin"]
    for k in range(3):
        raw_, rsm = oracle.profile(cake[k].reshape(-1), area, g["n_r"], g["n_eta"])
        np.testing.assert_allclose(aw[k].cpu().numpy(), raw_, rtol=1e-12, atol=1e-12)
        np.testing.assert_allclose(sm[k].cpu().numpy(), rsm, rtol=1e-12, atol=1e-12)


def test_cast_kernel(cuda):
    rng = np.random.default_rng(8)
    for dt, code in ((np.uint16, L.DT_U16), (np.int32, L.DT_I32), (np.uint8, L.DT_U8), (np.float64, L.DT_F64)):
        for n in (4096, 4099):
            x = torch.from_numpy(rng.integers(0, 200, size=(3, n)).astype(dt)).to(cuda)
            d = torch.from_numpy(rng.standard_normal(n).astype(np.float32)).to(cuda)
            out = torch.empty((3, n), dtype=torch.float32, device=cuda)
            L.check(L.lib().mi_cast_dark(x.data_ptr(), code, n, 3, d.data_ptr(), out.data_ptr(), None), "cast")
            torch.cuda.synchronize()
            assert torch.equal(out, x.to(torch.float32) - d[None])


def test_bad_map_raises(cuda):
    g = load_kernels_case("c")
    nmap = g["nmap"].copy()
    nmap[3, 1] = g["records"].size            # offset past the end
    with pytest.raises(L.MidasError) as e:
        CakePlan(from_arrays(g["records"], nmap), n_r=g["n_r"], n_eta=g["n_eta"], n_pixels_y=g["ny"],
                 n_pixels_z=g["nz"], device=cuda)
    assert e.value.code == L.MI_E_MAP


def test_empty_map_and_empty_batch(cuda):
    nmap = np.zeros((12, 2), np.int32)
    recs = np.zeros(0, dtype=oracle.REC_DTYPE)
    plan = CakePlan(from_arrays(recs, nmap), n_r=3, n_eta=4, n_pixels_y=8, n_pixels_z=8, device=cuda)
    ck, aw, sm = plan.integrate(torch.ones((2, 8, 8), dtype=torch.uint16, device=cuda))
    assert torch.count_nonzero(ck) == 0 and torch.count_nonzero(aw) == 0
    ck, aw, sm = plan.integrate(torch.ones((0, 8, 8), dtype=torch.uint16, device=cuda))
    assert ck.shape[0] == 0


def test_upload_copies_the_referenced_columns(cuda):
    """CakePlan.upload moves only the referenced columns of each 16-row group of the
    referenced band (upload_pixels per frame, fewer than the band's full rows); caking the
    uploaded frames equals caking the full frames."""
    from midas_b200 import synth
    from midas_b200.mapper import build_map
    w = synth.scaled(synth.sweep_2880(), 8)
    m = w.mapper
    pm, _ = build_map(m, device=0)
    plan = CakePlan(pm, n_r=w.n_r, n_eta=w.n_eta, n_pixels_y=m.NrPixelsY, n_pixels_z=m.NrPixelsZ, mode=w.mode,
                    bc_y=m.BC_y, bc_z=m.BC_z, device=cuda)
    info = plan.info
    lo, hi = info["ref_row_lo"], info["ref_row_hi"]
    assert 0 < lo < hi < m.NrPixelsZ
    fr = w.frames(0, 6)
    f32 = fr.cpu().int()   # uint16 reductions and masks are compared on the host
    sentinel = int(f32.max()) + 1
    assert sentinel < 65536
    host = fr.cpu().pin_memory()
    dev = torch.full_like(fr, sentinel)
    plan.upload(host, dev)
    torch.cuda.synchronize()
    d32 = dev.cpu().int()
    copied = d32 != sentinel
    assert int(copied.sum()) == fr.shape[0] * info["upload_pixels"]
    assert 0 < info["upload_pixels"] < (hi - lo) * m.NrPixelsY
    assert torch.equal(d32[copied], f32[copied])
    assert not bool(copied[:, :lo].any()) and not bool(copied[:, hi:].any())
    for x, y in zip(plan.integrate(dev), plan.integrate(fr)):
        assert torch.equal(x, y)
    # host staging of exactly the pixels the upload sends, then the upload: the same caking
    staged = torch.full((fr.shape[0],) + tuple(fr.shape[1:]), sentinel, dtype=fr.dtype).pin_memory()
    plan.stage_host(host.numpy(), staged)
    s32 = staged.int()
    moved = s32 != sentinel
    assert int(moved.sum()) == fr.shape[0] * info["upload_pixels"]
    assert torch.equal(moved, copied) and torch.equal(s32[moved], f32[moved])
    dev2 = torch.full_like(fr, sentinel)
    plan.upload(staged, dev2)
    for x, y in zip(plan.integrate(dev2), plan.integrate(fr)):
        assert torch.equal(x, y)


def test_graph_replay_equals_direct_calls(cuda):
    """A batch captured as a CUDA graph (staging, caking, lineouts) replays to the same results
    on new frames copied into the captured buffers."""
    from midas_b200 import synth
    from midas_b200.mapper import build_map
    w = synth.scaled(synth.sweep_2880(), 8)
    m = w.mapper
    pm, _ = build_map(m, device=0)
    plan = CakePlan(pm, n_r=w.n_r, n_eta=w.n_eta, n_pixels_y=m.NrPixelsY, n_pixels_z=m.NrPixelsZ, mode=w.mode,
                    bc_y=m.BC_y, bc_z=m.BC_z, device=cuda)
    plan.set_dark(w.dark().cpu().numpy())
    buf = w.frames(0, 40)
    out = {"cake": torch.empty((40, w.n_r, w.n_eta), dtype=torch.float32, device=cuda),
           "lineout_aw": torch.empty((40, w.n_r), dtype=torch.float64, device=cuda),
           "lineout_sm": torch.empty((40, w.n_r), dtype=torch.float64, device=cuda)}
    g = plan.capture(buf, out)
    for first in (100, 300):
        nxt = w.frames(first, 40)
        buf.copy_(nxt)
        g.replay()
        torch.cuda.synchronize()
        ref = plan.integrate(nxt)
        for k, r in zip(("cake", "lineout_aw", "lineout_sm"), ref):
            assert torch.equal(out[k], r)
    assert plan.status() == 0


def test_autotuner_picks_the_fastest_buildable_plan(cuda):
    from midas_b200 import autotune, synth
    from midas_b200.mapper import build_map
    w = synth.scaled(synth.sweep_2880(), 8)
    m = w.mapper
    pm, _ = build_map(m, device=0)
    fr = w.frames(0, 64)
    cands = [{"tile_rows": 16, "run_len": 0, "tile_pixels": 0}, {"tile_rows": 8, "run_len": 4, "tile_pixels": 0},
             {"tile_rows": 16, "run_len": 2, "tile_pixels": 0}]     # run_len 2 with 16 rows is refused
    res = autotune.tune(pm, fr, n_r=w.n_r, n_eta=w.n_eta, n_pixels_y=m.NrPixelsY, n_pixels_z=m.NrPixelsZ,
                        mode=w.mode, bc_y=m.BC_y, bc_z=m.BC_z, candidates=cands, device=cuda)
    timed = [r for r in res.table if "ms" in r]
    assert len(timed) == 2 and "error" in res.table[2]
    assert res.best_ms == min(r["ms"] for r in timed)
    again = autotune.tune(pm, fr, n_r=w.n_r, n_eta=w.n_eta, n_pixels_y=m.NrPixelsY, n_pixels_z=m.NrPixelsZ,
                          mode=w.mode, bc_y=m.BC_y, bc_z=m.BC_z, candidates=cands, device=cuda)
    assert again is res                                             # cached per map and batch
