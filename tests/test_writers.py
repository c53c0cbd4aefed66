"""Output files byte-compatible with the reference's (no GPU): lineout.bin and
lineout_simple_mean.bin as (R, I) float64 pairs, Int2D.bin as float64 cakes, fit.bin as 7
float64 per peak in ascending bin order, RTthEtaAreaMap.bin as five blocks of n_bins float64
(IntegratorFitPeaksGPUStream.cu:506-565, 2436-2450, 2616-2688), the OpenMP integrator's
n_r-double lineout.bin (IntegratorZarrOMP.c:1845-1849), and the serving loop writing them."""
import numpy as np

from midas_b200 import writers as W
from midas_b200.server import CakeServer

from test_server import HostTestBackend, _cfg, _drive


def test_stream_files_layout(tmp_path):
    n_r, n_eta = 6, 4
    table = np.zeros((n_r * n_eta, 5))
    table[:, 0] = np.repeat(10.0 + np.arange(n_r), n_eta) + 0.5    # R mean
    table[:, 1] = 0.1 * table[:, 0]
    table[:, 2] = np.tile(-135.0 + 90.0 * np.arange(n_eta), n_r)
    table[:, 3] = 1.5
    table[:, 4] = 0.2 * table[:, 0]
    r_axis = W.lineout_r_axis(table, n_eta)
    np.testing.assert_array_equal(r_axis, 10.5 + np.arange(n_r))
    rng = np.random.default_rng(0)
    aws, sms, cakes, fits = [], [], [], []
    with W.StreamOutputs(tmp_path, r_axis, write_2d=True, write_fit=True, bin_table=table) as out:
        for f in range(3):
            aw, sm = rng.random(n_r), rng.random(n_r)
            ck = rng.random((n_r, n_eta)).astype(np.float32)
            ft = rng.random((2, 7))
            out.write_frame(aw, sm, ck, ft)
            aws.append(aw); sms.append(sm); cakes.append(ck); fits.append(ft)
    sizes = W.file_sizes(tmp_path)
    assert sizes == {"Int2D.bin": 3 * n_r * n_eta * 8, "RTthEtaAreaMap.bin": 5 * n_r * n_eta * 8,
                     "fit.bin": 3 * 2 * 7 * 8, "lineout.bin": 3 * n_r * 16, "lineout_simple_mean.bin": 3 * n_r * 16}
    lo = W.read_lineouts(tmp_path / "lineout.bin", n_r)
    np.testing.assert_array_equal(lo[:, :, 0], np.tile(r_axis, (3, 1)))
    np.testing.assert_array_equal(lo[:, :, 1], np.array(aws))
    raw = np.fromfile(tmp_path / "lineout_simple_mean.bin", np.float64)
    np.testing.assert_array_equal(raw[1::2], np.concatenate(sms))          # interleaved R, I
    np.testing.assert_array_equal(W.read_cakes(tmp_path / "Int2D.bin", n_r, n_eta),
                                  np.array(cakes).astype(np.float64))
    np.testing.assert_array_equal(W.read_fits(tmp_path / "fit.bin"), np.concatenate(fits))
    bt = W.read_bin_table(tmp_path / "RTthEtaAreaMap.bin", n_r * n_eta)
    np.testing.assert_array_equal(bt, table.T)


def test_omp_lineout_layout(tmp_path):
    with W.StreamOutputs(tmp_path, np.arange(5.0), lineout_layout="omp") as out:
        out.write_frame(None, np.arange(5.0))
        out.write_frame(None, np.arange(5.0) * 2)
    assert W.file_sizes(tmp_path) == {"lineout.bin": 2 * 5 * 8}
    np.testing.assert_array_equal(W.read_lineouts(tmp_path / "lineout.bin", 5, "omp"),
                                  [np.arange(5.0), 2 * np.arange(5.0)])


def test_fit_rows_keep_fitted_peaks_in_bin_order():
    x = 0.5 + np.arange(100.0)
    peaks = np.array([60.2, 10.4, 500.0, 30.6])            # 500 is off the grid
    params = np.arange(4 * 11, dtype=np.float64).reshape(4, 11)
    iters = np.array([5, 7, -1, 3])
    rows = W.fit_rows(params, iters, x, peaks)
    np.testing.assert_array_equal(rows, params[[1, 3, 0], :7])


def test_server_writes_the_stream_files_in_frame_order(tmp_path):
    be = HostTestBackend(max_batch=3, max_inflight=2)
    srv = CakeServer(backend=be, hbm_budget=10**8)
    cfg = _cfg("a", n_r=5)
    cfg.output_dir = str(tmp_path / "a")
    cfg.r_axis = 100.0 + np.arange(5.0)
    sid = srv.admit(cfg)
    rng = np.random.default_rng(3)
    frames = [rng.integers(0, 50, (3, 4)) for _ in range(8)]
    futs = [srv.submit(sid, f) for f in frames]
    _drive(srv, futs)
    srv.remove(sid)
    lo = W.read_lineouts(tmp_path / "a" / "lineout.bin", 5)
    assert lo.shape == (8, 5, 2)
    for f, fr in enumerate(frames):
        np.testing.assert_array_equal(lo[f, :, 0], cfg.r_axis)
        np.testing.assert_array_equal(lo[f, :, 1], np.arange(1, 6) * fr.sum())
    sm = W.read_lineouts(tmp_path / "a" / "lineout_simple_mean.bin", 5)
    np.testing.assert_array_equal(sm[:, :, 1], [np.arange(5) + fr.max() for fr in frames])
