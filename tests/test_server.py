"""Scheduling logic of the continuous-batching server, on the CPU.

The device work is replaced by a test backend that "computes" a frame's lineouts as
fixed functions of its pixels and finishes a batch a few scheduling passes after it was
dispatched, so batching, slot reuse, admission by footprint, draining, cancellation
and latency accounting are exercised without a GPU.  (The product backend has no host
path; the GPU test of the same server is test_gpu_server.py.)"""
import threading
import time
from dataclasses import dataclass

import numpy as np
import pytest

from midas_b200.server import AdmissionError, CakeServer, PinnedPool, StreamConfig


@dataclass
class _PM:                        # the two attributes the server reads from a PixelMap
    n_entries: int
    n_bins: int


class HostTestBackend:
    """Backend double: lineout_aw[i] = sum(frame) * (i + 1), lineout_sm[i] = max(frame) + i."""

    def __init__(self, max_batch=4, max_inflight=2, delay_passes=2, free=10**9):
        self.max_batch, self.max_inflight, self.delay = max_batch, max_inflight, delay_passes
        self.free = free
        self.dispatched = []          # (stream name, batch size)
        self.opened, self.closed = [], []

    def free_bytes(self):
        return self.free

    def footprint_estimate(self, cfg):
        return cfg.pixmap.n_entries * 10

    def open(self, cfg):
        self.opened.append(cfg.name)
        return {"free": list(range(self.max_inflight)), "polls": {}}, cfg.pixmap.n_entries * 8

    def batch_limit(self, st):
        return self.max_batch

    def can_dispatch(self, st):
        return bool(st["free"])

    def dispatch(self, st, cfg, frames):
        k = st["free"].pop()
        self.dispatched.append((cfg.name, len(frames)))
        res = [(np.arange(1, cfg.n_r + 1) * float(f.sum()), np.arange(cfg.n_r) + float(f.max()), None, None)
               for f in frames]
        st["polls"][k] = 0
        return (k, res)

    def ready(self, st, handle):
        st["polls"][handle[0]] += 1
        return st["polls"][handle[0]] > self.delay

    def collect(self, st, cfg, handle):
        st["free"].append(handle[0])
        return handle[1]

    def close(self, st):
        self.closed.append(st)


def _cfg(name, entries=1000, n_r=5, ny=4, nz=3):
    return StreamConfig(name=name, pixmap=_PM(entries, n_r), n_r=n_r, n_eta=1, n_pixels_y=ny, n_pixels_z=nz)


def _drive(srv, futs, limit=10000):
    for _ in range(limit):
        if all(f.done() for f in futs):
            return
        srv._pass()
    raise AssertionError("scheduler did not complete the requests")


def test_frames_are_batched_per_stream_and_results_follow_their_frames():
    be = HostTestBackend(max_batch=4, max_inflight=2)
    srv = CakeServer(backend=be, hbm_budget=10**8)
    a, b = srv.admit(_cfg("a")), srv.admit(_cfg("b", n_r=3, ny=2, nz=2))
    rng = np.random.default_rng(0)
    fa = [rng.integers(0, 100, (3, 4)) for _ in range(11)]
    fb = [rng.integers(0, 100, (2, 2)) for _ in range(5)]
    futs_a = [srv.submit(a, f) for f in fa]
    futs_b = [srv.submit(b, f) for f in fb]
    _drive(srv, futs_a + futs_b)
    for f, fut in zip(fa, futs_a):
        r = fut.result()
        assert r.stream == "a"
        np.testing.assert_array_equal(r.lineout_aw, np.arange(1, 6) * f.sum())
        np.testing.assert_array_equal(r.lineout_sm, np.arange(5) + f.max())
    assert [fut.result().seq for fut in futs_a] == list(range(11))
    # all frames that were queued when a slot freed go in one launch, at most max_batch
    sizes_a = [n for s, n in be.dispatched if s == "a"]
    assert sum(sizes_a) == 11 and max(sizes_a) == 4 and len(sizes_a) == 3
    assert [n for s, n in be.dispatched if s == "b"] == [4, 1]
    assert srv.completed == 16 and srv.latency_ms()["n"] == 16


def test_later_arrivals_join_the_next_batch_while_slots_are_busy():
    be = HostTestBackend(max_batch=8, max_inflight=1, delay_passes=3)
    srv = CakeServer(backend=be, hbm_budget=10**8)
    s = srv.admit(_cfg("s"))
    first = srv.submit(s, np.ones((3, 4)))
    srv._pass()                                     # dispatches the single frame
    later = [srv.submit(s, np.full((3, 4), i)) for i in range(5)]
    _drive(srv, [first] + later)
    assert be.dispatched == [("s", 1), ("s", 5)]
    assert all(f.result().batch_size == 5 for f in later)


def test_admission_by_footprint_and_readmission_after_removal():
    be = HostTestBackend()
    srv = CakeServer(backend=be, hbm_budget=25_000)
    a = srv.admit(_cfg("a", entries=1000))          # estimate 10000, holds 8000
    srv.admit(_cfg("b", entries=1000))              # 16000 held
    with pytest.raises(AdmissionError):
        srv.admit(_cfg("c", entries=1000))          # 16000 + 10000 > 25000
    assert be.opened == ["a", "b"]
    srv.remove(a)
    assert srv.used == 8000
    srv.admit(_cfg("c", entries=1000))
    assert be.opened == ["a", "b", "c"] and len(be.closed) == 1


def test_remove_drains_queued_frames_or_cancels_them():
    be = HostTestBackend(max_batch=2, max_inflight=1)
    srv = CakeServer(backend=be, hbm_budget=10**8)
    a = srv.admit(_cfg("a"))
    futs = [srv.submit(a, np.ones((3, 4))) for _ in range(5)]
    srv.remove(a, drain=True)
    assert all(f.done() and not f.cancelled() for f in futs)
    b = srv.admit(_cfg("b"))
    futs = [srv.submit(b, np.ones((3, 4))) for _ in range(5)]
    srv.remove(b, drain=False)
    assert all(f.cancelled() for f in futs)
    late = srv.submit(b, np.ones((3, 4)))
    with pytest.raises(KeyError):
        late.result(timeout=1)


def test_bad_frame_size_is_rejected_on_submit():
    srv = CakeServer(backend=HostTestBackend(), hbm_budget=10**8)
    s = srv.admit(_cfg("s"))
    with pytest.raises(ValueError, match="expects 12"):
        srv.submit(s, np.ones((5, 5))).result(timeout=1)


def test_pinned_pool_first_fit_alignment_and_coalescing():
    import torch
    pool = PinnedPool(4096, pin=False)            # the allocator logic; page-locking needs a GPU
    a, ta = pool.alloc((10,), torch.float64)       # 80 B -> one 256 B block
    b, tb = pool.alloc((3, 100), torch.int32)      # 1200 B -> 1280
    c, tc = pool.alloc((5,), torch.uint16)
    assert (ta, tb, tc) == ((0, 256), (256, 1280), (1536, 256))
    assert b.shape == (3, 100) and b.dtype == torch.int32
    assert b.data_ptr() - pool.buf.data_ptr() == 256
    with pytest.raises(AdmissionError):
        pool.alloc((4096,), torch.uint8)
    pool.release(tb)
    d, td = pool.alloc((1000,), torch.uint8)       # first fit reuses the freed range
    assert td == (256, 1024)
    for t in (ta, tc, td):
        pool.release(t)
    assert pool.free == [(0, 4096)] and pool.free_bytes() == 4096


def test_threaded_server_with_concurrent_submitters():
    be = HostTestBackend(max_batch=6, max_inflight=2, delay_passes=1)
    with CakeServer(backend=be, hbm_budget=10**8, tick_s=1e-4) as srv:
        ids = [srv.admit(_cfg(f"s{i}")) for i in range(3)]
        out = {}

        def producer(sid):
            rng = np.random.default_rng(sid)
            frames = [rng.integers(0, 50, (3, 4)) for _ in range(40)]
            futs = []
            for f in frames:
                futs.append(srv.submit(sid, f))
                time.sleep(rng.exponential(2e-4))
            out[sid] = (frames, [fu.result(timeout=10) for fu in futs])

        th = [threading.Thread(target=producer, args=(sid,)) for sid in ids]
        for t in th:
            t.start()
        for t in th:
            t.join()
    for sid, (frames, res) in out.items():
        assert [r.seq for r in res] == list(range(40))
        for f, r in zip(frames, res):
            np.testing.assert_array_equal(r.lineout_aw, np.arange(1, 6) * f.sum())
    lat = srv.latency_ms()
    assert lat["n"] == 120 and lat["p99"] >= lat["p50"] > 0
    ps = srv.pass_stats()
    assert ps["passes"] > 0 and ps["max_pass_ms"] > 0 and ps["max_dispatch_ms"] > 0
    assert ps["max_pass_ms"] >= max(ps["max_ready_ms"], ps["max_collect_ms"], ps["max_dispatch_ms"])
    srv.reset_pass_stats()
    assert srv.pass_stats()["passes"] == 0


def test_peak_rows_two_theta_and_d_spacing():
    """pfio_make_row (PeakFitIO.c:52-82): 2-theta from the centre in px, Bragg d-spacing."""
    import math
    from midas_b200.peakfit import peak_rows
    params = np.zeros((2, 3, 11))
    params[..., 0] = 5.0
    params[..., 1] = [[300.0, 512.5, 0.0], [301.0, 700.0, 1e-9]]
    params[..., 4] = 0.01
    rows = peak_rows(params, px_um=200.0, lsd_um=1e6, wavelength_a=0.172979, first_frame=10)
    assert rows.shape == (6,)
    assert list(rows["frame_idx"]) == [10, 10, 10, 11, 11, 11]
    assert list(rows["peak_nr"]) == [0, 1, 2, 0, 1, 2]
    for r, c in zip(rows, params[..., 1].reshape(-1)):
        tth = math.atan(c * 200.0 / 1e6) * 180.0 / math.pi
        th = tth * math.pi / 360.0
        assert r["center_2theta"] == tth
        assert r["d_spacing_A"] == (0.172979 / (2.0 * math.sin(th)) if th > 1e-10 else 0.0)
    assert rows["d_spacing_A"][2] == 0.0 and rows["d_spacing_A"][5] == 0.0
    assert np.all(rows["area"] == 5.0) and np.all(rows["FWHM_deg"] == 0.01)


class HostRingBackend(HostTestBackend):
    """HostTestBackend with the staging protocol of DeviceBackend: frames are copied into a
    ring of ``R`` entries by the submitting thread (``reserve`` + ``stage``), batches name
    their entries, and a batch's entries are released when it is collected."""

    def __init__(self, R=6, slow=None, **kw):
        super().__init__(**kw)
        self.R, self.slow = R, slow or {}
        self.rings = []

    def open(self, cfg):
        st, fp = super().open(cfg)
        st.update(ring=[None] * self.R, R=self.R, head=0, tail=0, cv=threading.Condition(), n_staged=0)
        return st, fp

    def reserve(self, st, timeout=10.0):
        with st["cv"]:
            if not st["cv"].wait_for(lambda: st["head"] - st["tail"] < st["R"], timeout):
                raise TimeoutError("ring full")
            i = st["head"] % st["R"]
            st["head"] += 1
            return i

    def stage(self, st, idx, frame, cfg):
        k = st["n_staged"]
        st["n_staged"] += 1
        if k in self.slow:
            time.sleep(self.slow[k])
        st["ring"][idx] = np.array(frame, copy=True)

    def dispatch(self, st, cfg, frames, ring=None):
        assert ring is not None
        assert all((b - a) % st["R"] == 1 for a, b in zip(ring, ring[1:])), ring
        self.rings.append(list(ring))
        return super().dispatch(st, cfg, [st["ring"][i] for i in ring])

    def collect(self, st, cfg, handle):
        res = super().collect(st, cfg, handle)
        with st["cv"]:
            st["tail"] += len(res)
            st["cv"].notify_all()
        return res


def test_frames_staged_at_submission_in_ring_order_with_wraparound():
    be = HostRingBackend(R=6, max_batch=4, max_inflight=1)
    srv = CakeServer(backend=be, hbm_budget=10**8)
    a = srv.admit(_cfg("a"))
    rng = np.random.default_rng(1)
    frames = [rng.integers(0, 100, (3, 4)) for _ in range(6)]
    futs = [srv.submit(a, f) for f in frames[:4]]
    _drive(srv, futs)                       # ring entries 0-3
    futs += [srv.submit(a, f) for f in frames[4:]]
    _drive(srv, futs)                       # entries 4, 5
    more = [rng.integers(0, 100, (3, 4)) for _ in range(3)]
    futs2 = [srv.submit(a, f) for f in more]
    _drive(srv, futs2)                      # entries 0, 1, 2 again
    for f, fut in zip(frames + more, futs + futs2):
        np.testing.assert_array_equal(fut.result().lineout_aw, np.arange(1, 6) * f.sum())
    assert be.rings == [[0, 1, 2, 3], [4, 5], [0, 1, 2]]


def test_full_ring_holds_the_submitter_back_until_a_batch_finishes():
    be = HostRingBackend(R=4, max_batch=4, max_inflight=1, delay_passes=2)
    srv = CakeServer(backend=be, hbm_budget=10**8)
    a = srv.admit(_cfg("a"))
    futs = [srv.submit(a, np.full((3, 4), i)) for i in range(4)]
    done = threading.Event()
    extra = []

    def late():
        extra.append(srv.submit(a, np.full((3, 4), 9)))
        done.set()

    t = threading.Thread(target=late)
    t.start()
    assert not done.wait(0.2)               # all four entries hold frames not yet uploaded
    _drive(srv, futs)
    assert done.wait(5.0)
    t.join()
    _drive(srv, extra)
    assert extra[0].result().lineout_sm[0] == 9 and be.rings == [[0, 1, 2, 3], [0]]


def test_a_frame_still_being_staged_holds_back_the_frames_behind_it():
    be = HostRingBackend(R=8, max_batch=8, max_inflight=1, slow={1: 0.3})
    srv = CakeServer(backend=be, hbm_budget=10**8)
    a = srv.admit(_cfg("a"))
    first = srv.submit(a, np.full((3, 4), 1))
    box = []
    t = threading.Thread(target=lambda: box.append(srv.submit(a, np.full((3, 4), 2))))
    t.start()
    while not srv.streams[a].pending or len(srv.streams[a].pending) < 2:
        time.sleep(0.01)
    third = srv.submit(a, np.full((3, 4), 3))
    srv._pass()                             # only the first frame is staged ahead of the slow one
    assert be.dispatched == [("a", 1)]
    t.join()
    _drive(srv, [first, box[0], third])
    assert be.dispatched == [("a", 1), ("a", 2)]
    assert [f.result().lineout_sm[0] for f in (first, box[0], third)] == [1, 2, 3]
