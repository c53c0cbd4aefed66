"""TCP ingest with the reference's framing (<u16 dataset, u16 dtype> + payload; hybrid dtype 6),
on the CPU with a test backend: frames reach their streams in order, hybrid payloads decode
as the reference decodes them, and the failure forms end one connection without stopping
the server -- an unknown dtype code, a truncated payload, a producer killed mid-frame --
while a full pending window holds the producer back."""
import socket
import struct
import threading
import time

import numpy as np
import pytest

from midas_b200.ingest import HEADER, FrameIngest, decode_frame, send_frame
from midas_b200.server import CakeServer

from test_server import HostTestBackend, _cfg

NY, NZ = 4, 3


def _wait(pred, timeout=10.0):
    t0 = time.time()
    while time.time() - t0 < timeout:
        if pred():
            return True
        time.sleep(0.01)
    return False


@pytest.fixture
def served():
    be = HostTestBackend(max_batch=4, max_inflight=2, delay_passes=1)
    srv = CakeServer(backend=be, hbm_budget=10**8).start()
    sids = {0: srv.admit(_cfg("a", ny=NY, nz=NZ)), 7: srv.admit(_cfg("b", ny=NY, nz=NZ))}
    got = []
    ing = FrameIngest(srv, sids.get, n_pixels_y=NY, n_pixels_z=NZ, max_pending=8,
                      on_result=lambda d, r: got.append((d, r))).start()
    yield srv, ing, got
    ing.stop()
    srv.stop()


def _connect(ing):
    return socket.create_connection(ing.address, timeout=5)


def test_frames_of_every_dtype_reach_their_streams(served):
    srv, ing, got = served
    rng = np.random.default_rng(0)
    sent = []
    with _connect(ing) as s:
        for k, dt in enumerate([np.uint8, np.uint16, np.uint32, np.int64, np.float32, np.float64]):
            f = rng.integers(0, 200, (NZ, NY)).astype(dt)
            send_frame(s, 7 if k % 2 else 0, f)
            sent.append((7 if k % 2 else 0, f))
        assert _wait(lambda: len(got) == len(sent))
    by_ds = {0: [f for d, f in sent if d == 0], 7: [f for d, f in sent if d == 7]}
    for d in (0, 7):
        res = sorted([r for dd, r in got if dd == d], key=lambda r: r.seq)
        assert [r.stream for r in res] == ["a" if d == 0 else "b"] * len(res)
        for r, f in zip(res, by_ds[d]):
            np.testing.assert_allclose(r.lineout_aw, np.arange(1, 6) * float(f.sum()))
    assert ing.stats.frames == 6 and ing.stats.rejected == 0


def test_hybrid_payload_decodes_like_the_reference():
    rng = np.random.default_rng(1)
    base = rng.integers(0, 65535, (NZ, NY)).astype(np.uint16)
    idx = np.array([0, 5, 11], np.int32)
    val = np.array([70000, 123456789, -5], np.int64)
    payload = struct.pack("<I", 3) + base.tobytes() + idx.tobytes() + val.tobytes()
    out = decode_frame(6, payload, NY, NZ)
    want = base.astype(np.float32).reshape(-1)
    want[idx] = val.astype(np.float32)
    np.testing.assert_array_equal(out.reshape(-1), want)
    with pytest.raises(ValueError):
        decode_frame(6, payload[:-1], NY, NZ)


def test_hybrid_frame_over_the_socket(served):
    srv, ing, got = served
    base = np.full((NZ, NY), 3, np.uint16)
    with _connect(ing) as s:
        send_frame(s, 0, base, hybrid_overflow=([2], [100000]))
        assert _wait(lambda: len(got) == 1)
    want = base.astype(np.float32).reshape(-1)
    want[2] = 100000
    np.testing.assert_allclose(got[0][1].lineout_aw, np.arange(1, 6) * float(want.sum()))


def test_unknown_dtype_ends_that_connection_only(served):
    srv, ing, got = served
    with _connect(ing) as bad:
        bad.sendall(HEADER.pack(0, 9) + b"\0" * 16)
        assert _wait(lambda: ing.stats.rejected == 1)
        bad.settimeout(5)
        assert bad.recv(1) == b""                       # the server closed it
    with _connect(ing) as good:
        send_frame(good, 0, np.ones((NZ, NY), np.uint16))
        assert _wait(lambda: len(got) == 1)
    assert "unknown dtype code 9" in ing.stats.errors


def test_truncated_payload_and_killed_producer_drop_one_frame(served):
    srv, ing, got = served
    f = np.arange(NY * NZ, dtype=np.uint16).reshape(NZ, NY)
    with _connect(ing) as s:
        send_frame(s, 0, f)
        s.sendall(HEADER.pack(0, 1) + f.tobytes()[:5])      # then the producer dies mid-frame
    assert _wait(lambda: ing.stats.dropped_partial == 1 and len(got) == 1)
    with _connect(ing) as s:
        s.sendall(HEADER.pack(7, 1)[:3])                     # killed inside the header
    assert _wait(lambda: ing.stats.dropped_partial == 2)
    with _connect(ing) as s:                                 # the server still takes frames
        send_frame(s, 7, f)
        assert _wait(lambda: len(got) == 2)
    assert ing.stats.frames == 2


def test_full_pending_window_holds_the_producer_back():
    gate = threading.Event()

    class Held(HostTestBackend):
        def ready(self, st, handle):
            return gate.is_set() and super().ready(st, handle)

    be = Held(max_batch=2, max_inflight=1, delay_passes=0)
    srv = CakeServer(backend=be, hbm_budget=10**8).start()
    sid = srv.admit(_cfg("a", ny=NY, nz=NZ))
    done = []
    ing = FrameIngest(srv, sid, n_pixels_y=NY, n_pixels_z=NZ, max_pending=3,
                      on_result=lambda d, r: done.append(r.seq)).start()
    try:
        with _connect(ing) as s:
            for i in range(10):
                send_frame(s, 0, np.full((NZ, NY), i, np.uint16))
            assert _wait(lambda: ing.stats.waits >= 1)
            time.sleep(0.2)
            assert ing.stats.frames == 3 and not done         # three pending, the rest held
            gate.set()
            assert _wait(lambda: len(done) == 10)
        assert sorted(done) == list(range(10))
    finally:
        ing.stop()
        srv.stop()
