"""TCP frame ingest with the reference's framing, feeding a CakeServer.

The producer boundary of IntegratorFitPeaksGPUStream (handle_client,
FF_HEDM/src/IntegratorFitPeaksGPUStream.cu:588-689) and of midas_integrate's FrameServer
(_FrameTCPHandler, packages/midas_integrate/midas_integrate/server.py:80-102): each frame on
a connection is

    <u16 dataset_num, u16 dtype_code>                       (little endian)
    dtype 0..5: ny * nz pixels of u8, u16, u32, i64, f32, f64
    dtype 6 (hybrid): <u32 C>, then ny * nz u16 base pixels, C i32 indices, C i64 values

Frames are decoded on the host (midas_integrate image.py:83-123 for the hybrid layout: the
base as float32 with the overflow values overlaid) and submitted to the stream that
``route(dataset_num)`` names.  An unknown dtype code or a hybrid overflow count that cannot
fit ends the connection (the C server would read a wrong-sized payload; the Python one
raises); a connection that closes mid-frame drops that frame only.  ``max_pending`` bounds
the frames submitted and not yet finished: a handler that would exceed it stops reading its
socket until a frame completes, so a fast producer is held back by TCP flow control, as the
reference's bounded process queue does.
"""
from __future__ import annotations

import socket
import socketserver
import struct
import threading
import time
from dataclasses import dataclass, field
from typing import Callable, Dict, Optional

import numpy as np

HEADER = struct.Struct("<HH")
DTYPES = {0: np.uint8, 1: np.uint16, 2: np.uint32, 3: np.int64, 4: np.float32, 5: np.float64}
HYBRID = 6


def decode_frame(dtype_code: int, payload: bytes, ny: int, nz: int) -> np.ndarray:
    """One frame's pixels as an (nz, ny) array: the code's dtype, or float32 for hybrid."""
    n = ny * nz
    if dtype_code == HYBRID:
        if len(payload) < 4 + 2 * n:
            raise ValueError("hybrid payload shorter than its count and base")
        c = struct.unpack_from("<I", payload, 0)[0]
        if len(payload) != 4 + 2 * n + 12 * c:
            raise ValueError(f"hybrid payload of {len(payload)} B for {c} overflow pixels")
        out = np.frombuffer(payload, np.uint16, n, 4).astype(np.float32)
        if c:
            idx = np.frombuffer(payload, np.int32, c, 4 + 2 * n)
            val = np.frombuffer(payload, np.int64, c, 4 + 2 * n + 4 * c)
            ok = (idx >= 0) & (idx < n)
            out[idx[ok]] = val[ok].astype(np.float32)
        return out.reshape(nz, ny)
    dt = np.dtype(DTYPES[dtype_code])
    if len(payload) != n * dt.itemsize:
        raise ValueError(f"payload of {len(payload)} B, expected {n * dt.itemsize}")
    return np.frombuffer(payload, dt).reshape(nz, ny)


@dataclass
class IngestStats:
    connections: int = 0
    frames: int = 0
    bytes: int = 0
    dropped_partial: int = 0       # frames cut off by a closed connection
    rejected: int = 0              # connections ended by a malformed header or payload
    unrouted: int = 0              # frames whose dataset has no stream
    waits: int = 0                 # times a handler waited for a free pending slot
    errors: Dict[str, int] = field(default_factory=dict)


class _Handler(socketserver.BaseRequestHandler):
    def handle(self) -> None:
        ing: FrameIngest = self.server.ingest  # type: ignore[attr-defined]
        ing._count("connections")
        sock = self.request
        sock.settimeout(ing.client_timeout)
        while not ing._stop.is_set():
            try:
                hdr = _read(sock, HEADER.size)
            except EOFError as e:
                if e.args and e.args[0] > 0:
                    ing._count("dropped_partial")
                return
            except (OSError, socket.timeout):
                return
            dataset, code = HEADER.unpack(hdr)
            n = ing.ny * ing.nz
            try:
                if code == HYBRID:
                    cb = _read(sock, 4)
                    c = struct.unpack("<I", cb)[0]
                    if c > n:
                        ing._reject(f"hybrid overflow count {c} above {n} pixels")
                        return
                    payload = cb + _read(sock, 2 * n + 12 * c)
                elif code in DTYPES:
                    payload = _read(sock, n * np.dtype(DTYPES[code]).itemsize)
                else:
                    ing._reject(f"unknown dtype code {code}")
                    return
            except EOFError:
                ing._count("dropped_partial")
                return
            except (OSError, socket.timeout):
                ing._count("dropped_partial")
                return
            t_arrival = time.perf_counter()
            try:
                frame = decode_frame(code, payload, ing.ny, ing.nz)
            except ValueError as e:
                ing._reject(str(e))
                return
            if not ing._deliver(dataset, frame, t_arrival, len(payload) + HEADER.size):
                return


def _read(sock: socket.socket, n: int) -> bytes:
    """Exactly n bytes; EOFError(bytes read) when the peer closes first."""
    buf = bytearray(n)
    view = memoryview(buf)
    got = 0
    while got < n:
        k = sock.recv_into(view[got:], n - got)
        if k == 0:
            raise EOFError(got)
        got += k
    return bytes(buf)


class _TCPServer(socketserver.ThreadingMixIn, socketserver.TCPServer):
    daemon_threads = True
    allow_reuse_address = True


class FrameIngest:
    """Accepts producer connections and submits their frames to ``server``.

    route: dataset_num -> stream id of ``server`` (None: drop the frame), or one stream id
    for every dataset.  on_result(dataset_num, FrameResult) runs when a frame's result is
    ready (on the server's thread)."""

    def __init__(self, server, route, *, n_pixels_y: int, n_pixels_z: int, host: str = "127.0.0.1",
                 port: int = 0, max_pending: int = 64, client_timeout: Optional[float] = None,
                 frame_dtype: Optional[str] = None,
                 on_result: Optional[Callable[[int, object], None]] = None):
        self.server = server
        self.route = route if callable(route) else (lambda _d, sid=route: sid)
        self.ny, self.nz = int(n_pixels_y), int(n_pixels_z)
        self.client_timeout = client_timeout
        self.frame_dtype = np.dtype(frame_dtype) if frame_dtype else None
        self.on_result = on_result
        self.stats = IngestStats()
        self._lock = threading.Lock()
        self._slots = threading.BoundedSemaphore(max_pending)
        self._stop = threading.Event()
        self._tcp = _TCPServer((host, port), _Handler)
        self._tcp.ingest = self
        self.address = self._tcp.server_address
        self._thread: Optional[threading.Thread] = None

    # -- bookkeeping ----------------------------------------------------------
    def _count(self, key: str, k: int = 1) -> None:
        with self._lock:
            setattr(self.stats, key, getattr(self.stats, key) + k)

    def _reject(self, why: str) -> None:
        with self._lock:
            self.stats.rejected += 1
            self.stats.errors[why] = self.stats.errors.get(why, 0) + 1

    def _deliver(self, dataset: int, frame: np.ndarray, t_arrival: float, nbytes: int) -> bool:
        sid = self.route(dataset)
        if sid is None:
            self._count("unrouted")
            return True
        if self.frame_dtype is not None and frame.dtype != self.frame_dtype:
            frame = frame.astype(self.frame_dtype)
        if not self._slots.acquire(blocking=False):
            self._count("waits")
            while not self._slots.acquire(timeout=0.1):
                if self._stop.is_set():
                    return False
        try:
            fut = self.server.submit(sid, frame, t_arrival)
        except Exception as e:  # unknown or closing stream
            self._slots.release()
            self._reject(f"submit failed: {e}")
            return False
        with self._lock:
            self.stats.frames += 1
            self.stats.bytes += nbytes

        def done(f, dataset=dataset):
            self._slots.release()
            if self.on_result is not None and not f.cancelled() and f.exception() is None:
                try:
                    self.on_result(dataset, f.result())
                except Exception:
                    pass

        fut.add_done_callback(done)
        return True

    # -- lifecycle ------------------------------------------------------------
    def start(self) -> "FrameIngest":
        self._thread = threading.Thread(target=self._tcp.serve_forever, kwargs={"poll_interval": 0.05},
                                        name="midas-ingest", daemon=True)
        self._thread.start()
        return self

    def stop(self) -> None:
        self._stop.set()
        self._tcp.shutdown()
        self._tcp.server_close()
        if self._thread:
            self._thread.join(5.0)

    def __enter__(self) -> "FrameIngest":
        return self.start()

    def __exit__(self, *exc) -> None:
        self.stop()


def send_frame(sock: socket.socket, dataset: int, frame: np.ndarray, hybrid_overflow=None) -> None:
    """Producer side of the framing (what the reference's clients send): a frame of a plain
    dtype, or with ``hybrid_overflow`` = (indices, values) the dtype-6 layout of a u16 base."""
    if hybrid_overflow is not None:
        idx = np.asarray(hybrid_overflow[0], np.int32)
        val = np.asarray(hybrid_overflow[1], np.int64)
        base = np.ascontiguousarray(frame, np.uint16)
        sock.sendall(HEADER.pack(dataset, HYBRID) + struct.pack("<I", idx.size) + base.tobytes() + idx.tobytes()
                     + val.tobytes())
        return
    code = {np.dtype(v): k for k, v in DTYPES.items()}[np.dtype(frame.dtype)]
    sock.sendall(HEADER.pack(dataset, code) + np.ascontiguousarray(frame).tobytes())
