"""Serving: continuous batching of frames from several detector streams on one GPU.

Replaces the one-frame-at-a-time worker of the reference servers
(packages/midas_integrate/midas_integrate/server.py:113-179; the stream loop of
FF_HEDM/src/IntegratorFitPeaksGPUStream.cu:2571-2883, 4 CUDA streams round-robin,
one frame per submit) with a scheduler that

* keeps every admitted stream's map plan, dark and fit state resident on the device;
* admits a stream only if its HBM footprint (plan + device buffers) fits the budget
  left by the streams already admitted; a refused stream can be retried once others
  leave;
* on every scheduling tick, takes ALL frames that arrived for a stream since its last
  dispatch (up to ``max_batch``) and launches them as one batch -- H2D copy, batched
  caking with both lineouts, batched peak fits, D2H of lineouts and fits -- on that
  stream's own CUDA stream, with up to ``max_inflight`` batches per stream in flight, so
  work from different streams and successive batches overlaps on the device;
* completes each request's future when its batch's event has fired, with the latency
  arrival -> results on the host.

A frame's results do not depend on which other frames share its batch (each frame is
one lane of the batched kernels and is reduced in a fixed order), so a stream gets the
same answer alone and in the mix.

The device work goes through a backend; the default ``DeviceBackend`` runs
libmidas_b200.  There is no CPU path in the product: a backend that computes on the
host exists only in the tests, to exercise the scheduling logic without a GPU.
"""
from __future__ import annotations

import collections
import ctypes as C
import itertools
import os
import threading
import time
from concurrent.futures import Future
from dataclasses import dataclass, field
from typing import Dict, List, Optional

import numpy as np

from . import _lib as L
from .kernels import dtype_code
from .peakfit import MODELS


class AdmissionError(RuntimeError):
    """The stream's device footprint does not fit the remaining HBM budget (or its host
    staging does not fit the pinned pool)."""


class PinnedPool:
    """Page-locked host memory taken once, up front, and carved into staging buffers.

    Page-locking memory (cudaHostAlloc) takes a driver lock for a time proportional to
    the size, stalling the CUDA calls of every other thread; a stream admitted while
    others run must not do that, so its staging comes from this pool (first fit,
    256-byte aligned, coalescing free list)."""

    ALIGN = 256

    def __init__(self, nbytes: int, pin: bool = True):
        import torch
        self.torch = torch
        self.nbytes = int(nbytes)
        self.buf = torch.empty(self.nbytes, dtype=torch.uint8, pin_memory=pin)
        self.free = [(0, self.nbytes)]
        self._lock = threading.Lock()

    def alloc(self, shape, dtype):
        """(tensor view, token) or AdmissionError when no free range is large enough."""
        n = int(np.prod(shape)) * self.torch.empty((), dtype=dtype).element_size()
        n = max(self.ALIGN, (n + self.ALIGN - 1) // self.ALIGN * self.ALIGN)
        with self._lock:
            for i, (off, size) in enumerate(self.free):
                if size >= n:
                    self.free[i:i + 1] = [(off + n, size - n)] if size > n else []
                    t = self.buf[off:off + n].view(dtype)[:int(np.prod(shape))].view(shape)
                    return t, (off, n)
        raise AdmissionError(f"pinned staging pool ({self.nbytes / 1e9:.2f} GB) has no free {n / 1e6:.1f} MB range")

    def release(self, token) -> None:
        off, n = token
        with self._lock:
            self.free.append((off, n))
            self.free.sort()
            merged = []
            for o, s in self.free:
                if merged and merged[-1][0] + merged[-1][1] == o:
                    merged[-1] = (merged[-1][0], merged[-1][1] + s)
                else:
                    merged.append((o, s))
            self.free = merged

    def free_bytes(self) -> int:
        with self._lock:
            return sum(s for _, s in self.free)


@dataclass
class StreamConfig:
    name: str
    pixmap: object                 # bin_io.PixelMap
    n_r: int
    n_eta: int
    n_pixels_y: int
    n_pixels_z: int
    mode: str = "floor"
    bc_y: float = 0.0
    bc_z: float = 0.0
    dark: Optional[np.ndarray] = None
    frame_dtype: str = "uint16"    # numpy dtype name of the raw frames
    r_axis: Optional[np.ndarray] = None     # lineout x (R bin centres) for the fits
    peaks: Optional[np.ndarray] = None      # ring positions to fit (x units)
    fit_model: str = "pv"
    fit_half_window: int = 12
    x_bin: float = 1.0
    want_cake: bool = False
    tile_rows: int = 0             # run encoding only
    encoding: Optional[str] = None  # batched kernel (kernels.CakePlan encodings); None = the
                                    # backend's choice (DeviceBackend.encoding_for)
    max_batch: int = 0             # frames per launch at most (0 = the backend's default)
    output_dir: Optional[str] = None   # write the reference's per-frame files there (writers.py):
                                       # lineout.bin, lineout_simple_mean.bin, fit.bin (peaks
                                       # set), Int2D.bin (want_cake)


@dataclass
class FrameResult:
    stream: str
    seq: int
    lineout_aw: np.ndarray
    lineout_sm: np.ndarray
    fits: Optional[np.ndarray]     # [n_peaks, 11]
    cake: Optional[np.ndarray]
    latency_s: float
    batch_size: int
    t_arrival: float               # time.perf_counter() of the arrival,
    t_submit: float                # of the submit() call,
    t_dispatch: float              # of the launch of its batch,
    t_complete: float              # and of its completion


@dataclass
class _Req:
    seq: int
    frame: np.ndarray
    t_arrival: float
    fut: Future
    t_submit: float = 0.0
    t_dispatch: float = 0.0
    ring: int = -1                 # staging-ring entry holding the frame (backends that stage)
    staged: bool = True            # the frame is in its ring entry


@dataclass
class _Stream:
    sid: int
    cfg: StreamConfig
    state: object                  # backend-specific
    footprint: int
    pending: collections.deque = field(default_factory=collections.deque)
    inflight: collections.deque = field(default_factory=collections.deque)   # (handle, reqs)
    seq: itertools.count = field(default_factory=itertools.count)
    closing: bool = False
    writer: object = None          # writers.StreamOutputs when cfg.output_dir is set
    fit_valid: Optional[np.ndarray] = None
    submit_lock: threading.Lock = field(default_factory=threading.Lock)


class DeviceBackend:
    """Runs a stream's batches through libmidas_b200 on one CUDA device.

    Each admitted stream gets its plan (map, dark), its own CUDA stream, a ring of
    ``(max_inflight + 1) x batch limit`` pinned host frames and ``max_inflight`` slots of
    device buffers and pinned results; a batch is H2D -> ``mi_integrate_batch`` ->
    ``mi_fit_batch`` -> D2H, all on the stream's CUDA stream, and a slot is reused only after
    its event has fired.  A frame is copied into its ring entry by the thread that submits
    it (``reserve`` + ``stage``: the pixels the upload sends, in C without the interpreter
    lock), so the scheduler thread only uploads and launches; an entry is reused once the
    batch that uploaded it has finished.

    ``plain=True`` serves the same requests with the reference's algorithm, one frame
    per launch (``mi_integrate_plain`` and a one-frame fit per frame): the comparison
    arm of the serving benchmark.

    ``small_batch``: batches of at most this many frames go through that one-frame kernel
    too (the batched kernels' cost per launch hardly depends on the frame count, and for
    one frame the one-frame kernel is 1.5 to 4 times faster); larger batches use the
    stream's batched encoding.  A frame's result then depends on which path served it,
    never on the other frames of its batch.

    ``graph_batches``: for batches of up to this many frames (by default every batch size up
    to 32), the device part of a dispatch after the upload (caking, fits, result copies) is
    one CUDA graph per (slot, batch size), recorded when the stream is admitted and replayed
    with one launch, so a batch costs the scheduler thread the upload calls and one launch.
    """

    def __init__(self, device: int = 0, max_batch: int = 32, max_inflight: int = 2, plain: bool = False,
                 pinned_bytes: int = 2 << 30, build_threads: int = 0, graph_batches: int = 32,
                 small_batch: int = 1):
        import torch
        self.torch = torch
        self.device = torch.device("cuda", device)
        # host threads building an admitted stream's plan: a quarter of the cores (at most 4)
        self.build_threads = build_threads or max(1, min(4, (os.cpu_count() or 4) // 4))
        self._dmax = dict.fromkeys(("stage_ms", "upload_ms", "integrate_ms"), 0.0)
        self.max_batch = max_batch
        self.max_inflight = max_inflight
        self.plain = plain
        self.graph_batches = 0 if plain else int(graph_batches)
        self.small_batch = int(small_batch)
        self.pool = PinnedPool(pinned_bytes)
        self.alg_bytes = 0          # map bytes per launch + frame bytes, summed over dispatches
        self.launches = 0           # libmidas_b200 entry-point calls that launch kernels

    def free_bytes(self) -> int:
        free, _ = self.torch.cuda.mem_get_info(self.device)
        return int(free)

    @staticmethod
    def encoding_for(cfg: StreamConfig) -> str:
        """The stream's batched encoding: its own, else the tensor cores for 8/16-bit frames
        and the per-bin CSR kernel otherwise (both cost less per launch than the run
        encoding at serving batch sizes)."""
        if cfg.encoding:
            return cfg.encoding
        return "mma" if cfg.frame_dtype in ("uint8", "uint16") else "csr"

    def _one_frame(self, n: int) -> bool:
        return self.plain or n <= self.small_batch

    def batch_limit(self, st) -> int:
        return st["B"]

    def open(self, cfg: StreamConfig):
        torch = self.torch
        from .kernels import CakePlan
        fit = cfg.peaks is not None and len(cfg.peaks) > 0
        if fit and (cfg.r_axis is None or len(cfg.r_axis) != cfg.n_r):
            raise ValueError(f"stream {cfg.name!r}: fits need r_axis with n_r = {cfg.n_r} entries")
        tdt = getattr(torch, cfg.frame_dtype)
        B, nz, ny = cfg.max_batch or self.max_batch, cfg.n_pixels_z, cfg.n_pixels_y
        ck_dt = torch.float64 if self.plain else torch.float32
        tokens = []

        def pinned(shape, dtype):
            t, tok = self.pool.alloc(shape, dtype)
            tokens.append(tok)
            return t

        R = B * (self.max_inflight + 1)
        try:
            ring = pinned((R, nz, ny), tdt)
            host = []
            for _ in range(self.max_inflight):
                h = {"h_aw": pinned((B, cfg.n_r), torch.float64), "h_sm": pinned((B, cfg.n_r), torch.float64)}
                if cfg.want_cake:
                    h["h_cake"] = pinned((B, cfg.n_r, cfg.n_eta), ck_dt)
                if fit:
                    h["h_fit"] = pinned((B, len(cfg.peaks), L.FIT_NOUT), torch.float64)
                host.append(h)
        except AdmissionError:
            for tok in tokens:
                self.pool.release(tok)
            raise
        # a stream admitted while others are served builds its plan on a few host cores, so
        # the scheduler thread and the callers submitting frames keep theirs
        enc = self.encoding_for(cfg)
        plan = CakePlan(cfg.pixmap, n_r=cfg.n_r, n_eta=cfg.n_eta, n_pixels_y=cfg.n_pixels_y,
                        n_pixels_z=cfg.n_pixels_z, mode=cfg.mode, bc_y=cfg.bc_y, bc_z=cfg.bc_z,
                        device=self.device, tile_rows=cfg.tile_rows if enc == "runs" else 0, encoding=enc,
                        host_threads=self.build_threads)
        if cfg.dark is not None:
            plan.set_dark(cfg.dark)
        slots = []
        for h in host:
            s = dict(h)
            s.update({
                "d_frames": torch.empty((B, nz, ny), dtype=tdt, device=self.device),
                "d_aw": torch.empty((B, cfg.n_r), dtype=torch.float64, device=self.device),
                "d_sm": torch.empty((B, cfg.n_r), dtype=torch.float64, device=self.device),
                "event": torch.cuda.Event(),
            })
            if cfg.want_cake or self.plain:
                s["d_cake"] = torch.empty((B, cfg.n_r, cfg.n_eta), dtype=ck_dt, device=self.device)
            if not self.plain and self.small_batch > 0:
                # the one-frame kernel's FP64 cake of a small batch
                s["d_cake64"] = torch.empty((min(B, self.small_batch), cfg.n_r, cfg.n_eta), dtype=torch.float64,
                                            device=self.device)
            if fit:
                npk = len(cfg.peaks)
                s["d_fit"] = torch.empty((B, npk, L.FIT_NOUT), dtype=torch.float64, device=self.device)
                s["d_iters"] = torch.empty((B, npk), dtype=torch.int32, device=self.device)
            slots.append(s)
        st = {"plan": plan, "slots": slots, "free": list(range(self.max_inflight)), "B": B,
              "stream": torch.cuda.Stream(self.device), "map_bytes": int(plan.info["map_bytes"]),
              "frame_bytes": nz * ny * np.dtype(cfg.frame_dtype).itemsize, "tokens": tokens,
              "ring": ring, "R": R, "head": 0, "tail": 0, "ring_cv": threading.Condition()}
        if fit:
            st["x"] = torch.as_tensor(np.asarray(cfg.r_axis, np.float64), device=self.device)
            st["peaks"] = torch.as_tensor(np.asarray(cfg.peaks, np.float64), device=self.device)
            st["fit_opts"] = L.MiFitOpts(MODELS[cfg.fit_model], int(cfg.fit_half_window), 100,
                                         float(cfg.x_bin), 0.0, 0.0)
        fp = plan.info["device_bytes"]
        for s in slots:
            fp += sum(v.numel() * v.element_size() for k, v in s.items() if k.startswith("d_"))
        for s in slots:
            s["graphs"] = {}
            for n in range(1, min(B, self.graph_batches) + 1):
                s["graphs"][n] = self._record(st, cfg, s, n)
        return st, int(fp)

    def _upload(self, st, s, r0, n, strm):
        """H2D of ring entries r0 .. r0 + n - 1 (mod R) into the slot's first n device frames:
        the referenced pixels only, one call per contiguous piece of the ring."""
        R, ring, plan = st["R"], st["ring"], st["plan"]
        a = min(n, R - r0)
        plan.upload(ring[r0:r0 + a], s["d_frames"], stream=strm)
        if a < n:
            plan.upload(ring[:n - a], s["d_frames"][a:], stream=strm)

    def _device_work(self, st, cfg, s, n, strm):
        """Caking, fits and result copies of the slot's first n device frames on strm: the
        one-frame kernel per frame for small batches (and in plain mode), else one launch of
        the batched plan."""
        fit = "d_fit" in s
        if self._one_frame(n):
            code = dtype_code(s["d_frames"].dtype)
            ck = s["d_cake"] if self.plain else s["d_cake64"]
            for i in range(n):
                L.check(L.lib().mi_integrate_plain(st["plan"]._h, s["d_frames"][i].data_ptr(), code,
                                                   ck[i].data_ptr(), s["d_aw"][i].data_ptr(), s["d_sm"][i].data_ptr(),
                                                   L.stream_ptr(strm)), "mi_integrate_plain")
                if fit:
                    self._fit(st, cfg, s, i, 1, strm)
            if cfg.want_cake and not self.plain:
                s["d_cake"][:n].copy_(ck[:n])
        else:
            out = {"lineout_aw": s["d_aw"][:n], "lineout_sm": s["d_sm"][:n]}
            if cfg.want_cake:
                out["cake"] = s["d_cake"][:n]
            st["plan"].integrate(s["d_frames"][:n], cake=cfg.want_cake, out=out, stream=strm)
            if fit:
                self._fit(st, cfg, s, 0, n, strm)
        if fit:
            s["h_fit"][:n].copy_(s["d_fit"][:n], non_blocking=True)
        s["h_aw"][:n].copy_(s["d_aw"][:n], non_blocking=True)
        s["h_sm"][:n].copy_(s["d_sm"][:n], non_blocking=True)
        if cfg.want_cake:
            s["h_cake"][:n].copy_(s["d_cake"][:n], non_blocking=True)

    def _record(self, st, cfg, s, n):
        """The slot's device work for n frames (after their upload) as a CUDA graph, recorded
        on the stream's own CUDA stream (capture errors local to this thread: other threads
        keep their calls)."""
        torch = self.torch
        strm = st["stream"]
        launches = self.launches
        with torch.cuda.stream(strm):
            self._upload(st, s, 0, n, strm)
            self._device_work(st, cfg, s, n, strm)       # warm-up: kernels loaded, attributes set
        strm.synchronize()
        # capture_begin / capture_end directly: the torch.cuda.graph context would first
        # synchronise the device and empty the device and pinned-host caches (frees, which
        # stall every thread's CUDA calls) while the other streams are being served
        g = torch.cuda.CUDAGraph()
        with torch.cuda.stream(strm):
            g.capture_begin(capture_error_mode="thread_local")
            try:
                self._device_work(st, cfg, s, n, strm)
            finally:
                g.capture_end()
        strm.synchronize()
        self.launches = launches
        return g

    def footprint_estimate(self, cfg: StreamConfig) -> int:
        """Upper estimate before building anything: map + staging + buffers."""
        recs = cfg.pixmap.n_entries
        B = cfg.max_batch or self.max_batch
        item = np.dtype(cfg.frame_dtype).itemsize
        ck = 8 if self.plain else (4 if cfg.want_cake else 0)
        per_slot = B * (cfg.n_pixels_y * cfg.n_pixels_z * item + 16 * cfg.n_r + ck * cfg.n_r * cfg.n_eta)
        plan = recs * 60 + 256 * cfg.n_r * 12 * 16 + cfg.n_pixels_y * cfg.n_pixels_z * 8
        return int(plan + self.max_inflight * per_slot)

    # -- staging at submission ------------------------------------------------------
    def reserve(self, st, timeout: float = 60.0) -> int:
        """The next ring entry, in submission order; waits while every entry holds a frame
        not yet uploaded (a fast producer is held back)."""
        cv = st["ring_cv"]
        with cv:
            if not cv.wait_for(lambda: st["head"] - st["tail"] < st["R"], timeout):
                raise TimeoutError("staging ring full: no batch of the stream finished in time")
            i = st["head"] % st["R"]
            st["head"] += 1
            return i

    def stage(self, st, idx: int, frame: np.ndarray, cfg: StreamConfig) -> None:
        """Copy a frame into its ring entry (caller's thread)."""
        dst = st["ring"][idx]
        if frame.dtype == dst.numpy().dtype and frame.flags.c_contiguous:
            st["plan"].stage_host(frame, dst)      # the pixels the upload sends, without the GIL
        else:
            dst.numpy()[...] = frame.reshape(cfg.n_pixels_z, cfg.n_pixels_y)

    def _release(self, st, n: int) -> None:
        cv = st["ring_cv"]
        with cv:
            st["tail"] += n
            cv.notify_all()

    def can_dispatch(self, st) -> bool:
        return bool(st["free"])

    def _fit(self, st, cfg, s, first, n, strm):
        L.check(L.lib().mi_fit_batch(st["x"].data_ptr(), s["d_aw"][first].data_ptr(), n, cfg.n_r,
                                     st["peaks"].data_ptr(), st["peaks"].numel(), C.byref(st["fit_opts"]),
                                     s["d_fit"][first].data_ptr(), s["d_iters"][first].data_ptr(),
                                     L.stream_ptr(strm)), "mi_fit_batch")

    def dispatch_stats(self, reset: bool = False) -> Dict[str, float]:
        """Slowest step of dispatch() so far, per step (ms): the host staging copy (frames
        not staged at submission), the upload, and the device work (graph replay, or the
        caking and fit launches and result copies) with the event record."""
        out = dict(self._dmax)
        if reset:
            self._dmax = dict.fromkeys(self._dmax, 0.0)
        return out

    def dispatch(self, st, cfg: StreamConfig, frames: List[np.ndarray], ring: Optional[List[int]] = None):
        """Launch a batch: ``ring`` = the ring entries its frames were staged into (consecutive,
        in order); without it the frames are staged here first."""
        torch = self.torch
        clock, dm = time.perf_counter, self._dmax
        t0 = clock()
        k = st["free"].pop()
        s = st["slots"][k]
        n = len(frames)
        if ring is None:
            ring = [self.reserve(st) for _ in range(n)]
            for i, f in zip(ring, frames):
                self.stage(st, i, f, cfg)
        r0 = ring[0]
        strm = st["stream"]
        fit = "d_fit" in s
        t1 = clock()
        dm["stage_ms"] = max(dm["stage_ms"], (t1 - t0) * 1e3)
        g = s.get("graphs", {}).get(n)
        with torch.cuda.stream(strm):
            self._upload(st, s, r0, n, strm)             # referenced pixels only
            t2 = clock()
            dm["upload_ms"] = max(dm["upload_ms"], (t2 - t1) * 1e3)
            if g is not None:
                g.replay()                               # the recorded caking + fits + result copies
            else:
                self._device_work(st, cfg, s, n, strm)
            s["event"].record(strm)
        dm["integrate_ms"] = max(dm["integrate_ms"], (clock() - t2) * 1e3)
        one = self._one_frame(n)
        self.launches += (n if one else 1) * (2 if fit else 1)
        self.alg_bytes += (n * st["map_bytes"] if one else st["map_bytes"]) + n * st["frame_bytes"]
        return (k, n)

    def ready(self, st, handle) -> bool:
        return st["slots"][handle[0]]["event"].query()

    def collect(self, st, cfg: StreamConfig, handle):
        k, n = handle
        s = st["slots"][k]
        res = []
        for i in range(n):
            res.append((s["h_aw"][i].numpy().copy(), s["h_sm"][i].numpy().copy(),
                        s["h_fit"][i].numpy().copy() if "h_fit" in s else None,
                        s["h_cake"][i].numpy().copy() if cfg.want_cake else None))
        st["free"].append(k)
        self._release(st, n)
        return res

    def close(self, st):
        st["stream"].synchronize()
        st["plan"].close()
        st["slots"].clear()
        for tok in st["tokens"]:
            self.pool.release(tok)


def _fit_file_rows(s: "_Stream", fit: np.ndarray) -> np.ndarray:
    """fit.bin rows of one frame: the peaks within 2 bins of the grid, ascending by bin
    (IntegratorFitPeaksGPUStream.cu:2632-2688), first seven outputs."""
    if s.fit_valid is None:
        return np.zeros((0, 7))
    return np.ascontiguousarray(np.asarray(fit, np.float64)[s.fit_valid, :7])


class CakeServer:
    """Continuous-batching scheduler over admitted detector streams.

    Args:
        backend: executes batches (default: DeviceBackend on cuda:0).
        hbm_budget: bytes the admitted streams may hold on the device (default: 90 % of
            the device memory free at construction).
        tick_s: idle sleep between scheduling passes.
    """

    def __init__(self, backend=None, hbm_budget: Optional[int] = None, tick_s: float = 2e-4):
        self.backend = backend or DeviceBackend()
        self.budget = int(hbm_budget if hbm_budget is not None else 0.9 * self.backend.free_bytes())
        self.used = 0
        self.tick_s = tick_s
        self.streams: Dict[int, _Stream] = {}
        self._ids = itertools.count()
        self._lock = threading.Lock()
        self._wake = threading.Event()
        self._thread: Optional[threading.Thread] = None
        self._running = False
        self.latencies: List[float] = []
        self.completed = 0
        self.batches = 0
        self.reset_pass_stats()

    def reset_pass_stats(self) -> None:
        """Clear the scheduler-pass statistics (see pass_stats)."""
        self._ps = {"passes": 0, "slow_passes": 0, "max_pass_ms": 0.0, "max_pass_at": 0.0,
                    "max_ready_ms": 0.0, "max_collect_ms": 0.0, "max_dispatch_ms": 0.0}

    def pass_stats(self) -> Dict[str, float]:
        """Scheduler-thread statistics since the last reset: passes, passes over 20 ms, the
        slowest pass (ms, and its time.perf_counter() start), and the slowest single call of
        each kind (event query, result collection, dispatch of a batch)."""
        return dict(self._ps)

    # -- admission -----------------------------------------------------------
    def admit(self, cfg: StreamConfig) -> int:
        """Admit a stream if its footprint fits the remaining budget; AdmissionError otherwise."""
        with self._lock:
            est = self.backend.footprint_estimate(cfg)
            if self.used + est > self.budget:
                raise AdmissionError(f"stream {cfg.name!r} needs ~{est / 1e9:.2f} GB; "
                                     f"{(self.budget - self.used) / 1e9:.2f} GB of the budget left")
            self.used += est
        try:
            state, fp = self.backend.open(cfg)
        except Exception:
            with self._lock:
                self.used -= est
            raise
        writer, valid = None, None
        if cfg.output_dir:
            from .writers import StreamOutputs
            r_axis = cfg.r_axis if cfg.r_axis is not None else np.arange(cfg.n_r, dtype=np.float64)
            writer = StreamOutputs(cfg.output_dir, r_axis, write_2d=cfg.want_cake, write_fit=cfg.peaks is not None)
            if cfg.peaks is not None and cfg.r_axis is not None:
                xs = np.asarray(cfg.r_axis, np.float64)
                pk = np.asarray(cfg.peaks, np.float64).reshape(-1)
                bins = np.array([int(np.argmin(np.abs(xs - c))) for c in pk])
                ok = np.abs(xs[bins] - pk) < 2.0 * cfg.x_bin
                valid = np.array([k for k in np.argsort(bins, kind="stable") if ok[k]], dtype=np.int64)
        with self._lock:
            self.used += fp - est
            sid = next(self._ids)
            self.streams[sid] = _Stream(sid, cfg, state, fp, writer=writer, fit_valid=valid)
        return sid

    def remove(self, sid: int, *, drain: bool = True, timeout: float = 30.0) -> None:
        """Stop a stream; with drain, its queued frames are processed first."""
        with self._lock:
            s = self.streams.get(sid)
            if s is None:
                return
            s.closing = True
            if not drain:
                while s.pending:
                    s.pending.popleft().fut.cancel()
        t0 = time.time()
        while True:
            with self._lock:
                busy = bool(s.pending or s.inflight)
            if not busy or time.time() - t0 > timeout:
                break
            if self._running:
                time.sleep(self.tick_s)
            else:
                self._pass()
        with self._lock:
            while s.pending:
                s.pending.popleft().fut.cancel()
            del self.streams[sid]
            self.used -= s.footprint
        self.backend.close(s.state)
        if s.writer is not None:
            s.writer.close()

    # -- requests ---------------------------------------------------------------
    def submit(self, sid: int, frame: np.ndarray, t_arrival: Optional[float] = None) -> Future:
        """Queue one frame of a stream.  With a backend that stages (``reserve``/``stage``),
        the frame is copied into the stream's staging ring here, in the caller's thread, so
        the scheduler thread never copies frames; a full ring holds the caller back."""
        fut: Future = Future()
        with self._lock:
            s = self.streams.get(sid)
            if s is None or s.closing:
                fut.set_exception(KeyError(f"stream {sid} is not admitted"))
                return fut
            cfg = s.cfg
            if frame.size != cfg.n_pixels_y * cfg.n_pixels_z:
                fut.set_exception(ValueError(f"frame has {frame.size} pixels, stream {cfg.name!r} expects "
                                             f"{cfg.n_pixels_y * cfg.n_pixels_z}"))
                return fut
        now = time.perf_counter()
        t_arr = t_arrival if t_arrival is not None else now
        if not hasattr(self.backend, "reserve"):
            with self._lock:
                s.pending.append(_Req(next(s.seq), frame, t_arr, fut, now))
            self._wake.set()
            return fut
        with s.submit_lock:          # ring entries in the order the frames enter the queue
            try:
                idx = self.backend.reserve(s.state)
            except Exception as e:
                fut.set_exception(e)
                return fut
            req = _Req(next(s.seq), frame, t_arr, fut, now, ring=idx, staged=False)
            with self._lock:
                s.pending.append(req)
        try:
            self.backend.stage(s.state, idx, frame, cfg)
        finally:
            req.staged = True
            self._wake.set()
        return fut

    # -- scheduling ---------------------------------------------------------------
    def _pass(self) -> bool:
        """One scheduling pass: complete finished batches, dispatch pending frames."""
        did = False
        ps, clock = self._ps, time.perf_counter
        t_pass = clock()
        with self._lock:
            streams = list(self.streams.values())
        for s in streams:
            while s.inflight:
                t = clock()
                ok = self.backend.ready(s.state, s.inflight[0][0])
                t1 = clock()
                ps["max_ready_ms"] = max(ps["max_ready_ms"], (t1 - t) * 1e3)
                if not ok:
                    break
                handle, reqs = s.inflight.popleft()
                res = self.backend.collect(s.state, s.cfg, handle)
                now = clock()
                ps["max_collect_ms"] = max(ps["max_collect_ms"], (now - t1) * 1e3)
                for r, (aw, sm, fit, cake) in zip(reqs, res):
                    if s.writer is not None:
                        s.writer.write_frame(aw, sm, cake, None if fit is None else _fit_file_rows(s, fit))
                    lat = now - r.t_arrival
                    self.latencies.append(lat)
                    r.fut.set_result(FrameResult(s.cfg.name, r.seq, aw, sm, fit, cake, lat, len(reqs),
                                                 r.t_arrival, r.t_submit, r.t_dispatch, now))
                self.completed += len(reqs)
                did = True
            while s.pending and self.backend.can_dispatch(s.state):
                with self._lock:
                    # the longest staged prefix of the queue, up to the batch limit
                    lim = min(len(s.pending), self.backend.batch_limit(s.state))
                    n = 0
                    while n < lim and s.pending[n].staged:
                        n += 1
                    reqs = [s.pending.popleft() for _ in range(n)]
                if not reqs:
                    break
                t_disp = time.perf_counter()
                for r in reqs:
                    r.t_dispatch = t_disp
                if reqs[0].ring >= 0:
                    handle = self.backend.dispatch(s.state, s.cfg, [r.frame for r in reqs], ring=[r.ring for r in reqs])
                else:
                    handle = self.backend.dispatch(s.state, s.cfg, [r.frame for r in reqs])
                ps["max_dispatch_ms"] = max(ps["max_dispatch_ms"], (clock() - t_disp) * 1e3)
                s.inflight.append((handle, reqs))
                self.batches += 1
                did = True
        dt = (clock() - t_pass) * 1e3
        ps["passes"] += 1
        ps["slow_passes"] += dt > 20.0
        if dt > ps["max_pass_ms"]:
            ps["max_pass_ms"], ps["max_pass_at"] = dt, t_pass
        return did

    def _loop(self):
        while self._running:
            if not self._pass():
                self._wake.wait(self.tick_s)
                self._wake.clear()

    def start(self) -> "CakeServer":
        if not self._running:
            self._running = True
            self._thread = threading.Thread(target=self._loop, name="cake-server", daemon=True)
            self._thread.start()
        return self

    def stop(self, *, drain: bool = True, timeout: float = 30.0) -> None:
        if drain:
            t0 = time.time()
            while time.time() - t0 < timeout:
                with self._lock:
                    busy = any(s.pending or s.inflight for s in self.streams.values())
                if not busy:
                    break
                time.sleep(self.tick_s)
        self._running = False
        self._wake.set()
        if self._thread:
            self._thread.join(timeout)
        for sid in list(self.streams):
            self.remove(sid, drain=False)

    def __enter__(self):
        return self.start()

    def __exit__(self, *exc):
        self.stop()

    def latency_ms(self) -> Dict[str, float]:
        if not self.latencies:
            return {"p50": float("nan"), "p99": float("nan"), "n": 0}
        a = np.sort(np.asarray(self.latencies)) * 1e3
        return {"p50": float(np.percentile(a, 50)), "p99": float(np.percentile(a, 99)),
                "max": float(a[-1]), "n": int(a.size)}
