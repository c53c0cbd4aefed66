"""Frame preparation on the device, mirroring packages/midas_integrate/midas_integrate/image.py.

* ``decode_hybrid_payload``: a dtype-6 socket payload ([u32 C][u16 base][i32 idx, C]
  [i64 val, C]) -> float32 frame of raw counts on the device (image.py:83-123,
  ProcessImageGPU_Hybrid_Impl in IntegratorFitPeaksGPUStream.cu:1497-1560).  The payload
  crosses PCIe once, in the form it arrived; two kernels expand the base and overlay the
  overflow values.  Same size checks and ValueError messages as the reference.
* ``average_dark_frames``: per-pixel mean of a multi-frame dark file (image.py:161-184,
  the stream server's main(), IntegratorFitPeaksGPUStream.cu:2191-2238), summed in FP64 on
  the device and returned as the float32 dark the caking kernels subtract.
* ``average_frames``: the same mean over frames already on the device.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path
from typing import Optional, Union

import numpy as np
import torch

from . import _lib as L
from .kernels import _device_index, dtype_code


class HybridDecoder:
    """Reusable device buffers for decoding hybrid payloads of one detector shape.

    ``decode(payload)`` returns the (NZ, NY) float32 device frame (a view of a buffer the
    decoder owns and overwrites on the next call unless ``out`` is given).  Payload bytes
    are staged through a page-locked host buffer so the host->device copy is asynchronous.
    """

    def __init__(self, n_pixels_y: int, n_pixels_z: int, *, max_overflow: int = 1 << 16, device="cuda"):
        self.ny, self.nz = int(n_pixels_y), int(n_pixels_z)
        self.device = torch.device("cuda", _device_index(device))
        self.n_pixels = self.ny * self.nz
        self._cap = 0
        self._reserve(4 + 2 * self.n_pixels + 12 * int(max_overflow))
        self.frame = torch.empty((self.nz, self.ny), dtype=torch.float32, device=self.device)
        self.status = torch.zeros(1, dtype=torch.int32, device=self.device)

    def _reserve(self, nbytes: int) -> None:
        if nbytes <= self._cap:
            return
        cap = (nbytes + 4 + 255) // 256 * 256
        self._staging = torch.empty(cap, dtype=torch.uint8, device=self.device)
        self._host = torch.empty(cap, dtype=torch.uint8, pin_memory=True)
        self._cap = cap - 4

    def decode(self, payload: Union[bytes, bytearray, memoryview, np.ndarray], *,
               out: Optional[torch.Tensor] = None, stream=None) -> torch.Tensor:
        mv = memoryview(payload).cast("B")
        n = mv.nbytes
        if n < 4 + self.n_pixels * 2:
            raise ValueError("payload too small for hybrid base+count")
        count = int(np.frombuffer(mv[:4], dtype=np.uint32)[0])
        expected = 4 + self.n_pixels * 2 + count * (4 + 8)
        if n != expected:
            raise ValueError(f"hybrid payload size {n} != expected {expected} "
                             f"(N={self.n_pixels}, C={count})")
        self._reserve(n)
        s = stream if stream is not None else torch.cuda.current_stream(self.device)
        s.synchronize()                      # the pinned buffer may still feed the last copy
        self._host[:n].numpy()[:] = np.frombuffer(mv, dtype=np.uint8)
        dst = self.frame if out is None else out
        if dst.dtype != torch.float32 or dst.numel() != self.n_pixels or not dst.is_contiguous():
            raise ValueError("out must be a contiguous float32 tensor of NZ*NY pixels")
        L.check(L.lib().mi_decode_hybrid(self._host.data_ptr(), n, self.ny, self.nz, self._staging.data_ptr(),
                                         dst.data_ptr(), self.status.data_ptr(), C.c_void_p(s.cuda_stream)),
                "mi_decode_hybrid")
        return dst.view(self.nz, self.ny)

    def check(self) -> None:
        """Raise if a decoded payload held an overflow index outside the frame (reads the
        device status word, which synchronises, and clears it)."""
        st = int(self.status.item())
        if st:
            self.status.zero_()
            raise L.MidasError(st, "mi_decode_hybrid", "overflow index outside the frame")


def decode_hybrid_payload(payload: bytes, *, n_pixels_y: int, n_pixels_z: int, device="cuda") -> torch.Tensor:
    """Decode one dtype=6 hybrid payload to a (NZ, NY) float32 device frame of raw counts
    (image.py:decode_hybrid_payload).  For a stream of payloads keep a ``HybridDecoder``."""
    mv = memoryview(payload).cast("B")
    count = int(np.frombuffer(mv[:4], dtype=np.uint32)[0]) if mv.nbytes >= 4 else 0
    dec = HybridDecoder(n_pixels_y, n_pixels_z, max_overflow=count, device=device)
    frame = dec.decode(payload).clone()
    dec.check()
    return frame


def average_frames(frames: torch.Tensor, stream=None) -> torch.Tensor:
    """Per-pixel FP64 mean of device frames (K, NZ, NY) or (K, NZ*NY), as float32."""
    if frames.device.type != "cuda":
        raise ValueError("average_frames takes device frames")
    K = frames.shape[0]
    flat = frames.reshape(K, -1)
    if K and flat.stride(1) != 1:
        flat = flat.contiguous()
    out = torch.empty(frames.shape[1:], dtype=torch.float32, device=frames.device)
    with torch.cuda.device(frames.device):
        L.check(L.lib().mi_average_frames(flat.data_ptr(), dtype_code(flat.dtype), flat.shape[1], K,
                                          flat.stride(0), out.data_ptr(), L.stream_ptr(stream)),
                "mi_average_frames")
    return out


def average_dark_frames(path: Union[str, Path], *, n_pixels_y: int, n_pixels_z: int, dtype: str = "int64",
                        device="cuda") -> torch.Tensor:
    """Per-pixel mean of a multi-frame dark binary (image.py:average_dark_frames), computed on
    the device in FP64 and returned as the (NZ, NY) float32 dark."""
    path = Path(path)
    npdt = np.dtype(dtype)
    bytes_per_frame = n_pixels_y * n_pixels_z * npdt.itemsize
    sz = path.stat().st_size
    n_frames = sz // bytes_per_frame
    if n_frames == 0:
        raise ValueError(f"dark file {path} too small for one frame "
                         f"({sz} bytes, frame={bytes_per_frame})")
    raw = np.fromfile(path, dtype=npdt, count=n_pixels_y * n_pixels_z * n_frames)
    tdt = torch.from_numpy(raw[:0]).dtype
    host = torch.empty((n_frames, n_pixels_z, n_pixels_y), dtype=tdt, pin_memory=True)
    host.numpy()[:] = raw.reshape(n_frames, n_pixels_z, n_pixels_y)
    dev = torch.device("cuda", _device_index(device))
    return average_frames(host.to(dev, non_blocking=True))
