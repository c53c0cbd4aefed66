"""Output files of the integrators, byte-compatible with the reference's.

IntegratorFitPeaksGPUStream writes, per frame and in frame order, from a writer thread fed by
a bounded queue (FF_HEDM/src/IntegratorFitPeaksGPUStream.cu:506-565, files opened at
:2465-2469):

  lineout.bin              n_r (R, I) pairs of float64: R of the row's first bin, the
                           area-weighted eta average
  lineout_simple_mean.bin  the same with the simple mean over valid bins
  Int2D.bin                the n_r x n_eta cake as float64 (when 2-D output is on)
  fit.bin                  7 float64 per fitted peak (PF_PARAMS_PER_PEAK, PeakFit.h:40-48:
                           area, center, sig, gam, FWHM, eta, chi2/dof), the peaks placed
                           within 2 bins of the grid in ascending bin order (:2616-2619,
                           2686-2688)

and once, before the first frame, RTthEtaAreaMap.bin: five blocks of n_bins float64 -- R
mean, 2-theta, eta mean, area, Q -- in bin order (:2436-2450).  The OpenMP integrator writes
its lineout.bin as n_r float64 per frame, the mean of the nonzero, non-NaN bins, without an
R column (IntegratorZarrOMP.c:1845-1849): ``lineout_layout="omp"``.

``StreamOutputs`` is that writer: ``write_frame`` queues one frame's results (host arrays)
and a thread writes them in order; ``close`` drains the queue.  ``read_*`` read the files
back (they are what the reference's live viewer tails).
"""
from __future__ import annotations

import os
import queue
import threading
from pathlib import Path
from typing import Optional

import numpy as np

PF_PARAMS_PER_PEAK = 7


def bin_table_blocks(table: np.ndarray) -> np.ndarray:
    """[n_bins, 5] rows (mi_plan_bin_table) -> [5, n_bins] blocks (RTthEtaAreaMap.bin)."""
    t = np.asarray(table, np.float64)
    return np.ascontiguousarray(t.reshape(-1, 5).T)


def write_bin_table(path, table: np.ndarray) -> None:
    """RTthEtaAreaMap.bin: R, 2-theta, eta, area, Q blocks of n_bins float64."""
    with open(path, "wb") as f:
        f.write(bin_table_blocks(table).tobytes())


def lineout_r_axis(table: np.ndarray, n_eta: int) -> np.ndarray:
    """The R column of lineout.bin: R mean of each row's first bin (hR[r] = the table's R at
    bin r * n_eta, IntegratorFitPeaksGPUStream.cu:2438-2439)."""
    return np.ascontiguousarray(np.asarray(table, np.float64).reshape(-1, 5)[::n_eta, 0])


def fit_rows(params: np.ndarray, iters: np.ndarray, x: np.ndarray, peaks: np.ndarray) -> np.ndarray:
    """fit.bin rows of one frame: the first 7 outputs of each peak that was fit (iters >= 0),
    in ascending order of the peak's nearest bin, as fitPeaks returns them."""
    p = np.asarray(params, np.float64).reshape(-1, np.asarray(params).shape[-1])
    it = np.asarray(iters).reshape(-1)
    xs = np.asarray(x, np.float64)
    bins = np.array([int(np.argmin(np.abs(xs - c))) for c in np.asarray(peaks, np.float64).reshape(-1)])
    keep = [k for k in np.argsort(bins, kind="stable") if it[k] >= 0]
    return np.ascontiguousarray(p[keep, :PF_PARAMS_PER_PEAK])


class StreamOutputs:
    """The reference's per-frame output files of one stream, written by a thread in frame order."""

    def __init__(self, directory, r_axis: np.ndarray, *, write_2d: bool = False, write_fit: bool = False,
                 lineout_layout: str = "gpustream", queue_depth: int = 64, bin_table: Optional[np.ndarray] = None):
        if lineout_layout not in ("gpustream", "omp"):
            raise ValueError("lineout_layout is 'gpustream' or 'omp'")
        self.dir = Path(directory)
        self.dir.mkdir(parents=True, exist_ok=True)
        self.r_axis = np.ascontiguousarray(np.asarray(r_axis, np.float64))
        self.layout = lineout_layout
        if bin_table is not None:
            write_bin_table(self.dir / "RTthEtaAreaMap.bin", bin_table)
        self._f_lo = open(self.dir / "lineout.bin", "wb")
        self._f_sm = open(self.dir / "lineout_simple_mean.bin", "wb") if lineout_layout == "gpustream" else None
        self._f_2d = open(self.dir / "Int2D.bin", "wb") if write_2d else None
        self._f_fit = open(self.dir / "fit.bin", "wb") if write_fit else None
        self._q: "queue.Queue" = queue.Queue(maxsize=queue_depth)
        self._err: Optional[BaseException] = None
        self.frames_written = 0
        self._t = threading.Thread(target=self._run, name="midas-writer", daemon=True)
        self._t.start()

    def write_frame(self, lineout_aw=None, lineout_sm=None, cake=None, fits=None) -> None:
        """Queue one frame (host arrays; ``fits`` = fit.bin rows, see ``fit_rows``).  Blocks
        while the queue is full (the reference's writer_queue_push)."""
        if self._err is not None:
            raise RuntimeError(f"writer thread failed: {self._err}")
        self._q.put((lineout_aw, lineout_sm, cake, fits))

    def _run(self) -> None:
        n = self.r_axis.size
        pair = np.empty((n, 2), np.float64)
        pair[:, 0] = self.r_axis
        try:
            while True:
                job = self._q.get()
                if job is None:
                    break
                aw, sm, cake, fits = job
                if self.layout == "omp":
                    # IntegratorZarrOMP.c:1845-1849: n_r doubles, the mean of nonzero bins
                    if sm is not None:
                        self._f_lo.write(np.ascontiguousarray(np.asarray(sm, np.float64).reshape(n)).tobytes())
                        self._f_lo.flush()
                else:
                    if aw is not None:
                        pair[:, 1] = np.asarray(aw, np.float64).reshape(n)
                        self._f_lo.write(pair.tobytes())
                        self._f_lo.flush()
                    if sm is not None and self._f_sm is not None:
                        pair[:, 1] = np.asarray(sm, np.float64).reshape(n)
                        self._f_sm.write(pair.tobytes())
                        self._f_sm.flush()
                if cake is not None and self._f_2d is not None:
                    self._f_2d.write(np.ascontiguousarray(np.asarray(cake, np.float64)).tobytes())
                    self._f_2d.flush()
                if fits is not None and self._f_fit is not None and len(fits):
                    self._f_fit.write(np.ascontiguousarray(np.asarray(fits, np.float64)).tobytes())
                    self._f_fit.flush()
                self.frames_written += 1
        except BaseException as e:  # reported on the next write_frame / close
            self._err = e

    def close(self) -> None:
        """Write everything queued, then close the files."""
        if self._t.is_alive():
            self._q.put(None)
            self._t.join()
        for f in (self._f_lo, self._f_sm, self._f_2d, self._f_fit):
            if f is not None:
                f.close()
        if self._err is not None:
            raise RuntimeError(f"writer thread failed: {self._err}")

    def __enter__(self) -> "StreamOutputs":
        return self

    def __exit__(self, *exc) -> None:
        self.close()


def read_lineouts(path, n_r: int, layout: str = "gpustream") -> np.ndarray:
    """[F, n_r, 2] (R, I) pairs, or [F, n_r] for the OpenMP layout."""
    a = np.fromfile(path, dtype=np.float64)
    return a.reshape(-1, n_r, 2) if layout == "gpustream" else a.reshape(-1, n_r)


def read_cakes(path, n_r: int, n_eta: int) -> np.ndarray:
    return np.fromfile(path, dtype=np.float64).reshape(-1, n_r, n_eta)


def read_bin_table(path, n_bins: int) -> np.ndarray:
    return np.fromfile(path, dtype=np.float64).reshape(5, n_bins)


def read_fits(path) -> np.ndarray:
    return np.fromfile(path, dtype=np.float64).reshape(-1, PF_PARAMS_PER_PEAK)


def file_sizes(directory) -> dict:
    d = Path(directory)
    return {p.name: os.path.getsize(p) for p in sorted(d.glob("*.bin"))}
