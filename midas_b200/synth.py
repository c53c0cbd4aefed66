"""Seeded synthetic workloads of the caking benchmarks (no public dataset is used).

Each workload names a detector geometry, a cake binning, a map-builder setting and a
frame model; frames are generated on the device by ``mi_synth_frames`` (Philox
counter-based RNG, Poisson counts) so a 1440-frame 2880x2880 sweep never touches
the host.

  powder_2048      2048x2048 u16, 10 fcc rings, RBin 1 px, eta 5 deg (990x72 bins),
                   floor mode, no corrections
  sweep_2880       2880x2880 u16 omega sweep, rings with +-20 % per-frame drift and 50
                   Gaussian spots per frame, RBin 0.25 px, eta 1 deg (3960x360 bins),
                   gradient mode, solid-angle + polarisation (0.99) + parallax in the map
  sweep_2880_small the same model scaled down (for tests)
  pilatus_1679     1475x1679 int32, 172 um pixels, module gaps masked (serving mix)
  detector_1024    1024x1024 u16 panels (serving mix)
  powder_2048_fine 2048x2048 u16, RBin 0.5 px, eta 2 deg, gradient (serving mix)

``serving_mix`` lists the six concurrent streams of the serving load with their
Poisson frame rates; ``serving_stream`` turns a workload into a server stream.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field, replace
from typing import List, Optional

import numpy as np
import torch

from . import _lib as L
from .mapper import MapperParams

# Fm-3m (fluorite) a = 5.4116 A: ten of the twelve allowed reflections from 111 to 531
# (the weak h+k+l = 4n+2 all-even 222 and 420 are left out).
FCC_HKL = [(1, 1, 1), (2, 0, 0), (2, 2, 0), (3, 1, 1), (4, 0, 0), (3, 3, 1), (4, 2, 2),
           (5, 1, 1), (4, 4, 0), (5, 3, 1)]


def ring_radii_px(a_A: float, wavelength_A: float, lsd_um: float, px_um: float,
                  hkl=FCC_HKL) -> np.ndarray:
    """R = Lsd/px * tan(2 theta), sin(theta) = lambda / 2d, d = a / |hkl|."""
    out = []
    for h, k, l in hkl:
        d = a_A / math.sqrt(h * h + k * k + l * l)
        tth = 2.0 * math.asin(wavelength_A / (2.0 * d))
        out.append(lsd_um / px_um * math.tan(tth))
    return np.array(out)


@dataclass
class Workload:
    name: str
    mapper: MapperParams
    mode: str                      # integration mode
    fwhm_px: float = 1.5
    mix_eta: float = 0.5
    texture: float = 0.3
    background: float = 100.0
    amp_drift: float = 0.0
    n_spots: int = 0
    spot_sigma: float = 2.0
    spot_amp: float = 5.0e4
    dark_mean: float = 100.0
    dark_sigma: float = 5.0
    seed: int = 20251203
    wavelength_A: float = 0.172979
    lattice_A: float = 5.4116
    n_frames: int = 10
    tile_rows: int = 0
    frame_dtype: str = "uint16"    # raw frame type: "uint16" or "int32"
    module_gaps: Optional[tuple] = None   # (module_y, gap_y, module_z, gap_z) px, masked in the map

    @property
    def n_r(self) -> int:
        return self.mapper.n_r

    @property
    def n_eta(self) -> int:
        return self.mapper.n_eta

    @property
    def shape(self):
        return self.mapper.NrPixelsZ, self.mapper.NrPixelsY

    def mask(self) -> Optional[np.ndarray]:
        """(NZ, NY) uint8 mask (1 = excluded) of the inter-module gaps, or None."""
        if self.module_gaps is None:
            return None
        my, gy, mz, gz = self.module_gaps
        nz, ny = self.shape
        y = np.arange(ny) % (my + gy) >= my
        z = np.arange(nz) % (mz + gz) >= mz
        return (z[:, None] | y[None, :]).astype(np.uint8)

    def ring_radii(self) -> np.ndarray:
        return ring_radii_px(self.lattice_A, self.wavelength_A, self.mapper.Lsd, self.mapper.px)

    def ring_amps(self) -> np.ndarray:
        rng = np.random.default_rng(self.seed)
        return rng.uniform(1.0e3, 2.0e4, size=len(FCC_HKL))

    def synth_desc(self, poisson: bool = True) -> L.MiSynthDesc:
        m = self.mapper
        d = L.MiSynthDesc()
        d.ny, d.nz = m.NrPixelsY, m.NrPixelsZ
        d.bc_y, d.bc_z = m.BC_y, m.BC_z
        d.lsd_um, d.px_um = m.Lsd, m.px
        d.ty, d.tz = m.ty, m.tz
        rr, ra = self.ring_radii(), self.ring_amps()
        d.n_rings = len(rr)
        for i in range(len(rr)):
            d.ring_r_px[i] = float(rr[i])
            d.ring_amp[i] = float(ra[i])
        d.fwhm_px, d.mix_eta, d.texture = self.fwhm_px, self.mix_eta, self.texture
        d.background, d.amp_drift = self.background, self.amp_drift
        d.n_spots, d.spot_sigma, d.spot_amp = self.n_spots, self.spot_sigma, self.spot_amp
        d.dark_mean, d.dark_sigma = self.dark_mean, self.dark_sigma
        d.seed = self.seed
        d.poisson = 1 if poisson else 0
        return d

    def frames(self, first: int, n: int, *, out: Optional[torch.Tensor] = None, device="cuda",
               dtype=torch.uint16, stream=None) -> torch.Tensor:
        """Frames first..first+n-1 as a (n, NZ, NY) device tensor (raw counts incl. dark)."""
        nz, ny = self.shape
        if out is None:
            out = torch.empty((n, nz, ny), dtype=dtype, device=device)
        code = {torch.uint16: L.DT_U16, torch.int32: L.DT_I32}[out.dtype]
        d = self.synth_desc()
        L.check(L.lib().mi_synth_frames(C.byref(d), int(first), int(n), code, out.data_ptr(),
                                        out[0].numel() if n else ny * nz, L.stream_ptr(stream)),
                "mi_synth_frames")
        return out

    def dark(self, device="cuda", stream=None) -> torch.Tensor:
        nz, ny = self.shape
        out = torch.empty((nz, ny), dtype=torch.float32, device=device)
        d = self.synth_desc()
        L.check(L.lib().mi_synth_dark(C.byref(d), out.data_ptr(), L.stream_ptr(stream)),
                "mi_synth_dark")
        return out


def powder_2048() -> Workload:
    m = MapperParams(NrPixelsY=2048, NrPixelsZ=2048, px=200.0, Lsd=1.0e6, BC_y=1024.3,
                     BC_z=1022.7, ty=0.1, tz=-0.05, RMin=10.0, RMax=1000.0, RBinSize=1.0,
                     EtaMin=-180.0, EtaMax=180.0, EtaBinSize=5.0)
    return Workload("powder_2048x2048_u16_990x72_floor", m, "floor", n_frames=10, tile_rows=8)


def sweep_2880() -> Workload:
    # pixel size 200 um keeps all ten rings (R = 277..958 px) inside RMax = 1000 px
    m = MapperParams(NrPixelsY=2880, NrPixelsZ=2880, px=200.0, Lsd=1.0e6, BC_y=1440.3,
                     BC_z=1438.7, ty=0.1, tz=-0.05, RMin=10.0, RMax=1000.0, RBinSize=0.25,
                     EtaMin=-180.0, EtaMax=180.0, EtaBinSize=1.0, SolidAngleCorrection=1,
                     PolarizationCorrection=1, PolarizationFraction=0.99, Parallax=100.0)
    return Workload("sweep_2880x2880_u16_3960x360_gradient", m, "gradient", amp_drift=0.2,
                    n_spots=50, n_frames=1440, tile_rows=16)


def pilatus_1679() -> Workload:
    """PILATUS-2M-like panel: 1475x1679 int32, 172 um pixels, 3x8 modules of 487x195 px
    with 7 px (y) and 17 px (z) gaps masked in the map; RBin 1 px, eta 5 deg, floor."""
    m = MapperParams(NrPixelsY=1475, NrPixelsZ=1679, px=172.0, Lsd=8.0e5, BC_y=737.6,
                     BC_z=841.2, ty=0.2, tz=0.1, RMin=10.0, RMax=800.0, RBinSize=1.0,
                     EtaMin=-180.0, EtaMax=180.0, EtaBinSize=5.0)
    return Workload("pilatus_1475x1679_i32_790x72_floor", m, "floor", frame_dtype="int32",
                    module_gaps=(487, 7, 195, 17), tile_rows=8)


def pilatus3_2m_published() -> Workload:
    """The reference's published benchmark detector (run_benchmarks.py 'pilatus3_2m'): 1475x1679
    u16, 172 um pixels, Lsd 500 mm, beam centre (737.5, 839.5) px, no tilt, RMin 10 .. RMax
    1117.4 px at 1 px, eta -180 .. 180 at 5 deg (1108 x 72 bins), floor mode."""
    m = MapperParams(NrPixelsY=1475, NrPixelsZ=1679, px=172.0, Lsd=5.0e5, BC_y=737.5, BC_z=839.5, RMin=10.0,
                     RMax=1117.4, RBinSize=1.0, EtaMin=-180.0, EtaMax=180.0, EtaBinSize=5.0)
    return Workload("pilatus3_2m_1475x1679_u16_1108x72_floor", m, "floor", n_frames=512, tile_rows=8)


def detector_1024(variant: int = 0) -> Workload:
    """1024x1024 u16 panels of the serving mix: variant 0 = RBin 1 px, eta 8 deg (495x45 bins,
    floor); variant 1 = tilted, RBin 0.5 px, eta 5 deg (990x72 bins, bilinear)."""
    if variant == 0:
        m = MapperParams(NrPixelsY=1024, NrPixelsZ=1024, px=400.0, Lsd=1.0e6, BC_y=512.4,
                         BC_z=511.8, RMin=5.0, RMax=500.0, RBinSize=1.0, EtaMin=-180.0,
                         EtaMax=180.0, EtaBinSize=8.0)
        return Workload("detector_1024_u16_495x45_floor", m, "floor", tile_rows=8)
    m = MapperParams(NrPixelsY=1024, NrPixelsZ=1024, px=400.0, Lsd=1.1e6, BC_y=530.1,
                     BC_z=498.3, ty=0.4, tz=-0.3, RMin=5.0, RMax=500.0, RBinSize=0.5,
                     EtaMin=-180.0, EtaMax=180.0, EtaBinSize=5.0)
    return Workload("detector_1024_u16_990x72_bilinear", m, "bilinear", seed=77, tile_rows=8)


def powder_2048_fine() -> Workload:
    """2048x2048 u16, shifted centre and tilts, RBin 0.5 px, eta 2 deg (1980x180 bins), gradient."""
    m = MapperParams(NrPixelsY=2048, NrPixelsZ=2048, px=200.0, Lsd=1.05e6, BC_y=1010.7,
                     BC_z=1040.2, ty=-0.3, tz=0.25, RMin=10.0, RMax=1000.0, RBinSize=0.5,
                     EtaMin=-180.0, EtaMax=180.0, EtaBinSize=2.0)
    return Workload("powder_2048x2048_u16_1980x180_gradient", m, "gradient", seed=91, tile_rows=16)


def serving_mix() -> List[tuple]:
    """The six concurrent streams of the serving load, as (workload, Poisson rate in Hz):
    frame sizes 1024^2, 2048^2, 2880^2 and 1475x1679, 2.2e4 to 1.43e6 bins, 10-500 Hz."""
    return [(sweep_2880(), 10.0), (powder_2048(), 100.0), (powder_2048_fine(), 50.0),
            (pilatus_1679(), 200.0), (detector_1024(0), 500.0), (detector_1024(1), 200.0)]


def late_stream() -> tuple:
    """The stream with a fresh map admitted while the serving load runs."""
    m = MapperParams(NrPixelsY=2048, NrPixelsZ=2048, px=200.0, Lsd=0.95e6, BC_y=1030.9,
                     BC_z=1019.4, ty=0.15, tz=0.2, RMin=10.0, RMax=1000.0, RBinSize=1.0,
                     EtaMin=-180.0, EtaMax=180.0, EtaBinSize=5.0)
    return Workload("powder_2048x2048_u16_990x72_floor_late", m, "floor", seed=5, tile_rows=8), 30.0


def scaled(w: Workload, factor: int, name: Optional[str] = None) -> Workload:
    """The same workload on a detector `factor` times smaller in each direction."""
    m = w.mapper
    m2 = replace(m, NrPixelsY=m.NrPixelsY // factor, NrPixelsZ=m.NrPixelsZ // factor,
                 BC_y=m.BC_y / factor, BC_z=m.BC_z / factor, px=m.px * factor,
                 RMin=m.RMin / factor, RMax=m.RMax / factor)
    gaps = None
    if w.module_gaps is not None:
        my, gy, mz, gz = w.module_gaps
        gaps = (max(1, my // factor), max(1, gy // factor), max(1, mz // factor), max(1, gz // factor))
    return replace(w, name=name or f"{w.name}_div{factor}", mapper=m2,
                   fwhm_px=max(w.fwhm_px, 1.2), n_spots=min(w.n_spots, 8), module_gaps=gaps)


def panel_set(q_bin: float = 0.002, eta_bin: float = 2.0, mode: str = "floor") -> List[Workload]:
    """Uneven multi-panel detector sharing one Q binning (QMin 1.0, QMax 8.0 1/A): four
    2048x2048 u16 panels around the beam, each with its own beam centre, Lsd in 0.9-1.1 m
    and tilts <= 0.5 deg, plus one 1475x1679 int32 panel (172 um pixels, module gaps
    masked).  The rings are the same fcc lattice, so every panel sees them at the same Q."""
    lam = 0.172979
    q = dict(QMin=1.0, QMax=8.0, QBinSize=q_bin, Wavelength=lam, EtaMin=-180.0, EtaMax=180.0,
             EtaBinSize=eta_bin)
    geo = [(0.90e6, 2100.0, 2100.0, 0.3, -0.2), (1.00e6, -60.0, 2080.0, -0.4, 0.1),
           (1.05e6, 2090.0, -40.0, 0.2, 0.45), (1.10e6, -50.0, -70.0, -0.1, -0.35)]
    out = []
    for i, (lsd, by, bz, ty, tz) in enumerate(geo):
        m = MapperParams(NrPixelsY=2048, NrPixelsZ=2048, px=200.0, Lsd=lsd, BC_y=by, BC_z=bz, ty=ty, tz=tz, **q)
        out.append(Workload(f"panel{i}_2048x2048_u16", m, mode, seed=100 + i, tile_rows=16))
    m = MapperParams(NrPixelsY=1475, NrPixelsZ=1679, px=172.0, Lsd=0.95e6, BC_y=737.6, BC_z=-300.0, ty=0.2,
                     tz=0.1, **q)
    out.append(Workload("panel4_1475x1679_i32", m, mode, seed=104, tile_rows=16, frame_dtype="int32",
                        module_gaps=(487, 7, 195, 17)))
    return out


def scaled_panels(ws: List[Workload], factor: int) -> List[Workload]:
    """The panel set on detectors `factor` times smaller (same angular coverage and Q bins)."""
    out = []
    for w in ws:
        m = w.mapper
        m2 = replace(m, NrPixelsY=m.NrPixelsY // factor, NrPixelsZ=m.NrPixelsZ // factor,
                     BC_y=m.BC_y / factor, BC_z=m.BC_z / factor, px=m.px * factor)
        gaps = None
        if w.module_gaps is not None:
            my, gy, mz, gz = w.module_gaps
            gaps = (max(1, my // factor), max(1, gy // factor), max(1, mz // factor), max(1, gz // factor))
        out.append(replace(w, name=f"{w.name}_div{factor}", mapper=m2, fwhm_px=max(w.fwhm_px, 1.2),
                           module_gaps=gaps))
    return out


def ring_peaks(w: Workload, half_window: int = 15) -> np.ndarray:
    """Ring radii (px) whose +-half_window-bin fit window lies inside the R range."""
    m = w.mapper
    rr = w.ring_radii()
    lo, hi = m.RMin + (half_window + 1) * m.RBinSize, m.RMax - (half_window + 1) * m.RBinSize
    return rr[(rr > lo) & (rr < hi)]


def r_centres(w: Workload) -> np.ndarray:
    m = w.mapper
    return m.RMin + m.RBinSize * (np.arange(m.n_r, dtype=np.float64) + 0.5)


def serving_stream(w: Workload, *, device: int = 0, fit: bool = True, want_cake: bool = False,
                   half_window: int = 15):
    """StreamConfig of a workload for ``server.CakeServer``: map built on the device, the
    workload's dark, fits of its rings on the area-weighted lineout."""
    from .mapper import build_map
    from .server import StreamConfig
    pm, _ = build_map(w.mapper, device=device, mask=w.mask())
    dark = w.dark(device=torch.device("cuda", device)).cpu().numpy()
    m = w.mapper
    peaks = ring_peaks(w, half_window) if fit else None
    return StreamConfig(name=w.name, pixmap=pm, n_r=w.n_r, n_eta=w.n_eta, n_pixels_y=m.NrPixelsY,
                        n_pixels_z=m.NrPixelsZ, mode=w.mode, bc_y=m.BC_y, bc_z=m.BC_z, dark=dark,
                        frame_dtype=w.frame_dtype, r_axis=r_centres(w) if fit else None, peaks=peaks,
                        fit_half_window=half_window, x_bin=m.RBinSize, want_cake=want_cake,
                        tile_rows=w.tile_rows)


def host_frames(w: Workload, first: int, n: int, device: int = 0) -> np.ndarray:
    """Frames first..first+n-1 generated on the device and copied to host memory."""
    dt = {"uint16": torch.uint16, "int32": torch.int32}[w.frame_dtype]
    return w.frames(first, n, device=torch.device("cuda", device), dtype=dt).cpu().numpy()


WORKLOADS = {"powder_2048": powder_2048, "sweep_2880": sweep_2880, "pilatus_1679": pilatus_1679,
             "detector_1024": detector_1024, "powder_2048_fine": powder_2048_fine,
             "pilatus3_2m_published": pilatus3_2m_published}
