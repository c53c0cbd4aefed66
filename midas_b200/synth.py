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

    @property
    def n_r(self) -> int:
        return self.mapper.n_r

    @property
    def n_eta(self) -> int:
        return self.mapper.n_eta

    @property
    def shape(self):
        return self.mapper.NrPixelsZ, self.mapper.NrPixelsY

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


def scaled(w: Workload, factor: int, name: Optional[str] = None) -> Workload:
    """The same workload on a detector `factor` times smaller in each direction."""
    m = w.mapper
    m2 = replace(m, NrPixelsY=m.NrPixelsY // factor, NrPixelsZ=m.NrPixelsZ // factor,
                 BC_y=m.BC_y / factor, BC_z=m.BC_z / factor, px=m.px * factor,
                 RMin=m.RMin / factor, RMax=m.RMax / factor)
    return replace(w, name=name or f"{w.name}_div{factor}", mapper=m2,
                   fwhm_px=max(w.fwhm_px, 1.2), n_spots=min(w.n_spots, 8))


WORKLOADS = {"powder_2048": powder_2048, "sweep_2880": sweep_2880}
