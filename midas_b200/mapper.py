"""DetectorMapper through libmidas_b200: build Map.bin / nMap.bin on the GPU.

``build_map`` takes the mapper keys of the MIDAS parameter file (the subset
mapper_build_map uses: geometry, tilts, p0..p14 distortion, Parallax,
SolidAngleCorrection, PolarizationCorrection/Fraction, SubPixelLevel,
SubPixelCardinalWidth and the R / Q / eta binning) and returns a
``bin_io.PixelMap`` laid out exactly like DetectorMapper's output
(FF_HEDM/src/DetectorMapper.c:813-834).  ``device=-1`` runs the same code on the
host cores.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field
from typing import List, Optional, Tuple

import numpy as np

from . import _lib as L
from .bin_io import PixelMap, PXLIST_DTYPE


@dataclass
class MapperParams:
    NrPixelsY: int
    NrPixelsZ: int
    px: float                 # um
    Lsd: float                # um
    BC_y: float
    BC_z: float
    tx: float = 0.0
    ty: float = 0.0
    tz: float = 0.0
    RhoD: float = 2.0e5       # um
    p: List[float] = field(default_factory=lambda: [0.0] * 15)
    Parallax: float = 0.0
    SolidAngleCorrection: int = 0
    PolarizationCorrection: int = 0
    PolarizationFraction: float = 0.99
    SubPixelLevel: int = 1
    SubPixelCardinalWidth: float = 10.0
    RMin: float = 0.0
    RMax: float = 0.0
    RBinSize: float = 1.0
    EtaMin: float = -180.0
    EtaMax: float = 180.0
    EtaBinSize: float = 5.0
    QMin: float = 0.0
    QMax: float = 0.0
    QBinSize: float = 0.0
    Wavelength: float = 0.0

    @property
    def q_mode(self) -> bool:
        return self.QBinSize > 0 and self.Wavelength > 0

    @property
    def n_r(self) -> int:
        if self.q_mode:
            return int(math.ceil((self.QMax - self.QMin) / self.QBinSize))
        return int(math.ceil((self.RMax - self.RMin) / self.RBinSize))

    @property
    def n_eta(self) -> int:
        return int(math.ceil((self.EtaMax - self.EtaMin) / self.EtaBinSize))

    def edges(self) -> Tuple[np.ndarray, np.ndarray, np.ndarray, np.ndarray]:
        """(r_lo, r_hi, eta_lo, eta_hi); Q-mode R edges = Lsd/px * tan(2 asin(Q lambda / 4 pi))
        (DetectorMapper.c:712-755)."""
        n_r, n_eta = self.n_r, self.n_eta
        if self.q_mode:
            q = self.QMin + self.QBinSize * np.arange(n_r + 1, dtype=np.float64)
            r = (self.Lsd / self.px) * np.tan(2.0 * np.arcsin(q * self.Wavelength / (4.0 * np.pi)))
            r_lo, r_hi = r[:-1].copy(), r[1:].copy()
        else:
            r_lo = self.RMin + self.RBinSize * np.arange(n_r, dtype=np.float64)
            r_hi = self.RMin + self.RBinSize * (np.arange(n_r, dtype=np.float64) + 1)
        e_lo = self.EtaBinSize * np.arange(n_eta, dtype=np.float64) + self.EtaMin
        e_hi = self.EtaBinSize * (np.arange(n_eta, dtype=np.float64) + 1) + self.EtaMin
        return r_lo, r_hi, e_lo, e_hi


def build_map(p: MapperParams, *, device: int = 0, mask: Optional[np.ndarray] = None
              ) -> Tuple[PixelMap, np.ndarray]:
    """Build the pixel-split map -> (PixelMap, bin_mask_flag)."""
    geo = L.MiGeometry()
    geo.ny, geo.nz = int(p.NrPixelsY), int(p.NrPixelsZ)
    geo.px_um, geo.lsd_um = float(p.px), float(p.Lsd)
    geo.bc_y, geo.bc_z = float(p.BC_y), float(p.BC_z)
    geo.tx, geo.ty, geo.tz = float(p.tx), float(p.ty), float(p.tz)
    geo.rho_d = float(p.RhoD)
    for i in range(15):
        geo.p[i] = float(p.p[i]) if i < len(p.p) else 0.0
    geo.parallax_um = float(p.Parallax)
    geo.solid_angle = int(p.SolidAngleCorrection)
    geo.polarization = int(p.PolarizationCorrection)
    geo.pol_fraction = float(p.PolarizationFraction)
    geo.sub_pixel_level = int(p.SubPixelLevel)
    geo.sub_pixel_cardinal_width = float(p.SubPixelCardinalWidth)
    m = None
    if mask is not None:
        m = np.ascontiguousarray(np.asarray(mask).reshape(-1) != 0, dtype=np.uint8)
        if m.size != geo.ny * geo.nz:
            raise ValueError("mask size mismatch")
        geo.mask_host = m.ctypes.data
    r_lo, r_hi, e_lo, e_hi = (np.ascontiguousarray(a) for a in p.edges())
    b = L.MiBinning(r_lo.size, e_lo.size, r_lo.ctypes.data, r_hi.ctypes.data, e_lo.ctypes.data,
                    e_hi.ctypes.data)
    h = C.c_void_p()
    lib = L.lib()
    L.check(lib.mi_map_build(C.byref(geo), C.byref(b), int(device), C.byref(h)), "mi_map_build")
    try:
        nrec, nb = C.c_int64(), C.c_int64()
        L.check(lib.mi_map_sizes(h, C.byref(nrec), C.byref(nb)), "mi_map_sizes")
        recs = np.zeros(nrec.value, dtype=PXLIST_DTYPE)
        nmap = np.zeros((nb.value, 2), dtype=np.int32)
        bmask = np.zeros(nb.value, dtype=np.int32)
        L.check(lib.mi_map_copy(h, recs.ctypes.data if recs.size else None, nmap.ctypes.data,
                                bmask.ctypes.data), "mi_map_copy")
    finally:
        lib.mi_map_destroy(h)
    del m
    return PixelMap(recs, np.ascontiguousarray(nmap[:, 0]), np.ascontiguousarray(nmap[:, 1])), bmask
