"""The map builder's code, compiled for the host, reproduces the reference DetectorMapper
core (mapper_build_map, compiled unmodified from the MIDAS sources) record for record."""
import numpy as np
import pytest

from conftest import MAPPER_CASES, load_mapper_case
from midas_b200.mapper import MapperParams, build_map


def params_of(g):
    return MapperParams(NrPixelsY=g["ny"], NrPixelsZ=g["nz"], px=g["px"], Lsd=g["lsd"], BC_y=g["bc_y"],
                        BC_z=g["bc_z"], ty=g["ty"], tz=g["tz"], RhoD=g["rho_d"], Parallax=g["parallax"],
                        SolidAngleCorrection=g["sa"], PolarizationCorrection=g["pol"],
                        PolarizationFraction=0.99)


def build_with_edges(g, device):
    import ctypes as C
    from midas_b200 import _lib as L
    from midas_b200.bin_io import PXLIST_DTYPE
    p = params_of(g)
    geo = L.MiGeometry()
    geo.ny, geo.nz, geo.px_um, geo.lsd_um = p.NrPixelsY, p.NrPixelsZ, p.px, p.Lsd
    geo.bc_y, geo.bc_z, geo.ty, geo.tz, geo.rho_d = p.BC_y, p.BC_z, p.ty, p.tz, p.RhoD
    geo.parallax_um, geo.solid_angle, geo.polarization = p.Parallax, p.SolidAngleCorrection, p.PolarizationCorrection
    geo.pol_fraction, geo.sub_pixel_level, geo.sub_pixel_cardinal_width = 0.99, 1, 10.0
    e = [np.ascontiguousarray(g[k]) for k in ("r_lo", "r_hi", "eta_lo", "eta_hi")]
    b = L.MiBinning(e[0].size, e[2].size, *(a.ctypes.data for a in e))
    h = C.c_void_p()
    L.check(L.lib().mi_map_build(C.byref(geo), C.byref(b), device, C.byref(h)), "mi_map_build")
    nrec, nb = C.c_int64(), C.c_int64()
    L.lib().mi_map_sizes(h, C.byref(nrec), C.byref(nb))
    recs = np.zeros(nrec.value, PXLIST_DTYPE)
    nmap = np.zeros((nb.value, 2), np.int32)
    mask = np.zeros(nb.value, np.int32)
    L.lib().mi_map_copy(h, recs.ctypes.data, nmap.ctypes.data, mask.ctypes.data)
    L.lib().mi_map_destroy(h)
    return recs, nmap, mask


def assert_same_map(recs, nmap, g, exact=True):
    np.testing.assert_array_equal(nmap, g["nmap"])
    ref = g["records"]
    for f in ("y", "z", "frac", "deltaR", "areaWeight"):
        a = recs[f].astype(np.float64)
        b = ref[f].astype(np.float64)
        if exact:
            np.testing.assert_array_equal(a, b, err_msg=f)
        else:
            np.testing.assert_allclose(a, b, rtol=1e-6, atol=1e-6, err_msg=f)


@pytest.mark.parametrize("tag", MAPPER_CASES)
def test_host_mapper_bit_identical_to_reference(tag):
    g = load_mapper_case(tag)
    recs, nmap, mask = build_with_edges(g, -1)
    assert_same_map(recs, nmap, g, exact=True)
    np.testing.assert_array_equal(mask, g["bin_mask"])


def test_mapper_params_edges_match_reference_formula():
    p = MapperParams(NrPixelsY=10, NrPixelsZ=10, px=200.0, Lsd=1e6, BC_y=5, BC_z=5, RMin=10, RMax=20,
                     RBinSize=0.25, EtaBinSize=1.0)
    r_lo, r_hi, e_lo, e_hi = p.edges()
    assert r_lo.size == 40 and e_lo.size == 360
    np.testing.assert_array_equal(r_hi, 0.25 * (np.arange(40) + 1) + 10)
    q = MapperParams(NrPixelsY=10, NrPixelsZ=10, px=200.0, Lsd=1e6, BC_y=5, BC_z=5, QMin=1.0, QMax=8.0,
                     QBinSize=0.002, Wavelength=0.172979, EtaBinSize=2.0)
    assert q.n_r == 3500 and q.n_eta == 180
    r_lo, r_hi, _, _ = q.edges()
    assert np.all(np.diff(r_lo) > 0) and np.allclose(r_hi[:-1], r_lo[1:])


def test_build_map_small_geometry_on_host():
    p = MapperParams(NrPixelsY=40, NrPixelsZ=36, px=200.0, Lsd=2.5e5, BC_y=19.6, BC_z=17.2, ty=0.2,
                     RMin=2.0, RMax=18.0, RBinSize=1.0, EtaBinSize=15.0)
    pm, mask = build_map(p, device=-1)
    assert pm.n_bins == p.n_r * p.n_eta
    assert pm.counts.sum() == pm.n_entries > 0
    assert np.all(pm.offsets[1:] == np.cumsum(pm.counts)[:-1])
    # pixel-split areas of one pixel sum to <= 1 per sub-pixel (no double counting)
    assert pm.pxList["areaWeight"].max() <= 1.0 + 1e-6
    assert mask.sum() == 0
