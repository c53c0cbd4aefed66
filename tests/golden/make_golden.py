"""Generate the golden fixtures in tests/golden/ from the reference implementation.

Run where the MIDAS sources are checked out (read-only), naming the checkout:

    MIDAS_REF=<MIDAS checkout> python tests/golden/make_golden.py

It imports the reference's own Python package (packages/midas_integrate) --
without executing its __init__, which pulls in optional I/O dependencies -- and
the reference's C mapper and integrator compiled into oracle/_ref, and writes:

  kernels_*.npz   random pixel maps (empty bins, off-detector records, ragged
                  shapes) with images; cakes from build_csr + integrate and
                  lineouts from profile_1d, in FP64, for floor / bilinear /
                  gradient and normalize on/off
  mapper_*.npz    maps built by the reference DetectorMapper core
                  (mapper_build_map) for small detectors with tilt, solid-angle,
                  polarisation and parallax, plus the reference integrator's
                  (integration_apply_map) sums on a seeded image
  peakfit.npz     lineouts and the reference scipy TRF fit (peakfit.fit_peaks)
  header.npz      Map.bin header bytes and parameter hashes
  variance_*.npz  the kernels_* maps with a variance image: integrate_with_variance
                  (build_csr(compute_variance=True)) and profile_1d_with_variance, FP64,
                  every mode, normalize on/off
  image.npz       hybrid (dtype 6) payloads decoded by decode_hybrid_payload and a
                  multi-frame int64 dark averaged by average_dark_frames
  fused.npz       build_fused_geometry (4 R shifts) of a small tilted detector: the
                  shifted maps, their R axes, an image and the fused cakes

Selected groups only: python tests/golden/make_golden.py variance image

The fixtures are inputs/outputs only; nothing of the reference's source is copied.
"""
from __future__ import annotations

import importlib.util
import os
import sys
import types
from pathlib import Path

import numpy as np

OUT = Path(__file__).resolve().parent
REPO = OUT.parents[1]
if "MIDAS_REF" not in os.environ:
    sys.exit("make_golden.py: set MIDAS_REF to the MIDAS checkout whose outputs the fixtures record")
REF = Path(os.environ["MIDAS_REF"])
PKG = REF / "packages" / "midas_integrate" / "midas_integrate"


def ref_modules():
    pkg = types.ModuleType("midas_integrate")
    pkg.__path__ = [str(PKG)]
    sys.modules["midas_integrate"] = pkg
    mods = {}
    for name in ("bin_io", "kernels", "peakfit", "image"):
        spec = importlib.util.spec_from_file_location(f"midas_integrate.{name}", PKG / f"{name}.py")
        m = importlib.util.module_from_spec(spec)
        sys.modules[f"midas_integrate.{name}"] = m
        spec.loader.exec_module(m)
        mods[name] = m
    return mods


def random_pixmap(rng, ny, nz, n_r, n_eta, avg=6, oob_fraction=0.05, frac_y=False):
    """Random bin-major map: ~5 % empty bins, some records moved off the detector."""
    n_bins = n_r * n_eta
    recs, bins, cur = [], [], 0
    n_oob = int(n_bins * oob_fraction)
    oob = set(rng.choice(n_bins, size=n_oob, replace=False).tolist()) if n_oob else set()
    for b in range(n_bins):
        if rng.random() < 0.05:
            bins.append([])
            continue
        n = int(rng.poisson(avg)) + 1
        idx = []
        for _ in range(n):
            y = float(rng.integers(0, ny)) + (float(rng.uniform(-0.45, 0.45)) if frac_y else 0.0)
            z = float(rng.integers(0, nz)) + (float(rng.uniform(-0.45, 0.45)) if frac_y else 0.0)
            recs.append((y, z, float(rng.uniform(0.05, 1.0)), float(rng.uniform(-0.4, 0.4)),
                         float(rng.uniform(0.1, 1.0))))
            idx.append(cur)
            cur += 1
        if b in oob and idx:
            y0, z0, fr, dr, aw = recs[idx[-1]]
            recs[idx[-1]] = (float(ny + 5) if rng.random() < 0.5 else -3.0, z0, fr, dr, aw)
        bins.append(idx)
    return recs, bins


KERNEL_CASES = [
    ("a", 0xC0FFEE, 64, 48, 8, 12, False),
    ("b", 0xBEE, 33, 29, 5, 7, True),     # ragged shape, fractional sub-pixel y/z
    ("c", 0xDEAD, 16, 16, 4, 6, False),
    ("d", 123, 50, 70, 9, 11, True),
]


def variance_cases(M):
    """The kernels_* maps again (same seeds), each with a variance image."""
    import torch
    bin_io, kernels = M["bin_io"], M["kernels"]
    for tag, seed, ny, nz, n_r, n_eta, frac in KERNEL_CASES[:2] + KERNEL_CASES[3:]:
        rng = np.random.default_rng(seed)
        recs, bins = random_pixmap(rng, ny, nz, n_r, n_eta, frac_y=frac)
        counts = np.array([len(b) for b in bins], np.int32)
        offsets = np.zeros_like(counts)
        offsets[1:] = np.cumsum(counts[:-1])
        flat = [recs[i] for b in bins for i in b]
        px = np.array(flat, dtype=bin_io.PXLIST_DTYPE)
        pixmap = bin_io.PixelMap(pxList=px, counts=counts, offsets=offsets, map_header=None,
                                 nmap_header=None)
        vr = np.random.default_rng(seed + 1)
        image = vr.uniform(0, 1000, size=(nz, ny))
        var_image = image * vr.uniform(0.8, 1.5, size=(nz, ny)) + 4.0   # gain and read noise
        bc_y, bc_z = ny / 2 + 0.3, nz / 2 - 0.2
        geom = kernels.build_csr(pixmap, n_r=n_r, n_eta=n_eta, n_pixels_y=ny, n_pixels_z=nz,
                                 dtype=torch.float64, bc_y=bc_y, bc_z=bc_z, compute_variance=True)
        out = dict(records=px.view(np.uint8).copy(), counts=counts, offsets=offsets, image=image,
                   var_image=var_image, ny=ny, nz=nz, n_r=n_r, n_eta=n_eta, bc_y=bc_y, bc_z=bc_z,
                   area_per_bin=geom.area_per_bin.numpy())
        for mode in ("floor", "bilinear", "gradient"):
            for norm in (True, False):
                key = f"{mode}_{'n' if norm else 'r'}"
                I, V = kernels.integrate_with_variance(torch.from_numpy(image), geom, mode=mode, normalize=norm,
                                                       variance_image=torch.from_numpy(var_image))
                out[f"int_{key}"] = I.numpy().reshape(-1)
                out[f"var_{key}"] = V.numpy().reshape(-1)
                for pm in ("area_weighted", "simple_mean"):
                    i1, v1 = kernels.profile_1d_with_variance(I, V, geom, mode=pm)
                    out[f"i1_{pm}_{key}"] = i1.numpy()
                    out[f"v1_{pm}_{key}"] = v1.numpy()
        # Poisson default: variance_image=None uses the image itself
        I, V = kernels.integrate_with_variance(torch.from_numpy(image), geom, mode="bilinear", normalize=True)
        out["var_poisson_bilinear_n"] = V.numpy().reshape(-1)
        np.savez_compressed(OUT / f"variance_{tag}.npz", **out)
        print("wrote", OUT / f"variance_{tag}.npz", px.shape[0], "records")


def image_case(M):
    """Hybrid payloads (no overflow, a few overflows, overflows on the first and last
    pixel) and an int64 multi-frame dark file, through the reference's decoders."""
    import tempfile
    im = M["image"]
    rng = np.random.default_rng(606)
    ny, nz = 37, 23
    n = ny * nz
    out = dict(ny=ny, nz=nz)
    for k, n_over in enumerate((0, 9, 2)):
        base = rng.integers(0, 65535, size=n).astype(np.uint16)
        idx = rng.choice(n, size=n_over, replace=False).astype(np.int32)
        if k == 2:
            idx = np.array([0, n - 1], np.int32)
        val = rng.integers(65536, 1 << 40, size=n_over).astype(np.int64)
        payload = (np.array([n_over], np.uint32).tobytes() + base.tobytes() + idx.tobytes() + val.tobytes())
        out[f"payload_{k}"] = np.frombuffer(payload, np.uint8).copy()
        out[f"decoded_{k}"] = im.decode_hybrid_payload(payload, n_pixels_y=ny, n_pixels_z=nz)
    dark = rng.integers(90, 130, size=(7, nz, ny)).astype(np.int64)
    dark[:, 0, 0] = (1 << 40) + np.arange(7)        # large counts: the FP64 sum matters
    with tempfile.TemporaryDirectory() as td:
        f = Path(td) / "dark.bin"
        dark.tofile(f)
        out["dark_frames"] = dark
        out["dark_mean"] = im.average_dark_frames(f, n_pixels_y=ny, n_pixels_z=nz, dtype="int64")
    np.savez_compressed(OUT / "image.npz", **out)
    print("wrote", OUT / "image.npz")


def kernels_cases(M):
    import torch
    bin_io, kernels = M["bin_io"], M["kernels"]
    for tag, seed, ny, nz, n_r, n_eta, frac in KERNEL_CASES:
        rng = np.random.default_rng(seed)
        recs, bins = random_pixmap(rng, ny, nz, n_r, n_eta, frac_y=frac)
        counts = np.array([len(b) for b in bins], np.int32)
        offsets = np.zeros_like(counts)
        offsets[1:] = np.cumsum(counts[:-1])
        flat = [recs[i] for b in bins for i in b]
        px = np.array(flat, dtype=bin_io.PXLIST_DTYPE)
        pixmap = bin_io.PixelMap(pxList=px, counts=counts, offsets=offsets, map_header=None,
                                 nmap_header=None)
        image = rng.uniform(0, 1000, size=(nz, ny)).astype(np.float64)
        bc_y, bc_z = ny / 2 + 0.3, nz / 2 - 0.2
        geom = kernels.build_csr(pixmap, n_r=n_r, n_eta=n_eta, n_pixels_y=ny, n_pixels_z=nz,
                                 dtype=torch.float64, bc_y=bc_y, bc_z=bc_z)
        out = dict(records=px.view(np.uint8).copy(), counts=counts, offsets=offsets, image=image,
                   ny=ny, nz=nz, n_r=n_r, n_eta=n_eta, bc_y=bc_y, bc_z=bc_z,
                   area_per_bin=geom.area_per_bin.numpy())
        for mode in ("floor", "bilinear", "gradient"):
            for norm in (True, False):
                ck = kernels.integrate(torch.from_numpy(image), geom, mode=mode, normalize=norm)
                key = f"{mode}_{'n' if norm else 'r'}"
                out[f"cake_{key}"] = ck.numpy().reshape(-1)
                out[f"aw_{key}"] = kernels.profile_1d(ck, geom, mode="area_weighted").numpy()
                out[f"sm_{key}"] = kernels.profile_1d(ck, geom, mode="simple_mean").numpy()
        np.savez_compressed(OUT / f"kernels_{tag}.npz", **out)
        print("wrote", OUT / f"kernels_{tag}.npz", px.shape[0], "records")


def mapper_cases():
    sys.path.insert(0, str(REPO))
    import oracle
    if not oracle.ref_available():
        oracle.build()
    cases = [
        # tag, ny, nz, px, lsd, bcy, bcz, ty, tz, rmin, rmax, rbin, emin, emax, ebin, sa, pol, parallax
        ("m1", 96, 80, 200.0, 250000.0, 47.3, 41.8, 0.1, -0.05, 4.0, 44.0, 1.0, -180.0, 180.0, 10.0, 0, 0, 0.0),
        ("m2", 72, 72, 150.0, 200000.0, 36.6, 35.1, 0.3, 0.2, 3.0, 33.0, 0.25, -180.0, 180.0, 5.0, 1, 1, 0.0),
        ("m3", 64, 90, 172.0, 300000.0, 20.2, 70.9, -0.4, 0.5, 10.0, 60.0, 2.0, -170.0, 170.0, 20.0, 1, 0, 300.0),
    ]
    for tag, ny, nz, px, lsd, bcy, bcz, ty, tz, rmin, rmax, rbin, emin, emax, ebin, sa, pol, par in cases:
        n_r = int(np.ceil((rmax - rmin) / rbin))
        n_eta = int(np.ceil((emax - emin) / ebin))
        r_lo = rmin + rbin * np.arange(n_r)
        e_lo = emin + ebin * np.arange(n_eta)
        recs, nmap, mask = oracle.ref_build_map(ny=ny, nz=nz, px=px, lsd=lsd, bc_y=bcy, bc_z=bcz, ty=ty, tz=tz,
                                                rho_d=2.0e5,
                                                solid_angle=sa, polarization=pol, pol_fraction=0.99,
                                                parallax=par, r_lo=r_lo, r_hi=r_lo + rbin, eta_lo=e_lo,
                                                eta_hi=e_lo + ebin, n_threads=1)
        rng = np.random.default_rng(7)
        image = rng.uniform(50, 500, size=(nz, ny))
        dark = rng.uniform(0, 20, size=(nz, ny))
        sums_g, norms_g = oracle.ref_integrate(recs, nmap, n_r, n_eta, image, ny, nz, dark=dark, bc_y=bcy,
                                               bc_z=bcz, gradient=1, n_threads=1)
        sums_b, norms_b = oracle.ref_integrate(recs, nmap, n_r, n_eta, image, ny, nz, dark=dark, bc_y=bcy,
                                               bc_z=bcz, gradient=0, n_threads=1)
        np.savez_compressed(OUT / f"mapper_{tag}.npz", records=recs.view(np.uint8).copy(), nmap=nmap,
                            bin_mask=mask, ny=ny, nz=nz, px=px, lsd=lsd, bc_y=bcy, bc_z=bcz, ty=ty, tz=tz,
                            r_lo=r_lo, r_hi=r_lo + rbin, eta_lo=e_lo, eta_hi=e_lo + ebin, sa=sa, pol=pol,
                            parallax=par, rho_d=2.0e5, image=image, dark=dark, ic_sums_gradient=sums_g,
                            ic_norms_gradient=norms_g, ic_sums_bilinear=sums_b, ic_norms_bilinear=norms_b)
        print("wrote", OUT / f"mapper_{tag}.npz", recs.shape[0], "records")


def peakfit_case(M):
    pf = M["peakfit"]
    rng = np.random.default_rng(11)
    x = 100.0 + 0.25 * (np.arange(400) + 0.5)
    lineouts, fits = [], []
    centers = [130.3, 160.77, 171.2]
    for k in range(6):
        y = 80.0 + 0.05 * (x - x[0])
        for c in centers:
            sig_c, gam_c = 900.0 + 200 * k, 35.0 + 5 * k  # centi-x^2, centi-x
            p = [2000.0 * (1 + 0.1 * k), c + 0.013 * k, sig_c, gam_c]
            y = y + pf.pseudo_voigt(x, 1, p + [0.0, 0.0], x_lo=x[0], x_hi=x[-1])
        y = y + rng.normal(0, 0.5, size=x.size)
        out = pf.fit_peaks(x, y, centers, x_bin_size=0.25, fit_roi_padding=40) if hasattr(pf, "fit_peaks") else None
        lineouts.append(y)
        fits.append(np.asarray(out, dtype=np.float64).reshape(len(centers), -1) if out is not None else
                    np.zeros((len(centers), 7)))
    np.savez_compressed(OUT / "peakfit.npz", x=x, lineouts=np.array(lineouts), centers=np.array(centers),
                        ref_fits=np.array(fits))
    print("wrote", OUT / "peakfit.npz")


def header_case(M):
    bin_io = M["bin_io"]
    params = dict(Lsd=1e6, Ycen=1024.3, Zcen=1022.7, pxY=200.0, pxZ=200.0, tx=0.0, ty=0.1, tz=-0.05,
                  RhoD=2e5, RBinSize=1.0, EtaBinSize=5.0, RMin=10.0, RMax=1000.0, EtaMin=-180.0,
                  EtaMax=180.0, NrPixelsY=2048, NrPixelsZ=2048, Parallax=0.0, Wavelength=0.172979)
    h = bin_io.compute_param_hash(**params)
    hdr = bin_io.MapHeader(param_hash=h, q_mode=0, gradient_mode=1, wavelength=0.172979)
    np.savez_compressed(OUT / "header.npz", header=np.frombuffer(hdr.to_bytes(), np.uint8),
                        param_hash=np.frombuffer(h, np.uint8),
                        params=np.array([repr(params)]))
    print("wrote", OUT / "header.npz")


def fused_case(M):
    """build_fused_geometry (fused_csr.py) of a small tilted detector, 4 shifts: the shifted
    maps its own build_map made (captured as it runs), their R axes, an image and the
    integrate() cakes of the fused geometry for bilinear and gradient, FP64."""
    import importlib
    import torch
    kernels = M["kernels"]
    fc = importlib.import_module("midas_integrate.fused_csr")
    params_mod = importlib.import_module("midas_integrate.params")
    p = params_mod.IntegrationParams(NrPixelsY=56, NrPixelsZ=48, pxY=200.0, pxZ=200.0, Lsd=250000.0, BC_y=27.3,
                                     BC_z=23.8, RhoD=2.0e5, ty=0.1, tz=-0.05, RMin=3.0, RMax=27.0, RBinSize=1.5,
                                     EtaMin=-180.0, EtaMax=180.0, EtaBinSize=15.0)
    captured = []
    orig = fc.build_map

    def capture(pk, **kw):
        res = orig(pk, **kw)
        captured.append((float(pk.RMin), res.as_pixel_map()))
        return res

    fc.build_map = capture
    rng = np.random.default_rng(21)
    image = rng.uniform(20, 900, size=(p.NrPixelsZ, p.NrPixelsY))
    out = dict(image=image, ny=p.NrPixelsY, nz=p.NrPixelsZ, bc_y=p.BC_y, bc_z=p.BC_z, n_eta=p.n_eta_bins,
               rbin=p.RBinSize, n_shifts=4)
    for mode in ("bilinear", "gradient"):
        captured.clear()
        geom = fc.build_fused_geometry(p, n_shifts=4, mode=mode, dtype=torch.float64)
        cake = kernels.integrate(torch.from_numpy(image), geom, mode=mode, normalize=False)
        out[f"cake_{mode}"] = cake.numpy().reshape(-1)
        if mode == "gradient":
            for k, (rmin, pm) in enumerate(captured):
                out[f"records_{k}"] = np.ascontiguousarray(pm.pxList).view(np.uint8).copy()
                out[f"counts_{k}"] = np.asarray(pm.counts, np.int32)
                out[f"offsets_{k}"] = np.asarray(pm.offsets, np.int32)
                n_r = pm.counts.size // p.n_eta_bins
                out[f"r_axis_{k}"] = kernels.r_axis(n_r=n_r, RMin=rmin, RBinSize=p.RBinSize)
    fc.build_map = orig
    np.savez_compressed(OUT / "fused.npz", **out)
    print("wrote", OUT / "fused.npz", [out[f"records_{k}"].size // 24 for k in range(4)], "records")


def main():
    M = ref_modules()
    groups = {"kernels": lambda: kernels_cases(M), "mapper": mapper_cases, "peakfit": lambda: peakfit_case(M),
              "header": lambda: header_case(M), "variance": lambda: variance_cases(M),
              "image": lambda: image_case(M), "fused": lambda: fused_case(M)}
    for name in (sys.argv[1:] or list(groups)):
        groups[name]()


if __name__ == "__main__":
    main()
