"""FP64 CPU oracle of the MIDAS caking hot path -- TEST INFRASTRUCTURE ONLY.

Python (ctypes) access to:
  * liboracle.so: the FP64 C restatement in oracle.c (integrate in both reference
    semantics, the two profiles, the LM fitter twin);
  * _ref/libmidas_ref.so (when it was built from the reference sources):
    the reference's own mapper_build_map and integration_apply_map.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference legs
import this package; the library under test never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"
REF_LIB = HERE / "_ref" / "libmidas_ref.so"

REC_DTYPE = np.dtype([("y", "<f4"), ("z", "<f4"), ("frac", "<f8"), ("deltaR", "<f4"),
                      ("areaWeight", "<f4")])
MODES = {"floor": 0, "bilinear": 1, "gradient": 2}
SEMS = {"py": 0, "gpustream": 1, "ic": 2, "omp": 3}

_lib = None
_ref = None


def build() -> None:
    """Compile liboracle.so (and _ref when the reference sources exist)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True, capture_output=True)


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        L = C.CDLL(str(LIB))
        vp, i, d = C.c_void_p, C.c_int, C.c_double
        L.or_integrate.argtypes = [vp, vp, C.c_int64, i, i, d, d, vp, i, i, i, vp, vp]
        L.or_integrate.restype = i
        L.or_area_in.argtypes = [vp, vp, C.c_int64, i, i, vp]
        L.or_area_in.restype = None
        L.or_integrate_var.argtypes = [vp, vp, C.c_int64, i, i, d, d, vp, i, i, i, vp]
        L.or_integrate_var.restype = i
        L.or_profile.argtypes = [vp, vp, i, i, vp, vp]
        L.or_profile.restype = None
        L.or_profile_omp.argtypes = [vp, vp, i, i, vp, vp]
        L.or_profile_omp.restype = None
        L.or_snip_detect.argtypes = [vp, vp, i, i, d, i, vp, vp]
        L.or_snip_detect.restype = i
        L.or_fit.argtypes = [vp, vp, i, d, i, i, i, d, d, d, vp]
        L.or_fit.restype = i
        _lib = L
    return _lib


def ref_available() -> bool:
    return REF_LIB.exists()


def ref() -> C.CDLL:
    global _ref
    if _ref is None:
        if not REF_LIB.exists():
            raise RuntimeError("oracle/_ref/libmidas_ref.so was not built (reference sources absent)")
        R = C.CDLL(str(REF_LIB))
        vp, i, d = C.c_void_p, C.c_int, C.c_double
        R.ref_build_map.argtypes = [i, i, d, d, d, d, d, d, d, d, vp, d, i, i, d, i, d, vp, vp, vp, vp, i, i, i,
                                    C.POINTER(vp), C.POINTER(vp), C.POINTER(vp)]
        R.ref_build_map.restype = C.c_longlong
        R.ref_free.argtypes = [vp]
        R.ref_integrate.argtypes = [vp, vp, i, i, vp, i, i, vp, d, d, i, i, i, vp, vp]
        R.ref_integrate.restype = i
        R.ref_max_threads.restype = i
        _ref = R
    return _ref


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


def integrate(records, nmap, n_bins, ny, nz, image, *, mode="floor", semantics="py", normalize=True,
              bc_y=0.0, bc_z=0.0):
    """FP64 cake (n_bins,) and normaliser (n_bins,) of one dark-subtracted image."""
    rec = _c(records, REC_DTYPE)
    nm = _c(nmap, np.int32).reshape(-1)
    img = _c(image, np.float64).reshape(-1)
    cake = np.zeros(n_bins)
    area = np.zeros(n_bins)
    rc = lib().or_integrate(rec.ctypes.data if rec.size else None, nm.ctypes.data, n_bins, ny, nz, bc_y, bc_z,
                            img.ctypes.data, MODES[mode], SEMS[semantics], int(normalize), cake.ctypes.data,
                            area.ctypes.data)
    if rc:
        raise ValueError(f"or_integrate failed ({rc})")
    return cake, area


def integrate_var(records, nmap, n_bins, ny, nz, var_image, *, mode="floor", semantics="py", normalize=True,
                  bc_y=0.0, bc_z=0.0):
    """FP64 propagated bin variance (n_bins,) of a per-pixel variance image
    (integrate_with_variance, kernels.py:474-536)."""
    rec = _c(records, REC_DTYPE)
    nm = _c(nmap, np.int32).reshape(-1)
    img = _c(var_image, np.float64).reshape(-1)
    out = np.zeros(n_bins)
    rc = lib().or_integrate_var(rec.ctypes.data if rec.size else None, nm.ctypes.data, n_bins, ny, nz, bc_y, bc_z,
                                img.ctypes.data, MODES[mode], SEMS[semantics], int(normalize), out.ctypes.data)
    if rc:
        raise ValueError(f"or_integrate_var failed ({rc})")
    return out


def profile_var(var_cake, area, n_r, n_eta):
    """Variance halves of profile_1d_with_variance (kernels.py:604-645):
    sum(A^2 V) / (sum A)^2 and sum(V) / N^2 over the valid (A > 1e-9) eta bins."""
    v = _c(var_cake, np.float64).reshape(n_r, n_eta)
    a = _c(area, np.float64).reshape(n_r, n_eta)
    ok = a > 1e-9
    av = np.where(ok, a, 0.0)
    sa = av.sum(1)
    n = ok.sum(1).astype(np.float64)
    vaw = np.where(sa > 1e-9, (v * av * av).sum(1) / np.maximum(sa, 1e-9) ** 2, 0.0)
    vsm = np.where(n > 0, np.where(ok, v, 0.0).sum(1) / np.maximum(n, 1.0) ** 2, 0.0)
    return vaw, vsm


def average_frames(frames):
    """Per-pixel mean of k frames as the stream server's start-up computes it
    (IntegratorFitPeaksGPUStream.cu:2216-2232): sequential FP64 sum, divide, cast to float."""
    f = np.asarray(frames)
    acc = np.zeros(f.shape[1:], dtype=np.float64)
    for k in range(f.shape[0]):
        acc += f[k].astype(np.float64)
    return (acc / f.shape[0]).astype(np.float32)


def decode_hybrid(payload: bytes, ny: int, nz: int):
    """dtype-6 payload -> (nz, ny) float32 raw counts (image.py:83-123)."""
    n = ny * nz
    c = int(np.frombuffer(payload, dtype=np.uint32, count=1)[0])
    if len(payload) != 4 + 2 * n + 12 * c:
        raise ValueError("hybrid payload size mismatch")
    out = np.frombuffer(payload, dtype=np.uint16, count=n, offset=4).astype(np.float32)
    idx = np.frombuffer(payload, dtype=np.int32, count=c, offset=4 + 2 * n)
    val = np.frombuffer(payload, dtype=np.int64, count=c, offset=4 + 2 * n + 4 * c)
    out[idx] = val.astype(np.float32)
    return out.reshape(nz, ny)


def bin_table(records, nmap, n_r, n_eta, ny, nz, r_lo, r_hi, eta_lo, eta_hi, px, lsd, lam):
    """[n_r*n_eta, 5] R mean, 2-theta (deg), eta mean, area, Q: the static header of the GPU
    stream output (initialize_PerFrameArr_Area_kernel, IntegratorFitPeaksGPUStream.cu:817-899)."""
    rec = _c(records, REC_DTYPE)
    nm = _c(nmap, np.int32).reshape(-1, 2)
    out = np.zeros((n_r * n_eta, 5))
    for b in range(n_r * n_eta):
        j, k = divmod(b, n_eta)
        rm = (r_lo[j] + r_hi[j]) * 0.5
        em = (eta_lo[k] + eta_hi[k]) * 0.5
        tth = np.arctan(rm * px / lsd)
        area = 0.0
        for e in rec[nm[b, 1]:nm[b, 1] + max(nm[b, 0], 0)]:
            y, z = e["y"], e["z"]
            if y < 0 or y >= ny or z < 0 or z >= nz:
                continue
            flat = np.float32(np.float32(int(z) * ny) + y)
            if int(flat) >= ny * nz:
                continue
            area += float(e["areaWeight"])
        out[b] = (rm, (180.0 / np.pi) * tth, em, area,
                  (4.0 * np.pi / lam) * np.sin(tth / 2.0) if lam > 0 else 0.0)
    return out


def area_in(records, nmap, n_bins, ny, nz):
    rec = _c(records, REC_DTYPE)
    nm = _c(nmap, np.int32).reshape(-1)
    out = np.zeros(n_bins)
    lib().or_area_in(rec.ctypes.data if rec.size else None, nm.ctypes.data, n_bins, ny, nz, out.ctypes.data)
    return out


def snip_detect(x, y, *, n_iter=50, x_bin=1.0, max_sel=30):
    """fitPeaksAutoDetect's SNIP background and detection: (corrected profile, selected bins)."""
    xs = _c(x, np.float64)
    ys = _c(y, np.float64)
    corr = np.zeros(ys.size)
    sel = np.zeros(max(max_sel, 1), np.int32)
    k = lib().or_snip_detect(xs.ctypes.data, ys.ctypes.data, ys.size, int(n_iter), float(x_bin), int(max_sel),
                             corr.ctypes.data, sel.ctypes.data)
    return corr, sel[:k].copy()


def r_interp(r_src, r_tgt):
    """Linear interpolation in R of a cake on r_src onto r_tgt, per target row (j, w_lo,
    w_hi) over source rows j, j + 1: clamped to the first / last pair outside the axis
    (packages/midas_integrate/midas_integrate/fused_csr.py:63-104)."""
    src = np.asarray(r_src, np.float64)
    n = src.size
    out = []
    for r in np.asarray(r_tgt, np.float64):
        if r <= src[0]:
            out.append((0, 1.0, 0.0))
        elif r >= src[-1]:
            out.append((n - 2, 0.0, 1.0))
        else:
            j = min(max(int(np.searchsorted(src, r, side="right")) - 1, 0), n - 2)
            den = src[j + 1] - src[j]
            t = (r - src[j]) / den if den > 0 else 0.0
            out.append((j, 1.0 - t, t))
    return out


def fused_average(maps, r_axes, n_eta, ny, nz, image, *, mode="gradient", bc_y=0.0, bc_z=0.0):
    """Naive multi-map averaging, which the fused geometry folds into one matrix
    (fused_csr.py:1-37, 212-250): each shift's normalised py-semantics cake, interpolated
    in R onto shift 0's axis, averaged over the shifts.  maps: (records, nmap) per shift."""
    r0 = np.asarray(r_axes[0], np.float64)
    out = np.zeros((r0.size, n_eta))
    for (rec, nm), ax in zip(maps, r_axes):
        n_r = np.asarray(ax).size
        ck, _ = integrate(rec, nm, n_r * n_eta, ny, nz, image, mode=mode, semantics="py", normalize=True,
                          bc_y=bc_y, bc_z=bc_z)
        ck = ck.reshape(n_r, n_eta)
        for i, (j, wl, wh) in enumerate(r_interp(ax, r0)):
            out[i] += wl * ck[j] + wh * ck[j + 1]
    return (out / len(maps)).reshape(-1)


def profile_omp(cake, area, n_r, n_eta):
    """The OpenMP integrator's lineout (IntegratorZarrOMP.c:1829-1843): per row the mean of
    the nonzero, non-NaN bins (second) and the area-weighted mean over valid, non-NaN bins."""
    ck = _c(cake, np.float64).reshape(-1)
    ar = _c(area, np.float64).reshape(-1)
    aw = np.zeros(n_r)
    sm = np.zeros(n_r)
    lib().or_profile_omp(ck.ctypes.data, ar.ctypes.data, n_r, n_eta, aw.ctypes.data, sm.ctypes.data)
    return aw, sm


def profile(cake, area, n_r, n_eta):
    ck = _c(cake, np.float64).reshape(-1)
    ar = _c(area, np.float64).reshape(-1)
    aw = np.zeros(n_r)
    sm = np.zeros(n_r)
    lib().or_profile(ck.ctypes.data, ar.ctypes.data, n_r, n_eta, aw.ctypes.data, sm.ctypes.data)
    return aw, sm


def fit(x, y, peak, *, half_window=15, model=0, max_iter=200, x_bin=1.0, px_um=0.0, lsd_um=0.0):
    """FP64 LM fit of one window -> (11 outputs, iterations)."""
    xs = _c(x, np.float64)
    ys = _c(y, np.float64)
    out = np.zeros(11)
    it = lib().or_fit(xs.ctypes.data, ys.ctypes.data, xs.size, float(peak), int(half_window), int(model),
                      int(max_iter), float(x_bin), float(px_um), float(lsd_um), out.ctypes.data)
    return out, it


def ref_build_map(*, ny, nz, px, lsd, bc_y, bc_z, tx=0.0, ty=0.0, tz=0.0, rho_d=0.0, p=None, parallax=0.0,
                  solid_angle=0, polarization=0, pol_fraction=0.99, sub_pixel_level=1, sub_pixel_width=10.0,
                  r_lo, r_hi, eta_lo, eta_hi, n_threads=0):
    """The reference's mapper_build_map -> (records, nmap[n_bins, 2], bin_mask)."""
    R = ref()
    pp = _c(p if p is not None else np.zeros(15), np.float64)
    rl, rh, el, eh = (_c(a, np.float64) for a in (r_lo, r_hi, eta_lo, eta_hi))
    recs_p, nmap_p, mask_p = C.c_void_p(), C.c_void_p(), C.c_void_p()
    tot = R.ref_build_map(ny, nz, px, lsd, bc_y, bc_z, tx, ty, tz, rho_d, pp.ctypes.data, parallax,
                          int(solid_angle), int(polarization), pol_fraction, int(sub_pixel_level),
                          sub_pixel_width, rl.ctypes.data, rh.ctypes.data, el.ctypes.data, eh.ctypes.data,
                          rl.size, el.size, int(n_threads), C.byref(recs_p), C.byref(nmap_p), C.byref(mask_p))
    nb = rl.size * el.size
    recs = np.frombuffer((C.c_char * (24 * max(tot, 0))).from_address(recs_p.value), dtype=REC_DTYPE).copy() \
        if tot > 0 else np.empty(0, REC_DTYPE)
    nmap = np.frombuffer((C.c_int32 * (2 * nb)).from_address(nmap_p.value), dtype=np.int32).copy().reshape(nb, 2)
    mask = np.frombuffer((C.c_int32 * nb).from_address(mask_p.value), dtype=np.int32).copy()
    for q in (recs_p, nmap_p, mask_p):
        R.ref_free(q)
    return recs, nmap, mask


def ref_integrate(records, nmap, n_r, n_eta, image, ny, nz, *, dark=None, bc_y=0.0, bc_z=0.0, gradient=0,
                  n_threads=0, chunk_rows=8):
    """The reference's integration_apply_map over R-row chunks -> (sums, norms) per bin."""
    R = ref()
    rec = _c(records, REC_DTYPE)
    nm = _c(nmap, np.int32).reshape(-1)
    img = _c(image, np.float64).reshape(-1)
    dk = _c(dark, np.float64).reshape(-1) if dark is not None else None
    prof = np.zeros(n_r * n_eta)
    norm = np.zeros(n_r * n_eta)
    R.ref_integrate(rec.ctypes.data, nm.ctypes.data, n_r, n_eta, img.ctypes.data, ny, nz,
                    dk.ctypes.data if dk is not None else None, bc_y, bc_z, int(gradient), int(n_threads),
                    int(chunk_rows), prof.ctypes.data, norm.ctypes.data)
    return prof, norm
