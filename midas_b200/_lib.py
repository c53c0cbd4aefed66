"""ctypes binding of libmidas_b200.so (the C ABI declared in include/midas_b200.h).

The library is built in-tree by ``python -m midas_b200.build``.  There is no
fallback: if the shared library is missing every entry point raises.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

_HERE = Path(__file__).resolve().parent
LIB_PATH = _HERE / "libmidas_b200.so"

# ---- status codes ---------------------------------------------------------
MI_OK = 0
MI_E_ARG = -1
MI_E_MAP = -2
MI_E_OOM = -3
MI_E_CUDA = -4
MI_E_TIMEOUT = -5
MI_E_UNSUPPORTED = -6
MI_E_RANGE = -7

MODE = {"floor": 0, "bilinear": 1, "gradient": 2}
SEM = {"py": 0, "gpustream": 1, "ic": 2, "omp": 3}
DT_U8, DT_U16, DT_U32, DT_I64, DT_F32, DT_F64, DT_I32 = 0, 1, 2, 3, 4, 5, 7
FIT_PV, FIT_TCH = 0, 1
FIT_NOUT = 11
FIT_KIND_PEAKS, FIT_KIND_ETA = 0, 1
FIT_JOB_MAX_PEAKS = 8


class MiMapRecord(C.Structure):
    _fields_ = [("y", C.c_float), ("z", C.c_float), ("frac", C.c_double),
                ("deltaR", C.c_float), ("areaWeight", C.c_float)]


class MiMapDesc(C.Structure):
    _fields_ = [("records", C.c_void_p), ("n_records", C.c_int64), ("nmap", C.c_void_p),
                ("n_r", C.c_int32), ("n_eta", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
                ("bc_y", C.c_double), ("bc_z", C.c_double)]


class MiPlanOpts(C.Structure):
    _fields_ = [("mode", C.c_int32), ("normalize", C.c_int32), ("semantics", C.c_int32),
                ("tile_rows", C.c_int32), ("tile_pixels", C.c_int32),
                ("frames_per_lane", C.c_int32), ("encoding", C.c_int32), ("run_len", C.c_int32),
                ("variance", C.c_int32), ("host_threads", C.c_int32)]


ENC = {"auto": 0, "csr": 1, "runs": 2, "mma": 3, "mmad": 4}


class MiPlanInfo(C.Structure):
    _fields_ = [("n_bins", C.c_int64), ("n_r", C.c_int64), ("n_eta", C.c_int64),
                ("nnz", C.c_int64), ("n_records", C.c_int64), ("n_tiles", C.c_int64),
                ("n_items", C.c_int64), ("staged_pixels", C.c_int64), ("ref_pixels", C.c_int64),
                ("map_bytes", C.c_int64), ("device_bytes", C.c_int64), ("oob_records", C.c_int64),
                ("tile_rows", C.c_int32), ("tile_pixels", C.c_int32),
                ("frames_per_lane", C.c_int32), ("run_len", C.c_int32), ("xc_pixels", C.c_int64),
                ("ref_row_lo", C.c_int32), ("ref_row_hi", C.c_int32), ("upload_pixels", C.c_int64)]


class MiFitOpts(C.Structure):
    _fields_ = [("model", C.c_int32), ("half_window", C.c_int32), ("max_iter", C.c_int32),
                ("x_bin", C.c_double), ("px_um", C.c_double), ("lsd_um", C.c_double)]


class MiFitJobOpts(C.Structure):
    _fields_ = [("kind", C.c_int32), ("half_window", C.c_int32), ("max_iter", C.c_int32), ("pad", C.c_int32),
                ("x_bin", C.c_double), ("doublet_sep", C.c_double), ("px_um", C.c_double),
                ("lsd_um", C.c_double)]


class MiGeometry(C.Structure):
    _fields_ = [("ny", C.c_int32), ("nz", C.c_int32), ("px_um", C.c_double),
                ("lsd_um", C.c_double), ("bc_y", C.c_double), ("bc_z", C.c_double),
                ("tx", C.c_double), ("ty", C.c_double), ("tz", C.c_double),
                ("rho_d", C.c_double), ("p", C.c_double * 15), ("parallax_um", C.c_double),
                ("solid_angle", C.c_int32), ("polarization", C.c_int32),
                ("pol_fraction", C.c_double), ("sub_pixel_level", C.c_int32),
                ("sub_pixel_cardinal_width", C.c_double), ("mask_host", C.c_void_p)]


class MiBinning(C.Structure):
    _fields_ = [("n_r", C.c_int32), ("n_eta", C.c_int32), ("r_lo", C.c_void_p),
                ("r_hi", C.c_void_p), ("eta_lo", C.c_void_p), ("eta_hi", C.c_void_p)]


class MiSynthDesc(C.Structure):
    _fields_ = [("ny", C.c_int32), ("nz", C.c_int32), ("bc_y", C.c_double), ("bc_z", C.c_double),
                ("lsd_um", C.c_double), ("px_um", C.c_double), ("ty", C.c_double),
                ("tz", C.c_double), ("n_rings", C.c_int32), ("ring_r_px", C.c_double * 32),
                ("ring_amp", C.c_double * 32), ("fwhm_px", C.c_double), ("mix_eta", C.c_double),
                ("texture", C.c_double), ("background", C.c_double), ("amp_drift", C.c_double),
                ("n_spots", C.c_int32), ("spot_sigma", C.c_double), ("spot_amp", C.c_double),
                ("dark_mean", C.c_double), ("dark_sigma", C.c_double), ("seed", C.c_uint64),
                ("poisson", C.c_int32)]


# (name, restype, argtypes) for every exported entry point
SIGNATURES = [
    ("mi_plan_create", C.c_int, [C.POINTER(MiMapDesc), C.POINTER(MiPlanOpts), C.c_int,
                                 C.POINTER(C.c_void_p)]),
    ("mi_plan_set_dark", C.c_int, [C.c_void_p, C.c_void_p]),
    ("mi_plan_create_panels", C.c_int, [C.POINTER(MiMapDesc), C.c_int, C.POINTER(MiPlanOpts), C.c_int,
                                        C.POINTER(C.c_void_p)]),
    ("mi_plan_set_dark_panels", C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    ("mi_plan_create_fused", C.c_int, [C.POINTER(MiMapDesc), C.c_int, C.POINTER(C.c_void_p),
                                       C.POINTER(MiPlanOpts), C.c_int, C.POINTER(C.c_void_p)]),
    ("mi_fused_csr", C.c_int, [C.POINTER(MiMapDesc), C.c_int, C.POINTER(C.c_void_p), C.c_int, C.c_void_p,
                               C.c_void_p, C.c_void_p, C.c_int64, C.POINTER(C.c_int64)]),
    ("mi_integrate_panels", C.c_int, [C.c_void_p, C.POINTER(C.c_void_p), C.POINTER(C.c_int),
                                      C.POINTER(C.c_int64), C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                      C.c_void_p]),
    ("mi_plan_get_info", C.c_int, [C.c_void_p, C.POINTER(MiPlanInfo)]),
    ("mi_sum_cake", C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]),
    ("mi_plan_set_bin_mask", C.c_int, [C.c_void_p, C.c_void_p]),
    ("mi_plan_set_mma_pipeline", C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    ("mi_selftest_wait", C.c_int, [C.c_uint32, C.c_int, C.c_int, C.POINTER(C.c_int)]),
    ("mi_plan_bytes", C.c_int, [C.c_void_p, C.POINTER(C.c_size_t)]),
    ("mi_plan_status", C.c_int, [C.c_void_p, C.POINTER(C.c_int)]),
    ("mi_plan_destroy", None, [C.c_void_p]),
    ("mi_integrate_batch", C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int64,
                                     C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("mi_integrate_batch_static", C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int64,
                                            C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("mi_upload_frames", C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int64, C.c_void_p, C.c_int64,
                                   C.c_void_p]),
    ("mi_stage_host_frames", C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int64, C.c_void_p,
                                       C.c_int64]),
    ("mi_integrate_plain", C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p,
                                     C.c_void_p, C.c_void_p]),
    ("mi_profile_batch", C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p,
                                   C.c_void_p, C.c_void_p]),
    ("mi_cast_dark", C.c_int, [C.c_void_p, C.c_int, C.c_int64, C.c_int, C.c_void_p, C.c_void_p,
                               C.c_void_p]),
    ("mi_average_frames", C.c_int, [C.c_void_p, C.c_int, C.c_int64, C.c_int, C.c_int64, C.c_void_p,
                                    C.c_void_p]),
    ("mi_decode_hybrid", C.c_int, [C.c_void_p, C.c_size_t, C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                                   C.c_void_p, C.c_void_p]),
    ("mi_plan_bin_table", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_double,
                                    C.c_double, C.c_double, C.c_void_p]),
    ("mi_fit_batch", C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int,
                               C.POINTER(MiFitOpts), C.c_void_p, C.c_void_p, C.c_void_p]),
    ("mi_fit_plan_create", C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.POINTER(MiFitJobOpts), C.c_int,
                                     C.POINTER(C.c_void_p)]),
    ("mi_fit_plan_info", C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    ("mi_fit_plan_jobs", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    ("mi_fit_plan_run", C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int64, C.c_int64,
                                  C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("mi_fit_plan_destroy", None, [C.c_void_p]),
    ("mi_fit_autodetect", C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_double, C.c_int, C.c_int,
                                    C.c_double, C.c_double, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("mi_map_build", C.c_int, [C.POINTER(MiGeometry), C.POINTER(MiBinning), C.c_int,
                               C.POINTER(C.c_void_p)]),
    ("mi_map_sizes", C.c_int, [C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    ("mi_map_copy", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("mi_map_destroy", None, [C.c_void_p]),
    ("mi_synth_frames", C.c_int, [C.POINTER(MiSynthDesc), C.c_int64, C.c_int, C.c_int, C.c_void_p,
                                  C.c_int64, C.c_void_p]),
    ("mi_synth_dark", C.c_int, [C.POINTER(MiSynthDesc), C.c_void_p, C.c_void_p]),
    ("mi_last_error", C.c_char_p, []),
    ("mi_version", C.c_char_p, []),
]


class MidasError(RuntimeError):
    """Error returned by a libmidas_b200 entry point (status code + message)."""

    def __init__(self, code: int, where: str, msg: str):
        super().__init__(f"{where} failed ({code}): {msg}")
        self.code = code


_lib = None


def lib() -> C.CDLL:
    """Load libmidas_b200.so once; raise if it has not been built."""
    global _lib
    if _lib is None:
        path = os.environ.get("MIDAS_B200_LIB", str(LIB_PATH))
        if not Path(path).exists():
            raise RuntimeError(
                f"{path} not found: build the CUDA extension with `python -m midas_b200.build`")
        L = C.CDLL(path)
        for name, res, args in SIGNATURES:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(rc: int, where: str) -> None:
    if rc != MI_OK:
        msg = lib().mi_last_error()
        raise MidasError(rc, where, msg.decode() if msg else "")


def ptr(t) -> int:
    """Raw data pointer of a torch tensor / numpy array (or None -> 0)."""
    if t is None:
        return None
    if hasattr(t, "data_ptr"):
        return t.data_ptr()
    return t.ctypes.data


def stream_ptr(stream=None):
    """cudaStream_t of a torch.cuda.Stream (current stream when None)."""
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return C.c_void_p(s.cuda_stream)
