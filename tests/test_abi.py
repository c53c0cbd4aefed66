"""The C-ABI library loads, exports every entry point include/midas_b200.h declares, and
its host-side argument checks fail loudly (no GPU needed)."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

from midas_b200 import _lib as L

HEADER = Path(__file__).resolve().parents[1] / "include" / "midas_b200.h"


def declared_symbols():
    txt = HEADER.read_text()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(mi_[a-z0-9_]+)\s*\(", txt)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    assert "mi_integrate_batch" in syms and "mi_plan_create" in syms and "mi_fit_batch" in syms


def test_library_exports_every_declared_symbol():
    lib = L.lib()
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, f"not exported: {missing}"


def test_bindings_cover_every_declared_symbol():
    bound = {n for n, _, _ in L.SIGNATURES}
    assert set(declared_symbols()) <= bound


def test_version_and_empty_error():
    assert b"sm_100a" in L.lib().mi_version()
    assert isinstance(L.lib().mi_last_error(), bytes)


def test_null_arguments_are_rejected():
    lib = L.lib()
    h = C.c_void_p()
    assert lib.mi_plan_create(None, None, 0, C.byref(h)) == L.MI_E_ARG
    assert b"null" in lib.mi_last_error()
    assert lib.mi_integrate_batch(None, None, 1, 1, 1, None, None, None, None) == L.MI_E_ARG
    assert lib.mi_cast_dark(None, 1, 1, 1, None, None, None) == L.MI_E_ARG
    buf = np.zeros(16, np.uint16)
    assert lib.mi_upload_frames(None, buf.ctypes.data, 1, 1, 16, buf.ctypes.data, 16, None) == L.MI_E_ARG
    assert lib.mi_stage_host_frames(None, buf.ctypes.data, 1, 1, 16, buf.ctypes.data, 16) == L.MI_E_ARG
    assert b"mi_stage_host_frames" in lib.mi_last_error()
    opts = L.MiFitOpts(9, 15, 10, 1.0, 0.0, 0.0)
    x = np.zeros(4)
    assert lib.mi_fit_batch(x.ctypes.data, x.ctypes.data, 1, 4, x.ctypes.data, 1, C.byref(opts),
                            x.ctypes.data, x.ctypes.data, None) == L.MI_E_ARG
    lib.mi_plan_destroy(None)          # no-op
    lib.mi_map_destroy(None)


def test_plan_shape_errors_before_device_use():
    lib = L.lib()
    nmap = np.zeros((4, 2), np.int32)
    d = L.MiMapDesc(None, 0, nmap.ctypes.data, 2, 2, 1, 5, 0.0, 0.0)   # ny < 2
    h = C.c_void_p()
    assert lib.mi_plan_create(C.byref(d), None, 0, C.byref(h)) == L.MI_E_ARG
    assert b"bad shape" in lib.mi_last_error()


def test_error_code_raises_python_exception():
    with pytest.raises(L.MidasError) as e:
        L.check(L.lib().mi_cast_dark(None, 1, 1, 1, None, None, None), "mi_cast_dark")
    assert e.value.code == L.MI_E_ARG


def test_synth_descriptor_validation():
    d = L.MiSynthDesc()
    d.ny = 1
    assert L.lib().mi_synth_dark(C.byref(d), None, None) == L.MI_E_ARG


def test_frame_preparation_argument_checks():
    """Hybrid payload size and shape checks and the dark-average arguments are validated
    on the host before any device call (buffers here are host memory never touched)."""
    lib = L.lib()
    buf = np.zeros(64, np.uint8)
    p = buf.ctypes.data
    assert lib.mi_decode_hybrid(None, 0, 4, 4, p, p, p, None) == L.MI_E_ARG
    assert lib.mi_decode_hybrid(p, 10, 4, 4, p, p, p, None) == L.MI_E_ARG     # smaller than count + base
    assert b"smaller" in lib.mi_last_error()
    payload = np.zeros(4 + 2 * 16 + 12, np.uint8)
    payload[:4] = np.frombuffer(np.uint32(2).tobytes(), np.uint8)            # claims 2 overflows, holds 1
    assert lib.mi_decode_hybrid(payload.ctypes.data, payload.size, 4, 4, p, p, p, None) == L.MI_E_ARG
    assert b"need" in lib.mi_last_error()
    assert lib.mi_decode_hybrid(p, 40, 0, 4, p, p, p, None) == L.MI_E_ARG
    assert lib.mi_average_frames(None, 1, 16, 2, 16, None, None) == L.MI_E_ARG
    assert lib.mi_average_frames(p, 1, 16, 0, 16, p, None) == L.MI_E_ARG      # no frames
    assert lib.mi_average_frames(p, 1, 16, 2, 8, p, None) == L.MI_E_ARG       # stride < pixels
    assert lib.mi_average_frames(p, 6, 16, 2, 16, p, None) == L.MI_E_ARG      # hybrid is not a frame dtype
    assert lib.mi_plan_bin_table(None, p, p, p, p, 1.0, 1.0, 0.0, p) == L.MI_E_ARG


def test_plan_opts_layout_matches_header():
    """mi_plan_opts: ten int32 fields, host_threads last."""
    assert C.sizeof(L.MiPlanOpts) == 10 * 4
    assert [f for f, _ in L.MiPlanOpts._fields_][-2:] == ["variance", "host_threads"]


def test_without_a_gpu_plans_fail_loudly():
    """No CUDA device: the Python plan and the C ABI both refuse with an error; nothing falls
    back to a host computation."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("checks the behaviour on a host without a GPU")
    import oracle
    from midas_b200.bin_io import from_arrays
    from midas_b200.kernels import CakePlan
    recs = np.zeros(1, dtype=oracle.REC_DTYPE)
    recs["y"], recs["z"], recs["frac"], recs["areaWeight"] = 2.0, 3.0, 1.0, 1.0
    nmap = np.zeros((12, 2), np.int32)
    nmap[0] = (1, 0)
    with pytest.raises(RuntimeError, match="CUDA device"):
        CakePlan(from_arrays(recs, nmap), n_r=3, n_eta=4, n_pixels_y=8, n_pixels_z=8, device="cuda")
    desc = L.MiMapDesc(recs.ctypes.data, 1, nmap.ctypes.data, 3, 4, 8, 8, 0.0, 0.0)
    opts = L.MiPlanOpts(L.MODE["floor"], 1, L.SEM["py"], 0, 0, 0, L.ENC["auto"], 0, 0, 0)
    h = C.c_void_p()
    rc = L.lib().mi_plan_create(C.byref(desc), C.byref(opts), 0, C.byref(h))
    assert rc != 0 and not h.value
    assert L.lib().mi_last_error()
