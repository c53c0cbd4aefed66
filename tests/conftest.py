"""Shared pytest setup: the `gpu` marker, in-tree builds, golden-fixture loaders."""
from __future__ import annotations

import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

REPO = Path(__file__).resolve().parents[1]
GOLDEN = Path(__file__).resolve().parent / "golden"
if str(REPO) not in sys.path:
    sys.path.insert(0, str(REPO))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    config.addinivalue_line("markers", "slow: long-running")


def _ensure_built():
    lib = REPO / "midas_b200" / "libmidas_b200.so"
    if not lib.exists():
        from midas_b200 import build
        build.build()
    if not (REPO / "oracle" / "liboracle.so").exists():
        subprocess.run(["make", "-s", "-C", str(REPO / "oracle")], check=True)


_ensure_built()

REC_DTYPE = np.dtype([("y", "<f4"), ("z", "<f4"), ("frac", "<f8"), ("deltaR", "<f4"),
                      ("areaWeight", "<f4")])


def load_kernels_case(tag):
    g = dict(np.load(GOLDEN / f"kernels_{tag}.npz"))
    g["records"] = g["records"].view(REC_DTYPE)
    g["nmap"] = np.stack([g["counts"], g["offsets"]], 1).astype(np.int32)
    for k in ("ny", "nz", "n_r", "n_eta"):
        g[k] = int(g[k])
    for k in ("bc_y", "bc_z"):
        g[k] = float(g[k])
    return g


def load_variance_case(tag):
    g = dict(np.load(GOLDEN / f"variance_{tag}.npz"))
    g["records"] = g["records"].view(REC_DTYPE)
    g["nmap"] = np.stack([g["counts"], g["offsets"]], 1).astype(np.int32)
    for k in ("ny", "nz", "n_r", "n_eta"):
        g[k] = int(g[k])
    for k in ("bc_y", "bc_z"):
        g[k] = float(g[k])
    return g


def load_image_case():
    return dict(np.load(GOLDEN / "image.npz"))


def load_mapper_case(tag):
    g = dict(np.load(GOLDEN / f"mapper_{tag}.npz"))
    g["records"] = g["records"].view(REC_DTYPE)
    for k in ("ny", "nz", "sa", "pol"):
        g[k] = int(g[k])
    for k in ("px", "lsd", "bc_y", "bc_z", "ty", "tz", "parallax", "rho_d"):
        g[k] = float(g[k])
    return g


def load_fused_case():
    """fused.npz: the reference's shifted maps (PixelMaps), R axes, image and fused cakes."""
    from midas_b200.bin_io import from_arrays
    g = dict(np.load(GOLDEN / "fused.npz"))
    for k in ("ny", "nz", "n_eta", "n_shifts"):
        g[k] = int(g[k])
    for k in ("bc_y", "bc_z", "rbin"):
        g[k] = float(g[k])
    g["maps"], g["nmaps"], g["r_axes"] = [], [], []
    for k in range(g["n_shifts"]):
        rec = g[f"records_{k}"].view(REC_DTYPE)
        nm = np.stack([g[f"counts_{k}"], g[f"offsets_{k}"]], 1).astype(np.int32)
        g["maps"].append(from_arrays(rec, nm))
        g["nmaps"].append((rec, nm))
        g["r_axes"].append(g[f"r_axis_{k}"])
    return g


KERNEL_CASES = ["a", "b", "c", "d"]
MAPPER_CASES = ["m1", "m2", "m3"]
VARIANCE_CASES = ["a", "b", "d"]


def rel_err(x, ref, tau_frac=1e-3):
    """max / mean of |x - ref| / max(|ref|, tau), tau = tau_frac * median |ref| over nonzero."""
    x = np.asarray(x, np.float64).reshape(-1)
    ref = np.asarray(ref, np.float64).reshape(-1)
    nz = np.abs(ref[ref != 0])
    tau = tau_frac * (np.median(nz) if nz.size else 1.0)
    tau = max(tau, 1e-300)
    r = np.abs(x - ref) / np.maximum(np.abs(ref), tau)
    return float(r.max()) if r.size else 0.0, float(r.mean()) if r.size else 0.0


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("CUDA not available")
    return torch.device("cuda", 0)
