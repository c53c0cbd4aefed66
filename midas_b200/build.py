"""Build libmidas_b200.so (all CUDA sources, sm_100a) in-tree.

Usage: python -m midas_b200.build [--jobs N] [--force]

Each .cu file is compiled to an object with nvcc (``-gencode
arch=compute_100a,code=sm_100a``), then linked into one shared library next to
this file.  Objects are rebuilt only when a source or header is newer.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
INCLUDE = HERE.parent / "include"
OBJDIR = HERE / "_build"
LIB = HERE / "libmidas_b200.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [
    "-O3", "-lineinfo", "-std=c++17", "--expt-extended-lambda", "--expt-relaxed-constexpr",
    "-Xcompiler", "-fPIC,-fopenmp,-O3", f"-I{INCLUDE}", f"-I{CSRC}",
    "-Xptxas", "-warn-spills",
]


def nvcc() -> str:
    exe = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(exe).exists():
        raise RuntimeError("nvcc not found; the CUDA toolkit is required to build midas_b200")
    return exe


def sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu"))


def _newest_header() -> float:
    hs = list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h"))
    return max((h.stat().st_mtime for h in hs), default=0.0)


# per-file extra flags: the map builder's polygon clipping solves ill-conditioned
# quadratics near tangency; without FMA contraction the device build rounds like the
# host build of the same source
EXTRA = {"mi_mapper.cu": ["-fmad=false"]}


def _compile(src: Path, force: bool, verbose: bool) -> Path:
    obj = OBJDIR / (src.stem + ".o")
    if (not force and obj.exists()
            and obj.stat().st_mtime > max(src.stat().st_mtime, _newest_header())):
        return obj
    cmd = [nvcc(), *ARCH, *NVCC_FLAGS, *EXTRA.get(src.name, []), "-c", str(src), "-o", str(obj)]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src.name}:\n{r.stdout}\n{r.stderr}")
    if r.stderr.strip() and verbose:
        print(r.stderr, file=sys.stderr)
    return obj


def build(force: bool = False, jobs: int | None = None, verbose: bool = False) -> Path:
    OBJDIR.mkdir(exist_ok=True)
    srcs = sources()
    jobs = jobs or min(len(srcs), os.cpu_count() or 4)
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        objs = list(ex.map(lambda s: _compile(s, force, verbose), srcs))
    if (force or not LIB.exists()
            or LIB.stat().st_mtime < max(o.stat().st_mtime for o in objs)):
        cmd = [nvcc(), *ARCH, "-shared", "-Xcompiler", "-fopenmp", *map(str, objs),
               "-o", str(LIB), "-lgomp"]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--jobs", type=int, default=None)
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, jobs=a.jobs, verbose=a.verbose))


if __name__ == "__main__":
    main()
