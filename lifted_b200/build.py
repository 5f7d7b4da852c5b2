"""Builds liblifted_b200.so (CUDA kernels for sm_100a + host library + C ABI
+ drop-in C++ API) in-tree, next to this file.

    python -m lifted_b200.build [--force] [-j N]

Objects go to $LIFTED_BUILD_DIR, else lifted_b200_build/ under the system's
temporary directory, outside the source tree (only the linked library sits
in-tree).  Sources are recompiled when they or any header they may include
is newer than their object.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
import tempfile
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = Path(os.environ.get("LIFTED_BUILD_DIR") or
             Path(tempfile.gettempdir()) / "lifted_b200_build")
LIB = PKG / "liblifted_b200.so"

CUDA_HOME = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))
NVCC = str(CUDA_HOME / "bin" / "nvcc")
CXX = os.environ.get("CXX", "g++")

GENCODE = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = GENCODE + [
    "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
    "-fmad=false",  # every fused multiply-add is an explicit __fma_rn
    "--expt-relaxed-constexpr", "-Xptxas", "-warn-spills",
    f"-I{ROOT / 'include'}", f"-I{CSRC}",
]
CXX_FLAGS = ["-std=c++20", "-O2", "-fPIC", "-Wall", "-Wno-unused-function",
             "-ffp-contract=off", f"-I{CUDA_HOME / 'include'}",
             f"-I{ROOT / 'include'}", f"-I{CSRC}"]


def _sources():
    cu = sorted(CSRC.glob("*.cu"))
    cpp = sorted(CSRC.glob("*.cpp"))
    return cu, cpp


def _headers():
    hs = list(CSRC.glob("*.hpp")) + list(CSRC.glob("*.cuh")) + \
        list(CSRC.glob("*.inc")) + list((ROOT / "include").glob("*.h*"))
    return max((h.stat().st_mtime for h in hs), default=0.0)


def _stale(src: Path, obj: Path, hdr_mtime: float) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return src.stat().st_mtime > t or hdr_mtime > t


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build step failed:\n" + " ".join(cmd) + "\n" +
                           r.stdout + r.stderr)
    return r.stdout + r.stderr


def build(force: bool = False, jobs: int | None = None, verbose: bool = False) -> Path:
    """Compiles every CUDA/C++ source for sm_100a and links the library."""
    if shutil.which(NVCC) is None and not Path(NVCC).exists():
        raise RuntimeError(f"nvcc not found at {NVCC}")
    BUILD.mkdir(parents=True, exist_ok=True)
    cu, cpp = _sources()
    hdr = _headers()
    tasks = []
    objs = []
    for s in cu:
        o = BUILD / (s.stem + ".cu.o")
        objs.append(o)
        if force or _stale(s, o, hdr):
            tasks.append([NVCC] + NVCC_FLAGS + ["-c", str(s), "-o", str(o)])
    for s in cpp:
        o = BUILD / (s.stem + ".cpp.o")
        objs.append(o)
        if force or _stale(s, o, hdr):
            tasks.append([CXX] + CXX_FLAGS + ["-c", str(s), "-o", str(o)])
    if tasks:
        with cf.ThreadPoolExecutor(max_workers=jobs or os.cpu_count() or 4) as ex:
            for out in ex.map(_run, tasks):
                if verbose and out.strip():
                    print(out)
    newest = max(o.stat().st_mtime for o in objs)
    if force or tasks or not LIB.exists() or LIB.stat().st_mtime < newest:
        tmp = LIB.with_suffix(".so.tmp")
        _run([NVCC] + GENCODE + ["-shared", "-o", str(tmp)] +
             [str(o) for o in objs])
        os.replace(tmp, LIB)
    return LIB


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-j", "--jobs", type=int, default=None)
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args(argv)
    lib = build(a.force, a.jobs, a.verbose)
    print(lib)
    return 0


if __name__ == "__main__":
    sys.exit(main())
