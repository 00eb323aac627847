"""Build the sm_100a shared library in-tree: ultrasound_solver_b200/_lib/libusv_b200.so.

    python -m ultrasound_solver_b200.build [--force]

The library is plain CUDA C++ behind the C ABI of include/usv.h; it is
compiled with nvcc for sm_100a only and loaded with ctypes (no torch types
cross the boundary).
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INCLUDE = ROOT / "include"
LIBDIR = PKG / "_lib"
LIBNAME = "libusv_b200.so"
SOURCES = ("operator.cu", "gmres.cu", "scene.cu", "basis.cu", "losses.cu", "surface.cu",
           "dense.cpp")
HEADERS = ("usv_internal.cuh", "dense.h")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc_path() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: set NVCC or add /usr/local/cuda/bin to PATH")


def library_path() -> Path:
    return LIBDIR / LIBNAME


def _stale(target: Path) -> bool:
    if not target.exists():
        return True
    newest = max(p.stat().st_mtime for p in [*(CSRC / s for s in SOURCES),
                                              *(CSRC / h for h in HEADERS), INCLUDE / "usv.h"])
    return target.stat().st_mtime < newest


def build(force: bool = False, verbose: bool = False) -> Path:
    target = library_path()
    if not force and not _stale(target):
        return target
    LIBDIR.mkdir(exist_ok=True)
    nvcc = nvcc_path()
    objdir = LIBDIR / "obj"
    objdir.mkdir(exist_ok=True)
    common = [*ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
              "-I", str(INCLUDE), "-I", str(CSRC)]
    objs = []
    procs = []
    for src in SOURCES:
        obj = objdir / (Path(src).stem + ".o")
        cmd = [nvcc, *common, "-c", str(CSRC / src), "-o", str(obj)]
        if src.endswith(".cpp"):  # host dense algebra: plain complex arithmetic, finite data
            cmd.insert(1, "-Xcompiler=-fcx-limited-range")
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
            print(" ".join(cmd))
        procs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
        objs.append(obj)
    for cmd, proc in procs:
        out, _ = proc.communicate()
        if proc.returncode != 0:
            raise RuntimeError(f"nvcc failed ({' '.join(cmd)}):\n{out.decode(errors='replace')}")
        if verbose and out:
            print(out.decode(errors="replace"))
    tmp = target.with_suffix(".so.tmp")
    link = [nvcc, *ARCH, "-shared", "-o", str(tmp), *map(str, objs)]
    res = subprocess.run(link, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"link failed: {res.stdout}\n{res.stderr}")
    os.replace(tmp, target)
    return target


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    args = ap.parse_args(argv)
    print(build(force=args.force, verbose=args.verbose))


if __name__ == "__main__":
    sys.exit(main())
