"""Build the sm_100a shared library ``pfb200/_lib/libpfb200.so`` in-tree.

Every CUDA translation unit is compiled with
``nvcc -gencode arch=compute_100a,code=sm_100a -lineinfo -O3`` and linked with
the static CUDA runtime, so the library carries no dependency on the CUDA
runtime that PyTorch loads into the same process. Host code is compiled
without floating-point contraction (the initialisers' placement must be
reproducible bit for bit).

Usage: ``python phase-field-gh200_b200/build.py [--force] [--verbose]``.
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
OUT_DIR = HERE / "pfb200" / "_lib"
OBJ_DIR = HERE / "build" / "obj"
LIB = OUT_DIR / "libpfb200.so"
INCLUDE = HERE.parent / "include"

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = [
    "-std=c++17",
    "-O3",
    "-lineinfo",
    "--expt-relaxed-constexpr",
    "-Xcompiler", "-fPIC,-ffp-contract=off,-Wall",
    "-I", str(INCLUDE),
]
SOURCES = ["step2d.cu", "init2d.cu", "sim2d.cu", "host2d.cpp", "measure3d.cu", "update3d.cu",
           "step3d.cu", "promote3d.cu", "misc3d.cu", "sim3d.cu", "host3d.cpp", "conv2d_tc.cu",
           "relax2d.cu", "unet2d.cu", "ckpt2d.cpp",
           "ckpt3d.cpp", "velocity2d.cu", "boundary2d.cu", "boundary3d.cu",
           "order2d.cu"]
# command-line programs over the C ABI, linked against the library
CLI_SOURCES = {"pfb_cell": "cli2d.cpp", "pfb_cell_3d": "cli3d.cpp"}
CXX = os.environ.get("CXX", "g++")
HEADERS = ["pfb_common.cuh", "device_util.cuh", "pfb_internal.h", "step2d_common.cuh",
           "pfb3d_common.cuh", "ring3d.cuh", "storage2d.cuh", "measure3d_common.cuh",
           "update3d_common.cuh",
           "tc_util.cuh"]


def _newer(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _run(cmd: list[str], verbose: bool) -> str:
    if verbose:
        print(" ".join(cmd), flush=True)
    p = subprocess.run(cmd, capture_output=True, text=True)
    if p.returncode != 0:
        sys.stderr.write(p.stdout + p.stderr)
        raise RuntimeError(f"command failed ({p.returncode}): {' '.join(cmd[:3])} ...")
    return p.stdout + p.stderr


def build(force: bool = False, verbose: bool = False, ptxas_report: bool = False,
          defines: list[str] | None = None, out: Path | None = None) -> Path:
    """Compile changed sources and relink the library; returns its path.

    ``defines`` (``NAME=VALUE`` strings) and ``out`` build an alternative copy
    of the library (objects in their own folder) without touching the default
    one; such a copy is loaded by setting ``PFB_LIB`` to its path."""
    lib_path = LIB if out is None else Path(out).resolve()
    obj_dir = OBJ_DIR if out is None else lib_path.parent / (lib_path.stem + "_obj")
    defines = list(defines or [])
    if defines or out is not None:
        force = True
    lib_path.parent.mkdir(parents=True, exist_ok=True)
    obj_dir.mkdir(parents=True, exist_ok=True)
    headers = [CSRC / h for h in HEADERS] + [INCLUDE / "pfb200.h", INCLUDE / "pfb200_3d.h",
                                                 INCLUDE / "pfb200_surrogate.h",
                                                 INCLUDE / "pfb200_ckpt.h"]
    objs = []
    relink = force or not lib_path.exists()
    for src in SOURCES:
        s = CSRC / src
        o = obj_dir / (src + ".o")
        objs.append(o)
        if force or _newer(o, [s, *headers, Path(__file__)]):
            cmd = [NVCC, *ARCH, *COMMON, *(f"-D{d}" for d in defines), "-c", str(s), "-o", str(o)]
            if ptxas_report and src.endswith(".cu"):
                cmd += ["-Xptxas", "-v"]
            report = _run(cmd, verbose)
            if ptxas_report and report:
                print(report)
            relink = True
    if relink or _newer(lib_path, objs):
        tmp = lib_path.with_suffix(".so.tmp")
        _run([NVCC, *ARCH, "-shared", "-o", str(tmp), *map(str, objs), "-cudart", "static"],
             verbose)
        os.replace(tmp, lib_path)
    if out is None:
        for exe, src in CLI_SOURCES.items():
            target = lib_path.parent / exe
            s_path = CSRC / src
            if force or _newer(target, [s_path, lib_path, *headers]):
                _run([CXX, "-std=c++17", "-O2", "-Wall", "-ffp-contract=off", "-I", str(INCLUDE), str(s_path),
                      "-L", str(lib_path.parent), "-lpfb200", "-Wl,-rpath,$ORIGIN",
                      "-o", str(target)], verbose)
    return lib_path


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas", action="store_true", help="print the ptxas resource report")
    ap.add_argument("-D", dest="defines", action="append", default=[],
                    help="extra preprocessor definition NAME=VALUE (e.g. PFB_STEP2D_THREADS=256)")
    ap.add_argument("--out", default=None, help="write the library here instead")
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose, ptxas_report=a.ptxas, defines=a.defines,
                out=a.out))
