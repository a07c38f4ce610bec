"""Build step of the cfdgpu library (in-tree, sm_100a).

    python cfd-art_b200/build.py          # incremental
    python cfd-art_b200/build.py --force  # rebuild everything

Produces cfd-art_b200/lib/libcfdgpu.so (CUDA kernels + C ABI + host hooks,
CUDA runtime linked statically) and cfd-art_b200/lib/run-cfd-simulation (the
drop-in driver reading a reference settingsfile.txt).

The plain-FP64 translation units are compiled with --fmad=false: the
reference's x86-64 build never contracts a multiply-add, and bit-identical
results need the same rounding at every operation.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
LIB = PKG / "lib"
OBJ = LIB / "obj"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
CXX = "/usr/bin/g++"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
INC = [f"-I{ROOT / 'include'}", f"-I{PKG / 'csrc'}"]

# (source, extra flags)
CUDA_SOURCES = [
    ("csrc/cfd_api.cu", ["--fmad=false"]),
    ("csrc/cfd_noalloc.cu", ["--fmad=false"]),
    ("csrc/cfd_ic.cu", ["--fmad=false"]),
    # mixed precision: FP32 with contraction and flush-to-zero
    ("csrc/cfd_batch.cu", ["-ftz=true", "-prec-div=false", "-prec-sqrt=false"]),
]
HOST_SOURCES = ["host/ic.cpp", "host/io.cpp", "host/server.cpp"]
DRIVER = "host/driver.cpp"


def _newer(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return False
    t = target.stat().st_mtime
    return all(d.stat().st_mtime <= t for d in deps)


def _headers() -> list[Path]:
    return (sorted((PKG / "csrc").glob("*.cuh")) + sorted((PKG / "csrc").glob("*.h")) +
            sorted((ROOT / "include").glob("*.h")))


def _run(cmd: list[str], verbose: bool) -> None:
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build(force: bool = False, verbose: bool = False) -> Path:
    LIB.mkdir(parents=True, exist_ok=True)
    OBJ.mkdir(parents=True, exist_ok=True)
    hdrs = _headers()
    objs: list[Path] = []
    for src, extra in CUDA_SOURCES:
        s = PKG / src
        o = OBJ / (Path(src).stem + ".o")
        if force or not _newer(o, [s, *hdrs]):
            _run([NVCC, *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC",
                  "-Xcompiler", "-ffp-contract=off", *extra, *INC, "-c", str(s), "-o", str(o)],
                 verbose)
        objs.append(o)
    for src in HOST_SOURCES:
        s = PKG / src
        o = OBJ / (Path(src).stem + ".o")
        if force or not _newer(o, [s, *hdrs]):
            _run([CXX, "-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-Wall", *INC,
                  "-I/usr/local/cuda/include", "-pthread", "-c", str(s), "-o", str(o)], verbose)
        objs.append(o)
    so = LIB / "libcfdgpu.so"
    if force or not _newer(so, objs):
        _run([NVCC, *ARCH, "-shared", "-Xcompiler", "-pthread", "-o", str(so), *map(str, objs)],
             verbose)
    drv = PKG / DRIVER
    exe = LIB / "run-cfd-simulation"
    if drv.exists() and (force or not _newer(exe, [drv, so, *hdrs])):
        _run([CXX, "-O2", "-std=c++17", "-ffp-contract=off", *INC, str(drv), "-o", str(exe),
              f"-L{LIB}", "-lcfdgpu", f"-Wl,-rpath,$ORIGIN"], verbose)
    return so


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
