"""The headers are plain C: a C99 program (tests/abi/c_consumer.c) compiles
against include/*.h with -pedantic -Werror, links libcfdgpu.so, builds a
configuration and an initial condition through the host hooks, and gets
CFD_ERR_CUDA with a message from cfd_create where no GPU exists."""
import shutil
import subprocess

import pytest

from cfdtest import ROOT

LIBDIR = ROOT / "cfd-art_b200" / "lib"

pytestmark = pytest.mark.skipif(not (LIBDIR / "libcfdgpu.so").exists() or not shutil.which("gcc"),
                                reason="libcfdgpu.so or gcc absent")


def _has_device() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


def test_c99_consumer(tmp_path):
    exe = tmp_path / "c_consumer"
    subprocess.run(["gcc", "-std=c99", "-pedantic", "-Wall", "-Wextra", "-Werror",
                    f"-I{ROOT / 'include'}", "-o", str(exe), str(ROOT / "tests" / "abi" / "c_consumer.c"),
                    f"-L{LIBDIR}", "-lcfdgpu", f"-Wl,-rpath,{LIBDIR}"], check=True, timeout=120)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60, check=True).stdout
    lines = dict(line.split(" ", 1) for line in out.splitlines())
    assert lines["recipe_config"] == "0 nx 32 ny 24"
    assert lines["grid_elems"] == f"0 {(32 + 4) * (24 + 4) * 4}"
    assert lines["recipe_ic"] == "0 first_rho 0.13800000000000001"  # lower-left quadrant
    if _has_device():
        assert lines["create"].startswith("0") and lines["upload"] == "0"
    else:
        assert lines["create"] == "-2 no CUDA device available"
