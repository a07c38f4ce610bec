"""The reference's own main loop with the GPU problem adapter
(cfd-art_b200/adapter/gpu_problem.hpp) registered in place of its CPU problem.

oracle/Makefile's `adapter` target compiles the reference's main loop,
splitting schemes, set_ICs and writers from its sources with the adapter, in
two links: against the library (ref_main_gpu_*) and against a test-only device
stub whose device calls the CPU oracle answers (ref_main_stub_*,
tests/adapter/device_stub.cpp).  The stub build must write every output file
of the reference's own run byte for byte -- which checks the adapter's call
sequence (which call takes the step, when the state is read back, where the
masses go); the library build must write them on a GPU (the mass-change log
to the rounding of its sums) and fail loudly where no GPU exists.
"""
import os
import subprocess

import pytest

from cfdtest import GOLDEN, ROOT, load_golden, masschange_close

REF = ROOT / "oracle" / "_ref"
RUNS = sorted(p.stem for p in GOLDEN.glob("outputs_*.npz")) + \
    sorted("adapter/" + p.stem for p in (GOLDEN / "adapter").glob("*.npz"))
MODELS = {"adapter/godunov_totem_pole_2_20x20": "euler",
          "adapter/strang_circular_explosion_24x20": "euler",
          "adapter/naive_ST2_x_40x6": "allaire",
          "adapter/godunov_ST1_x_30x6": "allaire"}

pytestmark = pytest.mark.skipif(not (REF / "ref_main_stub_euler").exists(),
                                reason="adapter builds absent (need the reference sources)")


def _model(run: str) -> str:
    if run in MODELS:
        return MODELS[run]
    return "euler" if run.startswith("outputs_euler") else "allaire"


def _run(binary, fx, tmp_path, threads=2):
    out = tmp_path / "out"
    out.mkdir()
    sf = tmp_path / "settingsfile.txt"
    sf.write_text(str(fx["settings"]).format(out=str(out) + "/"))
    r = subprocess.run([str(binary), str(sf)], capture_output=True, text=True, timeout=300,
                       env={**os.environ, "OMP_NUM_THREADS": str(threads)})
    files = {p.name: p.read_bytes() for p in sorted(out.iterdir())}
    return r, files


@pytest.mark.parametrize("run", RUNS)
def test_adapter_on_device_stub_writes_reference_outputs(run, tmp_path):
    fx = load_golden(run)
    r, files = _run(REF / f"ref_main_stub_{_model(run)}", fx, tmp_path)
    assert r.returncode == 0, r.stderr
    expected = {k: bytes(v) for k, v in fx.items() if k != "settings"}
    assert sorted(files) == sorted(expected)
    for name, data in expected.items():
        assert files[name] == data, name


def _has_device() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_device(), reason="checks the no-device error path")
@pytest.mark.parametrize("model", ["euler", "allaire"])
def test_adapter_on_library_fails_loudly_without_device(model, tmp_path):
    run = next(r for r in RUNS if _model(r) == model)
    r, files = _run(REF / f"ref_main_gpu_{model}", load_golden(run), tmp_path)
    assert r.returncode == 1
    assert "cfd_create failed (-2)" in r.stderr
    assert files == {}


@pytest.mark.gpu
@pytest.mark.parametrize("run", RUNS)
def test_adapter_on_library_writes_reference_outputs(run, tmp_path):
    """The reference's unmodified main loop (E/sourcecode/main.cpp:17-49,
    E/headers/simulation.hpp:36-67) driving GpuProblem on the device: every
    output file of the reference's own run, states, schlieren frames and
    lineouts byte for byte, the mass-change log to the rounding of its sums
    (the reference sums serially, the device in a tree)."""
    fx = load_golden(run)
    r, files = _run(REF / f"ref_main_gpu_{_model(run)}", fx, tmp_path)
    assert r.returncode == 0, r.stderr[-2000:]
    expected = {k: bytes(v) for k, v in fx.items() if k != "settings"}
    assert sorted(files) == sorted(expected)
    for name, data in expected.items():
        if name.endswith("-masschange.dat"):
            assert masschange_close(files[name].decode(), data.decode()), name
        else:
            assert files[name] == data, name
