"""The CPU legs of bench.py, which need no GPU: the reference arm's JSON line,
the cpu_baseline record (all-threads and one-thread runs of the reference's
own code, oracle/_ref) on tiny budgets, and the density error measures the
served line reports."""
import json
import re
import subprocess
import sys

import pytest

import oracle_py as O
from cfdtest import ROOT

pytestmark = pytest.mark.skipif(not (O.ref_available("euler") and O.ref_available("allaire")),
                                reason="oracle/_ref (reference build) not built")


def test_cpu_baseline_record():
    sys.path.insert(0, str(ROOT))
    import bench

    r = bench.cpu_baseline("served", budget_s=0.5, single_thread_s=0.3)
    assert r["kind"] == "reference" and r["unit"] == bench.UNIT
    assert r["value"] > 0 and r["cores"] >= 1 and r["cpu_model"]
    assert "requests of the served workload" in r["sample"]
    st = r["single_thread"]
    assert st["cores"] == 1 and st["value"] > 0
    assert "1/4 size per side" in st["sample"]


def _reference_arm(workload, steps, warmup):
    """bench.py --impl reference in a fresh process; returns its JSON line and
    whether the shipped library was mapped into that process."""
    code = ("import sys, json; sys.argv = ['bench.py', '--impl', 'reference', '--workload', "
            f"'{workload}', '--steps', '{steps}', '--warmup', '{warmup}']; "
            f"sys.path.insert(0, {str(ROOT)!r}); import bench; bench.main(); "
            "print('LIBCFDGPU', 'libcfdgpu' in open('/proc/self/maps').read())")
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True,
                         timeout=600, check=True, cwd=ROOT)
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    mapped = [ln for ln in out.stdout.splitlines() if ln.startswith("LIBCFDGPU")]
    return json.loads(lines[0]), mapped == ["LIBCFDGPU True"]


@pytest.mark.parametrize("workload,unit", [("allaire2048", "one time step"),
                                           ("served", "one request")])
def test_reference_arm_line(workload, unit):
    r, lib_loaded = _reference_arm(workload, 2, 1)
    assert not lib_loaded, "the reference arm must not load the shipped library"
    assert r["impl"] == "reference" and r["steps"] == 2 and r["warmup"] == 1
    assert r["config"]["workload"] == workload and r["config"]["step"] == unit
    assert r["value"] > 0 and r["higher_is_better"] is True
    assert r["e2e"]["value"] == r["value"]
    assert r["e2e"]["h2d_bytes_per_step"] == 0 and r["e2e"]["d2h_bytes_per_step"] == 0
    assert r["cpu_baseline"]["value"] == r["value"] and r["cpu_baseline"]["cores"] >= 1
    # steps x ms_per_step is the timed loop time the sample states
    secs = float(re.search(r"\(([0-9.]+) s\)", r["config"]["sample"]).group(1))
    assert abs(r["ms_per_step"] * r["steps"] / 1e3 - secs) <= 0.05 + 0.01 * secs


def test_gpus_flag_must_match_world_size():
    out = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference",
                          "--gpus", "2"], capture_output=True, text=True, timeout=60, cwd=ROOT,
                         env={**__import__("os").environ, "WORLD_SIZE": "1", "RANK": "0"})
    assert out.returncode != 0 and "WORLD_SIZE=1" in out.stderr


def test_density_error_measures():
    sys.path.insert(0, str(ROOT))
    import numpy as np

    import bench

    rng = np.random.default_rng(3)
    for model, nv in ((0, 4), (1, 6)):
        ref = rng.uniform(0.5, 2.0, size=(12, 10, nv))
        got = ref.copy()
        assert bench._rel_l1_density(got, ref, model) == 0.0
        assert bench._rel_linf_density(got, ref, model) == 0.0
        got[5, 4, 0] += 1e-3  # one interior cell; ghost cells (first/last two) never count
        got[0, 0, 0] += 1.0
        rho = ref[2:-2, 2:-2, 0] if model == 0 else ref[2:-2, 2:-2, 0] + ref[2:-2, 2:-2, 1]
        assert np.isclose(bench._rel_l1_density(got, ref, model), 1e-3 / np.abs(rho).sum())
        assert np.isclose(bench._rel_linf_density(got, ref, model), 1e-3 / np.abs(rho).max())
