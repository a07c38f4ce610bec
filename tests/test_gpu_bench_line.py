"""bench.py on a small single-grid workload prints one JSON line with every
field the bench contract names (metric, value, timing, clocks, roofline of
the dominant kernel, end-to-end figure with its copied bytes, launch count)
and self-consistent numbers."""
import json
import subprocess
import sys

import pytest

from cfdtest import ROOT

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("workload", ["euler2048_mixed", "allaire2048_fast"])
def test_bench_line_fields(workload):
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--workload", workload, "--steps", "3",
                        "--warmup", "3", "--no-cpu-baseline", "--no-accuracy"],
                       cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "clocks", "roofline", "e2e",
              "gpu_launches"):
        assert k in line, k
    assert line["n_gpus"] == 1 and line["steps"] == 3 and line["warmup"] == 3
    assert line["config"]["workload"] == workload
    assert line["value"] > 0 and line["ms_per_step"] > 0 and line["gpu_launches"] > 0
    rl = line["roofline"]
    assert rl["bound"] == "hbm" and rl["unit"] == "GB/s"
    assert abs(rl["frac"] - rl["achieved"] / rl["peak"]) <= 1e-9 * rl["frac"]
    assert rl["traffic"] is None or rl["traffic"] > 0
    e2e = line["e2e"]
    assert e2e["value"] > 0 and e2e["unit"] == line["unit"]
    assert e2e["h2d_bytes_per_step"] > 0 and e2e["d2h_bytes_per_step"] > 0
    assert {"sm_mhz", "sm_max_mhz", "reasons"} <= set(line["clocks"])
