"""The drop-in driver (run-cfd-simulation) on a reference settings file writes
the same output files as the reference's own main() on that file: states,
schlieren frames (ghost cells included in their edge stencils) and Allaire
lineouts byte for byte; the mass-change log to the rounding of its sums
(the reference sums serially, the GPU in a tree).  The reference outputs are
committed fixtures made by tests/golden/make_golden.py."""
import os
import subprocess

import numpy as np
import pytest

from cfdtest import GOLDEN, ROOT, masschange_close

pytestmark = pytest.mark.gpu
DRIVER = ROOT / "cfd-art_b200" / "lib" / "run-cfd-simulation"
RUNS = sorted(p.stem for p in GOLDEN.glob("outputs_*.npz"))


@pytest.mark.parametrize("run", RUNS)
def test_driver_outputs_match_reference(tmp_path, run):
    with np.load(GOLDEN / f"{run}.npz", allow_pickle=False) as z:
        fx = {k: z[k] for k in z.files}
    out = tmp_path / "out"
    out.mkdir()
    sf = tmp_path / "settingsfile.txt"
    sf.write_text(str(fx.pop("settings")).format(out=str(out) + "/"))
    r = subprocess.run([str(DRIVER), str(sf)], capture_output=True, text=True, timeout=600,
                       cwd=tmp_path)
    assert r.returncode == 0, r.stderr[-2000:]
    assert sorted(os.listdir(out)) == sorted(fx)
    for name, ref in fx.items():
        data = (out / name).read_bytes()
        if name.endswith("-masschange.dat"):
            assert masschange_close(data.decode(), ref.tobytes().decode()), name
        else:
            assert data == ref.tobytes(), name
