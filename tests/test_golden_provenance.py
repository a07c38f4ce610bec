"""The committed golden fixtures are what tests/golden/make_golden.py makes
from the reference's own build: regenerated into a scratch directory, every
array of every fixture is identical.  Runs where the reference build
(oracle/_ref) exists."""
import subprocess
import sys

import numpy as np
import pytest

import oracle_py as O
from cfdtest import GOLDEN

pytestmark = pytest.mark.skipif(not (O.ref_available("euler") and O.ref_available("allaire")),
                                reason="reference build absent")


def test_fixtures_regenerate_identically(tmp_path):
    subprocess.run([sys.executable, str(GOLDEN / "make_golden.py"), "--out", str(tmp_path)],
                   check=True, stdout=subprocess.DEVNULL, timeout=900)
    committed = sorted(GOLDEN.glob("*.npz")) + sorted((GOLDEN / "adapter").glob("*.npz"))
    assert committed
    for f in committed:
        g = tmp_path / f.relative_to(GOLDEN)
        assert g.exists(), f.name
        with np.load(f) as a, np.load(g) as b:
            assert sorted(a.files) == sorted(b.files), f.name
            for k in a.files:
                assert np.array_equal(a[k], b[k]), (f.name, k)
