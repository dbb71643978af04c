"""The committed golden fixtures are the reference's own output.

Re-runs the reference oracle harnesses (oracle/_ref, built from the
reference sources by oracle/build_ref.py) on small golden cases and checks
that tests/golden/make_golden.py's packing of their dumps reproduces the
committed .npz files bit for bit.  Skipped where oracle/_ref is not built.
"""

import importlib.util
import os
import tempfile

import numpy as np
import pytest

from conftest import GOLDEN, ref_binary

spec = importlib.util.spec_from_file_location("make_golden", os.path.join(GOLDEN, "make_golden.py"))
make_golden = importlib.util.module_from_spec(spec)
spec.loader.exec_module(make_golden)


@pytest.mark.parametrize("name", ["hydro_bump_L2", "hydro_ppm_bump_L2", "grav_poly_L2", "ztwd_L2", "ztwd12_L2"])
def test_golden_is_reference_output(name, table_path):
    variant = make_golden.CASES[name][0]
    if ref_binary(variant) is None:
        pytest.skip("oracle/_ref/%s_harness not built" % variant)
    with tempfile.TemporaryDirectory() as td:
        if variant in ("ztwd", "ztwd12"):
            os.symlink(table_path, os.path.join(td, "helmholtz.table"))
        res = make_golden.run_case(name, td)
    g = np.load(os.path.join(GOLDEN, name + ".npz"))
    assert sorted(res) == sorted(g.files)
    for k in g.files:
        a, b = np.asarray(res[k]), g[k]
        assert a.shape == b.shape and a.dtype == b.dtype, k
        assert np.array_equal(a, b), k
