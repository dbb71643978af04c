import importlib.util
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "3d-eulerian-amr_b200")
ORACLE = os.path.join(ROOT, "oracle")
GOLDEN = os.path.join(ROOT, "tests", "golden")
REF_BIN = os.path.join(ORACLE, "_ref")

sys.path.insert(0, ORACLE)
sys.path.insert(0, os.path.join(ROOT, "tests"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built library")


def load_amr():
    spec = importlib.util.spec_from_file_location("amr_b200", os.path.join(PKG, "amr.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def gpu_available():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def amr_mod():
    return load_amr()


@pytest.fixture(scope="session")
def gpu(amr_mod):
    if not gpu_available():
        pytest.fail("GPU test run without a CUDA device")
    return amr_mod


def _load_pkg_module(name, fname):
    spec = importlib.util.spec_from_file_location(name, os.path.join(PKG, fname))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


@pytest.fixture(scope="session")
def table_path(tmp_path_factory):
    """The synthetic Helmholtz table (3d-eulerian-amr_b200/helm_table.py),
    written once per session."""
    helm_table = _load_pkg_module("helm_table", "helm_table.py")
    return helm_table.ensure_table(str(tmp_path_factory.mktemp("helm")))


def ref_binary(variant="g05"):
    p = os.path.join(REF_BIN, variant + "_harness")
    return p if os.path.exists(p) else None


def run_ref(args, workdir, variant="g05", threads=1, timeout=600):
    """Run the reference oracle harness (oracle/_ref) in workdir."""
    exe = ref_binary(variant)
    if exe is None:
        pytest.skip("reference oracle binary not built (oracle/build_ref.py)")
    env = dict(os.environ, OMP_NUM_THREADS=str(threads))
    r = subprocess.run([exe] + [str(a) for a in args], cwd=workdir, env=env, capture_output=True, text=True,
                       timeout=timeout)
    assert r.returncode == 0, r.stdout + r.stderr
    return r.stdout
