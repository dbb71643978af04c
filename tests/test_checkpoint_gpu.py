"""Checkpoint files in the reference's format (X.*.chk).

The reference's BINARY build (oracle/_ref/ztwd_harness) writes a checkpoint
of a binary after two BinaryDriver steps (Binary::write,
binary/binary.cpp:70-94); the library reads it (tree, every cell including
ghosts, time, root header) and writes it back byte for byte; and the Euler
form (no root header) round-trips through the library.
"""

import os
import subprocess

import numpy as np
import pytest

from conftest import ref_binary
from dumpio import read_dump
from test_ztwd_gpu import ztwd_config


@pytest.fixture(scope="module")
def ref_chk(tmp_path_factory, table_path):
    exe = ref_binary("ztwd")
    if exe is None:
        pytest.skip("oracle/_ref/ztwd_harness not built")
    d = str(tmp_path_factory.mktemp("chk"))
    os.symlink(table_path, os.path.join(d, "helmholtz.table"))
    env = dict(os.environ, OMP_NUM_THREADS="4")
    subprocess.run([exe, "ztwd_chk", "2", "2", "o.bin", "o.chk"], cwd=d, env=env, check=True, capture_output=True)
    return d


@pytest.mark.gpu
def test_read_reference_checkpoint_and_write_it_back(gpu, ref_chk):
    ref = read_dump(os.path.join(ref_chk, "o.bin"))
    a = gpu.AMR(**ztwd_config(2))
    hdr = a.read_checkpoint(os.path.join(ref_chk, "o.chk"), binary=True)
    t = a.get_tree()
    assert np.array_equal(t["level"], ref.level) and np.array_equal(t["loc"], ref.loc)
    assert np.array_equal(t["age"], ref.age)
    assert np.array_equal(a.download_state(), ref.U)
    assert a.get_time() == ref.time
    assert hdr.q == 0.7 and hdr.M1 == 2.4e-3 and hdr.Omega == hdr.Omega0 and hdr.Omega == ref.extra[4]
    out = os.path.join(ref_chk, "ours.chk")
    a.write_checkpoint(out, hdr, 1.0)
    with open(out, "rb") as f1, open(os.path.join(ref_chk, "o.chk"), "rb") as f2:
        assert f1.read() == f2.read()
    a.close()


@pytest.mark.gpu
def test_reference_reads_our_checkpoint(gpu, ref_chk):
    """A file written by the library after a step of its own is read by the
    reference's Binary::read to the same tree and state."""
    a = gpu.AMR(**ztwd_config(2))
    hdr = a.read_checkpoint(os.path.join(ref_chk, "o.chk"), binary=True)
    U = a.download_state()
    U[:, 7] *= 1.0 + 1e-3  # a state of our own, different from the reference's file
    a.upload_state(U)
    out = os.path.join(ref_chk, "mine.chk")
    a.write_checkpoint(out, hdr, 1.0)
    env = dict(os.environ, OMP_NUM_THREADS="4")
    subprocess.run([ref_binary("ztwd"), "read_chk", "mine.chk", "r.bin"], cwd=ref_chk, env=env, check=True,
                   capture_output=True)
    r = read_dump(os.path.join(ref_chk, "r.bin"))
    assert np.array_equal(r.level, a.get_tree()["level"])
    assert np.array_equal(r.U, U)
    a.close()


@pytest.mark.gpu
def test_euler_checkpoint_roundtrip(gpu, tmp_path):
    import importlib.util
    from conftest import PKG
    spec = importlib.util.spec_from_file_location("amr_initial", os.path.join(PKG, "initial.py"))
    initial = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(initial)
    a = gpu.AMR(max_refine_level=2, grid_dim=0.5, z_reflect=0, max_bricks=512)
    initial.build_tree(a, "bump", 3.0, 0.5, 0, 2, device=True)
    a.hydro_step(a.max_dt(), 3.0)
    path = str(tmp_path / "e.chk")
    a.write_checkpoint(path)
    b = gpu.AMR(max_refine_level=2, grid_dim=0.5, z_reflect=0, max_bricks=512)
    b.read_checkpoint(path)
    ta, tb = a.get_tree(), b.get_tree()
    for k in ("level", "loc", "age", "offset"):
        assert np.array_equal(ta[k], tb[k]), k
    assert np.array_equal(a.download_state(), b.download_state())
    assert np.array_equal(a.flow_off(), b.flow_off())
    assert a.get_time() == b.get_time()
    # a context of another ghost width rejects the file
    c = gpu.AMR(max_refine_level=2, grid_dim=0.5, z_reflect=0, max_bricks=512, bw=3)
    with pytest.raises(gpu.AmrError) as e:
        c.read_checkpoint(path)
    assert e.value.code == -6
    for x in (a, b, c):
        x.close()


@pytest.mark.gpu
def test_headless_output(gpu, tmp_path):
    """amr_write_output of a self-gravitating run: tree, interiors and the
    interior potential as the device holds them."""
    import importlib.util
    from conftest import PKG
    spec = importlib.util.spec_from_file_location("amr_initial", os.path.join(PKG, "initial.py"))
    initial = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(initial)
    a = gpu.AMR(physics=gpu.PHYSICS_EULER_GRAVITY, max_refine_level=2, grid_dim=0.5, z_reflect=0, max_bricks=512)
    initial.build_tree(a, "polytrope", 1e-6, 0.5, 0, 2, device=True)
    a.grav_step(a.max_dt(), 1e-6, 1e6, 0)
    path = str(tmp_path / "out.bin")
    a.write_output(path)
    o = gpu.read_output(path)
    t = a.get_tree()
    for k in ("level", "loc", "offset", "age", "child_mask", "h"):
        assert np.array_equal(o[k], t[k]), k
    bw = a.bw
    assert np.array_equal(o["U"], a.download_state()[:, :, bw:-bw, bw:-bw, bw:-bw])
    assert np.array_equal(o["phi"], a.download_poisson()[0][:, 1:-1, 1:-1, 1:-1])
    assert o["time"] == a.get_time()
    a.close()
