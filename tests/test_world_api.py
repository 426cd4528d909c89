"""pe's World / body-creation C++ API (include/pe_b200_world.hpp) driven by a C++ program
(tests/cpp/world_driver.cpp): argument checks on the CPU, and on the GPU the same trajectories as
the Engine binding and the oracle."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from helpers import load_golden, rel_err
from oracle.pe_oracle import OracleWorld
from pe_b200 import _abi
from pe_b200.engine import Engine

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "pe_b200")


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    if not os.path.exists(os.path.join(LIBDIR, "libpe_b200.so")):
        pytest.skip("libpe_b200.so not built")
    exe = str(tmp_path_factory.mktemp("cpp") / "world_driver")
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "world_driver.cpp"), "-L", LIBDIR,
                    "-lpe_b200", "-Wl,-rpath," + LIBDIR, "-o", exe], check=True)
    return exe


def test_world_api_argument_checks(driver):
    r = subprocess.run([driver, "errors"], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == "ok"


def run_driver(driver, tmp_path, s, solver, prec, steps):
    sp, out = str(tmp_path / "scene.bin"), str(tmp_path / "out.bin")
    s.save(sp)
    r = subprocess.run([driver, "run", sp, solver, prec, str(steps), out], capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    a = np.fromfile(out, "<f8").reshape(3, s.n, 3)
    return a[0], a[1], a[2]


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["small64_boxes", "lattice512"])
def test_world_api_dem_matches_engine_and_oracle(driver, tmp_path, name):
    s = load_golden(name)["scene"]
    x, v, w = run_driver(driver, tmp_path, s, "dem", "fp64", 10)
    e = Engine(solver=_abi.DEM, precision=_abi.FP64).load_scene(s)
    e.step(s.dt, 10)
    xe, ve, we = e.download()
    e.close()
    assert np.array_equal(x, xe) and np.array_equal(v, ve) and np.array_equal(w, we)
    o = OracleWorld(s)
    o.dem_step(s.dt, 10)
    assert rel_err(x, o.x) < 1e-12
    assert rel_err(v, o.v) < 1e-10


@pytest.mark.gpu
def test_world_api_hcsits_matches_engine(driver, tmp_path):
    s = load_golden("loose125_boxes")["scene"]
    x, v, w = run_driver(driver, tmp_path, s, "hcsits", "fp64", 4)
    e = Engine(solver=_abi.HCSITS, precision=_abi.FP64, relaxation_model=1,
               max_iterations=100).load_scene(s)
    e.step(s.dt, 4)
    xe, ve, we = e.download()
    e.close()
    assert np.array_equal(x, xe) and np.array_equal(v, ve) and np.array_equal(w, we)


@pytest.mark.gpu
def test_world_api_mixed_precision_runs(driver, tmp_path):
    s = load_golden("lattice512")["scene"]
    x, v, w = run_driver(driver, tmp_path, s, "dem", "mixed", 10)
    o = OracleWorld(s)
    o.dem_step(s.dt, 10)
    assert rel_err(x, o.x) < 1e-6


def test_world_api_checkpoint_bytes_match_pe_format(driver, tmp_path):
    """BodyBinaryWriter of the C++ API writes pe's checkpoint format byte for byte (the Python
    writer is itself checked byte-identical against pe's writer in test_checkpoint.py)."""
    from pe_b200 import checkpoint as ck
    s = load_golden("small64_boxes")["scene"]
    sp, out = str(tmp_path / "s.bin"), str(tmp_path / "cpp.peb")
    s.save(sp)
    r = subprocess.run([driver, "peb_write", sp, out], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    bodies, counter = ck.scene_bodies(s)
    ref = str(tmp_path / "py.peb")
    ck.write_peb(ref, bodies, counter)
    assert open(out, "rb").read() == open(ref, "rb").read()


@pytest.mark.gpu
def test_world_api_resumes_pe_checkpoint(driver, tmp_path):
    """pe's own checkpoint after 5 steps (tests/golden/peb_small64_boxes.peb), read by the C++
    API's BodyBinaryReader and advanced 5 more steps on the GPU, lands on pe's uninterrupted
    10-step state."""
    from helpers import GOLDEN
    g = load_golden("small64_boxes")
    s = g["scene"]
    sp, out = str(tmp_path / "s.bin"), str(tmp_path / "o.bin")
    s.save(sp)
    r = subprocess.run([driver, "peb_resume", sp, os.path.join(GOLDEN, "peb_small64_boxes.peb"),
                        "5", out], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    a = np.fromfile(out, "<f8").reshape(3, s.n, 3)
    assert rel_err(a[0], g["dem10_x"]) < 1e-12
    assert rel_err(a[1], g["dem10_v"]) < 1e-10


def run_driver_boxes(driver, tmp_path, s, solver, prec, steps):
    sp, out = str(tmp_path / "scene.bin"), str(tmp_path / "out.bin")
    s.save(sp)
    r = subprocess.run([driver, "run", sp, solver, prec, str(steps), out], capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    a = np.fromfile(out, "<f8")
    n, m = s.n, s.nmbox
    sph = a[:9 * n].reshape(3, n, 3)
    b = a[9 * n:]
    return sph, b[:9 * m].reshape(3, m, 3), b[9 * m:].reshape(m, 4)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["boxes27_tumbling", "boxes36_stack"])
def test_world_api_moving_boxes_dem(driver, tmp_path, name):
    """createBox without setFixed: the box moves (BoxTrait::move) and lands on pe's state."""
    g = load_golden(name)
    s = g["scene"]
    sph, box, q = run_driver_boxes(driver, tmp_path, s, "dem", "fp64", 10)
    e = Engine(solver=_abi.DEM, precision=_abi.FP64).load_scene(s)
    e.step(s.dt, 10)
    bx, bq, bv, bw = e.download_boxes()
    e.close()
    assert np.array_equal(box[0], bx) and np.array_equal(box[1], bv) and np.array_equal(q, bq)
    assert rel_err(box[0], g["dem10_bx"]) < 1e-13
    assert rel_err(q, g["dem10_bq"]) < 1e-13


@pytest.mark.gpu
def test_world_api_moving_boxes_hcsits(driver, tmp_path):
    g = load_golden("boxes36_stack")
    s = g["scene"]
    sph, box, q = run_driver_boxes(driver, tmp_path, s, "hcsits", "fp64", 4)
    e = Engine(solver=_abi.HCSITS, precision=_abi.FP64, relaxation_model=1,
               max_iterations=100).load_scene(s)
    e.step(s.dt, 4)
    bx, bq, bv, bw = e.download_boxes()
    e.close()
    assert np.array_equal(box[0], bx) and np.array_equal(box[1], bv) and np.array_equal(q, bq)
