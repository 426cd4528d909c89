"""Failure detection and consistency checks: the host checks behind pe_b200_validate on planted
inconsistencies (CPU), argument and allocation failures reported as status codes, the bounded
device wait that gives up with PE_B200_ERR_TIMEOUT and leaves the context usable, and validate()
on real colourings and neighbour lists (GPU)."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from helpers import load_golden
from pe_b200 import _abi, scenes
from pe_b200.engine import Engine, PeB200Error

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_host_checks_count_planted_inconsistencies(tmp_path):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    exe = str(tmp_path / "validate_test")
    subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-Werror", "-I",
                    os.path.join(ROOT, "pe_b200", "csrc"),
                    os.path.join(ROOT, "tests", "cpp", "validate_test.cpp"), "-o", exe], check=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout + r.stderr


def test_static_step_grid_plan_coarsens_instead_of_overflowing(tmp_path):
    """The allocation-free step's grid planner (pe_b200/csrc/static_grid.h) on wide domains and
    tiny radii (e.g. +-1e6 with r = 1e-3, whose finest grid would overflow int64) and on
    domains it must refuse."""
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    exe = str(tmp_path / "static_grid_test")
    subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-Werror", "-I",
                    os.path.join(ROOT, "pe_b200", "csrc"),
                    os.path.join(ROOT, "tests", "cpp", "static_grid_test.cpp"), "-o", exe],
                   check=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout + r.stderr


def test_contact_capacity_beyond_int32_is_rejected():
    with pytest.raises(PeB200Error) as ei:
        Engine(max_contacts=2 ** 31)
    assert ei.value.code == _abi.ERR_ARG
    with pytest.raises(PeB200Error) as ei:
        Engine(max_contacts=-1)
    assert ei.value.code == _abi.ERR_ARG


def test_corrupt_scene_bytes_are_rejected():
    s = load_golden("small64_boxes")["scene"]
    b = s.to_bytes()
    assert scenes.scene_from_bytes(b).n == s.n
    for bad in (b[:-9], b + b"\0", b[:20], b"XXXXXXXX" + b[8:]):
        with pytest.raises(ValueError):
            scenes.scene_from_bytes(bad)


@pytest.mark.gpu
def test_bounded_wait_times_out_and_context_stays_usable():
    s = load_golden("lattice512")["scene"]
    ref = Engine().load_scene(s)
    ref.step(s.dt, 5)
    xr, vr, wr = ref.download()
    ref.close()
    e = Engine().load_scene(s)
    e.step(s.dt, 2)
    assert e.selftest_timeout(polls=20000) == _abi.ERR_TIMEOUT
    assert "timed out" in e.last_error()
    e.step(s.dt, 3)
    x, v, w = e.download()
    e.close()
    assert np.array_equal(x, xr) and np.array_equal(v, vr) and np.array_equal(w, wr)


@pytest.mark.gpu
def test_selftest_rejects_bad_poll_counts():
    e = Engine()
    assert e.selftest_timeout(polls=0) == _abi.ERR_ARG
    assert e.selftest_timeout(polls=2 ** 25) == _abi.ERR_ARG
    e.close()


@pytest.mark.gpu
def test_allocation_failure_is_reported_and_other_contexts_work():
    """A contact capacity far beyond device memory (about 900 GB of HCSITS buffers) makes the
    allocation fail: the step returns PE_B200_ERR_NOMEM, and a new context still steps."""
    s = load_golden("loose125_boxes")["scene"]
    e = Engine(solver=_abi.HCSITS, max_contacts=2 ** 31 - 1).load_scene(s)
    with pytest.raises(PeB200Error) as ei:
        e.step(s.dt)
    assert ei.value.code == _abi.ERR_NOMEM
    e.close()
    f = Engine(solver=_abi.HCSITS).load_scene(s)
    f.step(s.dt, 2)
    x, _, _ = f.download()
    assert np.isfinite(x).all()
    f.close()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [_abi.FP64, _abi.MIXED])
def test_validate_hcsits_colouring(precision):
    s = load_golden("dense512")["scene"]
    e = Engine(solver=_abi.HCSITS, precision=precision, max_iterations=20).load_scene(s)
    for _ in range(3):
        e.step(s.dt)
        assert e.stats()["contacts"] > 0
        assert e.validate() == 0
    e.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["lattice512", "dense512"])
def test_validate_neighbour_lists(name):
    s = load_golden(name)["scene"]
    e = Engine().load_scene(s)
    e.step(s.dt, 20)
    assert e.neighbor_list_stats()["entries"] > 0
    assert e.validate() == 0
    e.close()
