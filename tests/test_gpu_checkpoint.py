"""Checkpoint and restart of the GPU step through pe's checkpoint format."""
import numpy as np
import pytest

from helpers import load_golden, rel_err
from pe_b200 import _abi, checkpoint as ck
from pe_b200.engine import Engine

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("lists", [False, True])
def test_restart_from_checkpoint_continues_the_run(tmp_path, lists):
    s = load_golden("small64_boxes")["scene"]
    e = Engine(solver=_abi.DEM, precision=_abi.FP64, neighbor_lists=lists).load_scene(s)
    e.step(s.dt, 5)
    x, v, w = e.download()
    e.step(s.dt, 5)
    ref = e.download()
    e.close()
    path = str(tmp_path / "c.peb")
    bodies, counter = ck.scene_bodies(s, x=x, v=v, w=w)
    ck.write_peb(path, bodies, counter)
    r = ck.restore_scene(path, s)
    e = Engine(solver=_abi.DEM, precision=_abi.FP64, neighbor_lists=lists).load_scene(r)
    e.step(s.dt, 5)
    out = e.download()
    e.close()
    if not lists:
        # the grid form does not depend on the history: the restart is exact
        for a, b in zip(out, ref):
            assert np.array_equal(a, b)
    else:
        # lists rebuilt at the restart sum in another order
        assert rel_err(out[0], ref[0]) < 1e-13 and rel_err(out[1], ref[1]) < 1e-10


def test_gpu_resumes_pe_box_checkpoint():
    """pe's own checkpoint of the tumbling-box scene after 5 DEM steps, restored and advanced 5
    more steps on the GPU, lands on pe's uninterrupted 10-step state (spheres and boxes)."""
    from helpers import GOLDEN
    import os
    g = load_golden("boxes27_tumbling")
    r = ck.restore_scene(os.path.join(GOLDEN, "peb_boxes27.peb"), g["scene"])
    e = Engine(solver=_abi.DEM, precision=_abi.FP64).load_scene(r)
    e.step(r.dt, 5)
    bx, bq, bv, bw = e.download_boxes()
    x, v, w = e.download()
    e.close()
    assert rel_err(bx, g["dem10_bx"]) < 1e-13
    assert rel_err(bq, g["dem10_bq"]) < 1e-13
    assert rel_err(bv, g["dem10_bv"]) < 1e-11
    assert rel_err(x, g["dem10_x"]) < 1e-13


def test_box_restart_is_exact(tmp_path):
    """Checkpoint the GPU's box scene after 5 steps and restart: the grid step does not depend
    on the history, so the restart equals the uninterrupted run bit for bit."""
    g = load_golden("boxes27_tumbling")
    s = g["scene"]
    e = Engine(solver=_abi.DEM, precision=_abi.FP64).load_scene(s)
    e.step(s.dt, 5)
    x, v, w = e.download()
    state = e.download_boxes()
    e.step(s.dt, 5)
    ref = e.download_boxes()
    e.close()
    path = str(tmp_path / "b.peb")
    bx, bq, bv, bw = state
    bodies, counter = ck.scene_bodies(s, x=x, v=v, w=w, box_state=(bx, bq, bv, bw))
    ck.write_peb(path, bodies, counter)
    r = ck.restore_scene(path, s)
    e = Engine(solver=_abi.DEM, precision=_abi.FP64).load_scene(r)
    e.step(s.dt, 5)
    out = e.download_boxes()
    e.close()
    for a, b in zip(out, ref):
        assert np.array_equal(a, b)
