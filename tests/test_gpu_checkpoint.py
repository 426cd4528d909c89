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
