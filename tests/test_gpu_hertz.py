"""pe's extended Hertz normal law (force_model 1) on the GPU against the compiled reference's
golden vectors (pe built with forceModel = hertz) and the oracle."""
import numpy as np
import pytest

from helpers import load_golden, rel_err, rel_err_w
from oracle.pe_oracle import OracleWorld
from pe_b200 import _abi, scenes
from pe_b200.engine import Engine

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["hertz64_boxes", "hertz64_planes"])
@pytest.mark.parametrize("lists", [False, True])
def test_hertz_fp64_matches_reference(name, lists):
    g = load_golden(name)
    s = g["scene"]
    for k in (1, 10):
        e = Engine(solver=_abi.DEM, precision=_abi.FP64, force_model=1,
                   neighbor_lists=lists).load_scene(s)
        e.step(s.dt, k)
        x, v, w = e.download()
        e.close()
        assert rel_err(x, g[f"dem{k}_x"]) < 1e-12
        assert rel_err(v, g[f"dem{k}_v"]) < 1e-10
        assert rel_err_w(w, g[f"dem{k}_w"], g[f"dem{k}_v"], s.r) < 1e-10


def test_hertz_mixed_close_to_fp64():
    s = load_golden("hertz64_planes")["scene"]
    out = []
    for prec in (_abi.FP64, _abi.MIXED):
        e = Engine(solver=_abi.DEM, precision=prec, force_model=1).load_scene(s)
        e.step(s.dt, 50)
        out.append(e.download()[0])
        e.close()
    assert rel_err(out[1], out[0]) < 1e-6


def test_hertz_lattice_against_oracle():
    s = scenes.dem_lattice(0, side=8)
    s.materials[:, 5] = 1e7     # Young's modulus
    e = Engine(solver=_abi.DEM, precision=_abi.FP64, force_model=1).load_scene(s)
    e.step(s.dt, 20)
    x, v, _ = e.download()
    e.close()
    o = OracleWorld(s, force_model=1)
    o.dem_step(s.dt, 20)
    assert rel_err(x, o.x) < 1e-12 and rel_err(v, o.v) < 1e-9


def test_adjoint_rejects_hertz():
    s = load_golden("hertz64_planes")["scene"]
    e = Engine(solver=_abi.DEM, precision=_abi.FP64, force_model=1).load_scene(s)
    with pytest.raises(_abi.PeB200Error):
        e.adjoint_forward(5, s.dt, 5)
    e.close()
