"""Edge cases of the sphere steps on the GPU against the oracle: no bodies at all, one body,
body counts that leave partial warps, blocks and list tiles, and spheres with exactly as many
list neighbours as the rebuild keeps from its counting pass (8) and one more."""
import numpy as np
import pytest

from helpers import rel_err
from oracle.pe_oracle import OracleWorld
from pe_b200 import _abi, scenes
from pe_b200.engine import Engine

pytestmark = pytest.mark.gpu

MAT = [scenes.material(1.0, 1e5, 50.0, 40.0, 0.3)]


def scene_of(x, v, r, name, dt=1e-4):
    x = np.asarray(x, float).reshape(-1, 3)
    n = len(x)
    return scenes._scene(x, np.asarray(v, float).reshape(-1, 3), np.asarray(r, float), np.zeros(n, np.int64),
                         scenes.box_planes([0, 0, 0], [8, 8, 8]), np.zeros(6, np.int64),
                         np.zeros((0, 15)), np.zeros(0), MAT, (0.0, 0.0, -9.81), dt, 100, name)


@pytest.mark.parametrize("solver,lists", [(_abi.DEM, True), (_abi.DEM, False), (_abi.HCSITS, False)])
def test_no_bodies(solver, lists):
    s = scene_of(np.zeros((0, 3)), np.zeros((0, 3)), np.zeros(0), "empty")
    e = Engine(solver=solver, precision=_abi.FP64, neighbor_lists=lists).load_scene(s)
    e.step(s.dt, 5)
    x, v, w = e.download()
    e.close()
    assert x.shape == (0, 3) and v.shape == (0, 3) and w.shape == (0, 3)


@pytest.mark.parametrize("precision", [_abi.FP64, _abi.MIXED])
@pytest.mark.parametrize("form", [0, 2])
def test_one_sphere_falls_onto_the_floor(precision, form):
    s = scene_of([[4.0, 4.0, 0.52]], [[0.3, 0.0, -1.0]], [0.5], "one")
    e = Engine(solver=_abi.DEM, precision=precision).load_scene(s)
    e.set_tuning(0, 0, 0.0, dem_split=form)
    e.step(s.dt, 600)
    x, v, _ = e.download()
    e.close()
    o = OracleWorld(s)
    o.dem_step(s.dt, 600)
    assert o.v[0, 2] > -0.5   # the floor stopped the fall
    tol = 1e-12 if precision == _abi.FP64 else 1e-5
    assert rel_err(x, o.x) < tol and rel_err(v, o.v) < (1e-10 if precision == _abi.FP64 else 1e-3)


@pytest.mark.parametrize("n", [2, 31, 33, 127, 129, 257, 1001])
@pytest.mark.parametrize("form", [0, 2])
def test_partial_warps_blocks_and_tiles(n, form):
    s = scenes.small_random(100 + n, n=n, overlap=0.03)
    e = Engine(solver=_abi.DEM, precision=_abi.FP64).load_scene(s)
    e.set_tuning(0, 0, 0.0, dem_split=form)
    e.step(s.dt, 30)
    x, v, _ = e.download()
    e.close()
    o = OracleWorld(s)
    o.dem_step(s.dt, 30)
    assert rel_err(x, o.x) < 1e-12 and rel_err(v, o.v) < 1e-9


@pytest.mark.parametrize("k", [8, 9])
def test_spheres_with_as_many_neighbours_as_kept_and_one_more(k):
    """A centre sphere with k neighbours 0.005 outside contact, spread over a sphere around it
    so that they are not each other's neighbours (and two lone spheres elsewhere): the rebuild
    copies the kept neighbours for k = 8 and searches again for k = 9; the lists are consistent
    and the steps match the oracle."""
    c = np.array([4.0, 4.0, 4.0])
    i = np.arange(k) + 0.5
    phi, th = np.arccos(1 - 2 * i / k), np.pi * (1 + 5 ** 0.5) * i
    u = np.stack([np.cos(th) * np.sin(phi), np.sin(th) * np.sin(phi), np.cos(phi)], 1)
    pts = c + 1.005 * u
    gaps = np.linalg.norm(pts[:, None] - pts[None], axis=-1) + 9 * np.eye(k)
    assert gaps.min() > 1.03
    x = np.concatenate([[c], pts, [[1.0, 1.0, 1.0], [7.0, 7.0, 7.0]]])
    v = np.zeros_like(x)
    v[0] = [0.02, -0.01, 0.03]
    s = scene_of(x, v, np.full(len(x), 0.5), f"star{k}")
    s.gravity = np.zeros(3)
    e = Engine(solver=_abi.DEM, precision=_abi.FP64, skin=0.02).load_scene(s)
    e.step(s.dt, 200)
    st = e.neighbor_list_stats()
    assert e.validate() == 0
    x1, v1, _ = e.download()
    e.close()
    assert st["entries"] == 2 * k
    o = OracleWorld(s)
    o.dem_step(s.dt, 200)
    assert rel_err(x1, o.x) < 1e-12 and rel_err(v1, o.v) < 1e-9
