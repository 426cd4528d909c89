"""DEM step on the GPU against the oracle (CPU restatement pinned to the compiled reference)
and the reference's own golden vectors."""
import numpy as np
import pytest

from helpers import GOLDEN_NAMES, load_golden, pair_set, rel_err, rel_err_w
from oracle.pe_oracle import OracleWorld
from pe_b200 import _abi, scenes
from pe_b200.engine import Engine, PeB200Error

pytestmark = pytest.mark.gpu


def engine_for(scene, precision=_abi.FP64, track_q=False, solver=_abi.DEM, **kw):
    e = Engine(solver=solver, precision=precision, track_orientation=track_q, **kw)
    return e.load_scene(scene)


@pytest.mark.parametrize("name", GOLDEN_NAMES)
def test_pair_set_bit_exact_vs_reference(name):
    g = load_golden(name)
    e = engine_for(g["scene"])
    ids, geom = e.contacts()
    ref = g["pairs"]
    assert pair_set(ids) == pair_set(np.stack([ref["b1"], ref["b2"]], 1))
    order = np.lexsort((ref["b2"], ref["b1"]))
    r = ref[order]
    if len(r):
        assert rel_err(geom[:, 0:3], r["gpos"]) < 1e-14
        assert rel_err(geom[:, 3:6], r["n"]) < 1e-14
        assert np.abs(geom[:, 6] - r["dist"]).max() < 1e-14


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_pair_set_random_scenes_vs_oracle(seed):
    s = scenes.small_random(20 + seed, n=1000, overlap=0.02, with_boxes=bool(seed % 2))
    e = engine_for(s)
    ids, _ = e.contacts()
    assert pair_set(ids) == pair_set(OracleWorld(s).pairs())


@pytest.mark.parametrize("name", GOLDEN_NAMES)
def test_dem_fp64_matches_reference(name):
    """One and several DEM steps agree with pe's FP64 step to 1e-12 relative."""
    g = load_golden(name)
    s = g["scene"]
    for key in sorted(k for k in g if k.startswith("dem") and k.endswith("_x")):
        k = int(key[3:-2])
        e = engine_for(s, track_q=True)
        e.step(s.dt, k)
        x, v, w, q = e.download()
        tol = 1e-12 if k <= 10 else 1e-10
        assert rel_err(x, g[f"dem{k}_x"]) < tol, (k, rel_err(x, g[f"dem{k}_x"]))
        assert rel_err(v, g[f"dem{k}_v"]) < tol, (k, rel_err(v, g[f"dem{k}_v"]))
        ew = rel_err_w(w, g[f"dem{k}_w"], g[f"dem{k}_v"], s.r)
        assert ew < tol, (k, ew)
        assert rel_err(q, g[f"dem{k}_q"]) < tol


def test_dem_lattice4096_vs_oracle():
    s = scenes.dem_lattice(0)
    o = OracleWorld(s)
    e = engine_for(s)
    for k in range(3):
        o.dem_step(s.dt, 10)
        e.step(s.dt, 10)
        x, v, w = e.download()
        assert rel_err(x, o.x) < 1e-12
        assert rel_err(v, o.v) < 1e-10
        assert rel_err_w(w, o.w, o.v, s.r) < 1e-10


def test_dem_deterministic_runs():
    s = scenes.small_random(7, n=2000, overlap=0.03)
    a = engine_for(s)
    b = engine_for(s)
    a.step(s.dt, 20)
    b.step(s.dt, 20)
    for u, w in zip(a.download(), b.download()):
        assert np.array_equal(u, w)


def test_dem_mixed_precision_error_bound():
    """FP32 contact forces and velocities (with their extension bytes) and FP64 positions stay
    within 1e-6 of the FP64 oracle relative to the largest displacement, on a scene where every
    sphere is in contact."""
    s = scenes.small_random(8, n=4000, overlap=0.03)
    o = OracleWorld(s)
    o.dem_step(s.dt, 200)
    e = engine_for(s, precision=_abi.MIXED)
    e.step(s.dt, 200)
    x, v, w = e.download()
    assert rel_err(x - s.x, o.x - s.x) < 1e-6
    assert rel_err(x, o.x) < 1e-7
    assert rel_err(v, o.v) < 1e-5


def test_batched_scenes_equal_single_runs():
    ss = [scenes.small_random(30 + k, n=200 + 50 * k, overlap=0.03, with_boxes=bool(k % 2))
          for k in range(4)]
    eb = Engine(solver=_abi.DEM).load_scenes(ss)
    eb.step(ss[0].dt, 5)
    xb, vb, wb = eb.download()
    off = 0
    for s in ss:
        e = engine_for(s)
        e.step(s.dt, 5)
        x, v, w = e.download()
        assert np.array_equal(x, xb[off:off + s.n])
        assert np.array_equal(v, vb[off:off + s.n])
        off += s.n


def test_invalid_arguments_are_rejected():
    s = scenes.small_random(1, n=27)
    e = engine_for(s)
    with pytest.raises(PeB200Error) as ei:
        e.step(0.0)
    assert ei.value.code == _abi.ERR_ARG
    with pytest.raises(PeB200Error) as ei:
        e.step(-1e-3)
    assert ei.value.code == _abi.ERR_ARG
    e2 = Engine()
    with pytest.raises(PeB200Error) as ei:
        e2.step(1e-3)
    assert ei.value.code == _abi.ERR_STATE
    bad = s.materials.copy()
    bad[0, 0] = -1.0
    with pytest.raises(PeB200Error):
        e2.set_materials(bad)
    with pytest.raises(PeB200Error):
        e2.set_materials(s.materials)
        e2.upload(s.x, s.v, s.w, -s.r, s.mat)


def test_nan_state_is_reported():
    s = scenes.small_random(1, n=27)
    e = engine_for(s)
    x = s.x.copy()
    x[0, 0] = np.nan
    e.set_state(x=x)
    e.step(s.dt)
    with pytest.raises(PeB200Error) as ei:
        e.download()
    assert ei.value.code == _abi.ERR_NAN


@pytest.mark.parametrize("precision", [_abi.FP64, _abi.MIXED])
def test_neighbor_lists_match_grid_search(precision):
    """Verlet lists (rebuilt whenever a sphere has moved skin/2) give the grid search's forces;
    a tiny skin forces a rebuild nearly every step, a large one almost never."""
    s = scenes.small_random(9, n=3000, overlap=0.03, with_boxes=True)
    g = Engine(solver=_abi.DEM, precision=precision, neighbor_lists=False).load_scene(s)
    g.step(s.dt, 60)
    xg, vg, wg = g.download()
    for skin in (1e-4, 0.05, 0.5):
        e = Engine(solver=_abi.DEM, precision=precision, neighbor_lists=True, skin=skin)
        e.load_scene(s)
        for _ in range(3):
            e.step(s.dt, 20)
        x, v, w = e.download()
        tol = 1e-12 if precision == _abi.FP64 else 1e-5
        assert rel_err(x, xg) < tol
        assert rel_err(v, vg) < (tol if precision == _abi.FP64 else 1e-3)


def test_neighbor_lists_vs_oracle_long_run():
    s = scenes.dem_lattice(1, side=10)
    o = OracleWorld(s)
    o.dem_step(s.dt, 300)
    e = engine_for(s)
    e.step(s.dt, 300)
    x, v, w = e.download()
    assert rel_err(x, o.x) < 1e-12
    assert rel_err(v, o.v) < 1e-9
