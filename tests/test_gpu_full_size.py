"""The benchmark workloads at their full sizes, where the oracle would take hours, checked
through properties that do not depend on size: repeated runs are bit-identical, the mixed
precision form stays within the stated 1e-6 of the FP64 form, the list step follows the FP64
grid step, every step of a 32k hard-contact scene has a race-free colouring, and scenes of the
512-scene ensemble step in the batch exactly as they do alone."""
import numpy as np
import pytest

from helpers import rel_err
from pe_b200 import _abi, scenes
from pe_b200.engine import Engine

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def large():
    return scenes.dem_large(0)


def run(s, steps, **kw):
    e = Engine(solver=_abi.DEM, **kw).load_scene(s)
    e.step(s.dt, steps)
    out = e.download()
    e.close()
    return out


def test_1m_runs_are_bit_identical(large):
    a = run(large, 60, precision=_abi.MIXED)
    b = run(large, 60, precision=_abi.MIXED)
    for u, w in zip(a, b):
        assert np.array_equal(u, w)


def test_1m_mixed_within_stated_error_of_fp64(large):
    """The stated error of the mixed-precision form: after 1000 steps of the 1M scene, every
    sphere's position is within 1e-6 of the FP64 run's, relative to the largest displacement
    (max |x_mixed - x_fp64| / max |x_fp64 - x_0|), and so is the RMS over spheres."""
    xm, _, _ = run(large, 1000, precision=_abi.MIXED)
    xd, _, _ = run(large, 1000, precision=_abi.FP64)
    d, disp = np.abs(xm - xd), np.abs(xd - large.x)
    assert d.max() / disp.max() < 1e-6
    assert np.sqrt((d ** 2).sum() / (disp ** 2).sum()) < 1e-6
    assert rel_err(xm, xd) < 1e-9


def test_1m_lists_follow_the_grid_step(large):
    xl, vl, _ = run(large, 100, precision=_abi.FP64)
    xg, vg, _ = run(large, 100, precision=_abi.FP64, neighbor_lists=False)
    assert rel_err(xl, xg) < 1e-12 and rel_err(vl, vg) < 1e-9


def test_32k_dense_hard_contacts_colour_race_free():
    s = scenes.nbgs_box(0, n=32768, dims=(32.0, 32.0, 120.0), dense=True)
    for precision in (_abi.MIXED, _abi.FP64):
        e = Engine(solver=_abi.HCSITS, precision=precision).load_scene(s)
        for _ in range(3):
            e.step(s.dt)
            assert e.stats()["contacts"] > 10000
            assert e.validate() == 0
        x, v, w = e.download()
        e.close()
        assert np.isfinite(x).all() and np.isfinite(v).all() and np.isfinite(w).all()


def test_ensemble_512_scenes_step_as_alone():
    ens = scenes.batched_ensemble(0)
    dt = ens[0].dt
    # one skin for the batch and the single runs (the default follows the smallest radius)
    eb = Engine(solver=_abi.DEM, precision=_abi.MIXED, skin=0.05).load_scenes(ens)
    eb.step(dt, 20)
    xb, vb, _ = eb.download()
    eb.close()
    offs = np.concatenate([[0], np.cumsum([s.n for s in ens])])
    for k in (0, 211, 511):
        s = ens[k]
        x, v, _ = run(s, 20, precision=_abi.MIXED, skin=0.05)
        assert np.array_equal(x, xb[offs[k]:offs[k + 1]])
        assert np.array_equal(v, vb[offs[k]:offs[k + 1]])
