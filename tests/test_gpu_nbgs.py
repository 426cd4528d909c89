"""Hard-contact (NBGS) step on the GPU against the compiled reference's converged solution and
the oracle."""
import numpy as np
import pytest

from helpers import CONVERGED_NAMES, load_golden, rel_err
from oracle.pe_oracle import APPROX_COULOMB_DECOUPLING, FRICTIONLESS, OracleWorld
from pe_b200 import _abi, scenes
from pe_b200.engine import Engine

pytestmark = pytest.mark.gpu


def hc_engine(scene, model, iters, precision=_abi.FP64):
    e = Engine(solver=_abi.HCSITS, precision=precision, relaxation_model=model,
               max_iterations=iters)
    return e.load_scene(scene)


@pytest.mark.parametrize("name", CONVERGED_NAMES)
def test_frictionless_converged_velocities_match_reference(name):
    g = load_golden(name)
    s = g["scene"]
    e = hc_engine(s, _abi.INELASTIC_FRICTIONLESS, 40000)
    e.step(s.dt)
    x, v, w = e.download()
    assert rel_err(v, g["hc0conv_v"]) < 1e-6
    assert rel_err(x, g["hc0conv_x"]) < 1e-9


@pytest.mark.parametrize("name", CONVERGED_NAMES)
def test_frictionless_mixed_precision_close_to_reference(name):
    g = load_golden(name)
    s = g["scene"]
    e = hc_engine(s, _abi.INELASTIC_FRICTIONLESS, 40000, precision=_abi.MIXED)
    e.step(s.dt)
    x, v, w = e.download()
    assert rel_err(v, g["hc0conv_v"]) < 1e-4
    # displacement of this step (x - x0 = v dt) to the same relative tolerance
    assert rel_err(x - s.x, g["hc0conv_x"] - s.x) < 1e-4


@pytest.mark.parametrize("precision,tol", [(_abi.FP64, 1e-6), (_abi.MIXED, 1e-4)])
def test_dense_packing_converged_velocities_match_reference(precision, tol):
    """4096 spheres on a 16x16x16 lattice of spacing 1.0 resting on the floor, 6,593 contacts
    (about half of the neighbours overlap): the GPU's colour-ordered frictionless sweeps converge
    to pe's converged velocities (pe: 20,000 sweeps in its detection order)."""
    g = load_golden("dense4096_conv")
    s = g["scene"]
    e = hc_engine(s, _abi.INELASTIC_FRICTIONLESS, 20000, precision=precision)
    e.step(s.dt)
    x, v, w = e.download()
    st = e.stats()
    assert st["contacts"] == int(g["contacts"])
    assert rel_err(v, g["hc0conv_v"]) < tol
    assert rel_err(x - s.x, g["hc0conv_x"] - s.x) < tol
    if precision == _abi.FP64:
        assert rel_err(x, g["hc0conv_x"]) < 1e-9


def test_dense_packing_friction_residual_like_oracle():
    """The same 4096-sphere packing with mu = 0.5 under pe's default model (approximate Coulomb
    friction by decoupling): after 1000 and 4000 sweeps the GPU's FP64 complementarity residual is
    of the oracle's size for the same sweep count (the fixed-point problem is the same; the sweep
    orders differ), and both shrink with the sweeps."""
    g = load_golden("dense4096_conv")
    s = scenes.nbgs_box(0, n=4096, mu=0.5, dims=(16.0, 16.0, 60.0), dense=True)
    assert np.array_equal(s.x, g["scene"].x)
    got = []
    for k, r_or in zip(g["mu05_sweeps"], g["mu05_residual_oracle"]):
        e = hc_engine(s, _abi.APPROX_INELASTIC_COULOMB_DECOUPLING, int(k))
        e.set_residual(True)
        e.step(s.dt)
        st = e.stats()
        e.close()
        got.append(st["residual"])
        if k >= 1000:
            assert st["residual"] < 10.0 * float(r_or) + 1e-9, (k, st["residual"], r_or)
    assert got[2] < got[1] < got[0]


def test_contact_count_matches_oracle():
    s = scenes.nbgs_box(0, n=2000, dims=(12.0, 12.0, 30.0), dense=True)
    e = hc_engine(s, _abi.APPROX_INELASTIC_COULOMB_DECOUPLING, 10)
    e.step(s.dt)
    st = e.stats()
    assert st["contacts"] == len(OracleWorld(s).contacts())
    assert 1 <= st["colors"] <= 64


@pytest.mark.parametrize("model", [_abi.INELASTIC_FRICTIONLESS,
                                   _abi.APPROX_INELASTIC_COULOMB_DECOUPLING])
def test_residual_reported_and_decreasing(model):
    s = scenes.small_random(3, n=125, overlap=0.0, mu=0.5)
    res = []
    for iters in (10, 100, 2000):
        e = hc_engine(s, model, iters)
        e.set_residual(True)
        e.step(s.dt)
        st = e.stats()
        assert st["residual"] >= 0.0 and st["delta_max"] >= 0.0
        res.append(st["residual"])
    assert res[2] < res[0]
    # the oracle's residual definition is the same; at 2000 sweeps both are small
    o = OracleWorld(s)
    _, _, r_or = o.hcsits_step(s.dt, FRICTIONLESS if model == 0 else APPROX_COULOMB_DECOUPLING, 2000)
    assert res[2] < max(10 * r_or, 1e-6)


def test_friction_converges_like_oracle():
    """Frictional contacts: the GPU solve reaches a complementarity residual as small as the
    oracle's with the same number of sweeps (different sweep orders, same fixed-point problem)."""
    s = scenes.small_random(5, n=216, overlap=-0.05, mu=0.5)
    e = hc_engine(s, _abi.APPROX_INELASTIC_COULOMB_DECOUPLING, 3000)
    e.set_residual(True)
    e.step(s.dt)
    st = e.stats()
    o = OracleWorld(s)
    _, _, r_or = o.hcsits_step(s.dt, APPROX_COULOMB_DECOUPLING, 3000)
    vscale = np.abs(o.v).max()
    assert st["residual"] < 1e-6 * vscale + 10 * r_or
    x, v, w = e.download()
    assert rel_err(x, o.x) < 1e-9
