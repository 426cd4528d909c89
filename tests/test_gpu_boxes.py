"""Moving boxes on the GPU against pe's own runs (tests/golden/boxes*.npz, made by the compiled
reference): the contact set of pe's box fine detection, DEM steps with BoxTrait::move, and the
hard-contact step with box bodies; plus the argument checks of pe_b200_upload_boxes."""
import numpy as np
import pytest

from helpers import load_golden, rel_err
from oracle.pe_oracle import OracleWorld
from pe_b200 import _abi, scenes
from pe_b200.engine import Engine, PeB200Error

BOX_GOLDENS = ["boxes27_tumbling", "boxes64_tilted", "boxes36_stack"]


def contact_key(ids, gpos, dist):
    return sorted(zip(ids[:, 0].tolist(), ids[:, 1].tolist(),
                      map(tuple, np.round(gpos, 10).tolist()), np.round(dist, 12).tolist()))


@pytest.mark.gpu
@pytest.mark.parametrize("name", BOX_GOLDENS)
def test_box_contacts_match_reference(name):
    """Every contact pe finds, in pe's body order, with its point, normal and distance."""
    g = load_golden(name)
    e = Engine(solver=_abi.HCSITS).load_scene(g["scene"])
    ids, geom = e.contacts()
    e.close()
    ref = g["pairs"]
    assert len(ids) == len(ref)
    assert contact_key(ids, geom[:, :3], geom[:, 6]) == \
        contact_key(np.stack([ref["b1"], ref["b2"]], 1), ref["gpos"], ref["dist"])
    oi = np.lexsort((np.round(geom[:, 2], 10), np.round(geom[:, 1], 10), np.round(geom[:, 0], 10),
                     ids[:, 1], ids[:, 0]))
    ri = np.lexsort((np.round(ref["gpos"][:, 2], 10), np.round(ref["gpos"][:, 1], 10),
                     np.round(ref["gpos"][:, 0], 10), ref["b2"], ref["b1"]))
    assert rel_err(geom[oi, 3:6], ref["n"][ri]) < 1e-14


@pytest.mark.gpu
@pytest.mark.parametrize("name", BOX_GOLDENS)
def test_box_dem_steps_match_reference(name):
    g = load_golden(name)
    s = g["scene"]
    for k in (1, 10):
        e = Engine(solver=_abi.DEM, precision=_abi.FP64).load_scene(s)
        e.step(s.dt, k)
        bx, bq, bv, bw = e.download_boxes()
        x, v, w = e.download() if s.n else (None, None, None)
        e.close()
        assert rel_err(bx, g[f"dem{k}_bx"]) < 1e-13
        assert rel_err(bv, g[f"dem{k}_bv"]) < 1e-11
        assert rel_err(bw, g[f"dem{k}_bw"]) < 1e-11
        assert rel_err(bq, g[f"dem{k}_bq"]) < 1e-13
        if s.n:
            assert rel_err(x, g[f"dem{k}_x"]) < 1e-13
            assert rel_err(v, g[f"dem{k}_v"]) < 1e-11


@pytest.mark.gpu
@pytest.mark.parametrize("name", BOX_GOLDENS)
def test_box_hcsits_converged_frictionless(name):
    """Converged frictionless velocities do not depend on the sweep order: the GPU's colour
    order reaches pe's converged step."""
    g = load_golden(name)
    s = g["scene"]
    e = Engine(solver=_abi.HCSITS, precision=_abi.FP64, relaxation_model=0,
               max_iterations=20000).load_scene(s)
    e.step(s.dt)
    bx, bq, bv, bw = e.download_boxes()
    assert e.validate() == 0
    assert e.stats()["contacts"] == len(g["hc_pairs"])
    x, v, w = e.download() if s.n else (None, None, None)
    e.close()
    assert rel_err(bv, g["hc0conv_bv"]) < 1e-6
    # angular velocities on the scale of the surface speeds (a stack's are rounding noise)
    wscale = max(np.abs(g["hc0conv_bw"]).max(), np.abs(g["hc0conv_bv"]).max() / s.mbox_len.min())
    assert np.abs(bw - g["hc0conv_bw"]).max() < 1e-5 * wscale
    assert rel_err(bx, g["hc0conv_bx"]) < 1e-9
    if s.n:
        assert rel_err(v, g["hc0conv_v"]) < 1e-6


@pytest.mark.gpu
@pytest.mark.parametrize("model", [1, 3, 5])
def test_box_hcsits_models_run_and_stay_consistent(model):
    """The friction models with box bodies over a few steps of a stack: finite state, unit
    quaternions and a race-free colouring."""
    g = load_golden("boxes36_stack")
    s = g["scene"]
    e = Engine(solver=_abi.HCSITS, precision=_abi.FP64, relaxation_model=model,
               max_iterations=100).load_scene(s)
    for _ in range(3):
        e.step(s.dt)
        assert e.validate() == 0
    bx, bq, bv, bw = e.download_boxes()
    e.close()
    assert np.isfinite(bx).all() and np.isfinite(bv).all() and np.isfinite(bq).all()
    assert np.allclose(np.linalg.norm(bq, axis=1), 1.0, atol=1e-12)


@pytest.mark.gpu
@pytest.mark.parametrize("model", [2, 4])
def test_box_hcsits_orthogonal_projection_models_break_down_as_in_pe(model):
    """pe's orthogonal-projection models (relaxation parameter 1) produce non-finite velocities
    within one step of the box stack (tests/golden/boxes36_stack.npz); the GPU step reports
    the same breakdown instead of a finite answer."""
    g = load_golden("boxes36_stack")
    assert not np.isfinite(g[f"hc{model}_bv"]).all()
    s = g["scene"]
    e = Engine(solver=_abi.HCSITS, precision=_abi.FP64, relaxation_model=model,
               max_iterations=100).load_scene(s)
    e.step(s.dt)
    with pytest.raises(PeB200Error) as ei:
        e.download_boxes()
    assert ei.value.code == _abi.ERR_NAN
    e.close()


@pytest.mark.gpu
def test_box_dem_long_run_against_oracle():
    """200 DEM steps of a tumbling scene (spheres and boxes), GPU against the oracle."""
    s = scenes.tumbling_boxes(5, side=3)
    e = Engine(solver=_abi.DEM, precision=_abi.FP64).load_scene(s)
    e.step(s.dt, 200)
    bx, bq, bv, bw = e.download_boxes()
    x, v, w = e.download()
    e.close()
    o = OracleWorld(s)
    o.dem_step(s.dt, 200)
    assert rel_err(bx, o.mb_x) < 1e-9
    assert rel_err(bq, o.mb_q) < 1e-9
    assert rel_err(x, o.x) < 1e-9


@pytest.mark.gpu
def test_box_upload_checks():
    s = scenes.tumbling_boxes(0)
    e = Engine(solver=_abi.DEM).load_scene(s)
    bad = s.mbox_len.copy()
    bad[3, 1] = 0.0
    with pytest.raises(PeB200Error) as ei:
        e.upload_boxes(s.mbox_x, s.mbox_q, s.mbox_v, s.mbox_w, bad, s.mbox_mat)
    assert ei.value.code == _abi.ERR_ARG and "side length" in str(ei.value)
    q = s.mbox_q.copy()
    q[0] *= 1.1
    with pytest.raises(PeB200Error) as ei:
        e.upload_boxes(s.mbox_x, q, s.mbox_v, s.mbox_w, s.mbox_len, s.mbox_mat)
    assert ei.value.code == _abi.ERR_ARG
    mat = s.mbox_mat.copy()
    mat[0] = 7
    with pytest.raises(PeB200Error) as ei:
        e.upload_boxes(s.mbox_x, s.mbox_q, s.mbox_v, s.mbox_w, s.mbox_len, mat)
    assert ei.value.code == _abi.ERR_ARG
    e.close()
    m = Engine(solver=_abi.DEM, precision=_abi.MIXED)
    t = s.copy()
    t.mbox_len = np.zeros((0, 3))
    m.load_scene(t)
    with pytest.raises(PeB200Error) as ei:
        m.upload_boxes(s.mbox_x, s.mbox_q, s.mbox_v, s.mbox_w, s.mbox_len, s.mbox_mat)
    assert ei.value.code == _abi.ERR_UNSUPPORTED
    m.close()
