"""Pins the CPU restatement (oracle/) against golden vectors produced by the compiled pe
reference (tests/golden/make_golden.py) and, when the reference build is present, against a
live run of it."""
import os
import subprocess

import numpy as np
import pytest

from helpers import CONVERGED_NAMES, GOLDEN_NAMES, load_golden, pair_set, rel_err, rel_err_w
from oracle.pe_oracle import APPROX_COULOMB_DECOUPLING, CONTACT_DTYPE, FRICTIONLESS, OracleWorld
from pe_b200 import scenes


@pytest.mark.parametrize("name", GOLDEN_NAMES)
def test_pairs_match_reference(name):
    g = load_golden(name)
    o = OracleWorld(g["scene"])
    c = o.contacts()
    ref = g["pairs"]
    assert pair_set(np.stack([c["b1"], c["b2"]], 1)) == pair_set(np.stack([ref["b1"], ref["b2"]], 1))
    # geometry of each contact (in canonical order)
    order = np.lexsort((ref["b2"], ref["b1"]))
    r = ref[order]
    if len(r):
        assert rel_err(c["gpos"], r["gpos"]) < 1e-15
        assert rel_err(c["n"], r["n"]) < 1e-15
        assert np.abs(c["dist"] - r["dist"]).max() < 1e-15


@pytest.mark.parametrize("name", GOLDEN_NAMES)
def test_dem_steps_match_reference(name):
    g = load_golden(name)
    for key in sorted(k for k in g if k.startswith("dem") and k.endswith("_x")):
        k = int(key[3:-2])
        o = OracleWorld(g["scene"], track_orientation=True)
        o.dem_step(g["scene"].dt, k)
        tol = 1e-13 if k <= 10 else 1e-11
        assert rel_err(o.x, g[f"dem{k}_x"]) < tol
        assert rel_err(o.v, g[f"dem{k}_v"]) < tol
        assert rel_err_w(o.w, g[f"dem{k}_w"], g[f"dem{k}_v"], g["scene"].r) < tol
        assert rel_err(o.q, g[f"dem{k}_q"]) < tol


@pytest.mark.parametrize("name", [n for n in GOLDEN_NAMES if n != "lattice512"])
@pytest.mark.parametrize("model", [0, 1, 2, 3, 4, 5])
def test_hcsits_step_bit_exact_in_reference_order(name, model):
    """Replaying pe's own contact order, the restated sweep of every relaxation model (pe's
    RelaxationModel 0-5) reproduces pe's step exactly -- including the NaNs pe's orthogonal
    projections produce for a friction coefficient of zero (dense512 has mu = 0)."""
    g = load_golden(name)
    o = OracleWorld(g["scene"], track_orientation=True)
    o.hcsits_step(g["scene"].dt, model, 100, contacts=g["hc_pairs"])
    assert np.array_equal(o.x, g[f"hc{model}_x"], equal_nan=True)
    assert np.array_equal(o.v, g[f"hc{model}_v"], equal_nan=True)
    assert np.array_equal(o.w, g[f"hc{model}_w"], equal_nan=True)


@pytest.mark.parametrize("name", CONVERGED_NAMES)
def test_hcsits_converged_frictionless_any_order(name):
    """Converged frictionless velocities do not depend on the sweep order."""
    g = load_golden(name)
    o = OracleWorld(g["scene"])
    o.hcsits_step(g["scene"].dt, FRICTIONLESS, 40000)
    assert rel_err(o.v, g["hc0conv_v"]) < 1e-6
    assert rel_err(o.x, g["hc0conv_x"]) < 1e-9


def test_dense_converged_frictionless_matches_reference():
    """The dense 4096-sphere packing (6,593 contacts): the oracle's converged frictionless
    velocities after 16,000 sweeps in its own order equal pe's after 20,000 to 1e-6."""
    g = load_golden("dense4096_conv")
    s = g["scene"]
    assert int(g["contacts"]) == len(OracleWorld(s).contacts())
    o = OracleWorld(s)
    o.hcsits_step(s.dt, FRICTIONLESS, 16000)
    assert rel_err(o.v, g["hc0conv_v"]) < 1e-6
    assert rel_err(o.x, g["hc0conv_x"]) < 1e-9


REF = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref")


@pytest.mark.skipif(not os.path.exists(os.path.join(REF, "ref_dem")),
                    reason="compiled reference not built (make -C oracle/ref)")
def test_live_reference_random_scenes(tmp_path):
    for seed in range(3):
        s = scenes.small_random(10 + seed, n=125, with_boxes=bool(seed % 2))
        p = tmp_path / "s.bin"
        s.save(str(p))
        out = tmp_path / "o.bin"
        subprocess.run([os.path.join(REF, "ref_dem"), "step", str(p), "5", str(out)], check=True)
        a = np.fromfile(out, "<f8")
        n = s.n
        o = OracleWorld(s)
        o.dem_step(s.dt, 5)
        assert rel_err(o.x, a[:3 * n].reshape(n, 3)) < 1e-13
        assert rel_err(o.v, a[3 * n:6 * n].reshape(n, 3)) < 1e-12


def test_oracle_finite_differences_match_reference():
    """The oracle's 40-step loss and its central differences (the checks the adjoint is held to)
    equal the compiled reference's."""
    from pe_b200.adjoint import LossSpec, set_params

    g = load_golden("adjoint_fd")
    s = g["scene"]
    spec = LossSpec.for_scene(s)

    def loss(t):
        o = OracleWorld(t)
        o.dem_step(t.dt, 40)
        return spec.value(o.x)

    assert abs(loss(s) - float(g["loss"])) < 1e-13
    fd = []
    for i, a in g["v_idx"]:
        sp, sm = s.copy(), s.copy()
        sp.v[i, a] += 1e-6
        sm.v[i, a] -= 1e-6
        fd.append((loss(sp) - loss(sm)) / 2e-6)
    assert np.abs(np.array(fd) - g["fd_v"]).max() < 1e-7 * np.abs(g["fd_v"]).max()
    p = {"k_n": 1e5, "c_n": 50.0, "c_t": 40.0, "mu": 0.3}
    for key, h in (("k_n", 1e-1), ("c_n", 1e-4), ("mu", 1e-6)):
        pp, pm = dict(p), dict(p)
        pp[key] += h
        pm[key] -= h
        f = (loss(set_params(s, **pp)) - loss(set_params(s, **pm))) / (2 * h)
        assert abs(f - float(g["fd_" + key])) < 1e-7 * abs(float(g["fd_" + key])) + 1e-12, key


@pytest.mark.parametrize("name", ["hertz64_boxes", "hertz64_planes"])
def test_hertz_dem_steps_match_reference(name):
    """pe's extended Hertz law (forceModel = hertz, compiled into ref_dem_hertz) against the
    oracle's restatement: sphere pairs use the Hertz law, walls the linear one."""
    g = load_golden(name)
    for k in (1, 10):
        o = OracleWorld(g["scene"], force_model=1)
        o.dem_step(g["scene"].dt, k)
        assert rel_err(o.x, g[f"dem{k}_x"]) < 1e-13
        assert rel_err(o.v, g[f"dem{k}_v"]) < 1e-12
        assert rel_err_w(o.w, g[f"dem{k}_w"], g[f"dem{k}_v"], g["scene"].r) < 1e-12
    # the linear law gives a different trajectory: the golden vectors do pin the Hertz branch
    o = OracleWorld(g["scene"], force_model=0)
    o.dem_step(g["scene"].dt, 10)
    assert rel_err(o.v, g["dem10_v"]) > 1e-3


# ---- moving boxes (box/box, box/plane, box/fixed-box and sphere/box contacts) ------------------
BOX_GOLDENS = ["boxes27_tumbling", "boxes64_tilted", "boxes36_stack"]


def contact_key(b1, b2, gpos, dist):
    return sorted(zip(b1.tolist(), b2.tolist(), map(tuple, np.round(gpos, 12).tolist()),
                      np.round(dist, 14).tolist()))


@pytest.mark.parametrize("name", BOX_GOLDENS)
def test_box_contacts_match_reference(name):
    """Same contacts as pe's fine detection (MaxContacts.h:589-668, 867-2250, 2380-2528):
    bodies in pe's orientation, contact points, normals and distances; several per box pair."""
    g = load_golden(name)
    c = OracleWorld(g["scene"]).contacts()
    ref = g["pairs"]
    assert len(c) == len(ref)
    assert contact_key(c["b1"], c["b2"], c["gpos"], c["dist"]) == \
        contact_key(ref["b1"], ref["b2"], ref["gpos"], ref["dist"])
    # normals, matched through the (stable) canonical order of both lists
    oi = np.lexsort((np.round(c["gpos"][:, 2], 12), np.round(c["gpos"][:, 1], 12),
                     np.round(c["gpos"][:, 0], 12), c["b2"], c["b1"]))
    ri = np.lexsort((np.round(ref["gpos"][:, 2], 12), np.round(ref["gpos"][:, 1], 12),
                     np.round(ref["gpos"][:, 0], 12), ref["b2"], ref["b1"]))
    assert rel_err(c["n"][oi], ref["n"][ri]) < 1e-15


@pytest.mark.parametrize("name", BOX_GOLDENS)
def test_box_dem_steps_match_reference(name):
    """DEM with moving boxes (BoxTrait::move, boxtrait/Default.h:149-220), including pe's zero
    stiffness at edge/edge contacts."""
    g = load_golden(name)
    s = g["scene"]
    for k in (1, 10):
        o = OracleWorld(s, track_orientation=True)
        o.dem_step(s.dt, k)
        assert rel_err(o.mb_x, g[f"dem{k}_bx"]) < 1e-14
        assert rel_err(o.mb_v, g[f"dem{k}_bv"]) < 1e-13
        assert rel_err(o.mb_w, g[f"dem{k}_bw"]) < 1e-13
        assert rel_err(o.mb_q, g[f"dem{k}_bq"]) < 1e-14
        if s.n:
            assert rel_err(o.x, g[f"dem{k}_x"]) < 1e-14
            assert rel_err(o.v, g[f"dem{k}_v"]) < 1e-13


@pytest.mark.parametrize("name", BOX_GOLDENS)
@pytest.mark.parametrize("model", [0, 1, 2, 3, 4, 5])
def test_box_hcsits_step_bit_exact_in_reference_order(name, model):
    """Hard contacts with moving boxes (world-frame inverse inertia R I^-1 R^T in the Delassus
    blocks and the impulse updates, gyroscopic term in the body cache) reproduce pe's step
    exactly in pe's contact order."""
    g = load_golden(name)
    s = g["scene"]
    o = OracleWorld(s, track_orientation=True)
    o.hcsits_step(s.dt, model, 100, contacts=g["hc_pairs"])
    for a, key in ((o.mb_x, "bx"), (o.mb_v, "bv"), (o.mb_w, "bw"), (o.mb_q, "bq"),
                   (o.x, "x"), (o.v, "v"), (o.w, "w")):
        assert np.array_equal(a, g[f"hc{model}_{key}"], equal_nan=True), key
