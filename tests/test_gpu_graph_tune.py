"""CUDA-graph replay and the launch-shape autotuner of the DEM neighbour-list step: neither may
change results (the skin may change the last bits), and the lists must hold every pair that can
touch before the next rebuild."""
import numpy as np
import pytest

from helpers import rel_err
from pe_b200 import _abi, scenes
from pe_b200.engine import Engine

pytestmark = pytest.mark.gpu


def run(s, precision, steps, graph_steps=16, tuning=None, scenes_list=None):
    e = Engine(solver=_abi.DEM, precision=precision)
    if scenes_list:
        e.load_scenes(scenes_list)
    else:
        e.load_scene(s)
    e.set_graph_steps(graph_steps)
    if tuning is not None:
        e.set_tuning(*tuning)
    e.step(s.dt, steps)
    out = e.download()
    active = e.graph_active()
    e.close()
    return out, active


@pytest.mark.parametrize("precision", [_abi.FP64, _abi.MIXED])
def test_graph_replay_matches_step_by_step(precision):
    s = scenes.dem_lattice(0, side=12)
    (x0, v0, w0), a0 = run(s, precision, 53, graph_steps=0)
    (x1, v1, w1), a1 = run(s, precision, 53, graph_steps=16)
    assert not a0 and a1
    assert np.array_equal(x0, x1) and np.array_equal(v0, v1) and np.array_equal(w0, w1)


def test_graph_replay_batched_scenes():
    ss = [scenes.small_random(s, n=64 + 16 * s, with_boxes=bool(s % 2)) for s in range(6)]
    for s in ss:
        s.dt = ss[0].dt
    (x0, v0, w0), _ = run(ss[0], _abi.MIXED, 40, graph_steps=0, scenes_list=ss)
    (x1, v1, w1), a1 = run(ss[0], _abi.MIXED, 40, graph_steps=8, scenes_list=ss)
    assert a1
    assert np.array_equal(x0, x1) and np.array_equal(v0, v1)


def test_launch_shapes_do_not_change_results():
    s = scenes.dem_lattice(1, side=10)
    e = Engine(solver=_abi.DEM, precision=_abi.MIXED).load_scene(s)
    skin = e.tuning()["skin"]
    nvar = e.tuning()["variants"]
    e.close()
    ref, _ = run(s, _abi.MIXED, 30)
    for v in range(nvar):
        for rb in (0, 1, 3):
            out, _ = run(s, _abi.MIXED, 30, tuning=(v, rb, skin))
            for a, b in zip(out, ref):
                assert np.array_equal(a, b), (v, rb)


def test_autotune_restores_state_and_keeps_physics():
    s = scenes.dem_lattice(2, side=12)
    e = Engine(solver=_abi.DEM, precision=_abi.FP64).load_scene(s)
    e.step(s.dt, 20)
    before = e.download()
    t = e.autotune(s.dt, 40)
    after = e.download()
    for a, b in zip(before, after):
        assert np.array_equal(a, b)
    assert 0 <= t["dem_variant"] < t["variants"] and t["rebuild_per_sm"] >= 0
    assert t["skin"] > 0 and t["ms_per_step"] > 0
    e.step(s.dt, 60)
    x, v, w = e.download()
    e.close()
    g = Engine(solver=_abi.DEM, precision=_abi.FP64, neighbor_lists=False).load_scene(s)
    g.step(s.dt, 80)
    xg, vg, wg = g.download()
    g.close()
    assert rel_err(x, xg) < 1e-12
    assert rel_err(v, vg) < 1e-9


@pytest.mark.parametrize("skin", [0.0, 0.2])
def test_lists_cover_pairs_beyond_one_cell(skin):
    """Two spheres 0.04 apart sit two grid cells apart along x when the cells are only 2 r_max
    wide; they close the gap before either has moved skin/2, so the list built at the start must
    already hold the pair (the cells are 2 r_max + skin wide)."""
    r = 0.5
    x = np.array([[1.99, 5.0, 5.0], [3.03, 5.0, 5.0]])
    v = np.array([[0.5, 0.0, 0.0], [-0.5, 0.0, 0.0]])
    s = scenes._scene(x, v, np.full(2, r), np.zeros(2, np.int64), scenes.box_planes([0, 0, 0], [10, 10, 10]),
                      np.zeros(6, np.int64), np.zeros((0, 15)), np.zeros(0), [scenes.material(1.0, 1e5, 50.0, 40.0, 0.3)],
                      (0.0, 0.0, 0.0), 1e-4, 600, "gap_pair")
    e = Engine(solver=_abi.DEM, precision=_abi.FP64, skin=skin).load_scene(s)
    e.step(s.dt, 600)
    xl, vl, _ = e.download()
    e.close()
    g = Engine(solver=_abi.DEM, precision=_abi.FP64, neighbor_lists=False).load_scene(s)
    g.step(s.dt, 600)
    xg, vg, _ = g.download()
    g.close()
    assert vg[0, 0] < 0.4   # the pair did collide
    assert rel_err(xl, xg) < 1e-12 and rel_err(vl, vg) < 1e-10


@pytest.mark.parametrize("precision", [_abi.FP64, _abi.MIXED])
@pytest.mark.parametrize("form", [0, 2])
def test_list_overflow_falls_back_to_the_grid(precision, form):
    """A list buffer far too small for the first rebuild: that step searches the grid, the
    library grows the buffer, and the trajectory is the grid path's (in the fused and the
    overlapped list-step forms)."""
    s = scenes.dem_lattice(3, side=8)
    e = Engine(solver=_abi.DEM, precision=precision, max_contacts=64).load_scene(s)
    e.set_tuning(0, 0, 0.0, dem_split=form)
    e.step(s.dt, 30)
    x, v, _ = e.download()
    st = e.neighbor_list_stats()
    e.close()
    assert st["capacity"] > 64
    g = Engine(solver=_abi.DEM, precision=precision, neighbor_lists=False).load_scene(s)
    g.step(s.dt, 30)
    xg, vg, _ = g.download()
    g.close()
    tol = 1e-12 if precision == _abi.FP64 else 1e-6
    assert rel_err(x, xg) < tol
    assert rel_err(v, vg) < (1e-9 if precision == _abi.FP64 else 1e-3)


@pytest.mark.parametrize("precision", [_abi.FP64, _abi.MIXED])
@pytest.mark.parametrize("model", [0, 1])
def test_nbgs_sweep_forms_agree(precision, model):
    """One cluster, one cooperative grid, one launch per colour and one cluster with the bodies
    in its shared memory run the same colour order, and the contacts of a colour share no body:
    the results are identical."""
    s = scenes.nbgs_box(0, n=4096, dims=(16.0, 16.0, 40.0), dense=True)
    out = []
    for mode in (1, 2, 3, 5):
        e = Engine(solver=_abi.HCSITS, precision=precision, relaxation_model=model,
                   max_iterations=30).load_scene(s)
        e.set_tuning(nbgs_sweeps=mode)
        e.step(s.dt, 3)
        out.append(e.download())
        e.close()
    for o in out[1:]:
        for a, b in zip(o, out[0]):
            assert np.array_equal(a, b)


@pytest.mark.parametrize("name", ["dense512", "boxes36_stack"])
def test_nbgs_single_block_form_agrees(name):
    """When every colour fits one block, all sweeps can run in that block with __syncthreads
    between colours; it gives the grid form's and the per-colour form's results bit for bit."""
    from helpers import load_golden
    s = load_golden(name)["scene"]
    out = []
    for mode in (2, 3, 4, 0):
        e = Engine(solver=_abi.HCSITS, precision=_abi.FP64, relaxation_model=1,
                   max_iterations=50).load_scene(s)
        e.set_tuning(nbgs_sweeps=mode)
        e.step(s.dt, 2)
        out.append(e.download_boxes() if s.nmbox else e.download())
        e.close()
    for o in out[1:]:
        for a, b in zip(o, out[0]):
            assert np.array_equal(a, b)


def _crowded_scene(seed=0):
    """One sphere of radius 1 among 4,096 of radius 0.05 packed 0.102 apart: the cells are sized
    for the large sphere, so a row of cells holds hundreds of small ones and every small sphere
    has up to 18 neighbours within a skin of 0.05."""
    rng = np.random.default_rng(seed)
    g = np.arange(16) * 0.102 + 0.06
    x = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    x = np.concatenate([x + rng.uniform(-0.001, 0.001, x.shape), [[1.0, 1.0, 3.2]]])
    r = np.concatenate([np.full(4096, 0.05), [1.0]])
    v = rng.normal(0.0, 0.05, x.shape)
    v[-1] = [0.0, 0.0, -2.0]
    return scenes._scene(x, v, r, np.zeros(len(r), np.int64),
                         scenes.box_planes([0, 0, 0], [2.5, 2.5, 5.0]), np.zeros(6, np.int64),
                         np.zeros((0, 15)), np.zeros(0), [scenes.material(1.0, 1e4, 5.0, 4.0, 0.3)],
                         (0.0, 0.0, -9.81), 1e-4, 300, "crowded_rows")


@pytest.mark.parametrize("name", ["dense512", "crowded"])
def test_list_rebuild_forms_agree(name):
    """The persistent rebuild keeps the first few neighbours of each sphere from its counting
    pass, searches again only for spheres with more, and takes rows of more than 32 candidates
    one candidate at a time; the rebuild in one launch per stage scans row by row.  Through
    several rebuilds of a dense packing and of a crowded one (cells sized for one large sphere,
    up to 18 neighbours each) both give the same lists, so the same trajectory bit for bit, and
    the grid path's trajectory up to summation order."""
    from helpers import load_golden
    s = load_golden("dense512")["scene"] if name == "dense512" else _crowded_scene()
    skin = 0.05 if name == "crowded" else 0.0
    steps = 300
    out = []
    for per_sm in (0, -1):
        e = Engine(solver=_abi.DEM, precision=_abi.FP64, skin=skin).load_scene(s)
        e.set_tuning(0, per_sm, skin)
        for _ in range(3):
            e.step(s.dt, steps // 3)
            assert e.validate() == 0
        st = e.neighbor_list_stats()
        assert st["rebuilds"] >= 2 and st["entries"] > (8 * s.n if name == "crowded" else 0)
        out.append(e.download())
        e.close()
    for a, b in zip(out[0], out[1]):
        assert np.array_equal(a, b)
    g = Engine(solver=_abi.DEM, precision=_abi.FP64, neighbor_lists=False).load_scene(s)
    g.step(s.dt, steps)
    xg, vg, _ = g.download()
    g.close()
    assert rel_err(out[0][0], xg) < 1e-9 and rel_err(out[0][1], vg) < 1e-6


def _crowded(seed=0, side=22, big=2.5):
    """Small spheres on a lattice around one large sphere: the large radius sets the cell edge
    (2 r_max), so a tile's neighbourhood holds far more candidates than the grid step stages in
    shared memory and those tiles search global memory instead."""
    s = scenes.small_random(seed, n=side ** 3, overlap=0.02, with_boxes=False)
    s.x = s.x * 0.22
    s.r = s.r * 0.22
    c = s.x.mean(0)
    keep = np.linalg.norm(s.x - c, axis=1) > big + 0.2
    t = s.copy()
    t.x = np.vstack([s.x[keep], c[None, :]])
    t.v = np.vstack([s.v[keep], np.zeros((1, 3))])
    t.w = np.vstack([s.w[keep], np.zeros((1, 3))])
    t.r = np.concatenate([s.r[keep], [big]])
    t.mat = np.concatenate([s.mat[keep], s.mat[:1]]).astype(np.int32)
    return t


def _grid_run(s, precision, form, steps=6, scenes_list=None, **kw):
    e = Engine(solver=_abi.DEM, precision=precision, neighbor_lists=False, **kw)
    if scenes_list:
        e.load_scenes(scenes_list)
    else:
        e.load_scene(s)
    e.set_tuning(dem_grid=form)
    e.step(s.dt, steps)
    out = e.download()
    boxes = e.download_boxes() if s.nmbox else None
    e.close()
    return out, boxes


@pytest.mark.parametrize("case", ["lattice", "dense", "boxes_walls", "moving_boxes", "hertz",
                                  "orientation", "mixed", "batched", "crowded"])
def test_grid_step_forms_agree_bitwise(case):
    """The tiled grid step (candidates staged in shared memory) and the one-thread-per-sphere
    grid step sum the same contact forces in the same order: identical trajectories."""
    kw, prec, ss = {}, _abi.FP64, None
    if case == "lattice":
        s = scenes.dem_lattice(2, side=14)
    elif case == "dense":
        s = scenes.nbgs_box(1, n=4096, dims=(16.0, 16.0, 60.0), dense=True)
        s.dt = 1e-4
    elif case == "boxes_walls":
        s = scenes.small_random(31, n=1000, overlap=0.03, with_boxes=True)
    elif case == "moving_boxes":
        s = scenes.tumbling_boxes(1)
    elif case == "hertz":
        s = scenes.small_random(32, n=512, overlap=0.03)
        kw["force_model"] = 1
    elif case == "orientation":
        s = scenes.small_random(33, n=512, overlap=0.03)
        kw["track_orientation"] = True
    elif case == "mixed":
        s = scenes.dem_lattice(3, side=12)
        prec = _abi.MIXED
    elif case == "batched":
        ss = [scenes.small_random(40 + k, n=100 + 50 * k, with_boxes=bool(k % 2)) for k in range(5)]
        for t in ss:
            t.dt = ss[0].dt
        s = ss[0]
    else:
        s = _crowded()
    a, ab = _grid_run(s, prec, 0, scenes_list=ss, **kw)
    b, bb = _grid_run(s, prec, 1, scenes_list=ss, **kw)
    assert np.isfinite(a[0]).all()
    for u, w in zip(a, b):
        assert np.array_equal(u, w), case
    if ab is not None:
        for u, w in zip(ab, bb):
            assert np.array_equal(u, w), case


@pytest.mark.parametrize("precision", [_abi.FP64, _abi.MIXED])
def test_hard_contact_graph_replay_matches_step_by_step(precision):
    """Hard-contact steps queued without host waits and replayed as captured graphs of 16
    steps give the step-by-step results, on a packing with contacts (including a step where
    the scene's first contacts appear after contact-free steps)."""
    s = scenes.nbgs_box(2, n=2000, dims=(12.0, 12.0, 30.0), dense=True)
    loose = scenes.nbgs_box(3, n=1000, dims=(12.0, 12.0, 40.0))
    for sc in (s, loose):
        out = []
        for gsteps in (0, 16):
            e = Engine(solver=_abi.HCSITS, precision=precision, relaxation_model=1,
                       max_iterations=30).load_scene(sc)
            e.set_graph_steps(gsteps)
            e.step(sc.dt, 3)
            e.step(sc.dt, 37)
            out.append(e.download())
            e.close()
        for a, b in zip(out[0], out[1]):
            assert np.array_equal(a, b)


@pytest.mark.gpu
def test_hard_contact_graphs_are_kept_across_calls():
    """Calls of 32 hard-contact steps replay the graphs captured by earlier calls: the plan
    (with or without contacts) and the sweep grid each key a graph of their own."""
    sc = scenes.nbgs_box(2, n=2000, dims=(12.0, 12.0, 30.0), dense=True)
    e = Engine(solver=_abi.HCSITS, precision=_abi.MIXED, relaxation_model=1,
               max_iterations=30).load_scene(sc)
    e.step(sc.dt, 2)
    e.step(sc.dt, 32)
    g0 = e.graph_stats()
    assert g0["captures"] >= 1
    for _ in range(6):
        e.step(sc.dt, 32)
    g1 = e.graph_stats()
    assert g1["replays"] - g0["replays"] >= 12
    assert g1["captures"] - g0["captures"] <= 3
    e.close()


@pytest.mark.parametrize("precision", [_abi.FP64, _abi.MIXED])
@pytest.mark.parametrize("track,law", [(False, 0), (True, 0), (False, 1)])
def test_split_list_step_matches_two_kernel_form(precision, track, law):
    """The split list step (the marked spheres' forces and integration on a second stream, the
    other spheres' integration beside them) and the overlapped form (the same on one stream: the
    integration of the unmarked spheres starts while the marked ones are computed) give the
    results of the two-kernel form bit for bit, step by step and through graph replays, over
    several rebuilds (a small skin): on a sparse lattice (few spheres marked) and on an agitated
    dense packing (every sphere marked)."""
    for s in (scenes.dem_lattice(4, side=12), scenes.dem_dense(4, 16, 16, 8)):
        out = []
        for split, gs in ((0, 0), (1, 0), (1, 16), (2, 0), (2, 16)):
            e = Engine(solver=_abi.DEM, precision=precision, track_orientation=track,
                       skin=0.004, force_model=law).load_scene(s)
            e.set_graph_steps(gs)
            e.set_tuning(0, 0, 0.0, dem_split=split)
            e.step(s.dt, 3)
            e.step(s.dt, 61)
            out.append(e.download())
            st = e.neighbor_list_stats()
            e.close()
            assert st["rebuilds"] >= 1
        for o in out[1:]:
            for a, b in zip(o, out[0]):
                assert np.array_equal(a, b)


@pytest.mark.parametrize("precision", [_abi.FP64, _abi.MIXED])
def test_list_forms_agree_on_batched_scenes(precision):
    """Six scenes of different sizes in one context, some with fixed boxes, each scene its own
    material (the kernels read every sphere's scene and material through its tag): the three
    list-step forms give the same results bit for bit, step by step and through graph
    replays."""
    ss = [scenes.small_random(s, n=64 + 16 * s, with_boxes=bool(s % 2)) for s in range(6)]
    for s in ss:
        s.dt = ss[0].dt
    out = []
    for split, gs in ((0, 0), (1, 0), (2, 0), (2, 8)):
        e = Engine(solver=_abi.DEM, precision=precision, skin=0.01)
        e.load_scenes(ss)
        e.set_graph_steps(gs)
        e.set_tuning(0, 0, 0.0, dem_split=split)
        e.step(ss[0].dt, 3)
        e.step(ss[0].dt, 45)
        out.append(e.download())
        e.close()
    for o in out[1:]:
        for a, b in zip(o, out[0]):
            assert np.array_equal(a, b)


def test_list_forms_switched_between_graph_replays_on_a_large_scene():
    """One context of 196,608 spheres switches, between graph replays, between the fused
    rebuild-and-contacts form, the two-stream split form and the overlapped form (dem_split 0, 1,
    2), at the rebuild grids of several CTA counts per SM.  The scene needs more rebuild blocks than either kernel keeps resident, so the
    two forms' cooperative grids differ (the fused kernel holds fewer CTAs per SM); the rebuild's
    per-block buffer must serve both without being reallocated (a step captured into a graph
    allocates nothing).  The result is that of a fresh context stepping in the two-kernel form
    without graphs, bit for bit."""
    s = scenes.dem_dense(4, 64, 64, 48)
    plan = ((0, 0), (1, 0), (2, 0), (0, 4), (1, 4), (2, 4), (0, 1), (2, 2), (1, 2))
    e = Engine(solver=_abi.DEM, precision=_abi.MIXED, skin=0.004).load_scene(s)
    e.set_graph_steps(16)
    e.step(s.dt, 3)
    for split, per_sm in plan:
        e.set_tuning(0, per_sm, 0.0, dem_split=split)
        e.step(s.dt, 32)
    got = e.download()
    gs = e.graph_stats()
    st = e.neighbor_list_stats()
    e.close()
    assert gs["replays"] >= len(plan) and st["rebuilds"] >= 2
    r = Engine(solver=_abi.DEM, precision=_abi.MIXED, skin=0.004).load_scene(s)
    r.set_graph_steps(0)
    r.set_tuning(0, -1, 0.0)
    r.step(s.dt, 3 + 32 * len(plan))
    want = r.download()
    r.close()
    for a, b in zip(got, want):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("precision", [_abi.MIXED, _abi.FP64])
@pytest.mark.parametrize("model", [0, 1])
def test_nbgs_compact_form_agrees(precision, model):
    """A scene of 32k spheres whose first few contacts appear after free fall: the compact
    single-block form (only the bodies with contacts in shared memory, asked for with 4), the
    whole-scene single-block form (what the queued grid mode runs for colours this small) and one
    launch per colour give identical results."""
    s = scenes.nbgs_box(0, mu=0.5 if model else 0.0)
    out = []
    for mode in (4, 2, 3):
        e = Engine(solver=_abi.HCSITS, precision=precision, relaxation_model=model,
                   max_iterations=40).load_scene(s)
        e.set_tuning(nbgs_sweeps=mode)
        e.step(s.dt, s.steps)
        st = e.stats()
        assert 0 < st["contacts"] <= 768
        out.append(e.download())
        e.close()
    for o in out[1:]:
        for a, b in zip(o, out[0]):
            assert np.array_equal(a, b)
