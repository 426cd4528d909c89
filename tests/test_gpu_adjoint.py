"""Adjoint of the FP64 DEM step (pe_b200_adjoint_forward/backward) against central finite
differences: of the GPU forward, of the oracle (CPU restatement pinned to pe), and of the compiled
reference (golden vectors), plus torch.autograd.gradcheck through a torch.autograd.Function that
is only the gradient-check harness."""
import numpy as np
import pytest

from helpers import load_golden, load_golden_arrays
from oracle.pe_oracle import OracleWorld, sphere_mass
from pe_b200 import _abi, scenes
from pe_b200.adjoint import LossSpec, difference_ladder, make_single_material, set_params
from pe_b200.engine import Engine

pytestmark = pytest.mark.gpu

K, EVERY = 40, 10


def scene(seed=2, n=64, boxes=False):
    s = make_single_material(scenes.small_random(seed, n=n, overlap=0.04, with_boxes=boxes),
                             k_n=1e5, c_n=50.0, c_t=40.0, mu=0.3)
    return s


def gpu_loss(s, spec):
    e = Engine(solver=_abi.DEM, precision=_abi.FP64, neighbor_lists=False).load_scene(s)
    e.step(s.dt, K)
    x, v, w = e.download()
    e.close()
    return spec.value(x)


def oracle_loss(s, spec):
    o = OracleWorld(s)
    o.dem_step(s.dt, K)
    return spec.value(o.x)


def adjoint(s, spec):
    e = Engine(solver=_abi.DEM, precision=_abi.FP64).load_scene(s)
    e.adjoint_forward(K, s.dt, EVERY)
    x, v, w = e.download()
    gx = spec.grad(x)
    gx0, gv0, gw0, gp = e.adjoint_backward(gx, np.zeros_like(gx), np.zeros_like(gx))
    e.close()
    return spec.value(x), gx0, gv0, gw0, gp


def fd_velocity(s, spec, idx, h, loss):
    out = []
    for (i, a) in idx:
        sp, sm = s.copy(), s.copy()
        sp.v[i, a] += h
        sm.v[i, a] -= h
        out.append((loss(sp, spec) - loss(sm, spec)) / (2 * h))
    return np.array(out)


def fd_param(s, spec, name, h, loss):
    p = {"k_n": 1e5, "c_n": 50.0, "c_t": 40.0, "mu": 0.3}
    pp, pm = dict(p), dict(p)
    pp[name] += h
    pm[name] -= h
    return (loss(set_params(s, **pp), spec) - loss(set_params(s, **pm), spec)) / (2 * h)


@pytest.mark.parametrize("boxes", [False, True])
def test_adjoint_matches_central_differences(boxes):
    s = scene(boxes=boxes)
    spec = LossSpec.for_scene(s)
    L, gx0, gv0, gw0, gp = adjoint(s, spec)
    assert abs(L - gpu_loss(s, spec)) < 1e-12
    rng = np.random.default_rng(0)
    idx = [(int(i), int(a)) for i, a in zip(rng.integers(0, s.n, 8), rng.integers(0, 3, 8))]
    fd = fd_velocity(s, spec, idx, 1e-6, gpu_loss)
    ad = np.array([gv0[i, a] for i, a in idx])
    scale = np.abs(fd).max()
    assert np.abs(ad - fd).max() < 1e-4 * scale + 1e-10, (ad, fd)
    # the same derivatives by finite differences of the oracle
    fdo = fd_velocity(s, spec, idx[:3], 1e-6, oracle_loss)
    assert np.abs(ad[:3] - fdo).max() < 1e-4 * scale + 1e-10
    for k, name, h in ((0, "k_n", 1e-1), (1, "c_n", 1e-4), (3, "mu", 1e-6)):
        f = fd_param(s, spec, name, h, gpu_loss)
        assert abs(gp[k] - f) < 1e-4 * abs(f) + 1e-9, (name, gp[k], f)


def test_adjoint_matches_reference_finite_differences():
    g = load_golden("adjoint_fd")
    s = g["scene"]
    spec = LossSpec.for_scene(s)
    L, gx0, gv0, gw0, gp = adjoint(s, spec)
    assert abs(L - float(g["loss"])) < 1e-10
    idx = [tuple(map(int, t)) for t in g["v_idx"]]
    ad = np.array([gv0[i, a] for i, a in idx])
    ref = g["fd_v"]
    assert np.abs(ad - ref).max() < 1e-4 * np.abs(ref).max() + 1e-10, (ad, ref)
    for k, key in ((0, "fd_k_n"), (1, "fd_c_n"), (3, "fd_mu")):
        assert abs(gp[k] - float(g[key])) < 1e-4 * abs(float(g[key])) + 1e-9, key


def test_adjoint_checkpoint_interval_does_not_matter():
    s = scene(seed=3)
    spec = LossSpec.for_scene(s)
    res = []
    for every in (1, 7, K):
        e = Engine(solver=_abi.DEM, precision=_abi.FP64).load_scene(s)
        e.adjoint_forward(K, s.dt, every)
        x, v, w = e.download()
        res.append(e.adjoint_backward(spec.grad(x), np.zeros_like(x), np.zeros_like(x)))
        e.close()
    for r in res[1:]:
        for a, b in zip(r, res[0]):
            assert np.array_equal(a, b)


def test_torch_gradcheck_harness():
    torch = pytest.importorskip("torch")
    from pe_b200.adjoint import dem_loss

    s = scene(seed=4, n=27)
    spec = LossSpec.for_scene(s)
    v0 = torch.tensor(s.v, dtype=torch.float64, requires_grad=True)
    scales = torch.ones(3, dtype=torch.float64, requires_grad=True)  # of k_n, c_n, mu
    f = lambda v, p: dem_loss(v, p, s, spec, K, EVERY)
    assert torch.autograd.gradcheck(f, (v0, scales), eps=1e-6, atol=1e-7, rtol=1e-4,
                                    nondet_tol=0.0)


# finite-difference steps of the hopper checks, largest first (as tests/golden/make_golden.py)
HOPPER_PARAM_STEPS = {"k_n": (1e-1, 1e-2, 1e-3), "c_n": (1e-4, 1e-5, 1e-6),
                      "mu": (1e-5, 1e-6, 1e-7)}
HOPPER_V_STEPS = (1e-6, 1e-7, 1e-8)


def test_hopper_full_horizon_gradient_matches_finite_differences():
    """The differentiable workload over its whole horizon: 16,384 spheres falling through the
    hopper for 2000 FP64 steps, checkpointed every 100.  The adjoint gradient of the loss with
    respect to k_n, c_n and mu and to the four initial-velocity components with the largest
    adjoint agrees to 1e-4 with finite differences of the GPU forward and, for the parameters,
    with pe's own FP64 finite differences (tests/golden/hopper_fd.npz).  Each difference is taken
    at the largest step of a ladder whose forward and backward one-sided differences agree: pe's
    dashpot force jumps when a contact starts, and a step that moves some contact's start across
    a time step measures that jump instead of the derivative (at h = 1e-6 one of the four velocity
    components does, by a factor of 8)."""
    g = load_golden_arrays("hopper_fd")
    s0 = scenes.hopper(0)
    m = s0.materials[0]
    p = {"k_n": m[6] / 2, "c_n": m[7] / 2, "c_t": m[8] / 2, "mu": 2 * m[2]}
    s = make_single_material(s0, **p)
    spec = LossSpec.for_scene(s, z_open=10.0)
    steps = s.steps
    assert int(g["steps"]) == steps and int(g["spheres"]) == s.n
    e = Engine(solver=_abi.DEM, precision=_abi.FP64).load_scene(s)
    e.adjoint_forward(steps, s.dt, 100)
    x = e.download()[0]
    z = np.zeros_like(x)
    _, gv0, _, gp = e.adjoint_backward(spec.grad(x), z, z)
    e.close()
    cache = {}

    def final(key, off, make):
        key = "base" if off == 0.0 else key
        if (key, off) not in cache:
            t = make(off)
            f = Engine(solver=_abi.DEM, precision=_abi.FP64, neighbor_lists=False).load_scene(t)
            f.step(t.dt, steps)
            cache[(key, off)] = f.download()[0]
            f.close()
        return cache[(key, off)]

    def ladder(key, hs, make):
        return difference_ladder(lambda a, b: spec.diff(final(key, a, make), final(key, b, make)),
                                 hs)

    for k, key in ((0, "k_n"), (1, "c_n"), (3, "mu")):
        rows, ch = ladder(key, HOPPER_PARAM_STEPS[key],
                          lambda off, key=key: set_params(s, **dict(p, **{key: p[key] + off})))
        assert abs(gp[k] - ch["central"]) < 1e-4 * abs(ch["central"]), (key, gp[k], rows)
        # pe's differences at the same ladder, with the same choice of step
        hs, fw, bw = g["h_" + key], g["fwd_" + key], g["bwd_" + key]
        assert np.allclose(hs, HOPPER_PARAM_STEPS[key])
        cen = 0.5 * (fw + bw)
        smooth = np.abs(fw - bw) <= 1e-4 * np.abs(cen)
        j = int(np.argmax(smooth)) if smooth.any() else len(hs) - 1
        assert abs(gp[k] - cen[j]) < 1e-4 * abs(cen[j]), (key, gp[k], cen, smooth)
    flat = np.argsort(-np.abs(gv0).ravel())[:4]
    for f in flat:
        i, a = int(f // 3), int(f % 3)

        def mv(off, i=i, a=a):
            t = s.copy()
            t.v[i, a] += off
            return t
        rows, ch = ladder(f"v{i}_{a}", HOPPER_V_STEPS, mv)
        assert abs(gv0[i, a] - ch["central"]) < 1e-4 * abs(ch["central"]), (i, a, gv0[i, a], rows)
