"""pe_b200_dem_step_static: the allocation-free DEM step for callers that cannot allocate device
memory (applications that own all device memory through their own pool, real-time loops that
must not stall on an allocation).  Its scratch is a fixed array inside the library.

Checked through the C ABI against the allocating entry point (pe_b200_step) on two calls in a
row, with the tolerance of the other DEM parity tests (1e-12 relative).  This file is collected
last so that a run stopping at the first failure has run every other test before it."""
import ctypes as C

import numpy as np
import pytest

from helpers import rel_err, rel_err_w
from pe_b200 import _abi, scenes
from pe_b200.engine import Engine

pytestmark = pytest.mark.gpu


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def _static_step(torch, s, x, v, w, r, mat, xo, vo, wo, n=None, lo=None, hi=None,
                 max_radius=None):
    L = _abi.load()
    mats = (_abi.Material * s.materials.shape[0])()
    for k in range(s.materials.shape[0]):
        for f, val in zip(_abi.Material._fields_, s.materials[k]):
            setattr(mats[k], f[0], float(val))
    planes = np.ascontiguousarray(s.planes, np.float64)
    pmat = np.ascontiguousarray(s.plane_mat, np.int32)
    boxes = np.ascontiguousarray(s.boxes, np.float64).reshape(-1, 15)
    bmat = np.ascontiguousarray(s.box_mat, np.int32)
    g = (C.c_double * 3)(*[float(a) for a in s.gravity])
    lo = (C.c_double * 3)(*[float(a) for a in (s.x.min(0) - 2.0 if lo is None else lo)])
    hi = (C.c_double * 3)(*[float(a) for a in (s.x.max(0) + 2.0 if hi is None else hi)])
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    return L.pe_b200_dem_step_static(
        s.n if n is None else n, _ptr(x), _ptr(v), _ptr(w), _ptr(r), _ptr(mat),
        s.materials.shape[0], mats, planes.shape[0], planes.ctypes.data, pmat.ctypes.data,
        boxes.shape[0], boxes.ctypes.data if boxes.size else None,
        bmat.ctypes.data if bmat.size else None, g, float(s.damping), float(s.dt), lo, hi,
        float(s.r.max() if max_radius is None else max_radius), _ptr(xo), _ptr(vo), _ptr(wo),
        stream)


def test_static_step_matches_allocating_step_twice():
    torch = pytest.importorskip("torch")
    s = scenes.small_random(11, n=1000, overlap=0.03, with_boxes=True)
    dev = torch.device("cuda", 0)
    t = lambda a, dt=torch.float64: torch.as_tensor(np.ascontiguousarray(a), dtype=dt, device=dev)
    x, v, w = t(s.x), t(s.v), t(s.w)
    r, mat = t(s.r), t(s.mat, torch.int32)
    xo, vo, wo = torch.empty_like(x), torch.empty_like(v), torch.empty_like(w)

    ref = Engine(solver=_abi.DEM, precision=_abi.FP64).load_scene(s)
    for call in range(2):
        free_before = torch.cuda.mem_get_info(dev)[0]
        rc = _static_step(torch, s, x, v, w, r, mat, xo, vo, wo)
        assert rc == _abi.OK, _abi.STATUS_NAMES.get(rc, rc)
        if call == 1:
            # the set-up happened on the first call; later calls allocate nothing
            assert torch.cuda.mem_get_info(dev)[0] == free_before
        ref.step(s.dt)
        rx, rv, rw = ref.download()
        gx, gv, gw = xo.cpu().numpy(), vo.cpu().numpy(), wo.cpu().numpy()
        assert rel_err(gx, rx) < 1e-12
        assert rel_err(gv, rv) < 1e-12
        assert rel_err_w(gw, rw, rv, s.r) < 1e-12
        # the output of this call is the input of the next one
        x, v, w = xo.clone(), vo.clone(), wo.clone()
    ref.close()


def test_static_step_rejects_oversize_requests():
    torch = pytest.importorskip("torch")
    s = scenes.small_random(12, n=64)
    dev = torch.device("cuda", 0)
    t = lambda a, dt=torch.float64: torch.as_tensor(np.ascontiguousarray(a), dtype=dt, device=dev)
    x, v, w, r, mat = t(s.x), t(s.v), t(s.w), t(s.r), t(s.mat, torch.int32)
    xo, vo, wo = torch.empty_like(x), torch.empty_like(v), torch.empty_like(w)
    rc = _static_step(torch, s, x, v, w, r, mat, xo, vo, wo, n=_abi.STATIC_MAX_SPHERES + 1)
    assert rc == _abi.ERR_ARG
    # a request within the limit still works afterwards
    assert _static_step(torch, s, x, v, w, r, mat, xo, vo, wo) == _abi.OK


def _tensors(torch, s):
    dev = torch.device("cuda", 0)
    t = lambda a, dt=torch.float64: torch.as_tensor(np.ascontiguousarray(a), dtype=dt, device=dev)
    x, v, w, r, mat = t(s.x), t(s.v), t(s.w), t(s.r), t(s.mat, torch.int32)
    return x, v, w, r, mat, torch.empty_like(x), torch.empty_like(v), torch.empty_like(w)


@pytest.mark.parametrize("case", ["wide_domain", "bodies_outside_domain"])
def test_static_step_coarse_or_clamped_grid_matches_allocating_step(case):
    """A domain much wider than the bodies (its finest grid exceeds PE_B200_STATIC_MAX_CELLS,
    so the grid is coarsened), and a domain smaller than the bodies' extent (bodies outside are
    clamped into border cells): both stay exact."""
    torch = pytest.importorskip("torch")
    s = scenes.small_random(13, n=500, overlap=0.03)
    x, v, w, r, mat, xo, vo, wo = _tensors(torch, s)
    c = s.x.mean(0)
    if case == "wide_domain":
        lo, hi = c - 1e4, c + 1e4        # ~1e4 cells per axis at the finest edge
    else:
        lo, hi = c - 1.0, c + 1.0        # most bodies outside
    ref = Engine(solver=_abi.DEM, precision=_abi.FP64, neighbor_lists=False).load_scene(s)
    for _ in range(2):
        rc = _static_step(torch, s, x, v, w, r, mat, xo, vo, wo, lo=lo, hi=hi)
        assert rc == _abi.OK, _abi.STATUS_NAMES.get(rc, rc)
        ref.step(s.dt)
        rx, rv, rw = ref.download()
        assert rel_err(xo.cpu().numpy(), rx) < 1e-12
        assert rel_err(vo.cpu().numpy(), rv) < 1e-12
        assert rel_err_w(wo.cpu().numpy(), rw, rv, s.r) < 1e-12
        x, v, w = xo.clone(), vo.clone(), wo.clone()
    ref.close()


@pytest.mark.parametrize("bad", ["radius_above_max", "material_out_of_range"])
def test_static_step_device_checks_reject_and_leave_outputs_alone(bad):
    torch = pytest.importorskip("torch")
    s = scenes.small_random(14, n=200, overlap=0.03)
    x, v, w, r, mat, xo, vo, wo = _tensors(torch, s)
    kw = {}
    if bad == "radius_above_max":
        kw["max_radius"] = float(s.r.max()) * 0.99
    else:
        mat[17] = s.materials.shape[0]
    for o in (xo, vo, wo):
        o.fill_(7.0)
    rc = _static_step(torch, s, x, v, w, r, mat, xo, vo, wo, **kw)
    assert rc == _abi.ERR_ARG
    for o in (xo, vo, wo):
        assert bool((o == 7.0).all())
    # a valid call afterwards succeeds
    mat[17] = 0
    assert _static_step(torch, s, x, v, w, r, mat, xo, vo, wo) == _abi.OK
