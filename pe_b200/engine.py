"""Python handle over the C ABI: one context = one World (or a batch of independent scenes).

Mirrors pe's usage pattern (materials, bodies and walls first, then World::simulationStep in a
loop, then body getters) with numpy arrays instead of per-body objects.
"""
from __future__ import annotations

import ctypes as C
from typing import List, Optional, Sequence

import numpy as np

from . import _abi
from ._abi import PeB200Error


def _p(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data


class Engine:
    def __init__(self, solver: int = _abi.DEM, precision: int = _abi.FP64,
                 relaxation_model: int = _abi.APPROX_INELASTIC_COULOMB_DECOUPLING,
                 max_iterations: int = 100, erp: float = 0.7, gravity=(0.0, 0.0, 0.0),
                 damping: float = 1.0, device: int = 0, track_orientation: bool = False,
                 max_contacts: int = 0, neighbor_lists: bool = True, skin: float = 0.0,
                 force_model: int = 0):
        self._L = _abi.load()
        p = _abi.default_params()
        p.solver, p.precision = solver, precision
        p.relaxation_model, p.max_iterations, p.erp = relaxation_model, max_iterations, erp
        for a in range(3):
            p.gravity[a] = float(gravity[a])
        p.damping, p.device = damping, device
        p.track_orientation = 1 if track_orientation else 0
        p.max_contacts = max_contacts
        p.neighbor_lists = 1 if neighbor_lists else 0
        p.skin = float(skin)
        p.force_model = int(force_model)
        h = C.c_void_p()
        self._check(self._L.pe_b200_create(C.byref(p), C.byref(h)), ctx=None)
        self._h = h
        self.track_orientation = track_orientation
        self.n = 0

    # -- lifecycle ----------------------------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None):
            self._L.pe_b200_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, rc: int, ctx="self"):
        if rc != _abi.OK:
            msg = ""
            if ctx == "self" and getattr(self, "_h", None):
                m = self._L.pe_b200_last_error(self._h)
                msg = m.decode() if m else ""
            raise PeB200Error(rc, msg)

    # -- setup ----------------------------------------------------------------------------------
    def set_materials(self, mats: np.ndarray):
        mats = np.ascontiguousarray(mats, np.float64).reshape(-1, 9)
        arr = (_abi.Material * mats.shape[0])()
        for k in range(mats.shape[0]):
            for f, val in zip(_abi.Material._fields_, mats[k]):
                setattr(arr[k], f[0], float(val))
        self._check(self._L.pe_b200_set_materials(self._h, mats.shape[0], arr))

    def set_walls(self, scene: int, planes, plane_mat, boxes, box_mat):
        planes = np.ascontiguousarray(planes, np.float64).reshape(-1, 4)
        plane_mat = np.ascontiguousarray(plane_mat, np.int32).reshape(-1)
        boxes = np.ascontiguousarray(boxes, np.float64).reshape(-1, 15)
        box_mat = np.ascontiguousarray(box_mat, np.int32).reshape(-1)
        self._check(self._L.pe_b200_set_walls(self._h, scene, planes.shape[0], _p(planes),
                                              _p(plane_mat), boxes.shape[0], _p(boxes),
                                              _p(box_mat)))

    def upload(self, x, v, w, r, mat, scene=None, nscenes: int = 1):
        x = np.ascontiguousarray(x, np.float64).reshape(-1, 3)
        v = np.ascontiguousarray(v, np.float64).reshape(-1, 3)
        w = np.ascontiguousarray(w, np.float64).reshape(-1, 3)
        r = np.ascontiguousarray(r, np.float64).reshape(-1)
        mat = np.ascontiguousarray(mat, np.int32).reshape(-1)
        sc = None if scene is None else np.ascontiguousarray(scene, np.int32).reshape(-1)
        self._check(self._L.pe_b200_upload_bodies(self._h, r.shape[0], _p(x), _p(v), _p(w),
                                                  _p(r), _p(mat), _p(sc), nscenes))
        self.n = r.shape[0]

    def load_scene(self, scene) -> "Engine":
        """Materials, walls, gravity and bodies of a pe_b200.scenes.Scene."""
        self.set_materials(scene.materials)
        self.set_walls(0, scene.planes, scene.plane_mat, scene.boxes, scene.box_mat)
        self.set_gravity(scene.gravity)
        self.set_damping(scene.damping)
        self.upload(scene.x, scene.v, scene.w, scene.r, scene.mat)
        if getattr(scene, "nmbox", 0):
            self.upload_boxes(scene.mbox_x, scene.mbox_q, scene.mbox_v, scene.mbox_w,
                              scene.mbox_len, scene.mbox_mat)
        return self

    def upload_boxes(self, x, q, v, w, lengths, mat, scene=None):
        """Moving boxes (after the spheres): centres, unit quaternions (w x y z), velocities,
        side lengths, material ids, optional scene ids grouped by scene."""
        x = np.ascontiguousarray(x, np.float64).reshape(-1, 3)
        q = np.ascontiguousarray(q, np.float64).reshape(-1, 4)
        v = np.ascontiguousarray(v, np.float64).reshape(-1, 3)
        w = np.ascontiguousarray(w, np.float64).reshape(-1, 3)
        lengths = np.ascontiguousarray(lengths, np.float64).reshape(-1, 3)
        mat = np.ascontiguousarray(mat, np.int32).reshape(-1)
        sc = None if scene is None else np.ascontiguousarray(scene, np.int32).reshape(-1)
        self._check(self._L.pe_b200_upload_boxes(self._h, x.shape[0], _p(x), _p(q), _p(v), _p(w),
                                                 _p(lengths), _p(mat), _p(sc)))
        self.nbox = x.shape[0]

    def download_boxes(self):
        """(x, q, v, w) of the moving boxes."""
        m = int(self._L.pe_b200_box_count(self._h))
        x, q = np.zeros((m, 3)), np.zeros((m, 4))
        v, w = np.zeros((m, 3)), np.zeros((m, 3))
        self._check(self._L.pe_b200_download_boxes(self._h, _p(x), _p(q), _p(v), _p(w)))
        return x, q, v, w

    def load_scenes(self, scenes: Sequence) -> "Engine":
        """A batch of independent scenes (each keeps its own walls and grid); materials are
        concatenated and re-indexed, gravity is taken from the first scene."""
        mats, xs, vs, ws, rs, ms, sc = [], [], [], [], [], [], []
        off = 0
        for s in scenes:
            mats.append(s.materials)
        self.set_materials(np.concatenate(mats))
        for k, s in enumerate(scenes):
            self.set_walls(k, s.planes, s.plane_mat + off, s.boxes, s.box_mat + off)
            xs.append(s.x); vs.append(s.v); ws.append(s.w); rs.append(s.r)
            ms.append(s.mat + off)
            sc.append(np.full(s.n, k, np.int32))
            off += s.materials.shape[0]
        self.set_gravity(scenes[0].gravity)
        self.set_damping(scenes[0].damping)
        self.upload(np.concatenate(xs), np.concatenate(vs), np.concatenate(ws),
                    np.concatenate(rs), np.concatenate(ms), np.concatenate(sc), len(scenes))
        return self

    def set_gravity(self, g):
        arr = (C.c_double * 3)(*[float(a) for a in g])
        self._check(self._L.pe_b200_set_gravity(self._h, arr))

    def set_damping(self, d: float):
        self._check(self._L.pe_b200_set_damping(self._h, float(d)))

    def set_max_iterations(self, n: int):
        self._check(self._L.pe_b200_set_max_iterations(self._h, int(n)))

    def set_relaxation_model(self, m: int):
        self._check(self._L.pe_b200_set_relaxation_model(self._h, int(m)))

    def set_error_reduction(self, erp: float):
        self._check(self._L.pe_b200_set_error_reduction(self._h, float(erp)))

    def set_residual(self, on: bool = True):
        self._check(self._L.pe_b200_set_residual(self._h, 1 if on else 0))

    def set_state(self, x=None, v=None, w=None):
        cv = lambda a: None if a is None else np.ascontiguousarray(a, np.float64).reshape(-1, 3)
        x, v, w = cv(x), cv(v), cv(w)
        self._check(self._L.pe_b200_set_state(self._h, _p(x), _p(v), _p(w)))

    # -- stepping -------------------------------------------------------------------------------
    def step(self, dt: float, nsteps: int = 1):
        self._check(self._L.pe_b200_step(self._h, int(nsteps), float(dt)))

    def download(self, out=None):
        """(x, v, w[, q]) in upload order.  out: arrays to fill instead of new ones (e.g. pinned
        host buffers reused across calls); each must be C-contiguous float64 of shape (n, 3)."""
        n = self.n
        if out is not None:
            x, v, w = out[0], out[1], out[2]
            for a in (x, v, w):
                if a.dtype != np.float64 or a.shape != (n, 3) or not a.flags["C_CONTIGUOUS"]:
                    raise ValueError("download buffers must be C-contiguous float64 (n, 3)")
        else:
            x, v, w = np.empty((n, 3)), np.empty((n, 3)), np.empty((n, 3))
        q = np.empty((n, 4)) if self.track_orientation else None
        self._check(self._L.pe_b200_download_bodies(self._h, _p(x), _p(v), _p(w), _p(q)))
        return (x, v, w, q) if self.track_orientation else (x, v, w)

    def contacts(self):
        """Contacts of the current state sorted by (body1, body2): (ids (k,2), geom (k,7))."""
        nout = C.c_int64(0)
        self._check(self._L.pe_b200_find_contacts(self._h, 0, None, None, C.byref(nout)))
        k = nout.value
        ids = np.zeros((max(k, 1), 2), np.int64)
        geom = np.zeros((max(k, 1), 7), np.float64)
        self._check(self._L.pe_b200_find_contacts(self._h, k, _p(ids), _p(geom), C.byref(nout)))
        return ids[:k], geom[:k]

    def stats(self):
        nc, ncol = C.c_int64(), C.c_int32()
        d, r = C.c_double(), C.c_double()
        self._check(self._L.pe_b200_last_step_stats(self._h, C.byref(nc), C.byref(ncol),
                                                    C.byref(d), C.byref(r)))
        return {"contacts": nc.value, "colors": ncol.value, "delta_max": d.value,
                "residual": r.value}

    def set_profiling(self, on: bool = True):
        self._check(self._L.pe_b200_set_profiling(self._h, 1 if on else 0))

    def profile(self) -> dict:
        """Stage name -> (total ms, timed launches) since profiling was enabled."""
        cap = 16
        names = (C.c_char_p * cap)()
        ms = (C.c_double * cap)()
        cnt = (C.c_int64 * cap)()
        n = C.c_int32()
        self._check(self._L.pe_b200_profile(self._h, cap, names, ms, cnt, C.byref(n)))
        return {names[k].decode(): (ms[k], cnt[k]) for k in range(min(n.value, cap))}

    def adjoint_forward(self, nsteps: int, dt: float, checkpoint_every: int = 100):
        """Runs nsteps FP64 DEM steps keeping checkpoints for adjoint_backward."""
        self._check(self._L.pe_b200_adjoint_forward(self._h, int(nsteps), float(dt),
                                                    int(checkpoint_every)))

    def adjoint_backward(self, gx, gv, gw):
        """Gradient of a loss w.r.t. the initial state and the contact coefficients, given its
        gradient w.r.t. the final state. Returns (gx0, gv0, gw0, gparams[k_n, c_n, c_t, mu])."""
        n = self.n
        cv = lambda a: np.ascontiguousarray(a, np.float64).reshape(n, 3)
        gx, gv, gw = cv(gx), cv(gv), cv(gw)
        ox, ov, ow = np.empty((n, 3)), np.empty((n, 3)), np.empty((n, 3))
        gp = np.zeros(4)
        self._check(self._L.pe_b200_adjoint_backward(self._h, _p(gx), _p(gv), _p(gw), _p(ox),
                                                     _p(ov), _p(ow), _p(gp)))
        return ox, ov, ow, gp

    def set_graph_steps(self, steps: int):
        """DEM list steps per CUDA-graph replay (0 = launch every step)."""
        self._check(self._L.pe_b200_set_graph_steps(self._h, int(steps)))

    def graph_active(self) -> bool:
        return bool(self._L.pe_b200_graph_active(self._h))

    def graph_stats(self) -> dict:
        """Graphs captured and graph launches since the context was created."""
        cap, rep = C.c_int64(), C.c_int64()
        self._check(self._L.pe_b200_graph_stats(self._h, C.byref(cap), C.byref(rep)))
        return {"captures": cap.value, "replays": rep.value}

    def tuning(self) -> dict:
        t = _abi.Tuning()
        self._check(self._L.pe_b200_get_tuning(self._h, C.byref(t)))
        return {k: getattr(t, k) for k, _ in _abi.Tuning._fields_}

    def set_tuning(self, dem_variant: int = 0, rebuild_per_sm: int = 0, skin: float = 0.0,
                   nbgs_sweeps: int = 0, dem_grid: int = 0, dem_split: int = 0):
        """skin <= 0 keeps the current skin."""
        if skin <= 0:
            skin = self.tuning()["skin"]
        t = _abi.Tuning(dem_variant=dem_variant, rebuild_per_sm=rebuild_per_sm, skin=skin,
                        nbgs_sweeps=nbgs_sweeps, dem_grid=dem_grid, dem_split=dem_split)
        self._check(self._L.pe_b200_set_tuning(self._h, C.byref(t)))

    def autotune(self, dt: float, trial_steps: int = 100) -> dict:
        """Times candidate launch shapes and skins from the current state and keeps the fastest
        (the state is restored)."""
        t = _abi.Tuning()
        self._check(self._L.pe_b200_autotune(self._h, float(dt), int(trial_steps), C.byref(t)))
        return {k: getattr(t, k) for k, _ in _abi.Tuning._fields_}

    def neighbor_list_stats(self) -> dict:
        r, e, c = C.c_int64(), C.c_int64(), C.c_int64()
        sk = C.c_double()
        self._check(self._L.pe_b200_neighbor_list_stats(self._h, C.byref(r), C.byref(e),
                                                        C.byref(c), C.byref(sk)))
        return {"rebuilds": r.value, "entries": e.value, "capacity": c.value, "skin": sk.value}

    def last_error(self) -> str:
        m = self._L.pe_b200_last_error(self._h)
        return m.decode() if m else ""

    def validate(self) -> int:
        """Number of inconsistencies in the device state: a body twice in one colour of the last
        HCSITS step, or a malformed / asymmetric DEM neighbour list (0 = consistent)."""
        p = C.c_int64()
        self._check(self._L.pe_b200_validate(self._h, C.byref(p)))
        return int(p.value)

    def selftest_timeout(self, polls: int = 100000) -> int:
        """Runs the bounded-wait self-test kernel; returns its status code (expected:
        _abi.ERR_TIMEOUT) without raising."""
        return int(self._L.pe_b200_selftest_timeout(self._h, int(polls)))

    def kernel_launches(self) -> int:
        return int(self._L.pe_b200_kernel_launches(self._h))

    def stream_ptr(self) -> int:
        return int(self._L.pe_b200_stream(self._h) or 0)
