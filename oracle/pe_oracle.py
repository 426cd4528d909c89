"""ctypes binding of the CPU restatement (oracle/pe_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, the smoke check and the CPU-baseline leg of
bench.py as the checker.  The product path (pe_b200) never imports this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libpe_oracle.so")

FRICTIONLESS = 0
APPROX_COULOMB_DECOUPLING = 1
APPROX_COULOMB_ORTHOGONAL = 2
COULOMB_DECOUPLING = 3
COULOMB_ORTHOGONAL = 4
GENERALIZED_MAX_DISSIPATION = 5


class Material(C.Structure):
    _fields_ = [(f, C.c_double) for f in ("density", "cor", "csf", "cdf", "poisson", "young",
                                          "stiffness", "dampingN", "dampingT")]


class World(C.Structure):
    _fields_ = [("n", C.c_int64), ("x", C.c_void_p), ("v", C.c_void_p), ("w", C.c_void_p),
                ("q", C.c_void_p), ("r", C.c_void_p), ("mat", C.c_void_p),
                ("nplanes", C.c_int32), ("planes", C.c_void_p), ("plane_mat", C.c_void_p),
                ("nboxes", C.c_int32), ("boxes", C.c_void_p), ("box_mat", C.c_void_p),
                ("nmat", C.c_int32), ("mats", C.c_void_p), ("gravity", C.c_double * 3),
                ("damping", C.c_double), ("force_model", C.c_int32),
                ("nmboxes", C.c_int32), ("mb_x", C.c_void_p), ("mb_q", C.c_void_p),
                ("mb_v", C.c_void_p), ("mb_w", C.c_void_p), ("mb_len", C.c_void_p),
                ("mb_mat", C.c_void_p)]


class Contact(C.Structure):
    _fields_ = [("b1", C.c_int64), ("b2", C.c_int64), ("gpos", C.c_double * 3),
                ("n", C.c_double * 3), ("dist", C.c_double), ("kind", C.c_int64)]


# kind: 0 vertex/face, 1 edge/edge (no DEM force: pe's edge/edge contacts have zero stiffness)
CONTACT_DTYPE = np.dtype([("b1", "<i8"), ("b2", "<i8"), ("gpos", "<f8", 3), ("n", "<f8", 3),
                          ("dist", "<f8"), ("kind", "<i8")])


def as_contacts(c) -> np.ndarray:
    """A contact array in CONTACT_DTYPE (records without a kind are vertex/face contacts)."""
    c = np.asarray(c)
    out = np.zeros(c.shape[0], CONTACT_DTYPE)
    for f in CONTACT_DTYPE.names:
        if f in c.dtype.names:
            out[f] = c[f]
    return out

_lib = None


def build() -> str:
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        L.pe_or_find_contacts.restype = C.c_int64
        L.pe_or_find_contacts.argtypes = [C.POINTER(World), C.c_void_p, C.c_int64]
        L.pe_or_dem_step.restype = C.c_int64
        L.pe_or_dem_step.argtypes = [C.POINTER(World), C.c_double]
        L.pe_or_hcsits_step.restype = C.c_int64
        L.pe_or_hcsits_step.argtypes = [C.POINTER(World), C.c_double, C.c_int, C.c_int,
                                        C.c_double, C.c_void_p, C.c_int64,
                                        C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.pe_or_hcsits_step_contacts.restype = C.c_int64
        L.pe_or_hcsits_step_contacts.argtypes = [C.POINTER(World), C.c_double, C.c_int, C.c_int,
                                                 C.c_double, C.c_void_p, C.c_int64,
                                                 C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.pe_or_sphere_mass.restype = None
        L.pe_or_sphere_mass.argtypes = [C.c_double, C.c_double, C.POINTER(C.c_double),
                                        C.POINTER(C.c_double), C.POINTER(C.c_double)]
        _lib = L
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data


class OracleWorld:
    """FP64 CPU world holding a copy of a pe_b200.scenes.Scene."""

    def __init__(self, scene, track_orientation: bool = False, force_model: int = 0):
        """force_model: pe's DEMConfig forceModel, 0 basic (linear), 1 hertz."""
        s = scene
        self.force_model = int(force_model)
        self.x = np.ascontiguousarray(s.x, np.float64).copy()
        self.v = np.ascontiguousarray(s.v, np.float64).copy()
        self.w = np.ascontiguousarray(s.w, np.float64).copy()
        self.q = None
        if track_orientation:
            self.q = np.zeros((s.n, 4))
            self.q[:, 0] = 1.0
        self.r = np.ascontiguousarray(s.r, np.float64)
        self.mat = np.ascontiguousarray(s.mat, np.int32)
        self.planes = np.ascontiguousarray(s.planes, np.float64).reshape(-1, 4)
        self.plane_mat = np.ascontiguousarray(s.plane_mat, np.int32)
        self.boxes = np.ascontiguousarray(s.boxes, np.float64).reshape(-1, 15)
        self.box_mat = np.ascontiguousarray(s.box_mat, np.int32)
        self.mats = np.ascontiguousarray(s.materials, np.float64).reshape(-1, 9)
        self.gravity = np.asarray(s.gravity, np.float64)
        self.damping = float(s.damping)
        self.n = s.n
        self.nwalls = self.planes.shape[0] + self.boxes.shape[0]
        # moving boxes (bodies n + nwalls + m)
        nmb = int(getattr(s, "nmbox", 0))
        self.nmbox = nmb
        self.mb_x = np.ascontiguousarray(s.mbox_x if nmb else np.zeros((0, 3)), np.float64).copy()
        self.mb_q = np.ascontiguousarray(s.mbox_q if nmb else np.zeros((0, 4)), np.float64).copy()
        self.mb_v = np.ascontiguousarray(s.mbox_v if nmb else np.zeros((0, 3)), np.float64).copy()
        self.mb_w = np.ascontiguousarray(s.mbox_w if nmb else np.zeros((0, 3)), np.float64).copy()
        self.mb_len = np.ascontiguousarray(s.mbox_len if nmb else np.zeros((0, 3)), np.float64)
        self.mb_mat = np.ascontiguousarray(s.mbox_mat if nmb else np.zeros(0), np.int32)

    def _struct(self) -> World:
        w = World()
        w.n = self.n
        w.x, w.v, w.w, w.q = _ptr(self.x), _ptr(self.v), _ptr(self.w), _ptr(self.q)
        w.r, w.mat = _ptr(self.r), _ptr(self.mat)
        w.nplanes, w.planes, w.plane_mat = self.planes.shape[0], _ptr(self.planes), _ptr(self.plane_mat)
        w.nboxes, w.boxes, w.box_mat = self.boxes.shape[0], _ptr(self.boxes), _ptr(self.box_mat)
        w.nmat, w.mats = self.mats.shape[0], _ptr(self.mats)
        for a in range(3):
            w.gravity[a] = self.gravity[a]
        w.damping = self.damping
        w.force_model = self.force_model
        w.nmboxes = self.nmbox
        w.mb_x, w.mb_q, w.mb_v, w.mb_w = (_ptr(self.mb_x), _ptr(self.mb_q), _ptr(self.mb_v),
                                          _ptr(self.mb_w))
        w.mb_len, w.mb_mat = _ptr(self.mb_len), _ptr(self.mb_mat)
        return w

    def contacts(self) -> np.ndarray:
        s = self._struct()
        n = lib().pe_or_find_contacts(C.byref(s), None, 0)
        if n < 0:
            raise MemoryError("oracle contact detection failed")
        out = np.zeros(n, dtype=CONTACT_DTYPE)
        m = lib().pe_or_find_contacts(C.byref(s), _ptr(out) if n else None, n)
        assert m == n
        return out

    def pairs(self) -> np.ndarray:
        c = self.contacts()
        return np.stack([c["b1"], c["b2"]], axis=1).astype(np.int64)

    def dem_step(self, dt: float, steps: int = 1) -> int:
        s = self._struct()
        nc = 0
        for _ in range(steps):
            nc = lib().pe_or_dem_step(C.byref(s), dt)
            if nc < 0:
                raise MemoryError("oracle DEM step failed")
        return nc

    def hcsits_step(self, dt: float, model: int = FRICTIONLESS, max_iter: int = 100,
                    erp: float = 0.7, order=None, contacts=None):
        s = self._struct()
        delta, resid = C.c_double(0.0), C.c_double(0.0)
        if contacts is not None:
            contacts = as_contacts(contacts)
            nc = lib().pe_or_hcsits_step_contacts(C.byref(s), dt, model, max_iter, erp,
                                                  _ptr(contacts), contacts.shape[0],
                                                  C.byref(delta), C.byref(resid))
        else:
            o = None if order is None else np.ascontiguousarray(order, np.int64)
            nc = lib().pe_or_hcsits_step(C.byref(s), dt, model, max_iter, erp, _ptr(o),
                                         0 if o is None else o.shape[0], C.byref(delta),
                                         C.byref(resid))
        if nc < 0:
            raise RuntimeError(f"oracle hard-contact step failed ({nc})")
        return nc, delta.value, resid.value


def sphere_mass(r: float, density: float):
    im, ii, I = C.c_double(), C.c_double(), C.c_double()
    lib().pe_or_sphere_mass(r, density, C.byref(im), C.byref(ii), C.byref(I))
    return im.value, ii.value, I.value
