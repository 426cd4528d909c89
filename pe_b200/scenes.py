"""Seeded synthetic scenes for the rigid-body step.

A scene is the input of one pe ``World``: spheres (FP64 position, velocity, angular velocity,
radius, material id), fixed walls (planes and boxes), a material table and the global gravity.
The generators below build the benchmark workloads with the shapes, sizes and value
distributions of the reference configurations; all randomness comes from a numpy ``Generator``
seeded by the caller, so both sides of every parity test see byte-identical inputs.

Material parameters follow pe's composition rules (pe/core/Materials.h:633-715,
src/core/Materials.cpp:232-246): contact stiffness and damping are harmonic means of the two
materials' values and friction is the sum, so a same-material contact with normal stiffness
``k_n``, damping ``c_n`` and friction ``mu`` needs material stiffness ``2 k_n``, damping
``2 c_n`` and static = dynamic friction ``mu / 2``.
"""
from __future__ import annotations

import dataclasses
import struct
from typing import List, Optional

import numpy as np

# one material record = the argument list of pe's createMaterial (src/core/Materials.cpp:175)
MATERIAL_FIELDS = ("density", "cor", "csf", "cdf", "poisson", "young", "stiffness",
                   "dampingN", "dampingT")

SCENE_MAGIC = b"PEB2SCN\0"
SCENE_VERSION = 1


def material(density: float, k_n: float, c_n: float, c_t: float, mu: float,
             cor: float = 0.0, poisson: float = 0.25, young: float = 1e9) -> np.ndarray:
    """Material record whose same-material contact has the given k_n, c_n, c_t and mu."""
    return np.array([density, cor, 0.5 * mu, 0.5 * mu, poisson, young, 2.0 * k_n, 2.0 * c_n,
                     2.0 * c_t], dtype=np.float64)


@dataclasses.dataclass
class Scene:
    x: np.ndarray            # (n, 3) f64 sphere centres
    v: np.ndarray            # (n, 3) f64 linear velocities
    w: np.ndarray            # (n, 3) f64 angular velocities
    r: np.ndarray            # (n,)   f64 radii
    mat: np.ndarray          # (n,)   i32 material ids
    planes: np.ndarray       # (P, 4) f64 unit normal + displacement (n.x = d on the plane)
    plane_mat: np.ndarray    # (P,)   i32
    boxes: np.ndarray        # (B, 15) f64 centre, side lengths, rotation (row-major 3x3)
    box_mat: np.ndarray      # (B,)   i32
    materials: np.ndarray    # (M, 9) f64, fields MATERIAL_FIELDS
    gravity: np.ndarray      # (3,)   f64
    dt: float
    steps: int
    name: str = ""
    damping: float = 1.0     # pe Settings::damping (1 = no drag)
    # moving (non-fixed) boxes, created in pe after the fixed boxes
    mbox_x: np.ndarray = dataclasses.field(default_factory=lambda: np.zeros((0, 3)))
    mbox_q: np.ndarray = dataclasses.field(default_factory=lambda: np.zeros((0, 4)))  # w x y z
    mbox_v: np.ndarray = dataclasses.field(default_factory=lambda: np.zeros((0, 3)))
    mbox_w: np.ndarray = dataclasses.field(default_factory=lambda: np.zeros((0, 3)))
    mbox_len: np.ndarray = dataclasses.field(default_factory=lambda: np.zeros((0, 3)))
    mbox_mat: np.ndarray = dataclasses.field(default_factory=lambda: np.zeros(0, np.int32))

    @property
    def n(self) -> int:
        return int(self.r.shape[0])

    @property
    def nmbox(self) -> int:
        return int(self.mbox_len.shape[0])

    def copy(self) -> "Scene":
        return dataclasses.replace(self, **{f.name: (getattr(self, f.name).copy()
                                                     if isinstance(getattr(self, f.name), np.ndarray)
                                                     else getattr(self, f.name))
                                            for f in dataclasses.fields(self)})

    # --- binary scene file (read by the compiled-reference driver and the C++ host layer) ---
    def to_bytes(self) -> bytes:
        """Version 1 without moving boxes (the layout the compiled-reference driver reads);
        version 2 appends uint32 M and the moving boxes' x, q, v, w, side lengths, materials."""
        ver = SCENE_VERSION if self.nmbox == 0 else 2
        hdr = struct.pack("<8sIIQII3dddI", SCENE_MAGIC, ver, self.materials.shape[0],
                          self.n, self.planes.shape[0], self.boxes.shape[0],
                          *[float(g) for g in self.gravity], float(self.dt),
                          float(self.damping), int(self.steps))
        parts = [hdr,
                 np.ascontiguousarray(self.materials, "<f8").tobytes(),
                 np.ascontiguousarray(self.planes, "<f8").tobytes(),
                 np.ascontiguousarray(self.plane_mat, "<i4").tobytes(),
                 np.ascontiguousarray(self.boxes, "<f8").tobytes(),
                 np.ascontiguousarray(self.box_mat, "<i4").tobytes(),
                 np.ascontiguousarray(self.x, "<f8").tobytes(),
                 np.ascontiguousarray(self.v, "<f8").tobytes(),
                 np.ascontiguousarray(self.w, "<f8").tobytes(),
                 np.ascontiguousarray(self.r, "<f8").tobytes(),
                 np.ascontiguousarray(self.mat, "<i4").tobytes()]
        if ver == 2:
            parts += [struct.pack("<I", self.nmbox),
                      np.ascontiguousarray(self.mbox_x, "<f8").tobytes(),
                      np.ascontiguousarray(self.mbox_q, "<f8").tobytes(),
                      np.ascontiguousarray(self.mbox_v, "<f8").tobytes(),
                      np.ascontiguousarray(self.mbox_w, "<f8").tobytes(),
                      np.ascontiguousarray(self.mbox_len, "<f8").tobytes(),
                      np.ascontiguousarray(self.mbox_mat, "<i4").tobytes()]
        return b"".join(parts)

    def save(self, path: str) -> None:
        with open(path, "wb") as f:
            f.write(self.to_bytes())


def scene_from_bytes(buf: bytes, name: str = "") -> Scene:
    fmt = "<8sIIQII3dddI"
    hs = struct.calcsize(fmt)
    if len(buf) < hs:
        raise ValueError("truncated scene file")
    magic, ver, nm, n, npl, nbx, gx, gy, gz, dt, damping, steps = struct.unpack_from(fmt, buf, 0)
    if magic != SCENE_MAGIC or ver not in (1, 2):
        raise ValueError("not a scene file")
    base = hs + 72 * nm + 36 * npl + 124 * nbx + 84 * n
    nmb = 0
    if ver == 2:
        if len(buf) < base + 4:
            raise ValueError("truncated scene file")
        nmb, = struct.unpack_from("<I", buf, base)
    if len(buf) != base + (4 + 132 * nmb if ver == 2 else 0):
        raise ValueError("scene file size does not match its header")
    off = hs

    def take(dtype, count, shape):
        nonlocal off
        a = np.frombuffer(buf, dtype=dtype, count=count, offset=off).reshape(shape).copy()
        off += a.nbytes
        return a

    materials = take("<f8", nm * 9, (nm, 9))
    planes = take("<f8", npl * 4, (npl, 4))
    plane_mat = take("<i4", npl, (npl,))
    boxes = take("<f8", nbx * 15, (nbx, 15))
    box_mat = take("<i4", nbx, (nbx,))
    x = take("<f8", n * 3, (n, 3))
    v = take("<f8", n * 3, (n, 3))
    w = take("<f8", n * 3, (n, 3))
    r = take("<f8", n, (n,))
    mat = take("<i4", n, (n,))
    s = Scene(x=x, v=v, w=w, r=r, mat=mat, planes=planes, plane_mat=plane_mat, boxes=boxes,
              box_mat=box_mat, materials=materials, gravity=np.array([gx, gy, gz]), dt=dt,
              steps=steps, name=name, damping=damping)
    if ver == 2:
        off += 4
        s.mbox_x = take("<f8", nmb * 3, (nmb, 3))
        s.mbox_q = take("<f8", nmb * 4, (nmb, 4))
        s.mbox_v = take("<f8", nmb * 3, (nmb, 3))
        s.mbox_w = take("<f8", nmb * 3, (nmb, 3))
        s.mbox_len = take("<f8", nmb * 3, (nmb, 3))
        s.mbox_mat = take("<i4", nmb, (nmb,))
    return s


def load_scene(path: str) -> Scene:
    with open(path, "rb") as f:
        return scene_from_bytes(f.read(), name=path)


# ------------------------------------------------------------------------------------------
# geometry helpers
# ------------------------------------------------------------------------------------------

def box_planes(lo, hi) -> np.ndarray:
    """Six inward-facing planes bounding the box [lo, hi] (pe createPlane(normal, d))."""
    lo = np.asarray(lo, float)
    hi = np.asarray(hi, float)
    p = []
    for a in range(3):
        e = np.zeros(3)
        e[a] = 1.0
        p.append(np.r_[e, lo[a]])        # e.x >= lo
        p.append(np.r_[-e, -hi[a]])      # -e.x >= -hi
    return np.array(p)


def aabox(centre, lengths) -> np.ndarray:
    """Axis-aligned fixed box record: centre, side lengths, identity rotation."""
    return np.r_[np.asarray(centre, float), np.asarray(lengths, float),
                 np.eye(3).ravel()].astype(np.float64)


def _jittered_lattice(rng, n, lo, counts, spacing, r, pick_random=True):
    """Place n spheres on distinct random sites of a lattice, each jittered inside its slack.

    Sites are ``lo + (idx + 0.5) * spacing``; a sphere of radius r_i moves by at most
    ``(min(spacing) - 2 r_max)/2`` per axis, so no two spheres overlap."""
    counts = np.asarray(counts)
    spacing = np.asarray(spacing, float)
    nsites = int(np.prod(counts))
    if nsites < n:
        raise ValueError("lattice too small")
    sites = rng.choice(nsites, size=n, replace=False) if pick_random else np.arange(n)
    iz = sites // (counts[0] * counts[1])
    iy = (sites // counts[0]) % counts[1]
    ix = sites % counts[0]
    idx = np.stack([ix, iy, iz], axis=1).astype(float)
    x = np.asarray(lo, float) + (idx + 0.5) * spacing
    slack = np.maximum(0.0, 0.5 * spacing.min() - r)[:, None]
    x += rng.uniform(-1.0, 1.0, size=(n, 3)) * slack * 0.98
    return x


def _scene(x, v, r, mat, planes, plane_mat, boxes, box_mat, materials, gravity, dt, steps,
           name) -> Scene:
    n = r.shape[0]
    return Scene(x=np.ascontiguousarray(x, np.float64), v=np.ascontiguousarray(v, np.float64),
                 w=np.zeros((n, 3)), r=np.ascontiguousarray(r, np.float64),
                 mat=np.ascontiguousarray(mat, np.int32),
                 planes=np.asarray(planes, np.float64).reshape(-1, 4),
                 plane_mat=np.asarray(plane_mat, np.int32).reshape(-1),
                 boxes=np.asarray(boxes, np.float64).reshape(-1, 15),
                 box_mat=np.asarray(box_mat, np.int32).reshape(-1),
                 materials=np.asarray(materials, np.float64).reshape(-1, 9),
                 gravity=np.asarray(gravity, np.float64), dt=float(dt), steps=int(steps),
                 name=name)


G = (0.0, 0.0, -9.81)


# ------------------------------------------------------------------------------------------
# the workloads
# ------------------------------------------------------------------------------------------

def dem_lattice(seed: int = 0, side: int = 16, c_t: float = 50.0) -> Scene:
    """Plain DEM, CPU-runnable: side^3 monodisperse spheres (r=0.5, density 1) on a lattice of
    spacing 1.05 with uniform jitter +-0.02, velocities N(0, 0.1^2), closed box of six planes,
    linear spring-dashpot k_n=1e5, c_n=50, mu=0.3, dt=1e-4, 1000 steps.  pe has no tangential
    spring; its tangential law is damping-limited Coulomb with damping c_t (default 50)."""
    rng = np.random.default_rng(seed)
    n = side ** 3
    spacing = 1.05
    idx = np.stack(np.meshgrid(np.arange(side), np.arange(side), np.arange(side),
                               indexing="ij"), axis=-1).reshape(-1, 3)[:, ::-1].astype(float)
    x = (idx + 0.5) * spacing + rng.uniform(-0.02, 0.02, size=(n, 3))
    v = rng.normal(0.0, 0.1, size=(n, 3))
    r = np.full(n, 0.5)
    L = side * spacing
    planes = box_planes([0, 0, 0], [L, L, L])
    mats = [material(1.0, 1e5, 50.0, c_t, 0.3)]
    return _scene(x, v, r, np.zeros(n), planes, np.zeros(6), np.zeros((0, 15)), [], mats, G,
                  1e-4, 1000, f"dem_lattice_{n}")


def nbgs_box(seed: int = 0, n: int = 32768, mu: float = 0.0, dims=(40.0, 40.0, 120.0),
             dense: bool = False) -> Scene:
    """Hard-contact workload: n spheres with radii U[0.4, 0.6] at random non-overlapping
    positions in a box of plane walls, settling under gravity, dt=1e-3, 200 steps.

    dense=True packs the spheres at the bottom of the box on a lattice of spacing 1.0 (radii
    U[0.45, 0.55], so neighbouring spheres start in contact) to exercise the contact sweeps."""
    rng = np.random.default_rng(seed)
    dims = np.asarray(dims, float)
    if dense:
        r = rng.uniform(0.45, 0.55, size=n)
        nx = int(dims[0] // 1.0)
        ny = int(dims[1] // 1.0)
        nz = int(np.ceil(n / (nx * ny)))
        x = _jittered_lattice(rng, n, [0.0, 0.0, 0.0], [nx, ny, nz], [1.0, 1.0, 1.0],
                              r, pick_random=False)
        x += 0.002 * rng.uniform(-1, 1, size=x.shape)
        name = f"nbgs_dense_{n}"
    else:
        r = rng.uniform(0.4, 0.6, size=n)
        nx = ny = int(dims[0] // 1.8)
        nz = int(np.ceil(n / (nx * ny)))
        sp = np.array([dims[0] / nx, dims[1] / ny, dims[2] / nz])
        x = _jittered_lattice(rng, n, [0, 0, 0], [nx, ny, nz], sp, r)
        name = f"nbgs_box_{n}"
    planes = box_planes([0, 0, 0], dims)
    mats = [material(1.0, 1e5, 50.0, 50.0, mu)]
    return _scene(x, np.zeros((n, 3)), r, np.zeros(n), planes, np.zeros(6), np.zeros((0, 15)),
                  [], mats, G, 1e-3, 200, name + ("_mu%.2g" % mu))


def _layered_pack(rng, r, lo, width, solid_fraction):
    """Non-overlapping packing of spheres with radii r: radii sorted descending are laid out
    in horizontal square-lattice layers whose spacing follows the largest radius of the layer,
    scaled to reach the requested solid fraction.  Returns centres in the input order."""
    n = r.shape[0]
    order = np.argsort(-r, kind="stable")
    f = (np.pi / 6.0 / solid_fraction) ** (1.0 / 3.0)
    x = np.empty((n, 3))
    z = lo[2]
    i = 0
    while i < n:
        rmax = r[order[i]]
        s = 2.0 * rmax * f
        m = int(width[0] // s)
        k = int(width[1] // s)
        cnt = min(m * k, n - i)
        ids = order[i:i + cnt]
        sites = rng.permutation(m * k)[:cnt]
        x[ids, 0] = lo[0] + (sites % m + 0.5) * s
        x[ids, 1] = lo[1] + (sites // m + 0.5) * s
        x[ids, 2] = z + 0.5 * s
        slack = np.maximum(0.0, 0.5 * s - r[ids])[:, None]
        x[ids] += rng.uniform(-1, 1, size=(cnt, 3)) * slack * 0.98
        z += s
        i += cnt
    return x


def dem_large(seed: int = 0, n: int = 1048576, dims=(200.0, 200.0, 400.0)) -> Scene:
    """Large DEM: n spheres with log-normal radii (median 0.5, sigma_log 0.2, clipped to
    [0.3, 0.9]) in a random non-overlapping packing at 30% solid fraction filling a slab at the
    bottom of a 200x200x400 box of planes; k_n=1e5, c_n=50, mu=0.4, dt=5e-5, 1000 steps."""
    rng = np.random.default_rng(seed)
    dims = np.asarray(dims, float)
    r = np.clip(np.exp(np.log(0.5) + 0.2 * rng.standard_normal(n)), 0.3, 0.9)
    x = _layered_pack(rng, r, np.array([0.0, 0.0, 0.0]), dims, 0.30)
    v = rng.normal(0.0, 0.1, size=(n, 3))
    planes = box_planes([0, 0, 0], dims)
    mats = [material(1.0, 1e5, 50.0, 50.0, 0.4)]
    return _scene(x, v, r, np.zeros(n), planes, np.zeros(6), np.zeros((0, 15)), [], mats, G,
                  5e-5, 1000, f"dem_large_{n}")


def dem_dense(seed: int = 0, nx: int = 128, ny: int = 128, nz: int = 64) -> Scene:
    """Contact-dense DEM: nx*ny*nz spheres (1,048,576 by default) on a simple cubic lattice of
    spacing 1.0 with radii U[0.495, 0.505], so most lattice neighbours start in contact, filling
    the lower half of a box of planes whose side walls touch the outer spheres; velocities
    N(0, 0.5^2); k_n=1e5, c_n=50, mu=0.4, dt=5e-5.  Every sphere feels contact forces every step
    and the released overlaps keep the packing agitated, so the lists are rebuilt often."""
    rng = np.random.default_rng(seed)
    n = nx * ny * nz
    idx = np.stack(np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij"),
                   axis=-1).reshape(-1, 3).astype(float)
    x = idx + 0.5
    r = rng.uniform(0.495, 0.505, size=n)
    v = rng.normal(0.0, 0.5, size=(n, 3))
    dims = np.array([float(nx), float(ny), 2.0 * nz])
    planes = box_planes([0, 0, 0], dims)
    mats = [material(1.0, 1e5, 50.0, 50.0, 0.4)]
    return _scene(x, v, r, np.zeros(n), planes, np.zeros(6), np.zeros((0, 15)), [], mats, G,
                  5e-5, 1000, f"dem_dense_{n}")


def batched_ensemble(seed: int = 0, scenes: int = 512, nmin: int = 1024,
                     nmax: int = 65536) -> List[Scene]:
    """Batched ensemble: independent DEM scenes with body counts log-uniform in [nmin, nmax],
    radii U[0.45, 0.55], per-scene mu ~ U[0.1, 0.8] and c_n ~ U[10, 100], k_n=1e5, each in its
    own box with gravity, dt=1e-4, 500 steps."""
    rng = np.random.default_rng(seed)
    counts = np.exp(rng.uniform(np.log(nmin), np.log(nmax), size=scenes)).astype(np.int64)
    out = []
    for s in range(scenes):
        n = int(counts[s])
        mu = float(rng.uniform(0.1, 0.8))
        c_n = float(rng.uniform(10.0, 100.0))
        r = rng.uniform(0.45, 0.55, size=n)
        side = int(np.ceil((n / 2.0) ** (1.0 / 3.0)))
        nz = int(np.ceil(n / (side * side)))
        sp = 1.15
        x = _jittered_lattice(rng, n, [0, 0, 0], [side, side, nz], [sp, sp, sp], r)
        dims = np.array([side * sp, side * sp, nz * sp * 1.5])
        v = rng.normal(0.0, 0.1, size=(n, 3))
        mats = [material(1.0, 1e5, c_n, c_n, mu)]
        out.append(_scene(x, v, r, np.zeros(n), box_planes([0, 0, 0], dims), np.zeros(6),
                          np.zeros((0, 15)), [], mats, G, 1e-4, 500, f"ens{s}_{n}"))
    return out


def hopper(seed: int = 0, n: int = 16384) -> Scene:
    """Differentiable DEM workload: n spheres (r ~ U[0.45, 0.55]) released from a random packing
    in a 30x30x60 hopper of fixed boxes whose bottom plate has a centred 6x6 opening above a
    floor plane; dt=1e-4, 2000 steps."""
    rng = np.random.default_rng(seed)
    r = rng.uniform(0.45, 0.55, size=n)
    zb = 10.0                       # bottom plate top surface
    W, H, t = 30.0, 60.0, 1.0       # inner width, height, wall thickness
    hole = 6.0
    sp = 1.12
    m = int(W // sp)
    nz = int(np.ceil(n / (m * m)))
    x = _jittered_lattice(rng, n, [0.0, 0.0, zb], [m, m, nz], [sp, sp, sp], r)
    boxes = []
    c = W / 2.0
    # side walls
    boxes.append(aabox([-t / 2, c, zb + H / 2], [t, W + 2 * t, H]))
    boxes.append(aabox([W + t / 2, c, zb + H / 2], [t, W + 2 * t, H]))
    boxes.append(aabox([c, -t / 2, zb + H / 2], [W, t, H]))
    boxes.append(aabox([c, W + t / 2, zb + H / 2], [W, t, H]))
    # bottom plate made of four slabs around the opening
    a = (W - hole) / 2.0
    boxes.append(aabox([a / 2, c, zb - t / 2], [a, W, t]))
    boxes.append(aabox([W - a / 2, c, zb - t / 2], [a, W, t]))
    boxes.append(aabox([c, a / 2, zb - t / 2], [hole, a, t]))
    boxes.append(aabox([c, W - a / 2, zb - t / 2], [hole, a, t]))
    planes = np.array([[0.0, 0.0, 1.0, 0.0]])
    mats = [material(1.0, 1e5, 50.0, 50.0, 0.4)]
    return _scene(x, np.zeros((n, 3)), r, np.zeros(n), planes, [0], np.array(boxes),
                  np.zeros(len(boxes)), mats, G, 1e-4, 2000, f"hopper_{n}")


def small_random(seed: int, n: int = 64, box: float = 4.0, overlap: float = 0.05,
                 mu: float = 0.3, with_boxes: bool = False, spin: float = 1.0) -> Scene:
    """Small scene with many simultaneous contacts (spheres start slightly overlapping each
    other and the walls) for unit parity tests."""
    rng = np.random.default_rng(seed)
    side = int(np.ceil(n ** (1.0 / 3.0)))
    r = rng.uniform(0.4, 0.6, size=n)
    sp = 1.0 - overlap
    idx = np.stack(np.meshgrid(np.arange(side), np.arange(side), np.arange(side),
                               indexing="ij"), axis=-1).reshape(-1, 3)[:n, ::-1].astype(float)
    x = (idx + 0.5) * sp + rng.uniform(-0.05, 0.05, size=(n, 3))
    v = rng.normal(0.0, 0.5, size=(n, 3))
    L = side * sp
    planes = box_planes([0, 0, 0], [L, L, L + 2.0])
    boxes = np.zeros((0, 15))
    if with_boxes:
        boxes = np.array([aabox([L / 2, L / 2, -0.45 + 0.1], [L / 2, L / 2, 1.0]),
                          aabox([-0.4, L / 2, L / 2], [1.0, L, L])])
    mats = [material(1.0, 1e5, 50.0, 40.0, mu), material(2.0, 2e5, 30.0, 20.0, mu * 0.5)]
    mat = rng.integers(0, 2, size=n)
    s = _scene(x, v, r, mat, planes, np.arange(6) % 2, boxes, np.zeros(len(boxes)), mats, G,
               1e-4, 10, f"small_{seed}_{n}")
    s.w = rng.normal(0.0, spin, size=(n, 3))
    return s


def random_quaternions(rng, m: int) -> np.ndarray:
    """m uniformly distributed unit quaternions (w, x, y, z)."""
    q = rng.normal(size=(m, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    q[q[:, 0] < 0] *= -1.0
    return q


def small_rotations(rng, m: int, max_angle: float) -> np.ndarray:
    """m unit quaternions (w, x, y, z) of rotations by U[0, max_angle] about random axes."""
    ax = rng.normal(size=(m, 3))
    ax /= np.linalg.norm(ax, axis=1, keepdims=True)
    ang = rng.uniform(0.0, max_angle, size=m)
    return np.concatenate([np.cos(ang / 2)[:, None], np.sin(ang / 2)[:, None] * ax], axis=1)


def tumbling_boxes(seed: int = 0, side: int = 3, max_angle: float = 0.3, mu: float = 0.3,
                   spheres: bool = True) -> Scene:
    """side^3 moving boxes (side lengths U[0.75, 0.95], tilted by up to max_angle about random
    axes) on a unit lattice resting on a floor plane, a fixed box against one column, and one
    sphere in every lattice corner between eight boxes; random velocities and spins, gravity.
    Tilted neighbours overlap slightly, so the first steps have face/face, edge/edge,
    box/plane, box/fixed-box and sphere/box contacts."""
    rng = np.random.default_rng(seed)
    nbox = side ** 3
    idx = np.stack(np.meshgrid(np.arange(side), np.arange(side), np.arange(side),
                               indexing="ij"), axis=-1).reshape(-1, 3)[:, ::-1].astype(float)
    bx = idx + np.array([1.5, 1.5, 0.5]) + rng.uniform(-0.02, 0.02, size=(nbox, 3))
    blen = rng.uniform(0.75, 0.95, size=(nbox, 3))
    bq = small_rotations(rng, nbox, max_angle)
    bv = rng.normal(0.0, 0.2, size=(nbox, 3))
    bw = rng.normal(0.0, 0.5, size=(nbox, 3))
    if spheres:
        cidx = np.stack(np.meshgrid(np.arange(side - 1), np.arange(side - 1),
                                    np.arange(side - 1), indexing="ij"),
                        axis=-1).reshape(-1, 3)[:, ::-1].astype(float)
        sx = cidx + np.array([2.0, 2.0, 1.0]) + rng.uniform(-0.02, 0.02, size=cidx.shape)
    else:
        sx = np.zeros((0, 3))
    ns = sx.shape[0]
    r = rng.uniform(0.3, 0.4, size=ns)
    L = side + 3.0
    planes = box_planes([0, 0, 0], [L, L, L + 4.0])
    boxes = np.array([aabox([0.5, 1.5 + (side - 1) / 2.0, 1.0], [1.0 - 0.02, side, 2.0])])
    mats = [material(1.0, 2e4, 20.0, 20.0, mu), material(0.5, 3e4, 10.0, 10.0, 0.5 * mu)]
    s = _scene(sx, rng.normal(0.0, 0.2, size=(ns, 3)), r, rng.integers(0, 2, size=ns),
               planes, np.arange(6) % 2, boxes, [1], mats, G, 1e-4, 20,
               f"tumbling_boxes_{seed}_{nbox}")
    s.w = rng.normal(0.0, 0.5, size=(ns, 3))
    s.mbox_x, s.mbox_q, s.mbox_v, s.mbox_w = bx, bq, bv, bw
    s.mbox_len = blen
    s.mbox_mat = rng.integers(0, 2, size=nbox).astype(np.int32)
    return s


def box_stack(layers: int = 4, per_side: int = 3, overlap: float = 1e-4) -> Scene:
    """pe's box-stack arrangement: layers of equal, axis-aligned cubes resting face to face on
    a floor plane (the degenerate, fully aligned case of the box/box test), plus one sphere
    flying into the stack."""
    a = 1.0
    pts = []
    for z in range(layers):
        for y in range(per_side):
            for x in range(per_side):
                pts.append([x * a, y * a, 0.5 * a + z * a - overlap * (z + 1)])
    bx = np.array(pts) + np.array([2.0, 2.0, 0.0])
    nb = bx.shape[0]
    planes = np.array([[0.0, 0.0, 1.0, 0.0]])
    mats = [material(1.0, 1e5, 50.0, 50.0, 0.4)]
    s = _scene(np.array([[2.0 + per_side * a / 2, -1.0, 1.5]]), np.array([[0.0, 3.0, 0.0]]),
               np.array([0.4]), [0], planes, [0], np.zeros((0, 15)), [], mats, G, 1e-4, 20,
               f"box_stack_{layers}x{per_side}")
    s.mbox_x = bx
    s.mbox_q = np.tile([1.0, 0.0, 0.0, 0.0], (nb, 1))
    s.mbox_v = np.zeros((nb, 3))
    s.mbox_w = np.zeros((nb, 3))
    s.mbox_len = np.full((nb, 3), a)
    s.mbox_mat = np.zeros(nb, np.int32)
    return s


def spheres_and_boxes(seed: int = 0, sphere_side: int = 48, box_side: int = 10) -> Scene:
    """A mixed DEM scene: the lattice of dem_lattice(seed, sphere_side) with box_side^3 moving
    boxes (side lengths U[0.5, 0.9] of their lattice spacing, tilted up to 0.5 rad) on a coarser
    lattice above the spheres, falling onto them; the box of planes is raised to hold them."""
    rng = np.random.default_rng(seed)
    s = dem_lattice(seed, side=sphere_side)
    nb = box_side ** 3
    idx = np.stack(np.meshgrid(*[np.arange(box_side)] * 3, indexing="ij"),
                   axis=-1).reshape(-1, 3).astype(float)
    top = s.x[:, 2].max() + 2.0
    lo = s.x[:, 0].min()
    sp = (s.x[:, 0].max() - lo) / box_side
    s.mbox_x = np.c_[idx[:, 0] * sp + sp / 2 + lo, idx[:, 1] * sp + sp / 2 + lo,
                     top + idx[:, 2] * sp]
    s.mbox_q = small_rotations(rng, nb, 0.5)
    s.mbox_v = rng.normal(0.0, 0.1, size=(nb, 3))
    s.mbox_w = rng.normal(0.0, 0.1, size=(nb, 3))
    s.mbox_len = rng.uniform(0.5, 0.9, size=(nb, 3)) * sp
    s.mbox_mat = np.zeros(nb, np.int32)
    s.planes[s.planes[:, 2] < -0.5, 3] = -(top + box_side * sp + 5.0)
    s.name = f"spheres_and_boxes_{s.n}_{nb}"
    return s


WORKLOADS = {
    "dem_lattice_4096": lambda seed=0: dem_lattice(seed),
    "nbgs_box_32768": lambda seed=0: nbgs_box(seed),
    "dem_large_1m": lambda seed=0: dem_large(seed),
    "hopper_16384": lambda seed=0: hopper(seed),
}
