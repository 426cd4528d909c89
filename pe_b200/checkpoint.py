"""pe's binary checkpoint files (".peb"), read and written in pe's own format.

The format is that of pe's BodyBinaryWriter / BodyBinaryReader (src/core/BodyBinaryWriter.cpp,
src/core/BodyBinaryReader.cpp) for one process, all values big-endian (pe's network-order send
buffers, pe/core/BodyBinaryWriter.h:68):

    header   'P' 'E' 0 1, sizeof(real) = 8, sizeof(int) = 4, sizeof(size_t) = 8,
             sizeof(id_t) = 8, sizeof(bool) = 1, uint32 processes = 1,
             uint32 offset of the global chunk, uint32 offset of the local chunk,
             uint32 end of the local chunk
    global   id_t counter, then for the types sphere 1, box 2, capsule 3, cylinder 4, plane 5,
             mesh 6, union 7: byte type, uint32 count, bodies
    local    id_t counter, then the same without planes (pe writes only global planes)
    body     id_t sid, id_t uid, bool visible, bool fixed, position (3 doubles), quaternion
             (w x y z), linear and angular velocity (3 doubles each), MaterialID (size_t);
             a sphere adds its radius, a box its side lengths (pe/core/Marshalling.h:184-200,
             290-293, 321-324, 498-501)

Material ids refer to pe's material table, whose first five entries are pe's predefined
materials (iron, copper, granite, oak, fir); a scene's material k is pe's 5 + k when the scene's
materials are created in order after them, as pe_b200_world.hpp and the compiled reference do.
"""
from __future__ import annotations

import dataclasses
import struct
from typing import List, Optional

import numpy as np

PREDEFINED_MATERIALS = 5
SPHERE, BOX, CAPSULE, CYLINDER, PLANE, MESH, UNION = 1, 2, 3, 4, 5, 6, 7
_GLOBAL_TYPES = (SPHERE, BOX, CAPSULE, CYLINDER, PLANE, MESH, UNION)
_LOCAL_TYPES = (SPHERE, BOX, CAPSULE, CYLINDER, MESH, UNION)


@dataclasses.dataclass
class Body:
    kind: int
    sid: int
    uid: int
    visible: bool
    fixed: bool
    x: np.ndarray           # (3,)
    q: np.ndarray           # (4,) w x y z
    v: np.ndarray           # (3,)
    w: np.ndarray           # (3,)
    material: int
    radius: float = 0.0             # spheres
    lengths: Optional[np.ndarray] = None   # boxes
    global_: bool = False


def _body_bytes(b: Body) -> bytes:
    out = struct.pack(">QQ??", b.sid, b.uid, bool(b.visible), bool(b.fixed))
    out += struct.pack(">3d4d3d3dQ", *np.asarray(b.x, float), *np.asarray(b.q, float),
                       *np.asarray(b.v, float), *np.asarray(b.w, float), b.material)
    if b.kind == SPHERE:
        out += struct.pack(">d", float(b.radius))
    elif b.kind == BOX:
        out += struct.pack(">3d", *np.asarray(b.lengths, float))
    elif b.kind != PLANE:
        raise ValueError("only spheres, boxes and planes are written")
    return out


def _chunk(counter: int, bodies: List[Body], types) -> bytes:
    out = struct.pack(">Q", counter)
    for t in types:
        sel = [b for b in bodies if b.kind == t]
        out += struct.pack(">BI", t, len(sel))
        for b in sel:
            out += _body_bytes(b)
    return out


def write_peb(path: str, bodies: List[Body], counter: int, global_counter: int = 0) -> None:
    """Writes bodies as pe's BodyBinaryWriter::writeFile does on one process (bodies flagged
    global go to the global chunk; planes are written only when global, as in pe)."""
    glob = _chunk(global_counter, [b for b in bodies if b.global_], _GLOBAL_TYPES)
    loc = _chunk(counter, [b for b in bodies if not b.global_ and b.kind != PLANE], _LOCAL_TYPES)
    head = b"PE" + bytes([0, 1, 8, 4, 8, 8, 1]) + struct.pack(">I", 1)
    header_size = len(head) + 3 * 4
    offset = header_size + len(glob)
    head += struct.pack(">III", header_size, offset, offset + len(loc))
    with open(path, "wb") as f:
        f.write(head + glob + loc)


def read_peb(path: str) -> dict:
    """Parses a one-process pe checkpoint: {"counter", "global_counter", "bodies"}; raises
    ValueError with pe's messages for files pe's reader rejects."""
    b = open(path, "rb").read()
    if len(b) < 13 or b[:2] != b"PE":
        raise ValueError("Invalid file format.")
    if (b[2], b[3]) != (0, 1):
        raise ValueError("Unsupported file format version.")
    if b[4] != 8:
        raise ValueError("Invalid size of floating point data.")
    if b[5] != 4 or b[6] != 8 or b[7] != 8 or b[8] != 1:
        raise ValueError("Size of a data type does not match the one used to produce the file.")
    procs, = struct.unpack_from(">I", b, 9)
    if procs != 1:
        raise ValueError("Number of processes differ from the number of processes used to "
                         "produce the file.")
    goff, loff, lend = struct.unpack_from(">III", b, 13)
    if loff < goff or lend < loff or lend > len(b):
        raise ValueError("Invalid body data offset.")

    def parse(p, end, is_global):
        counter, = struct.unpack_from(">Q", b, p)
        p += 8
        out = []
        while p < end:
            kind, count = struct.unpack_from(">BI", b, p)
            p += 5
            for _ in range(count):
                sid, uid, vis, fixed = struct.unpack_from(">QQ??", b, p)
                p += 18
                vals = struct.unpack_from(">3d4d3d3dQ", b, p)
                p += 13 * 8 + 8
                body = Body(kind, sid, uid, vis, fixed, np.array(vals[0:3]), np.array(vals[3:7]),
                            np.array(vals[7:10]), np.array(vals[10:13]), int(vals[13]),
                            global_=is_global)
                if kind == SPHERE:
                    body.radius, = struct.unpack_from(">d", b, p)
                    p += 8
                elif kind == BOX:
                    body.lengths = np.array(struct.unpack_from(">3d", b, p))
                    p += 24
                elif kind != PLANE:
                    raise ValueError("Unsupported geometry type in checkpoint: %d" % kind)
                out.append(body)
        return counter, out

    gc, gb = parse(goff, loff, True)
    lc, lb = parse(loff, lend, False)
    return {"counter": lc, "global_counter": gc, "bodies": gb + lb}


def scene_bodies(scene, x=None, v=None, w=None, q=None,
                 material_offset: int = PREDEFINED_MATERIALS, box_state=None) -> tuple:
    """The bodies of a pe_b200.scenes.Scene in the order pe creates them in the compiled
    reference's driver: spheres (system id = user id = index), then planes, then fixed
    axis-aligned boxes, then moving boxes; returns (bodies, next system id).  x, v, w, q
    override the spheres' state, box_state = (x, q, v, w) the moving boxes'."""
    n = scene.n
    x = scene.x if x is None else x
    v = scene.v if v is None else v
    w = scene.w if w is None else w
    ident = np.array([1.0, 0.0, 0.0, 0.0])
    out = []
    for i in range(n):
        out.append(Body(SPHERE, i, i, True, False, np.asarray(x[i], float),
                        ident if q is None else np.asarray(q[i], float), np.asarray(v[i], float),
                        np.asarray(w[i], float), int(scene.mat[i]) + material_offset,
                        radius=float(scene.r[i])))
    npl = scene.planes.shape[0]
    for p in range(npl):
        nrm, d = scene.planes[p, :3], scene.planes[p, 3]
        out.append(Body(PLANE, n + p, n + p, True, True, nrm * d, ident, np.zeros(3), np.zeros(3),
                        int(scene.plane_mat[p]) + material_offset))
    nb = scene.boxes.shape[0]
    for k in range(nb):
        bx = scene.boxes[k]
        if not np.array_equal(bx[6:], np.eye(3).ravel()):
            raise ValueError("axis-aligned boxes only")
        out.append(Body(BOX, n + npl + k, n + npl + k, True, True, bx[:3].copy(), ident,
                        np.zeros(3), np.zeros(3), int(scene.box_mat[k]) + material_offset,
                        lengths=bx[3:6].copy()))
    # moving boxes, created after the fixed ones; state overrides as for the spheres
    m = getattr(scene, "nmbox", 0)
    bx_, bq_, bv_, bw_ = (scene.mbox_x, scene.mbox_q, scene.mbox_v, scene.mbox_w) if m else (
        None, None, None, None)
    if box_state is not None:
        bx_, bq_, bv_, bw_ = box_state
    for k in range(m):
        sid = n + npl + nb + k
        out.append(Body(BOX, sid, sid, True, False, np.asarray(bx_[k], float),
                        np.asarray(bq_[k], float), np.asarray(bv_[k], float),
                        np.asarray(bw_[k], float), int(scene.mbox_mat[k]) + material_offset,
                        lengths=np.asarray(scene.mbox_len[k], float)))
    return out, n + npl + nb + m


def restore_scene(path: str, scene, material_offset: int = PREDEFINED_MATERIALS):
    """A copy of scene whose spheres are the checkpoint's (in system-id order), keeping the
    scene's materials, planes and gravity; the checkpoint's fixed boxes replace the scene's
    walls and its moving boxes the scene's moving boxes."""
    data = read_peb(path)
    sph = sorted([b for b in data["bodies"] if b.kind == SPHERE], key=lambda b: b.sid)
    box = sorted([b for b in data["bodies"] if b.kind == BOX and b.fixed], key=lambda b: b.sid)
    mov = sorted([b for b in data["bodies"] if b.kind == BOX and not b.fixed],
                 key=lambda b: b.sid)
    s = scene.copy()
    s.x = np.array([b.x for b in sph]).reshape(-1, 3)
    s.v = np.array([b.v for b in sph]).reshape(-1, 3)
    s.w = np.array([b.w for b in sph]).reshape(-1, 3)
    s.r = np.array([b.radius for b in sph])
    s.mat = np.array([b.material - material_offset for b in sph], dtype=s.mat.dtype)
    if box:
        s.boxes = np.array([np.r_[b.x, b.lengths, np.eye(3).ravel()] for b in box])
        s.box_mat = np.array([b.material - material_offset for b in box], dtype=s.box_mat.dtype)
    else:
        s.boxes = np.zeros((0, 15))
        s.box_mat = np.zeros(0, dtype=s.box_mat.dtype)
    s.mbox_x = np.array([b.x for b in mov]).reshape(-1, 3)
    s.mbox_q = np.array([b.q for b in mov]).reshape(-1, 4)
    s.mbox_v = np.array([b.v for b in mov]).reshape(-1, 3)
    s.mbox_w = np.array([b.w for b in mov]).reshape(-1, 3)
    s.mbox_len = np.array([b.lengths for b in mov]).reshape(-1, 3)
    s.mbox_mat = np.array([b.material - material_offset for b in mov], dtype=np.int32)
    return s
