"""pe's binary checkpoint format (.peb): files written here are byte-identical to pe's own
BodyBinaryWriter output, pe's files read back exactly, and pe's BodyBinaryReader resumes from a
file written here (against the compiled reference when it is built; the fixture made by
tests/golden/make_golden.py otherwise)."""
import os
import subprocess

import numpy as np
import pytest

from helpers import GOLDEN, load_golden, rel_err
from pe_b200 import checkpoint as ck

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref", "ref_dem")
live = pytest.mark.skipif(not os.path.exists(REF), reason="compiled reference not built")


def test_fixture_bytes_identical_to_pe():
    """The pe-written fixture (small64_boxes after 5 steps) equals what write_peb produces from
    the same state."""
    g = load_golden("peb_small64_boxes")
    s = g["scene"]
    bodies, counter = ck.scene_bodies(s, x=g["x"], v=g["v"], w=g["w"], q=g["q"])
    path = os.path.join(GOLDEN, "peb_small64_boxes.peb")
    mine = os.path.join(os.path.dirname(path), "_tmp_written.peb")
    try:
        ck.write_peb(mine, bodies, counter)
        assert open(mine, "rb").read() == open(path, "rb").read()
    finally:
        if os.path.exists(mine):
            os.unlink(mine)


def test_fixture_reads_back_pe_state():
    g = load_golden("peb_small64_boxes")
    d = ck.read_peb(os.path.join(GOLDEN, "peb_small64_boxes.peb"))
    sph = sorted([b for b in d["bodies"] if b.kind == ck.SPHERE], key=lambda b: b.sid)
    assert len(sph) == g["scene"].n and d["counter"] == g["scene"].n + 6 + 2
    assert np.array_equal(np.array([b.x for b in sph]), g["x"])
    assert np.array_equal(np.array([b.v for b in sph]), g["v"])
    assert np.array_equal(np.array([b.w for b in sph]), g["w"])
    assert np.array_equal(np.array([b.q for b in sph]), g["q"])
    assert sum(b.kind == ck.BOX for b in d["bodies"]) == 2
    assert not any(b.kind == ck.PLANE for b in d["bodies"])   # pe writes only global planes


def test_rejects_what_pe_rejects(tmp_path):
    bad = tmp_path / "bad.peb"
    bad.write_bytes(b"XX" + bytes(30))
    with pytest.raises(ValueError, match="Invalid file format"):
        ck.read_peb(str(bad))
    good = open(os.path.join(GOLDEN, "peb_small64_boxes.peb"), "rb").read()
    bad.write_bytes(good[:4] + bytes([4]) + good[5:])
    with pytest.raises(ValueError, match="floating point"):
        ck.read_peb(str(bad))


@live
@pytest.mark.parametrize("steps", [0, 7])
def test_live_bytes_identical_to_pe(tmp_path, steps):
    s = load_golden("small64_planes")["scene"]
    sp, peb = str(tmp_path / "s.bin"), str(tmp_path / "pe.peb")
    s.save(sp)
    subprocess.run([REF, "peb_write", sp, str(steps), peb], check=True)
    out = str(tmp_path / "st.bin")
    subprocess.run([REF, "step", sp, str(steps), out], check=True)
    a = np.fromfile(out, "<f8")
    n = s.n
    x, v, w, q = (a[:3 * n].reshape(n, 3), a[3 * n:6 * n].reshape(n, 3),
                  a[6 * n:9 * n].reshape(n, 3), a[9 * n:].reshape(n, 4))
    bodies, counter = ck.scene_bodies(s, x=x, v=v, w=w, q=q)
    mine = str(tmp_path / "mine.peb")
    ck.write_peb(mine, bodies, counter)
    assert open(mine, "rb").read() == open(peb, "rb").read()


@live
def test_pe_resumes_from_our_checkpoint(tmp_path):
    """pe's reader restarts from a file written here; its continuation matches pe's own
    restart from its own file (pe re-creates contacts on restart, so not bitwise against the
    uninterrupted run)."""
    s = load_golden("small64_boxes")["scene"]
    sp = str(tmp_path / "s.bin")
    s.save(sp)
    peb_pe, peb_us = str(tmp_path / "pe.peb"), str(tmp_path / "us.peb")
    subprocess.run([REF, "peb_write", sp, "5", peb_pe], check=True)
    d = ck.read_peb(peb_pe)
    ck.write_peb(peb_us, d["bodies"], d["counter"], d["global_counter"])
    o1, o2 = str(tmp_path / "o1.bin"), str(tmp_path / "o2.bin")
    subprocess.run([REF, "peb_read", sp, peb_pe, "5", o1], check=True)
    subprocess.run([REF, "peb_read", sp, peb_us, "5", o2], check=True)
    assert open(o1, "rb").read() == open(o2, "rb").read()
    oc = str(tmp_path / "oc.bin")
    subprocess.run([REF, "step", sp, "10", oc], check=True)
    a, c = np.fromfile(o1, "<f8"), np.fromfile(oc, "<f8")
    assert rel_err(a[:3 * s.n], c[:3 * s.n]) < 1e-12


# ---- moving boxes ----------------------------------------------------------------------------
def test_box_fixture_bytes_identical_to_pe():
    """pe's checkpoint of the tumbling-box scene after 5 steps (moving boxes with orientation
    and velocities) equals what write_peb produces from the same state."""
    g = load_golden("peb_boxes27")
    s = g["scene"]
    bodies, counter = ck.scene_bodies(s, x=g["x"], v=g["v"], w=g["w"], q=g["q"],
                                      box_state=(g["bx"], g["bq"], g["bv"], g["bw"]))
    path = os.path.join(GOLDEN, "peb_boxes27.peb")
    mine = os.path.join(os.path.dirname(path), "_tmp_written_boxes.peb")
    try:
        ck.write_peb(mine, bodies, counter)
        assert open(mine, "rb").read() == open(path, "rb").read()
    finally:
        if os.path.exists(mine):
            os.unlink(mine)


def test_box_fixture_restores_moving_boxes():
    g = load_golden("peb_boxes27")
    s = ck.restore_scene(os.path.join(GOLDEN, "peb_boxes27.peb"), g["scene"])
    assert s.nmbox == g["scene"].nmbox and s.boxes.shape[0] == g["scene"].boxes.shape[0]
    for a, key in ((s.mbox_x, "bx"), (s.mbox_q, "bq"), (s.mbox_v, "bv"), (s.mbox_w, "bw")):
        assert np.array_equal(a, g[key])
    assert np.array_equal(s.mbox_len, g["scene"].mbox_len)
    assert np.array_equal(s.mbox_mat, g["scene"].mbox_mat)


@live
def test_pe_resumes_boxes_from_our_checkpoint(tmp_path):
    """With moving boxes, pe's reader restarts from a file written here exactly as from its own
    file.  (pe's own restart is not its uninterrupted run here: Box::Box sets the orientation
    after BoxBase computed the bounding box of the unrotated box, Box.cpp:100-130, so the first
    step after a restart can miss box pairs.)"""
    from pe_b200 import scenes
    s = scenes.tumbling_boxes(0)
    sp = str(tmp_path / "s.bin")
    s.save(sp)
    peb_pe, peb_us = str(tmp_path / "pe.peb"), str(tmp_path / "us.peb")
    subprocess.run([REF, "peb_write", sp, "5", peb_pe], check=True)
    d = ck.read_peb(peb_pe)
    ck.write_peb(peb_us, d["bodies"], d["counter"], d["global_counter"])
    assert open(peb_us, "rb").read() == open(peb_pe, "rb").read()
    o1, o2 = str(tmp_path / "o1.bin"), str(tmp_path / "o2.bin")
    subprocess.run([REF, "peb_read", sp, peb_pe, "5", o1], check=True)
    subprocess.run([REF, "peb_read", sp, peb_us, "5", o2], check=True)
    assert open(o1, "rb").read() == open(o2, "rb").read()
