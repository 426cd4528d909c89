"""pe's own World::simulationStep (src/core/World.cpp:330-357) running on the GPU: pe compiled from
its unmodified sources with the B200 collision system (include/pe_b200_pe, selected by the
configuration of oracle/ref/config_b200_*.h) and linked to libpe_b200.so, driven by the same
driver program (oracle/ref/ref_driver.cpp, unchanged) and scenes that made the golden vectors
with pe's CPU collision systems.

Checked: pe's contact set through the B200 detector (bit-exact pairs), DEM steps within 1e-12 of
pe's CPU DEM step (spheres, and spheres with moving boxes), converged frictionless HCSITS
velocities within 1e-6 of pe's CPU hard-contact step, and a checkpoint pe writes after steps on
the GPU."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

from helpers import CONVERGED_NAMES, GOLDEN_NAMES, load_golden, pair_set, rel_err, rel_err_w

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref")
B200_DEM = os.path.join(REF, "b200_dem")
B200_HC = os.path.join(REF, "b200_hcsits")
CONTACT_DTYPE = np.dtype([("b1", "<i8"), ("b2", "<i8"), ("gpos", "<f8", 3), ("n", "<f8", 3),
                          ("dist", "<f8")])


def _need(exe):
    if not os.path.exists(exe):
        pytest.skip(f"pe with the B200 collision system not built ({exe}; make -C oracle/ref)")


def _run(exe, *args):
    r = subprocess.run([exe, *map(str, args)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr


def _state(path, n, nmb=0):
    a = np.fromfile(path, "<f8")
    sizes = [3 * n, 3 * n, 3 * n, 4 * n, 3 * nmb, 3 * nmb, 3 * nmb, 4 * nmb]
    parts = np.split(a, np.cumsum(sizes)[:-1])
    shapes = [(n, 3), (n, 3), (n, 3), (n, 4), (nmb, 3), (nmb, 3), (nmb, 3), (nmb, 4)]
    return [p.reshape(sh) for p, sh in zip(parts, shapes)]


@pytest.mark.parametrize("name", GOLDEN_NAMES)
def test_pe_world_contacts_through_b200_detector(name):
    """pe's CollisionSystem::getCoarseDetector().findContacts (HashGrids.h:1121) answered by the
    device: the same (body 1, body 2) pairs as pe's hash grids and MaxContacts, same geometry."""
    _need(B200_DEM)
    g = load_golden(name)
    s = g["scene"]
    with tempfile.TemporaryDirectory() as tmp:
        sp, out = os.path.join(tmp, "s.bin"), os.path.join(tmp, "p.bin")
        s.save(sp)
        _run(B200_DEM, "pairs", sp, out)
        b = open(out, "rb").read()
    nc = int(np.frombuffer(b[:8], "<i8")[0])
    got = np.frombuffer(b[8:], CONTACT_DTYPE, count=nc)
    ref = g["pairs"]
    assert pair_set(np.stack([got["b1"], got["b2"]], 1)) == \
        pair_set(np.stack([ref["b1"], ref["b2"]], 1))
    if nc:
        a = got[np.lexsort((got["b2"], got["b1"]))]
        r = ref[np.lexsort((ref["b2"], ref["b1"]))]
        assert rel_err(a["gpos"], r["gpos"]) < 1e-14
        assert np.abs(a["dist"] - r["dist"]).max() < 1e-14


@pytest.mark.parametrize("name", GOLDEN_NAMES)
def test_pe_world_dem_steps_match_pe_cpu(name):
    """World::simulationStep with pe's DEM response on the GPU against pe's own CPU DEM step."""
    _need(B200_DEM)
    g = load_golden(name)
    s = g["scene"]
    with tempfile.TemporaryDirectory() as tmp:
        sp, out = os.path.join(tmp, "s.bin"), os.path.join(tmp, "o.bin")
        s.save(sp)
        for key in sorted(k for k in g if k.startswith("dem") and k.endswith("_x")):
            k = int(key[3:-2])
            _run(B200_DEM, "step", sp, k, out)
            x, v, w, q = _state(out, s.n)[:4]
            tol = 1e-12 if k <= 10 else 1e-10
            assert rel_err(x, g[f"dem{k}_x"]) < tol, (k, rel_err(x, g[f"dem{k}_x"]))
            assert rel_err(v, g[f"dem{k}_v"]) < tol, (k, rel_err(v, g[f"dem{k}_v"]))
            assert rel_err_w(w, g[f"dem{k}_w"], g[f"dem{k}_v"], s.r) < tol
            assert rel_err(q, g[f"dem{k}_q"]) < tol


def test_pe_world_dem_with_moving_boxes_matches_pe_cpu():
    _need(B200_DEM)
    g = load_golden("boxes27_tumbling")
    s = g["scene"]
    with tempfile.TemporaryDirectory() as tmp:
        sp, out = os.path.join(tmp, "s.bin"), os.path.join(tmp, "o.bin")
        s.save(sp)
        for k in (1, 10):
            _run(B200_DEM, "step", sp, k, out)
            x, v, w, q, bx, bv, bw, bq = _state(out, s.n, s.nmbox)
            assert rel_err(bx, g[f"dem{k}_bx"]) < 1e-13
            assert rel_err(bv, g[f"dem{k}_bv"]) < 1e-11
            assert rel_err(bq, g[f"dem{k}_bq"]) < 1e-13
            assert rel_err(x, g[f"dem{k}_x"]) < 1e-13
            assert rel_err(v, g[f"dem{k}_v"]) < 1e-11


@pytest.mark.parametrize("name", CONVERGED_NAMES + ["dense4096_conv"])
def test_pe_world_hcsits_converged_velocities_match_pe_cpu(name):
    """World::simulationStep with pe's hard-contact response (frictionless model, 20,000 sweeps,
    set through pe's setRelaxationModel / setMaxIterations) on the GPU against pe's CPU step."""
    _need(B200_HC)
    g = load_golden(name)
    s = g["scene"]
    with tempfile.TemporaryDirectory() as tmp:
        sp, out = os.path.join(tmp, "s.bin"), os.path.join(tmp, "o.bin")
        s.save(sp)
        _run(B200_HC, "step", sp, 1, out, 0, 20000)
        x, v, w, q = _state(out, s.n)[:4]
    assert rel_err(v, g["hc0conv_v"]) < 1e-6
    assert rel_err(x, g["hc0conv_x"]) < 1e-9


def test_pe_checkpoint_written_after_gpu_steps():
    """pe's BodyBinaryWriter (src/core/BodyBinaryWriter.cpp) after five GPU steps of pe's World
    writes the same bodies, ids and materials as after five CPU steps, with states within the DEM
    tolerance: what pe's getters see after a GPU step is the device's state."""
    _need(B200_DEM)
    g = load_golden("small64_boxes")
    s = g["scene"]
    ref_exe = os.path.join(REF, "ref_dem")
    if not os.path.exists(ref_exe):
        pytest.skip("compiled reference not built")
    from pe_b200.checkpoint import read_peb
    with tempfile.TemporaryDirectory() as tmp:
        sp = os.path.join(tmp, "s.bin")
        s.save(sp)
        a, b = os.path.join(tmp, "gpu.peb"), os.path.join(tmp, "cpu.peb")
        _run(B200_DEM, "peb_write", sp, 5, a)
        _run(ref_exe, "peb_write", sp, 5, b)
        ga, gb = read_peb(a), read_peb(b)
    assert ga["counter"] == gb["counter"] and len(ga["bodies"]) == len(gb["bodies"])
    for p, q in zip(ga["bodies"], gb["bodies"]):
        assert (p.kind, p.sid, p.uid, p.fixed, p.material) == (q.kind, q.sid, q.uid, q.fixed,
                                                                q.material)
        scale = max(1.0, float(np.abs(q.x).max()))
        assert np.abs(p.x - q.x).max() < 1e-12 * scale
        assert np.abs(p.v - q.v).max() < 1e-11 * max(1.0, float(np.abs(q.v).max()))
        assert np.abs(p.q - q.q).max() < 1e-12
