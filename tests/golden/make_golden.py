"""Generates the golden vectors of tests/golden/ by running the compiled pe reference.

The reference is built from its own sources by oracle/ref/Makefile (into oracle/_ref/); this
script feeds it seeded scenes (pe_b200.scenes) through its public API (oracle/ref/ref_driver.cpp)
and stores inputs and outputs as compressed .npz files.  Run from the repository root:

    make -C oracle/ref -j8 && python tests/golden/make_golden.py
"""
import os
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from pe_b200 import scenes  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref")
OUT = os.path.dirname(os.path.abspath(__file__))
CONTACT_DTYPE = np.dtype([("b1", "<i8"), ("b2", "<i8"), ("gpos", "<f8", 3), ("n", "<f8", 3),
                          ("dist", "<f8")])


def run_pairs(exe, scene_path, tmp):
    out = os.path.join(tmp, "pairs.bin")
    subprocess.run([os.path.join(REF, exe), "pairs", scene_path, out], check=True)
    b = open(out, "rb").read()
    n = int(np.frombuffer(b[:8], "<i8")[0])
    return np.frombuffer(b[8:], CONTACT_DTYPE, count=n).copy()


def run_steps(exe, scene_path, n, steps, tmp, extra=()):
    out = os.path.join(tmp, "state.bin")
    subprocess.run([os.path.join(REF, exe), "step", scene_path, str(steps), out,
                    *[str(e) for e in extra]], check=True)
    a = np.fromfile(out, "<f8")
    return (a[:3 * n].reshape(n, 3), a[3 * n:6 * n].reshape(n, 3), a[6 * n:9 * n].reshape(n, 3),
            a[9 * n:].reshape(n, 4))


def golden(name, scene, dem_steps=(1, 10), hc=True, hc_converged=False, dem_exe="ref_dem"):
    with tempfile.TemporaryDirectory() as tmp:
        sp = os.path.join(tmp, "scene.bin")
        scene.save(sp)
        rec = {"scene": np.frombuffer(scene.to_bytes(), np.uint8)}
        rec["pairs"] = run_pairs(dem_exe, sp, tmp)
        for k in dem_steps:
            x, v, w, q = run_steps(dem_exe, sp, scene.n, k, tmp)
            rec[f"dem{k}_x"], rec[f"dem{k}_v"], rec[f"dem{k}_w"], rec[f"dem{k}_q"] = x, v, w, q
        if hc:
            rec["hc_pairs"] = run_pairs("ref_hcsits", sp, tmp)
            for model in (0, 1, 2, 3, 4, 5):
                x, v, w, q = run_steps("ref_hcsits", sp, scene.n, 1, tmp, (model, 100))
                rec[f"hc{model}_x"], rec[f"hc{model}_v"], rec[f"hc{model}_w"] = x, v, w
                rec[f"hc{model}_q"] = q
        if hc_converged:
            x, v, w, q = run_steps("ref_hcsits", sp, scene.n, 1, tmp, (0, 40000))
            rec["hc0conv_x"], rec["hc0conv_v"], rec["hc0conv_w"] = x, v, w
    path = os.path.join(OUT, name + ".npz")
    np.savez_compressed(path, **rec)
    print(path, os.path.getsize(path), "bytes,", len(rec["pairs"]), "contacts")


def hertz_scene(seed, n=64, with_boxes=False):
    """small_random with two materials whose Young's moduli and Poisson ratios differ, for pe's
    extended Hertz law (sphere-sphere contacts)."""
    s = scenes.small_random(seed, n=n, with_boxes=with_boxes)
    s.materials = np.stack([scenes.material(1.0, 1e5, 50.0, 40.0, 0.3, young=2e6, poisson=0.3),
                            scenes.material(2.0, 2e5, 30.0, 20.0, 0.15, young=5e6, poisson=0.2)])
    s.name = f"hertz_{seed}_{n}"
    return s


def adjoint_fd(name="adjoint_fd", seed=2, n=64, steps=40):
    """Central differences (h as in the adjoint tests) of the loss of pe_b200.adjoint.LossSpec after
    `steps` reference DEM steps, with respect to sampled initial velocities and to k_n, c_n, mu."""
    from pe_b200.adjoint import LossSpec, make_single_material, set_params

    p = {"k_n": 1e5, "c_n": 50.0, "c_t": 40.0, "mu": 0.3}
    s = make_single_material(scenes.small_random(seed, n=n, overlap=0.04, with_boxes=False), **p)
    spec = LossSpec.for_scene(s)
    with tempfile.TemporaryDirectory() as tmp:
        def loss(t):
            sp = os.path.join(tmp, "scene.bin")
            t.save(sp)
            return spec.value(run_steps("ref_dem", sp, t.n, steps, tmp)[0])

        rec = {"scene": np.frombuffer(s.to_bytes(), np.uint8), "loss": loss(s)}
        rng = np.random.default_rng(0)
        idx = np.stack([rng.integers(0, n, 8), rng.integers(0, 3, 8)], axis=1)
        fd = []
        for i, a in idx:
            sp_, sm_ = s.copy(), s.copy()
            sp_.v[i, a] += 1e-6
            sm_.v[i, a] -= 1e-6
            fd.append((loss(sp_) - loss(sm_)) / 2e-6)
        rec["v_idx"], rec["fd_v"] = idx, np.array(fd)
        for key, h in (("k_n", 1e-1), ("c_n", 1e-4), ("mu", 1e-6)):
            pp, pm = dict(p), dict(p)
            pp[key] += h
            pm[key] -= h
            rec["fd_" + key] = (loss(set_params(s, **pp)) - loss(set_params(s, **pm))) / (2 * h)
    path = os.path.join(OUT, name + ".npz")
    np.savez_compressed(path, **rec)
    print(path, os.path.getsize(path), "bytes, loss", rec["loss"])


def peb_fixture(steps=5):
    """pe's own checkpoint of small64_boxes after `steps` DEM steps, and that state."""
    s = scenes.small_random(1, n=64, with_boxes=True)
    with tempfile.TemporaryDirectory() as tmp:
        sp = os.path.join(tmp, "scene.bin")
        s.save(sp)
        peb = os.path.join(OUT, "peb_small64_boxes.peb")
        subprocess.run([os.path.join(REF, "ref_dem"), "peb_write", sp, str(steps), peb], check=True)
        x, v, w, q = run_steps("ref_dem", sp, s.n, steps, tmp)
    path = os.path.join(OUT, "peb_small64_boxes.npz")
    np.savez_compressed(path, scene=np.frombuffer(s.to_bytes(), np.uint8), x=x, v=v, w=w, q=q)
    print(peb, os.path.getsize(peb), "bytes")


def run_steps_boxes(exe, scene_path, n, nmb, steps, tmp, extra=()):
    """Sphere and moving-box states after `steps` reference steps."""
    out = os.path.join(tmp, "state.bin")
    subprocess.run([os.path.join(REF, exe), "step", scene_path, str(steps), out,
                    *[str(e) for e in extra]], check=True)
    a = np.fromfile(out, "<f8")
    sizes = [3 * n, 3 * n, 3 * n, 4 * n, 3 * nmb, 3 * nmb, 3 * nmb, 4 * nmb]
    parts = np.split(a, np.cumsum(sizes)[:-1])
    shapes = [(n, 3), (n, 3), (n, 3), (n, 4), (nmb, 3), (nmb, 3), (nmb, 3), (nmb, 4)]
    return [p.reshape(sh) for p, sh in zip(parts, shapes)]


def box_golden(name, scene, dem_steps=(1, 10), hc_converged_iters=20000):
    """Moving-box scene: pe's contacts (detection order), DEM states, one HCSITS step per
    relaxation model in pe's contact order, and a converged frictionless step."""
    keys = ("x", "v", "w", "q", "bx", "bv", "bw", "bq")
    with tempfile.TemporaryDirectory() as tmp:
        sp = os.path.join(tmp, "scene.bin")
        scene.save(sp)
        rec = {"scene": np.frombuffer(scene.to_bytes(), np.uint8)}
        rec["pairs"] = run_pairs("ref_dem", sp, tmp)
        for k in dem_steps:
            for key, a in zip(keys, run_steps_boxes("ref_dem", sp, scene.n, scene.nmbox, k, tmp)):
                rec[f"dem{k}_{key}"] = a
        rec["hc_pairs"] = run_pairs("ref_hcsits", sp, tmp)
        for model in (0, 1, 2, 3, 4, 5):
            st = run_steps_boxes("ref_hcsits", sp, scene.n, scene.nmbox, 1, tmp, (model, 100))
            for key, a in zip(keys, st):
                rec[f"hc{model}_{key}"] = a
        st = run_steps_boxes("ref_hcsits", sp, scene.n, scene.nmbox, 1, tmp,
                             (0, hc_converged_iters))
        for key, a in zip(keys, st):
            rec[f"hc0conv_{key}"] = a
    path = os.path.join(OUT, name + ".npz")
    np.savez_compressed(path, **rec)
    print(path, os.path.getsize(path), "bytes,", len(rec["pairs"]), "contacts")


def box_goldens():
    box_golden("boxes27_tumbling", scenes.tumbling_boxes(0))
    box_golden("boxes64_tilted", scenes.tumbling_boxes(2, side=4, spheres=False))
    box_golden("boxes36_stack", scenes.box_stack())


def peb_box_fixture(steps=5):
    """pe's own checkpoint of the tumbling-box scene (boxes27_tumbling) after `steps` DEM steps,
    and that state (spheres and moving boxes)."""
    s = scenes.tumbling_boxes(0)
    keys = ("x", "v", "w", "q", "bx", "bv", "bw", "bq")
    with tempfile.TemporaryDirectory() as tmp:
        sp = os.path.join(tmp, "scene.bin")
        s.save(sp)
        peb = os.path.join(OUT, "peb_boxes27.peb")
        subprocess.run([os.path.join(REF, "ref_dem"), "peb_write", sp, str(steps), peb], check=True)
        st = run_steps_boxes("ref_dem", sp, s.n, s.nmbox, steps, tmp)
    rec = {"scene": np.frombuffer(s.to_bytes(), np.uint8)}
    rec.update(dict(zip(keys, st)))
    path = os.path.join(OUT, "peb_boxes27.npz")
    np.savez_compressed(path, **rec)
    print(peb, os.path.getsize(peb), "bytes")


def hertz_goldens():
    golden("hertz64_boxes", hertz_scene(1, with_boxes=True), dem_steps=(1, 10), hc=False,
           dem_exe="ref_dem_hertz")
    golden("hertz64_planes", hertz_scene(2), dem_steps=(1, 10), hc=False, dem_exe="ref_dem_hertz")


def dense_converged(name="dense4096_conv", iters=20000):
    """A dense packing with thousands of contacts: 4096 spheres on a 16x16x16 lattice of spacing
    1.0 (radii U[0.45, 0.55], so about half of the neighbours touch or overlap) resting on the
    floor of a box of planes, 6,593 contacts.  pe's frictionless HCSITS step with `iters` sweeps
    (its velocities change by < 1e-13 relative between 16,000 and 64,000 sweeps, so they are the
    unique converged ones) and the scene."""
    s = scenes.nbgs_box(0, n=4096, dims=(16.0, 16.0, 60.0), dense=True)
    with tempfile.TemporaryDirectory() as tmp:
        sp = os.path.join(tmp, "scene.bin")
        s.save(sp)
        x, v, w, _ = run_steps("ref_hcsits", sp, s.n, 1, tmp, (0, iters))
        ncont = len(run_pairs("ref_hcsits", sp, tmp))
    rec = {"scene": np.frombuffer(s.to_bytes(), np.uint8), "hc0conv_x": x, "hc0conv_v": v,
           "hc0conv_w": w, "iters": iters, "contacts": ncont}
    # the same packing with mu = 0.5 under pe's default model (approximate Coulomb friction by
    # decoupling): pe reports no residual, so the oracle's complementarity residual (its
    # restatement of that model, pinned bit for bit to pe in pe's contact order) after a given
    # number of sweeps is the reference for the frictional runs
    from oracle.pe_oracle import APPROX_COULOMB_DECOUPLING, OracleWorld
    sf = scenes.nbgs_box(0, n=4096, mu=0.5, dims=(16.0, 16.0, 60.0), dense=True)
    assert np.array_equal(sf.x, s.x) and np.array_equal(sf.r, s.r)
    sweeps = np.array([100, 1000, 4000])
    res = []
    for k in sweeps:
        o = OracleWorld(sf)
        res.append(o.hcsits_step(sf.dt, APPROX_COULOMB_DECOUPLING, int(k))[2])
    rec["mu05_sweeps"], rec["mu05_residual_oracle"] = sweeps, np.array(res)
    path = os.path.join(OUT, name + ".npz")
    np.savez_compressed(path, **rec)
    print(path, os.path.getsize(path), "bytes,", ncont, "contacts")


# steps of the hopper's finite differences, largest first: k_n, c_n and mu (the composed
# coefficients; the hopper has k_n = 5e4, c_n = 25, mu = 0.4)
HOPPER_PARAM_STEPS = {"k_n": (1e-1, 1e-2, 1e-3), "c_n": (1e-4, 1e-5, 1e-6),
                      "mu": (1e-5, 1e-6, 1e-7)}


def hopper_fd(name="hopper_fd"):
    """pe's own FP64 finite differences of the hopper workload's loss over its full horizon
    (16,384 spheres, 2000 steps) with respect to k_n, c_n and mu: the scene of
    pe_b200.scenes.hopper(0) with one material whose composed coefficients equal the hopper's
    (so that a derivative with respect to the composed value is one with respect to the
    material's), the loss of pe_b200.adjoint.LossSpec with the opening at z = 10.  For every step
    of HOPPER_PARAM_STEPS the forward and backward one-sided differences are stored (their
    disagreement shows a contact onset crossed inside the step).  The runs go to parallel
    processes."""
    from concurrent.futures import ThreadPoolExecutor

    from pe_b200.adjoint import LossSpec, make_single_material, set_params

    s0 = scenes.hopper(0)
    m = s0.materials[0]
    p = {"k_n": m[6] / 2, "c_n": m[7] / 2, "c_t": m[8] / 2, "mu": 2 * m[2]}
    s = make_single_material(s0, **p)
    spec = LossSpec.for_scene(s, z_open=10.0)
    steps = s.steps
    with tempfile.TemporaryDirectory() as tmp:
        def final_x(args):
            tag, t = args
            d = os.path.join(tmp, tag)
            os.makedirs(d)
            sp = os.path.join(d, "scene.bin")
            t.save(sp)
            return run_steps("ref_dem", sp, t.n, steps, d)[0]

        jobs = [("base", s)]
        for key, hs in HOPPER_PARAM_STEPS.items():
            for k, h in enumerate(hs):
                pp, pm = dict(p), dict(p)
                pp[key] += h
                pm[key] -= h
                jobs.append((f"{key}_{k}_p", set_params(s, **pp)))
                jobs.append((f"{key}_{k}_m", set_params(s, **pm)))
        with ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
            xs = dict(zip([j[0] for j in jobs], ex.map(final_x, jobs)))
    rec = {"steps": steps, "spheres": s.n}
    for key, hs in HOPPER_PARAM_STEPS.items():
        rec["h_" + key] = np.array(hs)
        rec["fwd_" + key] = np.array([spec.diff(xs[f"{key}_{k}_p"], xs["base"]) / h
                                      for k, h in enumerate(hs)])
        rec["bwd_" + key] = np.array([spec.diff(xs["base"], xs[f"{key}_{k}_m"]) / h
                                      for k, h in enumerate(hs)])
    path = os.path.join(OUT, name + ".npz")
    np.savez_compressed(path, **rec)
    print(path, {k: v.tolist() if hasattr(v, "tolist") else v for k, v in rec.items()})


if __name__ == "__main__":
    if sys.argv[1:] == ["adjoint_fd"]:
        adjoint_fd()
        sys.exit(0)
    if sys.argv[1:] == ["hopper_fd"]:
        hopper_fd()
        sys.exit(0)
    if sys.argv[1:] == ["dense"]:
        dense_converged()
        sys.exit(0)
    if sys.argv[1:] == ["hertz"]:
        hertz_goldens()
        sys.exit(0)
    if sys.argv[1:] == ["peb"]:
        peb_fixture()
        sys.exit(0)
    if sys.argv[1:] == ["boxes"]:
        box_goldens()
        peb_box_fixture()
        sys.exit(0)
    golden("small64_boxes", scenes.small_random(1, n=64, with_boxes=True))
    golden("small64_planes", scenes.small_random(2, n=64, with_boxes=False))
    golden("lattice512", scenes.dem_lattice(0, side=8), dem_steps=(1, 10, 100))
    golden("dense512", scenes.nbgs_box(0, n=512, dims=(8.0, 8.0, 20.0), dense=True),
           dem_steps=(1,))
    # loose packings whose frictionless solve converges (contacts form short chains)
    golden("loose125_planes", scenes.small_random(3, n=125, overlap=0.0, with_boxes=False),
           dem_steps=(1,), hc_converged=True)
    golden("loose125_boxes", scenes.small_random(4, n=125, overlap=0.0, with_boxes=True),
           dem_steps=(1,), hc_converged=True)
    dense_converged()
    hopper_fd()
    adjoint_fd()
    hertz_goldens()
    peb_fixture()
    box_goldens()
    peb_box_fixture()
