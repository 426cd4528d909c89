"""Benchmark of the B200 rigid-body step (sphere-steps/s).

Default workload: the large DEM scene -- 1,048,576 spheres, 1000 steps, log-normal radii (median 0.5,
sigma_log 0.2, clipped to [0.3, 0.9]) in a random packing at 30% solid fraction at the bottom of a
200x200x400 box of planes, linear spring-dashpot k_n=1e5, c_n=50, mu=0.4, dt=5e-5 -- advanced by
the mixed-precision path (FP64 positions, FP32 velocities/forces).  Beside it, on the same scene,
the plain all-FP64 GPU path, the 32,768-sphere hard-contact (NBGS) scene, and the compiled pe
reference on the host cores.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload dem_large_1m|dem_lattice_4096|nbgs_box_32768|ensemble_512]

Under torchrun each rank advances its own replica of the scene (one scene does not shard
without spatial decomposition; the batched ensemble shards by scene): weak scaling, whole-job
throughput = spheres x steps x ranks / max-over-ranks device time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from pe_b200 import scenes  # noqa: E402
from pe_b200.shard import shard_scenes  # noqa: E402

METRIC = "sphere-steps/s (1M DEM, 32k NBGS) mixed+batched vs plain FP64 GPU at stated err"
UNIT = "sphere-steps/s"
# algorithmic bytes per sphere-step of the DEM step (positions, velocities, radius/mass, grid
# key+id read and written once): FP64 176 B; mixed 128 B (FP64 positions 48, FP32 velocities 48,
# their extension bytes 8, radius and mass 8, list offsets and grid key 16)
ALGO_BYTES = {"fp64": 176.0, "mixed": 128.0}
L2_FLUSH_BYTES = 256 << 20


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="dem_large_1m",
                    choices=["dem_large_1m", "dem_dense_1m", "dem_lattice_4096", "nbgs_box_32768",
                             "ensemble_512"])
    ap.add_argument("--no-extras", action="store_true", help="headline measurement only")
    ap.add_argument("--no-cpu-baseline", action="store_true",
                    help="skip the pe-on-one-core leg (minutes of set-up at 1M spheres)")
    ap.add_argument("--tuning", default=None,
                    help="dem_variant,rebuild_per_sm,skin[,dem_split] instead of running the "
                         "autotuner")
    ap.add_argument("--profile-case", default=None, choices=sorted(PROFILE_CASES),
                    help="run one small case of one stage for a profiler (prints a short JSON "
                         "line, not a bench line); see profile_case()")
    return ap.parse_args()


def build_workload(name, seed=0, rank=0, world=1):
    """The scenes this rank advances.  A single scene is replicated on every rank; the batched
    ensemble is partitioned by scene (largest first onto the least-loaded rank), so the ranks
    share one fixed job and exchange nothing."""
    if name == "dem_large_1m":
        return [scenes.dem_large(seed)], "dem"
    if name == "dem_dense_1m":
        return [scenes.dem_dense(seed)], "dem"
    if name == "dem_lattice_4096":
        return [scenes.dem_lattice(seed)], "dem"
    if name == "nbgs_box_32768":
        return [scenes.nbgs_box(seed)], "hcsits"
    if name == "ensemble_512":
        return shard_scenes(scenes.batched_ensemble(seed), rank, world), "dem"
    raise ValueError(name)


# ------------------------------------------------------------------------------------------
# reference (pe compiled from its own sources, oracle/_ref) on the host cores
# ------------------------------------------------------------------------------------------
REF_DIR = os.path.join(ROOT, "oracle", "_ref")


def ref_scene(workload):
    """The workload's scene for the single-threaded reference, and its executable.  The single
    scenes are the full configured scenes; for the ensemble, one median-size scene."""
    if workload == "dem_large_1m":
        return scenes.dem_large(0), "ref_dem", "the full 1,048,576-sphere scene"
    if workload == "dem_lattice_4096":
        return scenes.dem_lattice(0), "ref_dem", "the full 4096-sphere lattice scene"
    if workload == "nbgs_box_32768":
        return scenes.nbgs_box(0), "ref_hcsits", "the full 32768-sphere NBGS scene"
    if workload == "ensemble_512":
        ss = scenes.batched_ensemble(0)
        k = int(np.argsort([s.n for s in ss])[len(ss) // 2])
        return ss[k], "ref_dem", f"one median-size scene ({ss[k].n} spheres) of the ensemble"
    raise ValueError(workload)


# timed steps per reference process: pe needs ~3 minutes to set up the 1M-sphere scene (body
# creation and the first hash-grid insertion) and then ~3 s per step on one core
REF_STEPS = {"dem_large_1m": 6, "dem_lattice_4096": 200, "nbgs_box_32768": 10, "ensemble_512": 50}


class RefRun:
    """pe (oracle/_ref, compiled from pe's own sources) timing `steps` World::simulationStep
    calls on a workload's scene, after `warmup` untimed ones, in `procs` concurrent
    single-threaded processes that each advance their own copy of the scene (pe's step is
    single-threaded; the host's throughput is the sum).  Started at once, collected by result()."""

    def __init__(self, workload, steps, warmup=1, procs=1):
        self.err = None
        self.jobs = []
        self.t0 = time.perf_counter()
        sc, exe, what = ref_scene(workload)
        self.n, self.steps, self.warmup, self.what = sc.n, steps, warmup, what
        path = os.path.join(REF_DIR, exe)
        if not os.path.exists(path):
            self.err = f"compiled reference missing ({path}); build with make -C oracle/ref"
            return
        self.tmp = tempfile.TemporaryDirectory()
        sp = os.path.join(self.tmp.name, "scene.bin")
        sc.save(sp)
        extra = ["0", "100"] if exe == "ref_hcsits" else []
        self.procs = procs
        self.jobs = [subprocess.Popen([path, "time", sp, str(warmup), str(steps), *extra],
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)
                     for _ in range(procs)]

    def result(self):
        if self.err:
            return None, self.err
        res = []
        for j in self.jobs:
            out, err = j.communicate()
            if j.returncode != 0:
                return None, "reference run failed: " + err.strip()[-200:]
            res.append(json.loads(out.strip().splitlines()[-1]))
        wall = time.perf_counter() - self.t0
        self.tmp.cleanup()
        total = sum(x["sphere_steps_per_s"] for x in res)
        cores = os.cpu_count() or 1
        return {"sphere_steps_per_s": total, "steps": self.steps, "spheres": self.n,
                "seconds": max(x["seconds"] for x in res), "cores": self.procs, "wall_s": wall,
                "sample": f"{self.procs} concurrent single-threaded pe process(es), each on "
                          f"{self.what}; {self.steps} timed steps after {self.warmup} untimed, "
                          f"set-up excluded (whole run {wall:.1f} s); host has {cores} "
                          f"cores"}, None


def ref_procs(workload):
    """Processes for the reference arm: one per host core, as far as half the free memory
    allows (pe holds about 1.4 KB per sphere)."""
    cores = os.cpu_count() or 1
    try:
        avail = int([l for l in open("/proc/meminfo")
                     if l.startswith("MemAvailable")][0].split()[1]) * 1024
    except (OSError, IndexError, ValueError):
        avail = 8 << 30
    n = ref_scene(workload)[0].n
    return max(1, min(cores, int(0.5 * avail / max(1400 * n, 1 << 20))))


# ------------------------------------------------------------------------------------------
# clocks
# ------------------------------------------------------------------------------------------
class Clocks:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, uuid):
        self.uuid = uuid
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        try:
            cmd = ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                   "-lms", "20"]
            if self.uuid:
                cmd += ["-i", self.uuid]
            self.p = subprocess.Popen(cmd, stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        self.f.seek(0)
        rows = [r.split(",") for r in self.f.read().strip().splitlines() if r.count(",") >= 8]
        os.unlink(self.f.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4)
                          if r[5 + k].strip().lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(rows)}


# ------------------------------------------------------------------------------------------
# our arm
# ------------------------------------------------------------------------------------------
def make_engine(ss, kind, precision, iters=100, lists=True):
    from pe_b200 import _abi
    from pe_b200.engine import Engine
    solver = _abi.DEM if kind == "dem" else _abi.HCSITS
    model = _abi.INELASTIC_FRICTIONLESS
    if kind == "hcsits" and float(ss[0].materials[0, 2]) > 0:
        model = _abi.APPROX_INELASTIC_COULOMB_DECOUPLING
    e = Engine(solver=solver, precision=precision, relaxation_model=model, max_iterations=iters,
               neighbor_lists=lists)
    if len(ss) == 1:
        e.load_scene(ss[0])
    else:
        e.load_scenes(ss)
    return e


def stage_inputs(ss, torch):
    """The bodies of the scenes in pinned host arrays (materials re-indexed per scene), and the
    small per-scene tables, ready for one upload."""
    pin = lambda a, dtype: torch.from_numpy(np.ascontiguousarray(a, dtype)).pin_memory().numpy()
    off, mats, mat, walls = 0, [], [], []
    for s in ss:
        mats.append(s.materials)
        mat.append(s.mat + off)
        walls.append((s.planes, s.plane_mat + off, s.boxes, s.box_mat + off))
        off += s.materials.shape[0]
    scene = None
    if len(ss) > 1:
        scene = pin(np.concatenate([np.full(s.n, k, np.int32) for k, s in enumerate(ss)]), np.int32)
    return {"x": pin(np.concatenate([s.x for s in ss]), np.float64),
            "v": pin(np.concatenate([s.v for s in ss]), np.float64),
            "w": pin(np.concatenate([s.w for s in ss]), np.float64),
            "r": pin(np.concatenate([s.r for s in ss]), np.float64),
            "mat": pin(np.concatenate(mat), np.int32), "scene": scene,
            "materials": np.concatenate(mats), "walls": walls, "gravity": ss[0].gravity,
            "damping": ss[0].damping, "nscenes": len(ss)}


def engine_from_staged(st, kind, precision, iters=100, lists=True, skin=0.0):
    from pe_b200 import _abi
    from pe_b200.engine import Engine
    solver = _abi.DEM if kind == "dem" else _abi.HCSITS
    model = _abi.INELASTIC_FRICTIONLESS
    if kind == "hcsits" and float(st["materials"][0, 2]) > 0:
        model = _abi.APPROX_INELASTIC_COULOMB_DECOUPLING
    e = Engine(solver=solver, precision=precision, relaxation_model=model, max_iterations=iters,
               neighbor_lists=lists, skin=skin)
    e.set_materials(st["materials"])
    for k, (pl, pm, bx, bm) in enumerate(st["walls"]):
        e.set_walls(k, pl, pm, bx, bm)
    e.set_gravity(st["gravity"])
    e.set_damping(st["damping"])
    e.upload(st["x"], st["v"], st["w"], st["r"], st["mat"], st["scene"], st["nscenes"])
    return e


def spin_up(torch, flush_buf, stream, ms=20.0):
    """About `ms` of untimed GPU work (the flush kernels, no step of the workload), so that a
    short timed region does not start while the GPU's clocks are still rising after host-side
    work left it idle."""
    with torch.cuda.stream(stream):
        for _ in range(max(1, int(ms / 0.085))):
            flush_buf[0].add_(1)
            flush_buf[2].add_(flush_buf[1].sum())
    torch.cuda.synchronize()


def timed_steps(e, dt, steps, warmup, torch, flush_buf, stream, dist=None, per_step=None):
    """Per-step CUDA events on the library's stream; the L2 flush between steps is untimed.
    per_step (a list) receives the timed steps' times in ms."""
    spin_up(torch, flush_buf, stream)
    for _ in range(warmup):
        e.step(dt)
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()

    def one_pass(k_steps):
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(k_steps)]
        with torch.cuda.stream(stream):
            for k in range(k_steps):
                # L2 flush: write a 256 MiB buffer, then read another one, so the next step
                # finds neither its own data nor dirty flush lines in the 126 MB L2
                flush_buf[0].add_(1)
                flush_buf[2].add_(flush_buf[1].sum())
                evs[k][0].record(stream)
                e.step(dt)
                evs[k][1].record(stream)
        torch.cuda.synchronize()
        t = [a.elapsed_time(b) for a, b in evs]
        if per_step is not None and not per_step:
            per_step.extend(t)
        return sum(t)

    # the headline pass runs without the library's stage timers (their events cost time)
    launches0 = e.kernel_launches()
    ms = one_pass(steps)
    launches = e.kernel_launches() - launches0
    if dist is not None:
        dist.barrier()
    # a second, shorter pass with stage timers for the per-kernel roofline and the breakdown
    kprof = min(steps, 200)
    e.set_profiling(True)
    one_pass(kprof)
    prof = e.profile()
    e.set_profiling(False)
    prof = {k: (v[0] * steps / kprof, int(round(v[1] * steps / kprof))) for k, v in prof.items()}
    return ms, launches, prof


def timed_chunks(e, dt, chunks, chunk, warmup, torch, flush_buf, stream):
    """Steps in chunks of `chunk` (each one CUDA-graph replay), L2 flushed between chunks."""
    spin_up(torch, flush_buf, stream)
    e.set_graph_steps(chunk)
    e.step(dt, chunk * max(1, warmup))
    torch.cuda.synchronize()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(chunks)]
    l0 = e.kernel_launches()
    with torch.cuda.stream(stream):
        for k in range(chunks):
            flush_buf[0].add_(1)
            flush_buf[2].add_(flush_buf[1].sum())
            evs[k][0].record(stream)
            e.step(dt, chunk)
            evs[k][1].record(stream)
    torch.cuda.synchronize()
    return sum(a.elapsed_time(b) for a, b in evs), e.kernel_launches() - l0, e.graph_active()


# steps of the adjoint checks' finite differences, largest first (the first is the step the
# gradient checks use elsewhere): the composed k_n, c_n, mu, and initial velocities
HOPPER_PARAM_STEPS = {"k_n": (1e-1, 1e-2, 1e-3), "c_n": (1e-4, 1e-5, 1e-6),
                      "mu": (1e-5, 1e-6, 1e-7)}
HOPPER_V_STEPS = (1e-6, 1e-7, 1e-8)


def adjoint_extra(torch):
    """The differentiable-DEM workload: 16384 spheres in the hopper, 2000 FP64 steps with a
    checkpoint every 100, gradient of final centre-of-mass height plus mass fraction below the
    opening w.r.t. all initial velocities and k_n, c_n, mu.  Checked over the full horizon against
    central differences of the GPU forward (parameters, and the four initial-velocity components
    with the largest adjoint) and against pe's own FP64 central differences of the parameters
    (tests/golden/hopper_fd.npz, made by the compiled reference); and over the last 100-step
    segment, where every sphere near the floor is in contact, against GPU central differences."""
    from pe_b200 import _abi
    from pe_b200.adjoint import LossSpec, make_single_material, set_params
    from pe_b200.engine import Engine
    s0 = scenes.hopper(0)
    m = s0.materials[0]
    p = {"k_n": m[6] / 2, "c_n": m[7] / 2, "c_t": m[8] / 2, "mu": 2 * m[2]}
    s = make_single_material(s0, **p)
    spec = LossSpec.for_scene(s, z_open=10.0)
    K, EVERY = s.steps, 100
    e = Engine(solver=_abi.DEM, precision=_abi.FP64).load_scene(s)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e.adjoint_forward(K, s.dt, EVERY)
    x = e.download()[0]
    t1 = time.perf_counter()
    z = np.zeros_like(x)
    _, gv0, _, gp = e.adjoint_backward(spec.grad(x), z, z)
    t2 = time.perf_counter()
    out = {"spheres": s.n, "steps": K, "checkpoint_every": EVERY, "loss": spec.value(x),
           "forward_ms": 1e3 * (t1 - t0), "backward_ms": 1e3 * (t2 - t1),
           "grad_params": {"k_n": gp[0], "c_n": gp[1], "c_t": gp[2], "mu": gp[3]},
           "grad_v0_linf": float(np.abs(gv0).max())}
    e.close()

    def gpu_x(t, steps):
        g = Engine(solver=_abi.DEM, precision=_abi.FP64, neighbor_lists=False).load_scene(t)
        g.step(t.dt, steps)
        x = g.download()[0]
        g.close()
        return x

    from pe_b200.adjoint import difference_ladder
    pk = {"k_n": 0, "c_n": 1, "mu": 3}
    relerr = lambda a, b: abs(a - b) / max(abs(b), 1e-300)

    def check(start, steps, gv, gpar):
        """Adjoint against finite differences of the GPU forward from `start`: the parameters
        and the four initial-velocity components with the largest adjoint, each at a ladder
        of steps (the first is the step of the other checks; see difference_ladder)."""
        cache = {}

        def xs(key, off, make):
            if off == 0.0:
                key = "base"
            if (key, off) not in cache:
                cache[(key, off)] = gpu_x(make(off), steps)
            return cache[(key, off)]

        res = {}
        flat = np.argsort(-np.abs(gv).ravel())[:4]
        quantities = [(k, float(gpar[j]), HOPPER_PARAM_STEPS[k],
                       lambda off, k=k: set_params(start, **dict(p, **{k: p[k] + off})))
                      for k, j in pk.items()]
        for f in flat:
            i, a = int(f // 3), int(f % 3)

            def mv(off, i=i, a=a):
                t = start.copy()
                t.v[i, a] += off
                return t
            quantities.append((f"v[{i}][{a}]", float(gv[i, a]), HOPPER_V_STEPS, mv))
        for name, ad, hs, make in quantities:
            rows, ch = difference_ladder(
                lambda u, w, name=name, make=make: spec.diff(xs(name, u, make), xs(name, w, make)),
                hs)
            res[name] = {"adjoint": ad, "ladder": rows, "chosen_h": ch["h"],
                         "rel_err": relerr(ad, ch["central"]),
                         "rel_err_at_first_h": relerr(ad, rows[0]["central"])}
        return {"steps": steps, "quantities": res,
                "max_rel_err": max(q["rel_err"] for q in res.values())}

    full = check(s, K, gv0, gp)
    gold = os.path.join(ROOT, "tests", "golden", "hopper_fd.npz")
    if os.path.exists(gold):
        g = np.load(gold)
        if int(g["steps"]) == K and int(g["spheres"]) == s.n:
            ref = {}
            for k, j in pk.items():
                rows = [{"h": float(h), "forward": float(fw), "backward": float(bw),
                         "central": 0.5 * float(fw + bw),
                         "smooth": bool(abs(fw - bw) <= 1e-4 * abs(0.5 * (fw + bw)))}
                        for h, fw, bw in zip(g["h_" + k], g["fwd_" + k], g["bwd_" + k])]
                ch = next((r for r in rows if r["smooth"]), rows[-1])
                ref[k] = {"ladder": rows, "chosen_h": ch["h"],
                          "rel_err": relerr(float(gp[j]), ch["central"])}
            full["reference_params"] = ref
            full["reference_fd_source"] = ("pe compiled from its sources, FP64 one-sided "
                                           "differences over the full horizon "
                                           "(tests/golden/make_golden.py hopper_fd)")
    out["full_horizon_check"] = full
    # the last segment: state after K - 100 steps, adjoint of 100 steps vs central differences
    e = Engine(solver=_abi.DEM, precision=_abi.FP64, neighbor_lists=False).load_scene(s)
    e.step(s.dt, K - EVERY)
    xs, vs, ws = e.download()
    e.close()
    seg = s.copy()
    seg.x, seg.v, seg.w = xs, vs, ws
    e = Engine(solver=_abi.DEM, precision=_abi.FP64).load_scene(seg)
    e.adjoint_forward(EVERY, s.dt, 10)
    xe = e.download()[0]
    _, gvs, _, gps = e.adjoint_backward(spec.grad(xe), z, z)
    e.close()
    segment = check(seg, EVERY, gvs, gps)
    segment["from_step"] = K - EVERY
    out["segment_check"] = segment
    return out


def nsph_total(ss, dist, torch, dev):
    tot = torch.tensor([float(sum(s.n for s in ss))], dtype=torch.float64, device=dev)
    if dist is not None:
        dist.all_reduce(tot, op=dist.ReduceOp.SUM)
    return float(tot.item())


def end_to_end(ss, kind, precision, tuning, dt, steps, torch, dev, dist):
    """The public API end to end: a new context, the bodies uploaded from pinned host arrays,
    `steps` steps, the state downloaded into pinned host arrays; wall clock. One untimed pass
    first (host thread pools, first allocations), then the median of three passes, each taken
    as the max over ranks."""
    staged = stage_inputs(ss, torch)
    nsph = sum(s.n for s in ss)
    outs = [torch.zeros((nsph, 3), dtype=torch.float64).pin_memory().numpy() for _ in range(3)]
    runs = []
    for rep in range(4):
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        t0 = time.perf_counter()
        # the tuned skin sizes the cells at upload; the launch shapes follow
        e2 = engine_from_staged(staged, kind, precision,
                                skin=tuning["skin"] if tuning is not None else 0.0)
        if tuning is not None:
            e2.set_tuning(tuning["dem_variant"], tuning["rebuild_per_sm"], tuning["skin"],
                          dem_split=tuning.get("dem_split", 0))
        t1 = time.perf_counter()
        e2.step(dt, steps)
        t2 = time.perf_counter()
        out = e2.download(out=outs)
        torch.cuda.synchronize()
        t3 = time.perf_counter()
        e2.close()
        te = torch.tensor([t3 - t0, t1 - t0, t2 - t1, t3 - t2], dtype=torch.float64, device=dev)
        if dist is not None:
            dist.all_reduce(te, op=dist.ReduceOp.MAX)
        runs.append([float(a) for a in te.tolist()])
    h2d = sum(staged[k].nbytes for k in ("x", "v", "w", "r", "mat")) + \
        (staged["scene"].nbytes if staged["scene"] is not None else 0)
    d2h = sum(a.nbytes for a in out if a is not None)
    timed = sorted(runs[1:], key=lambda r: r[0])
    med = timed[len(timed) // 2]
    parts = {"setup_upload_ms": 1e3 * med[1], "steps_issue_ms": 1e3 * med[2],
             "download_sync_ms": 1e3 * med[3]}
    return med[0], parts, [1e3 * r[0] for r in runs], h2d, d2h


def our_arm(args):
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as tdist
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                 device_id=torch.device("cuda", local))
        dist = tdist
    from pe_b200 import _abi
    from pe_b200.engine import Engine

    ref_run = None
    ss, kind = build_workload(args.workload, rank=rank, world=world)
    nsph = sum(s.n for s in ss)
    dt = ss[0].dt
    dev = torch.device("cuda", local)
    flush = (torch.zeros(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev),
             torch.ones(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev),
             torch.zeros(1, dtype=torch.float32, device=dev))
    precision = _abi.MIXED
    e = make_engine(ss, kind, precision)
    # launch shapes and skin picked by the library's autotuner from the initial state (untimed;
    # the state is restored)
    tuning = None
    if kind == "dem" and args.tuning:
        parts = args.tuning.split(",")
        v, r, sk = parts[:3]
        e.set_tuning(int(v), int(r), float(sk), dem_split=int(parts[3]) if len(parts) > 3 else 0)
        tuning = dict(e.tuning(), source="--tuning")
    elif kind == "dem":
        tuning = e.autotune(dt, 100)
    stream = torch.cuda.ExternalStream(e.stream_ptr(), device=dev)
    uuid = None
    try:
        uuid = str(torch.cuda.get_device_properties(dev).uuid)
        uuid = uuid if uuid.startswith("GPU-") else "GPU-" + uuid
    except Exception:
        uuid = None
    # end to end first: nvidia-smi polling (the clock record of the device-timed region) slows
    # the driver calls that allocate and free, here and for a while after it stops
    e2e_s, e2e_parts, e2e_runs, h2d, d2h = end_to_end(ss, kind, precision, tuning, dt, args.steps,
                                                      torch, dev, dist)
    e2e_value = nsph_total(ss, dist, torch, dev) * args.steps / e2e_s
    clocks = Clocks(uuid)
    nl0 = e.neighbor_list_stats() if kind == "dem" else None
    clocks.start()
    step_ms = []
    ms, launches, prof = timed_steps(e, dt, args.steps, args.warmup, torch, flush, stream, dist,
                                     per_step=step_ms)
    clk = clocks.stop()
    nl1 = e.neighbor_list_stats() if kind == "dem" else None
    # the cpu_baseline leg: pe on one host core over the same scene, started once the headline
    # and end-to-end measurements are done (pe's set-up of a 1M-sphere scene takes minutes and
    # its host load slowed the end-to-end set-up) and collected after the other GPU lines
    if world == 1 and not args.no_cpu_baseline:
        ref_run = RefRun(args.workload, REF_STEPS[args.workload], warmup=1, procs=1)
    t = torch.tensor([ms], dtype=torch.float64, device=dev)
    tot = torch.tensor([float(nsph)], dtype=torch.float64, device=dev)
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dist.all_reduce(tot, op=dist.ReduceOp.SUM)
    ms_max = float(t.item())
    total_sph = float(tot.item())
    value = total_sph * args.steps / (ms_max / 1e3)


    if dist is not None:
        dist.destroy_process_group()
    if rank != 0:
        e.close()
        return None

    # roofline of the dominant work: the DEM list step as timed (its kernels overlap in the
    # overlapped form, so the step is the unit), or the NBGS sweeps
    peak, peak_src = _peak_gbs()
    stage_timed = None
    if kind == "dem":
        per = ALGO_BYTES["mixed"]
        algo = per * nsph
        kms, kcnt = ms_max, args.steps
        form = (tuning or {}).get("dem_split", 0)
        kname = {0: "the list step: k_rebuild_contacts (rebuild check, marked spheres' forces), "
                    "then k_dem_move (integration of every sphere)",
                 1: "the list step: k_rebuild (rebuild check), then k_dem_contacts (marked "
                    "spheres) on a second stream beside k_dem_move (the others)",
                 2: "the list step, overlapped: k_rebuild_contacts (rebuild check, marked "
                    "spheres' forces and integration) beside k_dem_move (integration of the "
                    "unmarked spheres), one stream"}.get(form, "the list step")
        sms, scnt = prof.get("dem_step", (0.0, 0))
        if scnt:
            sav = sms / scnt
            stage_timed = {"kernels": "k_dem_contacts + k_dem_move, run one after the other in "
                                      "the stage-timed pass (the library's stage timers keep "
                                      "the kernels apart)",
                           "avg_launch_ms": sav, "achieved": algo / (sav / 1e3) / 1e9,
                           "frac": algo / (sav / 1e3) / 1e9 / peak}
    else:
        kms, kcnt = prof.get("sweeps", (0.0, 0))
        st = e.stats()
        algo = 100 * (128.0 * st["contacts"] + 80.0 * nsph)
        kname = "k_sweep<float> (100 sweeps)"
    nls = None
    if kind == "dem":
        # rebuilds of the warm-up, timed and stage-timed steps (the autotuner's trials before
        # them rebuild too)
        nls = dict(nl1, rebuilds_in_measured_steps=nl1["rebuilds"] - nl0["rebuilds"],
                   measured_steps=args.warmup + args.steps + min(args.steps, 200))
    kavg = kms / max(kcnt, 1)
    achieved = algo / (kavg / 1e3) / 1e9 if kavg > 0 else None
    traffic = read_traffic(args.workload)
    roofline = {"bound": "hbm", "kernel": kname, "achieved": achieved, "peak": peak,
                "unit": "GB/s", "frac": (achieved / peak) if achieved else None,
                "traffic": traffic, "peak_source": peak_src,
                "algorithmic_bytes_per_launch": algo, "avg_launch_ms": kavg}
    if kind == "dem":
        roofline["timing"] = ("the step's CUDA events on the library's stream over the timed "
                              "region (every kernel of the step inside: rebuild check, forces, "
                              "integration)")
        roofline["stage_timed"] = stage_timed
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "strong" if args.workload == "ensemble_512" else "weak",
            "vs_baseline": None, "dtype": "f32 (f64 positions)", "data": "synthetic (seeded)",
            "config": {"workload": args.workload, "spheres": int(total_sph),
                       "spheres_per_rank": nsph, "scenes": len(ss),
                       "precision": "mixed", "dt": dt, "tuning": tuning,
                       "l2": "flushed between timed steps (256 MiB write + 256 MiB read, "
                             "untimed); the flush also writes back the lines each step left "
                             "dirty in L2, outside the timed region (graph_replay_16 runs 16 "
                             "steps back to back and pays for them)",
                       "parallelism": ("1 GPU" if world == 1 else
                                       f"scenes partitioned over {world} ranks"
                                       if args.workload == "ensemble_512" else
                                       f"replicas x{world}")},
            "clocks": clk, "gpu_launches": launches,
            "step_ms": {"min": min(step_ms), "median": float(np.median(step_ms)),
                        "max": max(step_ms), "first": step_ms[0],
                        "note": "this rank's timed steps, each between two L2 flushes; ~20 ms "
                                "of untimed flush kernels run before the warm-up steps"},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d / args.steps,
                    "d2h_bytes_per_step": d2h / args.steps,
                    "note": "new context, upload from pinned host arrays, steps, download into "
                            "pinned host arrays, through the C ABI; wall clock; median of 3 "
                            "passes after 1 untimed pass, max over ranks",
                    "parts": e2e_parts, "passes_ms": e2e_runs},
            "roofline": roofline,
            "stages_ms_per_step": {k: v[0] / args.steps for k, v in prof.items() if v[1]},
            "neighbor_lists": nls}
    e.close()
    if not args.no_extras:
        line.update(extras(args, torch, flush, dev, ss, kind, value))
    if ref_run is not None:
        ref, why = ref_run.result()
        if ref:
            line["cpu_baseline"] = {"value": ref["sphere_steps_per_s"], "unit": UNIT,
                                    "cores": ref["cores"], "kind": "reference",
                                    "sample": ref["sample"]}
        else:
            line["cpu_baseline"] = {"value": None, "unit": UNIT, "cores": 0,
                                    "kind": "reference", "sample": why}
    return line


def boxes_extra(torch, flush, dev):
    """Scenes with moving boxes (FP64, the only precision for boxes): a 6x6x6 stack of cubes
    resting face to face (every face contact held by gravity) under the hard-contact solver,
    and 110,592 spheres with 1,000 tilted boxes falling on them under DEM; body-steps/s on the
    GPU and in pe on one host core."""
    from pe_b200 import _abi
    out = {}
    for label, sc, kind in (("stack_216_hcsits", scenes.box_stack(6, 6, overlap=0.0), "hcsits"),
                            ("spheres110k_boxes1000_dem", scenes.spheres_and_boxes(0), "dem")):
        e = make_engine([sc], kind, _abi.FP64)
        st = torch.cuda.ExternalStream(e.stream_ptr(), device=dev)
        k = 20
        ms, _, prof = timed_steps(e, sc.dt, k, 3, torch, flush, st)
        stt = e.stats()
        e.close()
        nb = sc.n + sc.nmbox
        rec = {"bodies": nb, "spheres": sc.n, "boxes": sc.nmbox, "ms_per_step": ms / k,
               "body_steps_per_s": nb * k / (ms / 1e3), "precision": "fp64"}
        if kind == "hcsits":
            rec.update({"contacts": stt["contacts"], "colors": stt["colors"], "sweeps": 100})
        exe = os.path.join(REF_DIR, "ref_dem" if kind == "dem" else "ref_hcsits")
        if os.path.exists(exe):
            with tempfile.TemporaryDirectory() as tmp:
                sp = os.path.join(tmp, "s.bin")
                sc.save(sp)
                extra = ["1", "100"] if kind == "hcsits" else []
                r = subprocess.run([exe, "time", sp, "1", "5", *extra], capture_output=True,
                                   text=True, timeout=600)
                if r.returncode == 0:
                    sec = json.loads(r.stdout.strip().splitlines()[-1])["seconds"]
                    rec["pe_one_core"] = {"ms_per_step": sec / 5 * 1e3,
                                          "body_steps_per_s": nb * 5 / sec}
        out[label] = rec
    return out


def _peak_gbs():
    """The HBM roofline peak: MEASURED_PEAKS.json's copy bandwidth, else the pool's fallback."""
    pp = os.path.join(ROOT, "MEASURED_PEAKS.json")
    peak = json.load(open(pp)).get("hbm_gbs") if os.path.exists(pp) else None
    return (peak, "measured") if peak else (6650.0, "fallback")


def dense_extra(torch, flush, dev, steps):
    """The contact-dense DEM workload (every sphere in contact every step, lists rebuilt often):
    1,048,576 spheres, mixed precision, tuned launch shapes, stepped one call per step with the
    L2 flushed between steps, and through CUDA-graph replays of 16 steps."""
    from pe_b200 import _abi
    s = scenes.dem_dense(0)
    e = make_engine([s], "dem", _abi.MIXED)
    tu = e.autotune(s.dt, 50)
    st = torch.cuda.ExternalStream(e.stream_ptr(), device=dev)
    k = max(20, min(steps, 200))
    r0 = e.neighbor_list_stats()
    ms, launches, prof = timed_steps(e, s.dt, k, 3, torch, flush, st)
    r1 = e.neighbor_list_stats()
    msg, _, active = timed_chunks(e, s.dt, max(2, k // 16), 16, 1, torch, flush, st)
    kg = max(2, k // 16) * 16
    e.close()
    # the force stage's algorithmic bytes: the headline's per-sphere state traffic, plus the
    # list entries read and each sphere's stored force, written then read (every sphere of this
    # scene is marked)
    per = ALGO_BYTES["mixed"] + 4.0 * r1["entries"] / s.n + 2 * 24.0
    # over the timed step (every kernel of it, rebuilds included), as for the headline
    kavg = ms / k
    peak = _peak_gbs()
    achieved = per * s.n / (kavg / 1e3) / 1e9 if kavg > 0 else None
    return {"value": s.n * k / (ms / 1e3), "unit": "sphere-steps/s", "ms_per_step": ms / k,
            "roofline": {"bound": "hbm", "kernel": "the list step (form: tuning.dem_split)",
                         "achieved": achieved, "peak": peak[0], "unit": "GB/s",
                         "frac": achieved / peak[0] if achieved else None,
                         "peak_source": peak[1], "algorithmic_bytes_per_sphere": per,
                         "avg_launch_ms": kavg,
                         "timing": "the step's CUDA events over the timed region"},
            "graph_replay_16_value": s.n * kg / (msg / 1e3), "graph_active": active,
            "spheres": s.n, "precision": "mixed", "tuning": tu,
            "rebuilds_per_step": (r1["rebuilds"] - r0["rebuilds"]) / (k + min(k, 200) + 3),
            "list_entries_per_sphere": r1["entries"] / s.n,
            "stages_ms_per_step": {a: b[0] / k for a, b in prof.items() if b[1]}}


def nbgs_extra(torch, flush, dev):
    """The 32,768-sphere hard-contact workload as specified (free fall in the 40x40x120 box, few
    contacts) and a pre-settled dense variant (a lattice at the bottom of a 32x32x120 box, about
    20,000 contacts), each frictionless (pe's InelasticFrictionlessContact) and with mu = 0.5
    (pe's default ApproximateInelasticCoulombContactByDecoupling), 100 sweeps per step, mixed
    precision and FP64.  Frictional runs report the FP64 complementarity residual of the last
    step's impulses (one extra step with the residual enabled, after the timed ones); on the
    4096-sphere dense packing the GPU's residual is reported beside the oracle's for the same
    sweep counts (committed with the golden vectors)."""
    from pe_b200 import _abi
    out = {}
    variants = (("nbgs_32k", lambda mu: scenes.nbgs_box(0, mu=mu)),
                ("nbgs_32k_dense", lambda mu: scenes.nbgs_box(0, n=32768, mu=mu,
                                                              dims=(32.0, 32.0, 120.0),
                                                              dense=True)))
    for label, make in variants:
        for mu in (0.0, 0.5):
            sc = make(mu)
            key = label if mu == 0.0 else label + "_mu0.5"
            for prec, name in ((_abi.MIXED, "mixed"), (_abi.FP64, "fp64")):
                e = make_engine([sc], "hcsits", prec)
                st = torch.cuda.ExternalStream(e.stream_ptr(), device=dev)
                ksteps = 10
                ms, _, prof = timed_steps(e, sc.dt, ksteps, 2, torch, flush, st)
                stt = e.stats()
                # the same steps in calls of 16 (one CUDA-graph replay each), L2 flushed between
                msg, _, active = timed_chunks(e, sc.dt, 3, 16, 1, torch, flush, st)
                rec = {"value": sc.n * 48 / (msg / 1e3), "ms_per_step": msg / 48,
                       "graph_active": active, "graph_steps_timed": "39-86",
                       "ms_per_step_one_step_calls": ms / ksteps,
                       "contacts": stt["contacts"], "colors": stt["colors"], "sweeps": 100,
                       "model": "approx_coulomb_decoupling" if mu > 0 else "frictionless",
                       "stages_ms_per_step": {a: b[0] / ksteps for a, b in prof.items() if b[1]}}
                if label == "nbgs_32k":
                    # the free fall before the first contact (steps 19-34): steps planned
                    # without the contact stages, one graph replay of 16, L2 flushed before
                    f = make_engine([sc], "hcsits", prec)
                    f.step(sc.dt, 2)
                    fst = torch.cuda.ExternalStream(f.stream_ptr(), device=dev)
                    mcf, _, _ = timed_chunks(f, sc.dt, 1, 16, 0, torch, flush, fst)
                    rec["contact_free_ms_per_step"] = mcf / 16
                    rec["contact_free_contacts_after"] = f.stats()["contacts"]
                    f.close()
                    # the configured run whole: its 200 steps in one call (graph replays of
                    # 16) after one untimed step that allocates, L2 flushed before it
                    f = make_engine([sc], "hcsits", prec)
                    fst = torch.cuda.ExternalStream(f.stream_ptr(), device=dev)
                    f.step(sc.dt, 1)
                    torch.cuda.synchronize()
                    flush[0].add_(1)
                    flush[2].add_(flush[1].sum())
                    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    with torch.cuda.stream(fst):
                        a.record(fst)
                        f.step(sc.dt, sc.steps)
                        b.record(fst)
                    torch.cuda.synchronize()
                    rec["configured_run_ms_per_step"] = a.elapsed_time(b) / sc.steps
                    rec["configured_run_steps"] = sc.steps
                    rec["configured_run_contacts_at_end"] = f.stats()["contacts"]
                    f.close()
                if mu > 0:
                    e.set_residual(True)
                    e.step(sc.dt)
                    rec["residual_fp64"] = e.stats()["residual"]
                    rec["residual_note"] = ("max over contacts of the complementarity residual, "
                                            "velocity units, after 100 sweeps of one step")
                out.setdefault(key, {})[name] = rec
                e.close()
    gold = os.path.join(ROOT, "tests", "golden", "dense4096_conv.npz")
    if os.path.exists(gold):
        g = np.load(gold)
        sc = scenes.nbgs_box(0, n=4096, mu=0.5, dims=(16.0, 16.0, 60.0), dense=True)
        rows = []
        for k, r_or in zip(g["mu05_sweeps"], g["mu05_residual_oracle"]):
            e = make_engine([sc], "hcsits", _abi.FP64, iters=int(k))
            e.set_residual(True)
            e.step(sc.dt)
            stt = e.stats()
            e.close()
            rows.append({"sweeps": int(k), "residual_gpu_fp64": stt["residual"],
                         "residual_oracle": float(r_or)})
        out["nbgs_4096_dense_mu0.5_residual_vs_oracle"] = {
            "spheres": sc.n, "contacts": int(g["contacts"]), "rows": rows,
            "note": "same packing and model; the oracle sweeps in pe's detection order, the GPU "
                    "colour by colour"}
    return out


def extras(args, torch, flush, dev, ss, kind, mixed_value):
    """Beside the headline: the plain FP64 GPU path (grid search every step, the first CUDA
    form), the FP64 path with neighbour lists, the mixed-vs-FP64 position error after 1000 steps,
    the batched ensemble, the NBGS scenes, and the compiled reference."""
    from pe_b200 import _abi
    out = {}
    nsph = sum(s.n for s in ss)
    dt = ss[0].dt

    def timed(e, k, w=3):
        st = torch.cuda.ExternalStream(e.stream_ptr(), device=dev)
        ms, _, prof = timed_steps(e, dt if e is not None else dt, k, w, torch, flush, st)
        return ms, prof

    if kind == "dem":
        for label, prec, lists in (("plain_fp64", _abi.FP64, False), ("fp64", _abi.FP64, True)):
            k = max(10, min(args.steps, 200))
            e = make_engine(ss, kind, prec, lists=lists)
            ms, prof = timed(e, k)
            v = nsph * k / (ms / 1e3)
            out[label] = {"value": v, "ms_per_step": ms / k, "mixed_over_this": mixed_value / v,
                          "neighbor_lists": lists,
                          "stages_ms_per_step": {a: b[0] / k for a, b in prof.items() if b[1]}}
            e.close()
        # stated error: mixed against FP64 positions after 1000 steps from the same state
        em = make_engine(ss, kind, _abi.MIXED)
        ef = make_engine(ss, kind, _abi.FP64)
        em.step(dt, 1000)
        ef.step(dt, 1000)
        xm, xf = em.download()[0], ef.download()[0]
        x0 = np.concatenate([s.x for s in ss])
        d, disp = np.abs(xm - xf), np.abs(xf - x0)
        out["error_after_1000_steps"] = {
            "displacement_rel_linf": float(d.max() / max(disp.max(), 1e-300)),
            "displacement_rel_l2": float(np.sqrt((d ** 2).sum() / max((disp ** 2).sum(), 1e-300))),
            "position_rel_linf": float(d.max() / np.abs(xf).max()),
            "stated_measure": "displacement_rel_linf = max_i |x_mixed - x_fp64| / "
                              "max_i |x_fp64 - x_0| (the largest error against the largest "
                              "distance travelled); target <= 1e-6",
            "reference": "FP64 GPU path (itself within 1e-12 of pe's FP64 step)"}
        em.close()
        ef.close()
    if kind == "dem":
        # the same tuned mixed step through CUDA-graph replays of 16 steps, flushed between
        # replays (the scene's state and lists, > 126 MB, exceed L2 within a replay as well)
        e = make_engine(ss, kind, _abi.MIXED)
        tu = e.autotune(dt, 100)
        st = torch.cuda.ExternalStream(e.stream_ptr(), device=dev)
        chunks = max(2, min(args.steps, 400) // 16)
        ms, launches, active = timed_chunks(e, dt, chunks, 16, 3, torch, flush, st)
        out["graph_replay_16"] = {"value": nsph * chunks * 16 / (ms / 1e3),
                                  "ms_per_step": ms / (chunks * 16), "steps": chunks * 16,
                                  "graph_active": active, "gpu_launches": launches,
                                  "tuning": tu}
        e.close()
    if args.workload == "dem_large_1m":
        ens = scenes.batched_ensemble(0)
        ne = sum(s.n for s in ens)
        e = make_engine(ens, "dem", _abi.MIXED)
        tu = e.autotune(ens[0].dt, 50)
        st = torch.cuda.ExternalStream(e.stream_ptr(), device=dev)
        k = 48
        ms, _, prof = timed_steps(e, ens[0].dt, k, 3, torch, flush, st)
        msg, _, active = timed_chunks(e, ens[0].dt, 3, 16, 1, torch, flush, st)
        out["ensemble_512"] = {"value": ne * k / (ms / 1e3), "ms_per_step": ms / k,
                               "graph_replay_16_value": ne * 48 / (msg / 1e3),
                               "graph_replay_16_ms_per_step": msg / 48, "graph_active": active,
                               "spheres": ne, "scenes": len(ens), "precision": "mixed",
                               "tuning": tu,
                               "stages_ms_per_step": {a: b[0] / k for a, b in prof.items() if b[1]}}
        e.close()
        out["dem_dense_1m"] = dense_extra(torch, flush, dev, args.steps)
        out["adjoint_hopper_16384"] = adjoint_extra(torch)
        out.update(nbgs_extra(torch, flush, dev))
    if args.workload == "dem_large_1m":
        out["moving_boxes"] = boxes_extra(torch, flush, dev)
    return out


def read_traffic(workload):
    """DRAM bytes per launch of the dominant kernel from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", f"{workload}_launch_traffic.txt")
    if not os.path.exists(path):
        return None
    for line in open(path):
        if line.startswith("dram_bytes_per_launch:"):
            try:
                return float(line.split(":", 1)[1].split()[0])
            except ValueError:
                return None
    return None


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return None
    procs = ref_procs(args.workload)
    run = RefRun(args.workload, REF_STEPS[args.workload], warmup=1, procs=procs)
    ref, why = run.result()
    if not ref:
        return {"impl": "reference", "unavailable": why}
    v = ref["sphere_steps_per_s"]
    sc = ref_scene(args.workload)[0]
    return {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT,
            "n_gpus": int(os.environ.get("WORLD_SIZE", "1")), "steps": ref["steps"],
            "warmup": 1, "ms_per_step": 1e3 * ref["seconds"] / ref["steps"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded)",
            "config": {"workload": args.workload, "spheres": sc.n, "spheres_per_rank": sc.n,
                       "scenes": 1, "dt": sc.dt,
                       "precision": "fp64 (pe's real; compiled -O3 -DNDEBUG from its sources)",
                       "parallelism": f"{procs} host processes, each the whole scene"},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": ref["cores"], "kind": "reference",
                             "sample": ref["sample"]},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


# Small cases of the library's kernels, each a few launches on inputs larger than L2, for the
# committed ncu summaries (profiles/): python bench.py --profile-case NAME --steps K
PROFILE_CASES = {
    # the plain FP64 grid step (sort + k_dem_sorted) on the 1M scene
    "dem_grid_fp64": ("dem", 1048576, "fp64", False),
    "dem_grid_mixed": ("dem", 1048576, "mixed", False),
    # the headline list step (k_rebuild, k_dem_contacts, k_dem_move) on the full 1M scene
    "dem_list_mixed": ("dem", 1048576, "mixed", True),
    "dem_list_fp64": ("dem", 1048576, "fp64", True),
    # the contact-dense 1M scene (every sphere in contact, frequent rebuilds)
    "dem_dense_mixed": ("dense", 1048576, "mixed", True),
    # hard-contact step on the dense 32k packing (detection, colouring, cache, sweeps)
    "nbgs_dense_mixed": ("hcsits", 32768, "mixed", None),
    "nbgs_dense_fp64": ("hcsits", 32768, "fp64", None),
    # hard-contact step on the loose 32k scene (no contacts for most of its steps)
    "nbgs_free_mixed": ("hcsits_free", 32768, "mixed", None),
    # the 512-scene ensemble (list step)
    "ensemble_mixed": ("ensemble", 0, "mixed", True),
    # the adjoint of 100 steps of the hopper
    "adjoint_hopper": ("adjoint", 16384, "fp64", None),
}


def profile_case(args):
    """Runs --steps steps of one PROFILE_CASES entry after --warmup steps; prints the stage
    times (library events) as one JSON line."""
    import torch
    from pe_b200 import _abi
    from pe_b200.engine import Engine
    kind, n, prec, lists = PROFILE_CASES[args.profile_case]
    precision = _abi.FP64 if prec == "fp64" else _abi.MIXED
    if kind == "dem":
        side = 200.0 * (n / 1048576) ** 0.5
        sc = scenes.dem_large(0, n=n, dims=(side, side, 400.0)) if n != 1048576 else \
            scenes.dem_large(0)
        e = make_engine([sc], "dem", precision, lists=lists)
        dt = sc.dt
    elif kind == "dense":
        sc = scenes.dem_dense(0)
        e = make_engine([sc], "dem", precision, lists=lists)
        dt = sc.dt
    elif kind in ("hcsits", "hcsits_free"):
        sc = scenes.nbgs_box(0, n=n, dims=(32.0, 32.0, 120.0), dense=True) \
            if kind == "hcsits" else scenes.nbgs_box(0, n=n)
        e = make_engine([sc], "hcsits", precision)
        dt = sc.dt
    elif kind == "ensemble":
        ens = scenes.batched_ensemble(0)
        e = make_engine(ens, "dem", precision)
        dt = ens[0].dt
    else:
        from pe_b200.adjoint import make_single_material
        s0 = scenes.hopper(0)
        m = s0.materials[0]
        sc = make_single_material(s0, k_n=m[6] / 2, c_n=m[7] / 2, c_t=m[8] / 2, mu=2 * m[2])
        e = Engine(solver=_abi.DEM, precision=_abi.FP64).load_scene(sc)
        e.step(sc.dt, 1900)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e.adjoint_forward(args.steps, sc.dt, 10)
        x = e.download()[0]
        z = np.zeros_like(x)
        e.adjoint_backward(x * 0 + 1.0, z, z)
        torch.cuda.synchronize()
        print(json.dumps({"case": args.profile_case, "steps": args.steps,
                          "wall_ms": 1e3 * (time.perf_counter() - t0)}))
        e.close()
        return
    e.step(dt, args.warmup)
    torch.cuda.synchronize()
    e.set_profiling(True)
    e.step(dt, args.steps)
    prof = e.profile()
    print(json.dumps({"case": args.profile_case, "steps": args.steps,
                      "stages_ms_per_step": {k: v[0] / args.steps for k, v in prof.items()
                                             if v[1]}}))
    e.close()


def main():
    args = parse()
    if args.profile_case:
        profile_case(args)
        return
    line = reference_arm(args) if args.impl == "reference" else our_arm(args)
    if line is not None:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
