#!/usr/bin/env python
"""Benchmark of the B200 hybrid particle-grid substep (particle-steps/s).

Workload (one GPU): the FLIP dam break on a 128^3 MAC grid over the unit cube with solid walls; the
fluid block [0,0.4]x[0,0.6]x[0,1] is seeded with 8 jittered particles per cell (subcell rule, seed 0;
4,021,248 particles), FLIP ratio 0.95, gravity (0,-9.81,0), fixed dt = 1/240 s, pressure by FP32 CG
inside FP64 refinement to relative residual 1e-6.  A "step" is one substep of the whole hot path
(sort, P2G, marking, grid passes, pressure solve, G2P + advection) on the device-resident state.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--n 128]

Under torchrun every rank runs its own independent scene (replicas: a scene does not shard), the timed
region is bracketed by a barrier + synchronize, and the slowest rank's device time is used.  One JSON
line is printed by rank 0.  `--impl reference` times the reference's own CPU simulator (built from its
sources into oracle/_ref by oracle/build_ref.py) on the host cores, rank 0 only.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "particle-steps/s"
BOX = (0.0, 0.0, 0.0, 0.4, 0.6, 1.0)
DT = 1.0 / 240.0


# The --collider obstacle: a box in the dam break's path (TriangleMeshCollider on the scene's grid).
COLLIDER_BOX = (0.55, 0.0, 0.35, 0.8, 0.3, 0.65)


def box_mesh(b):
    """A closed box as (V (8,3), T (12,4): vertex ids and a normal id, N (12,3) unit face normals)."""
    import numpy as np

    lo, hi = np.array(b[:3], float), np.array(b[3:], float)
    V = np.array([[lo[0] if (c & 1) == 0 else hi[0], lo[1] if (c & 2) == 0 else hi[1], lo[2] if (c & 4) == 0 else hi[2]]
                  for c in range(8)])
    tri = []
    for a, b_, c, d in [(0, 2, 3, 1), (4, 5, 7, 6), (0, 1, 5, 4), (2, 6, 7, 3), (0, 4, 6, 2), (1, 3, 7, 5)]:
        tri += [(a, b_, c), (a, c, d)]
    T = np.array([[a, b_, c, t] for t, (a, b_, c) in enumerate(tri)], dtype=np.int64)
    N = np.cross(V[T[:, 1]] - V[T[:, 0]], V[T[:, 2]] - V[T[:, 0]])
    return V, T, N / np.linalg.norm(N, axis=1, keepdims=True)


def sphere_mesh(center, radius, subdiv=1):
    """An icosphere as (V, T (T,4)) for the --mesh-init report."""
    import numpy as np

    t = (1.0 + 5 ** 0.5) / 2.0
    V = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
         (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    F = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2), (10, 7, 6),
         (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10), (8, 6, 7),
         (9, 8, 1)]
    V = [np.array(v, float) / np.linalg.norm(v) for v in V]
    for _ in range(subdiv):
        cache, F2 = {}, []

        def mid(a, b):
            key = (min(a, b), max(a, b))
            if key not in cache:
                m = V[a] + V[b]
                V.append(m / np.linalg.norm(m))
                cache[key] = len(V) - 1
            return cache[key]

        for a, b, c in F:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            F2 += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        F = F2
    V = np.array(V) * radius + np.asarray(center, float)
    return V, np.array([[a, b, c, 0] for a, b, c in F], dtype=np.int64)


def workload_config(n, steps, warmup, n_gpus, np_, viscosity=0.0, collider=False):
    cfg = {
        "workload": "FLIP dam break %d^3, box [0,0.4]x[0,0.6]x[0,1], 8 particles/cell (seed 0), dt=1/240, "
                    "FP32 CG in FP64 refinement to rel 1e-6" % n + (", viscosity %g (backward Euler, Jacobi "
                                                                    "1000/5/1e-14)" % viscosity if viscosity else "")
                    + (", box collider [%g,%g]x[%g,%g]x[%g,%g] (TriangleMeshCollider on the %d^3 grid)"
                       % (COLLIDER_BOX[0], COLLIDER_BOX[3], COLLIDER_BOX[1], COLLIDER_BOX[4], COLLIDER_BOX[2],
                          COLLIDER_BOX[5], n) if collider else ""),
        "grid": [n, n, n], "particles": np_, "solver": "FLIP 0.95", "dt": DT, "cg_rel_tol": 1e-6, "max_cfl": 1.0,
        "substeps_timed": steps, "warmup": warmup, "parallelism": "replicas x%d" % n_gpus,
        "l2": "working set > 126 MB L2 (particles alone %.0f MB); no flush" % (np_ * 24 / 1e6),
    }
    if viscosity:
        cfg["viscosity"] = viscosity
    if collider:
        cfg["collider"] = list(COLLIDER_BOX)
    return cfg


def max_over_ranks(x, device):
    """The slowest rank's value of a time (every rank calls this at the same point); x itself on one rank."""
    import torch
    import torch.distributed as dist

    if not dist.is_initialized() or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(world, particles_per_rank, steps, seconds):
    """Whole-job particle-steps/s of `world` independent replicas timed by the slowest rank."""
    return world * particles_per_rank * steps / seconds


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def mg_coarse_cells(n):
    """Cells of the multigrid levels >= 1 for an n^3 grid (each axis halved, rounding up, until <= 8)."""
    dims, total = [n, n, n], 0
    while max(dims) > 8:
        dims = [(d + 1) // 2 for d in dims]
        total += dims[0] * dims[1] * dims[2]
    return total


def uses_multigrid(n, pressure_solver):
    return pressure_solver == "mgpcg" or (pressure_solver == "auto" and n ** 3 >= (1 << 15))


def solver_alg_bytes(fluid, its, refs, n, multigrid):
    """Algorithmic bytes of one pressure solve (numpy arrays per substep).  Plain CG: 41 B per FLUID cell per
    inner iteration.  Multigrid-preconditioned CG: 68 B per FLUID cell per inner iteration over the five
    level-0 passes (update + pre-smoothing residual 28, restriction read 4, pre-smoothed correction 8,
    post-smoothing 12, search direction 16) plus 30 B per cell of every coarser level (residual, restriction,
    correction, smoothing).  Both: 45 B per FLUID cell per FP64 residual pass (refinements + 1)."""
    if multigrid:
        return fluid * (its * 68.0 + (refs + 1.0) * 45.0) + its * 30.0 * mg_coarse_cells(n)
    return fluid * (its * 41.0 + (refs + 1.0) * 45.0)


def profile_traffic(multigrid=False):
    """DRAM bytes per unit of solver work from the committed ncu summary, or None."""
    path = os.path.join(ROOT, "profiles", "k_mgcg_traffic.txt" if multigrid else "k_cg_traffic.txt")
    try:
        with open(path) as f:
            for line in f:
                if line.startswith("dram_bytes_per_unit:"):
                    return float(line.split(":")[1])
    except Exception:
        pass
    return None


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "--query-gpu=" + self.Q, "--format=csv,noheader,nounits",
                                          "-i", str(self.gpu), "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        rows = []
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def reference_sample(n, steps, cores_hint=None, viscosity=0.0, collider=False, warmup=0):
    """Times the reference's own threaded CPU simulator on the workload: `warmup` untimed substeps from rest, then
    `steps` timed ones; returns (value, ms per substep, info)."""
    import numpy as np
    import oracle

    variant = "threaded" if oracle.ref_available("threaded") else None
    pos, vel = oracle.seed_regions([dict(kind=0, lo=BOX[:3], hi=BOX[3:])], (n, n, n), (0, 0, 0), (1, 1, 1), 0)
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    if variant:
        sim = oracle.RefSim((n, n, n), oracle.FLIP, max_cfl=1.0, cg_rel_tol=1e-6, cg_max_it=500, variant=variant,
                            viscosity=viscosity)
        kind = "reference"
        threads = os.cpu_count()  # std::thread::hardware_concurrency() threads per parallel loop
    else:
        sim = oracle.OracleSim((n, n, n), oracle.FLIP, max_cfl=1.0, cg_rel_tol=1e-6, cg_max_it=500,
                               viscosity=viscosity)
        kind = "port"
        threads = 1
    if collider:
        V, T, Nrm = box_mesh(COLLIDER_BOX)
        sim.add_mesh_collider(V, T, Nrm, (n, n, n), (0.0, 0.0, 0.0), (1.0 / n,) * 3)
    sim.set_particles(pos.astype(np.float64), vel.astype(np.float64))
    t_warm = time.perf_counter()
    for _ in range(warmup):
        sim.substep(DT)
    t_warm = time.perf_counter() - t_warm
    times = []
    for _ in range(steps):
        t0 = time.perf_counter()
        sim.substep(DT)
        times.append(time.perf_counter() - t0)
    total = sum(times)
    value = pos.shape[0] * steps / total
    window = ("substep%s %d%s after %d untimed warm-up substep(s) from rest"
              % ("s" if steps > 1 else "", warmup + 1, "-%d" % (warmup + steps) if steps > 1 else "", warmup)
              if warmup else "%d substep(s) from rest" % steps)
    info = {"value": value, "unit": METRIC, "cores": threads, "kind": kind, "window": window,
            "sample": "%s of the %d^3 FLIP dam break (%d particles)%s%s, %.1f s timed (+%.1f s warm-up); host has %d "
                      "cores" % (window, n, pos.shape[0], ", viscosity %g" % viscosity if viscosity else "",
                                 ", box collider" if collider else "", total, t_warm, cores)}
    return value, total / steps * 1e3, info


# Algorithmic bytes of one Jacobi relaxation per FLUID face (k_jacobi): list entry 8 B + right-hand side 4 B +
# iterate read 8 B (each neighbour value is read by its 6 neighbours, once per face algorithmically) + write 8 B.
JACOBI_BYTES_PER_FACE = 28


def diffusion_report(scene, stream, peak, peak_kind, reps=5):
    """The viscosity stage on the scene's current state, timed alone (FE_STAGE_DIFFUSE: band-SDF scatter, face
    markers, FLUID-face list, persistent Jacobi kernel), with the Jacobi kernel's relaxation count and an
    algorithmic-bandwidth figure for it.  Runs after the timed region; the state it leaves is not used."""
    import torch

    import fluide_engine_b200 as fe

    scene.run_stages(DT, fe.STAGE_SORT, fe.STAGE_PRE)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    times, passes = [], []
    for _ in range(reps):
        ev0.record(stream)
        scene.run_stages(DT, fe.STAGE_DIFFUSE, fe.STAGE_DIFFUSE)
        ev1.record(stream)
        torch.cuda.synchronize()
        times.append(ev0.elapsed_time(ev1))
        its, marks, npass = scene.diffusion_info()
        passes.append(npass)
    faces = int(sum(int(m.sum()) for m in marks))
    ms = sorted(times)[len(times) // 2]
    npass = passes[times.index(ms)]
    achieved = faces * npass * JACOBI_BYTES_PER_FACE / (ms / 1e3) / 1e9
    return {"stage_ms": ms, "stage_ms_all": times, "jacobi_iterations": list(its), "relaxation_passes": npass,
            "fluid_faces": faces,
            "roofline": {"bound": "latency (one grid barrier per relaxation)", "kernel": "k_jacobi",
                         "achieved": achieved, "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                         "frac": achieved / peak, "note": "algorithmic bytes = FLUID faces x passes x %d B; the "
                         "stage time includes the SDF scatter, face markers and list build" % JACOBI_BYTES_PER_FACE}}


def surface_report(scene, n, reps=5, reference=True):
    """GetSurface per frame: the band SDF of the last substep's particles and the marching-cubes mesh built on the
    device (fe_scene_build_surface, wall time of the synchronous call), the OBJ write of that mesh, and the
    reference's own CPU GetSurface (MarchingCubesSolver on its SDF of the same particles) for comparison."""
    import ctypes
    import tempfile

    import numpy as np

    import fluide_engine_b200 as fe

    L = fe.lib()
    nv, nt = ctypes.c_uint64(), ctypes.c_uint64()
    times = []
    for _ in range(reps):
        t0 = time.perf_counter()
        fe._abi.check(L.fe_scene_build_surface(scene.handle, ctypes.byref(nv), ctypes.byref(nt)))
        times.append((time.perf_counter() - t0) * 1e3)
    with tempfile.TemporaryDirectory() as d:
        t0 = time.perf_counter()
        fe._abi.check(L.fe_scene_write_surface_obj(scene.handle, os.path.join(d, "f.obj").encode(), b"fluid"))
        obj_ms = (time.perf_counter() - t0) * 1e3
        obj_bytes = os.path.getsize(os.path.join(d, "f.obj"))
    out = {"build_ms": sorted(times)[len(times) // 2], "build_ms_all": times, "vertices": int(nv.value),
           "triangles": int(nt.value), "obj_write_ms": obj_ms, "obj_bytes": obj_bytes,
           "path": "fe_scene_build_surface (device: SDF scatter, cube/cap counts, 2 scans, emit) + "
                   "fe_scene_write_surface_obj (host: OBJManager::Save format)"}
    if reference:
        try:
            import oracle

            variant = "threaded" if oracle.ref_available("threaded") else ("serial" if oracle.ref_available("serial") else None)
            if variant:
                P = scene.particles()[0].astype(np.float64)
                r = oracle.RefSim((n, n, n), oracle.FLIP, variant=variant)
                r.set_particles(P)
                r.stage("sdf")
                t0 = time.perf_counter()
                V, _, T = r.surface()
                out["reference_ms"] = (time.perf_counter() - t0) * 1e3
                out["reference_mesh"] = [int(V.shape[0]), int(T.shape[0])]
        except Exception as ex:  # reported, never required
            out["reference_ms"] = None
            out["reference_error"] = str(ex)[:200]
    return out


def mesh_init_report(n, device, reference=True, reps=3):
    """InitializeFromTriangleMesh on the GPU (fe_scene_init_from_mesh: Mesh2SDF band distances and winding signs,
    cell test, scan, particle writes; wall time of the synchronous call on a fresh scene) for an 80-triangle
    icosphere, and the reference's own InitializeFromTriangleMesh on the CPU for comparison."""
    import fluide_engine_b200 as fe

    V, T = sphere_mesh((0.5, 0.45, 0.5), 0.3, 1)
    times, count = [], 0
    for _ in range(reps):
        sc = fe.Scene((n, n, n), solver=fe.FLIP, max_cfl=1.0, device=device)
        t0 = time.perf_counter()
        sc.init_from_mesh(V, T, seed=1)
        times.append((time.perf_counter() - t0) * 1e3)
        count = sc.num_particles()
        sc.close()
    out = {"gpu_ms": sorted(times)[len(times) // 2], "gpu_ms_all": times, "particles": int(count),
           "triangles": int(T.shape[0]), "grid": [n, n, n],
           "path": "fe_scene_init_from_mesh (Mesh2SDF on the device, 16 particles per inside cell)"}
    if reference:
        try:
            import oracle

            variant = "threaded" if oracle.ref_available("threaded") else ("serial" if oracle.ref_available("serial") else None)
            if variant:
                r = oracle.RefSim((n, n, n), oracle.FLIP, variant=variant)
                t0 = time.perf_counter()
                r.init_from_mesh(V, T)
                out["reference_ms"] = (time.perf_counter() - t0) * 1e3
                out["reference_particles"] = int(r.particles()[0].shape[0])
        except Exception as ex:  # reported, never required
            out["reference_ms"] = None
            out["reference_error"] = str(ex)[:200]
    return out


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    n_gpus = args.gpus
    steps = max(1, min(args.steps, args.ref_steps))
    # the same untimed warm-up substeps as the GPU arm, so the timed substep is the first of the GPU arm's window
    warmup = max(args.warmup, 3)
    value, ms, info = reference_sample(args.n, steps, viscosity=args.viscosity, collider=args.collider, warmup=warmup)
    particles = int(round(value * ms / 1e3))
    line = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": n_gpus, "steps": steps, "warmup": warmup,
            "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded analytic scene)", "impl": "reference",
            "config": workload_config(args.n, steps, warmup, 1, particles, args.viscosity, args.collider),
            "window": info["window"], "cpu_baseline": info,
            "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_pool(args):
    """APIC sphere drop into a pool on a 256^3 grid (about 42M particles): the pool fills y < 0.3 and a sphere
    of radius 0.15 at (0.5, 0.7, 0.5) starts at velocity (0, -2, 0); 8 jittered particles per cell (seed 1),
    dt = 1/480, FP32 inner CG inside FP64 refinement to relative residual 1e-8.  The largest single-scene
    configuration: particle state (about 5 GB) and the solver's vectors exceed the 126 MB L2."""
    import numpy as np
    import torch

    import fluide_engine_b200 as fe

    torch.cuda.set_device(0)
    n = args.n or 256
    regions = [dict(kind=0, lo=(0.0, 0.0, 0.0), hi=(1.0, 0.3, 1.0)),
               dict(kind=1, lo=(0.5, 0.7, 0.5), hi=(0.15,), vel=(0.0, -2.0, 0.0))]
    t_seed = time.perf_counter()
    pos, vel = fe.seed_regions(regions, (n, n, n), seed=1)
    t_seed = time.perf_counter() - t_seed
    N = pos.shape[0]
    dt = 1.0 / 480.0
    scene = fe.Scene((n, n, n), solver=fe.APIC, max_cfl=1.0, cg_rel_tol=1e-8, cg_max_it=4000, max_refine=24,
                     cg_inner_tol=args.cg_inner_tol,
                     pressure_solver={"auto": fe.AUTO, "mgpcg": fe.MGPCG, "cg": fe.CG}[args.pressure_solver])
    stream = torch.cuda.Stream()
    scene.set_stream(stream.cuda_stream)
    scene.set_particles(pos, vel)
    del pos, vel
    scene.step(dt, args.warmup)
    torch.cuda.synchronize()
    sampler = ClockSampler(torch.cuda.current_device())
    sampler.start()
    launches0 = fe.kernel_launch_count()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    stats, phase_ms = scene.step_profiled(dt, args.steps)
    ev1.record(stream)
    torch.cuda.synchronize()
    launches = fe.kernel_launch_count() - launches0
    clocks = sampler.stop()
    ms = ev0.elapsed_time(ev1)
    value = N * args.steps / (ms / 1e3)
    cg_ms = phase_ms[:, 1].astype(np.float64)
    fluid = np.array([s["fluid_cells"] for s in stats], dtype=np.float64)
    its = np.array([s["cg_iterations"] for s in stats], dtype=np.float64)
    refs = np.array([s["refinements"] for s in stats], dtype=np.float64)
    multigrid = uses_multigrid(n, args.pressure_solver)
    alg_bytes = solver_alg_bytes(fluid, its, refs, n, multigrid)
    peak, peak_kind = peaks()
    achieved = alg_bytes.sum() / (cg_ms.sum() / 1e3) / 1e9
    phase_share = (phase_ms.sum(axis=0) / phase_ms.sum()).tolist()
    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 (FP64 refinement)", "data": "synthetic (seeded analytic scene)", "workload_kind": "pool256",
        "config": {"workload": "APIC sphere drop into a pool %d^3, pool y<0.3 + sphere r=0.15 at (0.5,0.7,0.5) "
                               "v=(0,-2,0), 8 particles/cell (seed 1), dt=1/480, FP32 CG in FP64 refinement to "
                               "rel 1e-8" % n, "grid": [n, n, n], "particles": N, "solver": "APIC",
                   "substeps_timed": args.steps, "warmup": args.warmup, "seeding_s": t_seed,
                   "l2": "working set > 126 MB L2 (particles alone %.0f MB); no flush" % (N * 60 / 1e6)},
        "roofline": {"bound": "hbm", "kernel": "k_mgcg" if multigrid else "k_cg",
                     "achieved": achieved, "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": None, "algorithmic_bytes_per_launch": float(alg_bytes.mean())},
        "phases": {"share": {"pre_solve": phase_share[0], "cg_solve": phase_share[1], "post_solve": phase_share[2]},
                   "ms_per_substep": (phase_ms.mean(axis=0)).tolist()},
        "solver": {"cg_iterations_mean": float(its.mean()), "cg_iterations_max": float(its.max()),
                   "refinements_mean": float(refs.mean()),
                   "rel_residual_max": float(max(s["rel_residual"] for s in stats)),
                   "converged_all": bool(all(s["converged"] for s in stats)), "fluid_cells_mean": float(fluid.mean())},
        "gpu_launches": int(launches), "clocks": clocks,
    }
    print(json.dumps(line), flush=True)
    scene.close()
    return 0


def tune_scenes(make_scene, keys, dt, device=0):
    """Runs the autotuner (all candidates) once per (grid, transfer) key on a scene make_scene(key) builds, a few
    substeps after it starts; the choices go into the library's table, so the scenes both arms create afterwards
    (automatic solver choice) start from them.  Returns {key: (choice, ms per substep)}."""
    from fluide_engine_b200 import autotune

    out = {}
    for key in keys:
        sc = make_scene(key)
        sc.step(dt, 2, stats=False)
        out[key] = autotune.tune(sc, dt, substeps=3, device=device, save=False)
        sc.close()
    return out


def batched_measure(n_scenes=48, steps=50, warmup=5, device=0, batch_family=None):
    """Batched independent scenes vs the same scenes one at a time on the plain single-scene path.

    Scenes: cubic grids drawn from {32,48,64,96,128}, a dam-break block with extents U[0.2,0.6] per axis,
    8 particles per cell, solver drawn from PIC / FLIP(0.95) / APIC (seed 2).  Both arms use the same
    pressure tolerance (rel 1e-6); times are wall clock around synchronised device work.  The one-at-a-time arm
    runs every scene with the autotuner's choice for its kind, and so does the batched arm by default;
    batch_family="cg" runs the batched arm's scenes on the plain CG body inside the multi-scene solve instead (with
    the current multigrid solver slower for this set: 12.29 against 11.31 ms per substep).  Returns a dict.
    """
    import numpy as np
    import torch

    import fluide_engine_b200 as fe

    rng = np.random.default_rng(2)
    specs = []
    for k in range(n_scenes):
        n = int(rng.choice([32, 48, 64, 96, 128]))
        ext = rng.uniform(0.2, 0.6, 3)
        solver = int(rng.integers(0, 3))
        specs.append((n, solver, tuple(float(e) for e in ext), k))

    def make(spec):
        n, solver, ext, k = spec
        pos, vel = fe.seed_regions([dict(kind=0, lo=(0.0, 0.0, 0.0), hi=ext)], (n, n, n), seed=k)
        sc = fe.Scene((n, n, n), solver=solver, max_cfl=1.0, cg_rel_tol=1e-6, device=device)
        sc.set_particles(pos, vel)
        return sc

    def build():
        return [make(sp) for sp in specs]

    # the autotuner's choice per (grid, transfer), tuned on the first scene of each kind; both arms use it
    first = {}
    for sp in specs:
        first.setdefault((sp[0], sp[1]), sp)
    t0 = time.perf_counter()
    tuned = tune_scenes(lambda key: make(first[key]), sorted(first), DT, device)
    tune_s = time.perf_counter() - t0

    # both arms time the same substep window: the batched arm's warm-up (at least the 8 substeps after which a batch
    # runs from its captured graph) plus the batch tuner's substeps come first in both
    from fluide_engine_b200 import autotune

    flat_candidates = autotune.FLAT_CANDIDATES
    tune_sub = 3
    pre = max(warmup, 8) + 2 * len(flat_candidates) * (tune_sub + 1)
    # one at a time (each scene's own graph-captured substeps, scene after scene)
    scenes = build()
    particles = sum(sc.num_particles() for sc in scenes)
    for sc in scenes:
        sc.step(DT, pre, stats=False)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    res_alone = []
    for sc in scenes:
        st = sc.step(DT, steps, stats=True)
        res_alone.append(max(x["rel_residual"] for x in st))
    torch.cuda.synchronize()
    t_alone = time.perf_counter() - t0
    for sc in scenes:
        sc.close()
    # batched
    scenes = build()
    if batch_family == "cg":
        for sc in scenes:
            sc.set_tuning(multigrid=0)
    batch = fe.Batch(scenes)
    batch.step(DT, max(warmup, 8), stats=False)
    # which scenes run in the flat (scene, block) launches: timed on the batch's own substeps
    flat_best, flat_ms = autotune.tune_batch(batch, DT, substeps=tune_sub, candidates=flat_candidates)
    torch.cuda.synchronize()
    launches0 = fe.kernel_launch_count()
    t0 = time.perf_counter()
    st = batch.step(DT, steps, stats=True)
    torch.cuda.synchronize()
    t_batch = time.perf_counter() - t0
    launches = fe.kernel_launch_count() - launches0
    res_batch = [max(x["rel_residual"] for x in s_) for s_ in st]
    conv = all(x["converged"] for s_ in st for x in s_)
    batch.close()
    for sc in scenes:
        sc.close()
    v_batch = particles * steps / t_batch
    v_alone = particles * steps / t_alone
    return {"value": v_batch, "unit": METRIC, "steps": steps, "warmup": pre,
            "ms_per_step": t_batch / steps * 1e3,
            "workload": "%d batched scenes, n in {32,48,64,96,128}, block extents U[0.2,0.6], solver "
                        "U{PIC,FLIP,APIC} (seed 2), dt=1/240, CG rel 1e-6, %d substeps after %d warm-up and tuning "
                        "substeps in both arms" % (len(specs), steps, pre),
            "scenes": [[n, ["PIC", "FLIP", "APIC"][sv]] for n, sv, _, _ in specs],
            "particles_total": particles, "timing": "wall clock around synchronised device work",
            "one_at_a_time": {"value": v_alone, "ms_per_step_all_scenes": t_alone / steps * 1e3},
            "batched_over_one_at_a_time": v_batch / v_alone, "batch_family": batch_family or "autotuned per kind",
            "flat_launches": {"max_cells": flat_best,
                              "note": "scenes of at most max_cells cells run each pre/post-solve pass as one launch "
                                      "for all of them over a (scene, block) work list, the rest on their own "
                                      "streams (0: none, -1: all); picked by timing each choice over %d substeps "
                                      "(ms per substep below); %d substeps precede both arms' timed window"
                                      % (tune_sub, pre),
                              "ms_per_substep": {str(k): v for k, v in flat_ms.items()}},
            "accuracy": {"rel_residual_max_batched": max(res_batch), "rel_residual_max_alone": max(res_alone),
                         "converged_all": conv},
            "tuning": {"%d^3 %s" % (n, ["PIC", "FLIP", "APIC"][sv]): choice for (n, sv), (choice, _) in tuned.items()},
            "tuning_s": tune_s,
            "gpu_launches": int(launches)}


def run_batch_only(args):
    """The batched workload's scenes stepped as one batch only (no tuning, no one-at-a-time arm): `--batch-flat`
    scenes' cells or fewer in the flat launches, `--warmup` untimed then `--steps` timed substeps; a profiling
    target for the batch's launches."""
    import numpy as np
    import torch

    import fluide_engine_b200 as fe

    torch.cuda.set_device(0)
    rng = np.random.default_rng(2)
    scenes = []
    for k in range(args.scenes):
        n = int(rng.choice([32, 48, 64, 96, 128]))
        ext = rng.uniform(0.2, 0.6, 3)
        solver = int(rng.integers(0, 3))
        pos, vel = fe.seed_regions([dict(kind=0, lo=(0.0, 0.0, 0.0), hi=tuple(float(e) for e in ext))], (n, n, n),
                                   seed=k)
        sc = fe.Scene((n, n, n), solver=solver, max_cfl=1.0, cg_rel_tol=1e-6, device=0)
        sc.set_particles(pos, vel)
        scenes.append(sc)
    particles = sum(sc.num_particles() for sc in scenes)
    batch = fe.Batch(scenes)
    flat = 0 if args.batch_flat is None else args.batch_flat
    batch.set_flat(flat)
    if args.warmup:
        batch.step(DT, args.warmup, stats=False)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    batch.step(DT, args.steps, stats=False)
    torch.cuda.synchronize()
    t = time.perf_counter() - t0
    line = {"metric": METRIC, "value": particles * args.steps / t, "unit": METRIC, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t / max(args.steps, 1) * 1e3, "workload_kind": "batched-only",
            "config": {"scenes": args.scenes, "particles_total": particles, "flat_max_cells": flat,
                       "timing": "wall clock around synchronised device work"}}
    print(json.dumps(line), flush=True)
    batch.close()
    for sc in scenes:
        sc.close()
    return 0


def run_batched(args):
    import torch

    torch.cuda.set_device(0)
    if args.batch_only:
        return run_batch_only(args)
    b = batched_measure(args.scenes, args.steps, args.warmup)
    line = {"metric": METRIC, "value": b["value"], "unit": METRIC, "n_gpus": 1, "steps": b["steps"],
            "warmup": b["warmup"], "ms_per_step": b["ms_per_step"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 (FP64 refinement)",
            "data": "synthetic (seeded analytic scenes)", "workload_kind": "batched",
            "config": {"workload": b["workload"], "scenes": b["scenes"], "particles_total": b["particles_total"],
                       "timing": b["timing"]},
            "one_at_a_time": b["one_at_a_time"], "batched_over_one_at_a_time": b["batched_over_one_at_a_time"],
            "flat_launches": b["flat_launches"], "accuracy": b["accuracy"], "gpu_launches": b["gpu_launches"]}
    print(json.dumps(line), flush=True)
    return 0


def served_measure(rate, seconds, res, fr, budget_gb, max_batch, device=0, batch_family=None):
    """A seeded Poisson trace of APIC pool + sphere jobs served with continuous batching, and the same trace run
    FIFO one job at a time through the plain single-scene path.  Returns a dict."""
    import numpy as np

    import fluide_engine_b200 as fe
    from fluide_engine_b200 import serving

    jobs = serving.poisson_trace(rate, seconds, 3, resolutions=res, frames=fr)
    # the autotuner's choice per job resolution (tuned on the first job of each), used by both arms' scenes
    first = {}
    for j in jobs:
        first.setdefault(j.n, j)

    def make(n):
        j = first[n]
        pos, vel = fe.seed_regions(j.regions, (n,) * 3, seed=j.seed)
        sc = fe.Scene((n,) * 3, solver=j.solver, max_cfl=1.0, cg_rel_tol=1e-6, device=device)
        sc.set_particles(pos, vel)
        return sc

    t0 = time.perf_counter()
    tuned = tune_scenes(make, sorted(first), jobs[0].dt, device)
    tune_s = time.perf_counter() - t0
    srv = serving.Server(hbm_budget_bytes=int(budget_gb * 1e9), max_batch=max_batch, device=device,
                         batch_family=batch_family)
    for j in jobs:
        srv.submit(j)
    wall, psteps = srv.run()
    p50, p99 = srv.latency_percentiles()
    served = psteps / wall
    # the same trace served one job at a time (FIFO) through the plain single-scene path: a job starts at
    # max(arrival, end of the previous job); setup (seeding, scene creation) is inside the measured time as
    # it is for the server
    clock, ps_alone, ms_alone = 0.0, 0, []
    alone_split = {"seed": 0.0, "create": 0.0, "step": 0.0, "retire": 0.0}
    for j in sorted(jobs, key=lambda x: x.arrival):
        start = max(j.arrival, clock)
        t_job = time.perf_counter()
        pos, vel = fe.seed_regions(j.regions, (j.n,) * 3, seed=j.seed)
        t1 = time.perf_counter()
        sc = fe.Scene((j.n,) * 3, solver=j.solver, max_cfl=1.0, cg_rel_tol=1e-6, device=device)
        sc.set_particles(pos, vel)
        t2 = time.perf_counter()
        for _ in range(j.frames):
            t0 = time.perf_counter()
            sc.step(j.dt, j.substeps_per_frame, stats=False)
            sc.synchronize()
            ms_alone.append((time.perf_counter() - t0) * 1e3)
            ps_alone += pos.shape[0] * j.substeps_per_frame
        t3 = time.perf_counter()
        sc.particles()
        sc.close()
        t4 = time.perf_counter()
        alone_split["seed"] += t1 - t_job
        alone_split["create"] += t2 - t1
        alone_split["step"] += t3 - t2
        alone_split["retire"] += t4 - t3
        clock = start + (time.perf_counter() - t_job)
    t_alone = clock
    return {"value": served, "unit": METRIC, "substeps_total": int(sum(j.frames * j.substeps_per_frame for j in jobs)),
            "workload": "Poisson %.0f jobs/s for %.0f s (seed 3), APIC pool+sphere, n in %s, %s frames x 4 substeps, "
                        "dt=1/480, HBM budget %.0f GB, batch <= %d" % (rate, seconds, list(res), list(fr), budget_gb,
                                                                         max_batch),
            "jobs": len(jobs), "frame_ms": {"p50": p50, "p99": p99},
            "one_at_a_time": {"value": ps_alone / t_alone, "makespan_s": t_alone,
                              "frame_ms_p50": float(np.percentile(ms_alone, 50)),
                              "frame_ms_p99": float(np.percentile(ms_alone, 99)),
                              "time_s": alone_split,
                              "note": "FIFO over the same arrival trace, one job at a time; frame latency excludes "
                                      "the queueing delay before a job starts"},
            "served_over_one_at_a_time": served / (ps_alone / t_alone), "wall_s": wall,
            "server_time_s": dict(srv.timing), "batch_rebuilds": srv.rebuilds, "scenes_reused": srv.reused,
            "device_step_ratio": alone_split["step"] / max(srv.timing["step"], 1e-9),
            "tuning": {"%d^3" % n: choice for n, (choice, _) in tuned.items()}, "tuning_s": tune_s}


def run_served(args):
    """Served request stream (the served configuration scaled down in duration and resolution; see --trace-*)."""
    import torch

    torch.cuda.set_device(0)
    res = tuple(int(x) for x in args.trace_res.split(","))
    fr = tuple(int(x) for x in args.trace_frames.split(","))
    m = served_measure(args.trace_rate, args.trace_seconds, res, fr, args.hbm_budget_gb, args.max_batch)
    line = {"metric": METRIC, "value": m["value"], "unit": METRIC, "n_gpus": 1, "steps": m["substeps_total"],
            "warmup": 0, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 (FP64 refinement)", "data": "synthetic (seeded Poisson trace)", "workload_kind": "served",
            "config": {"workload": m["workload"], "jobs": m["jobs"]}}
    line.update({k: v for k, v in m.items() if k not in ("value", "unit", "substeps_total", "workload", "jobs")})
    print(json.dumps(line), flush=True)
    return 0


def divergence_report(scene):
    """One substep of the scene's current state run stage by stage: ||div u||_2 over FLUID cells before the pressure
    stage and after it (the reference applies the pressure gradient one-sidedly, only toward +x/+y/+z from FLUID
    cells, so a FLUID cell with an AIR neighbour on its low side keeps part of its divergence: the post/pre ratio
    is bounded by that discretisation, not by the solver's residual).  Runs after the timed region."""
    import fluide_engine_b200 as fe

    scene.run_stages(DT, fe.STAGE_SORT, fe.STAGE_PRE)
    pre = scene.divergence()
    scene.run_stages(DT, fe.STAGE_DIFFUSE, fe.STAGE_PRESSURE)
    post = scene.divergence()
    scene.run_stages(DT, fe.STAGE_POST, fe.STAGE_MOVE)
    return {"div_l2_pre": pre, "div_l2_post": post, "div_post_over_pre": post / pre if pre > 0 else None}


def oracle_snapshot_report(n=64, later=30, device=0):
    """Per-substep error against the FP64 oracle on the same scene family at n^3: the GPU runs later-1 substeps,
    the oracle is seeded with the GPU's particles and pressure (warm start), and both run substep `later`
    (trajectories diverge chaotically, so errors are compared from an identical snapshot).  The oracle runs its
    substep stage by stage to report its own divergence before and after the pressure stage."""
    import numpy as np

    import fluide_engine_b200 as fe
    import oracle

    def rel(a, b):
        a = np.asarray(a, np.float64).ravel()
        b = np.asarray(b, np.float64).ravel()
        return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))

    pos, vel = fe.seed_regions([dict(kind=0, lo=BOX[:3], hi=BOX[3:])], (n, n, n), seed=0)
    g = fe.Scene((n, n, n), solver=fe.FLIP, max_cfl=1.0, cg_rel_tol=1e-6, device=device)
    g.set_particles(pos, vel)
    g.step(DT, later - 1, stats=False)
    P0, V0, _ = g.particles()
    p0 = g.grid()[3]
    o = oracle.OracleSim((n, n, n), oracle.FLIP, max_cfl=1.0, cg_rel_tol=1e-10, cg_max_it=20000)
    o.set_particles(P0.astype(np.float64), V0.astype(np.float64))
    o.set_pressure(p0)
    t0 = time.perf_counter()
    o.build_collider()
    for st_ in ("p2g", "sdf", "extrapolate", "bc"):
        o.stage(st_)
    o.stage("forces", DT)
    o.stage("markers")
    o_pre = o.divergence_l2()
    o.stage("pressure", DT)
    o_post = o.divergence_l2()
    o_res = o.cg_rel_residual()
    o.stage("advection", DT)
    t_oracle = time.perf_counter() - t0
    stats = g.step(DT, 1)
    P, V, _ = g.particles()
    u, v, w, p, m = g.grid()
    Po, Vo, _ = o.particles()
    out = {"scene": "FLIP dam break %d^3 (%d particles), substep %d from the GPU's state at substep %d"
                    % (n, pos.shape[0], later, later - 1),
           "particle_velocity_rel_l2": rel(V, Vo), "particle_position_rel_l2": rel(P, Po),
           "pressure_rel_l2": rel(p, o.pressure()),
           "grid_velocity_rel_l2": rel(np.concatenate([np.ravel(a) for a in (u, v, w)]),
                                       np.concatenate([np.ravel(a) for a in o.grid()])),
           "marks_bit_exact": bool(np.array_equal(m, o.marks())),
           "gpu_rel_residual": stats[0]["rel_residual"], "oracle_rel_residual": o_res,
           "oracle_div_post_over_pre": o_post / o_pre if o_pre > 0 else None,
           "oracle_seconds": t_oracle,
           "tolerances": {"particle_velocity": 1e-4, "grid": 1e-4, "pressure": 1e-3, "marks": "bit-exact"}}
    g.close()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=240)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=None, help="grid cells per axis (default 128; 256 for pool256)")
    ap.add_argument("--e2e-steps", type=int, default=10)
    ap.add_argument("--ref-steps", type=int, default=1, help="substeps of the CPU reference sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-autotune", action="store_true", help="single workload: keep the default launch shape")
    ap.add_argument("--no-extras", action="store_true",
                    help="single workload: skip the accuracy-vs-oracle, batched and served objects of the line")
    ap.add_argument("--cg-inner-tol", type=float, default=0.0,
                    help="inner FP32 CG residual reduction per refinement (0: the solver's default)")
    ap.add_argument("--pressure-solver", default="auto", choices=["auto", "mgpcg", "cg"],
                    help="inner pressure solver: auto (multigrid-preconditioned CG from 2^15 cells, plain CG below), "
                         "mgpcg or cg")
    ap.add_argument("--workload", default="single", choices=["single", "batched", "served", "pool256"])
    ap.add_argument("--surface", action="store_true",
                    help="single workload: also time GetSurface (device mesh + OBJ write) after the timed region")
    ap.add_argument("--viscosity", type=float, default=0.0,
                    help="single workload / reference arm: kinematic viscosity (0 = none, as the benchmark scenes)")
    ap.add_argument("--collider", action="store_true",
                    help="single workload / reference arm: a box TriangleMeshCollider in the dam break's path")
    ap.add_argument("--mesh-init", action="store_true",
                    help="single workload: also time InitializeFromTriangleMesh (GPU and reference CPU)")
    ap.add_argument("--scenes", type=int, default=48, help="batched workload: number of scenes")
    ap.add_argument("--batch-only", action="store_true",
                    help="batched workload: step the batch alone (no tuning, no one-at-a-time arm)")
    ap.add_argument("--batch-flat", type=int, default=None,
                    help="with --batch-only: scenes of at most this many cells in the flat launches (-1: all)")
    # served: 20 jobs/s as the served configuration, over 6 s instead of 10 min and with resolutions <= 128 so
    # that a run takes tens of seconds; the work still exceeds the arrival window several times (saturated)
    ap.add_argument("--trace-rate", type=float, default=20.0)
    ap.add_argument("--trace-seconds", type=float, default=6.0)
    ap.add_argument("--trace-res", default="32,48,64,96,128")
    ap.add_argument("--trace-frames", default="8,24")
    ap.add_argument("--hbm-budget-gb", type=float, default=150.0)
    ap.add_argument("--max-batch", type=int, default=32)
    args = ap.parse_args()
    if args.impl == "reference":
        args.n = args.n or 128
        return run_reference_arm(args)
    if args.workload == "batched":
        return run_batched(args)
    if args.workload == "served":
        return run_served(args)
    if args.workload == "pool256":
        return run_pool(args)
    args.n = args.n or 128
    args.warmup = max(args.warmup, 3)

    import numpy as np
    import torch
    import torch.distributed as dist

    import fluide_engine_b200 as fe

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        dist.init_process_group("nccl", device_id=torch.device("cuda", local),
                                timeout=__import__("datetime").timedelta(seconds=300))
    n = args.n
    pos, vel = fe.seed_regions([dict(kind=0, lo=BOX[:3], hi=BOX[3:])], (n, n, n), (0, 0, 0), (1, 1, 1), 0)
    N = pos.shape[0]
    scene = fe.Scene((n, n, n), solver=fe.FLIP, max_cfl=1.0, cg_rel_tol=1e-6, cg_inner_tol=args.cg_inner_tol,
                     device=local, pressure_solver={"auto": fe.AUTO, "mgpcg": fe.MGPCG, "cg": fe.CG}[args.pressure_solver],
                     viscosity=args.viscosity)
    if args.collider:
        CV, CT, CN = box_mesh(COLLIDER_BOX)
        scene.add_mesh_collider(CV, CT, CN, (n, n, n), (0.0, 0.0, 0.0), (1.0 / n,) * 3)
    stream = torch.cuda.Stream()
    scene.set_stream(stream.cuda_stream)
    scene.set_particles(pos, vel)
    scene.step(DT, args.warmup)
    # launch shape of the pressure solve picked by the autotuner on this scene's state after the warm-up (untimed;
    # the state is restored); the solver family stays the automatic choice, whose iteration count over a whole run
    # the first substeps do not predict
    tuning = None
    if not args.no_autotune:
        from fluide_engine_b200 import autotune

        t0 = time.perf_counter()
        choice, tuned_ms = autotune.tune(scene, DT, substeps=4, device=local, save=False, shape_only=True)
        tuning = {"choice": choice, "ms_per_substep_in_search": tuned_ms, "search_s": time.perf_counter() - t0,
                  "by": "fe_scene_autotune (FE_TUNE_SHAPE), 4 substeps per candidate"}

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    sampler = ClockSampler(torch.cuda.current_device())
    sampler.start()
    barrier()
    launches0 = fe.kernel_launch_count()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    stats, phase_ms = scene.step_profiled(DT, args.steps)
    ev1.record(stream)
    barrier()
    launches = fe.kernel_launch_count() - launches0
    clocks = sampler.stop()
    ms = max_over_ranks(ev0.elapsed_time(ev1), "cuda")
    value = replica_throughput(world, N, args.steps, ms / 1e3)

    # roofline of the dominant kernel: the persistent CG kernel (solve phase = exactly one launch)
    cg_ms = phase_ms[:, 1].astype(np.float64)
    fluid = np.array([s["fluid_cells"] for s in stats], dtype=np.float64)
    its = np.array([s["cg_iterations"] for s in stats], dtype=np.float64)
    refs = np.array([s["refinements"] for s in stats], dtype=np.float64)
    multigrid = uses_multigrid(n, args.pressure_solver) and not args.collider  # collider scenes use the plain CG
    alg_bytes = solver_alg_bytes(fluid, its, refs, n, multigrid)  # per launch
    peak, peak_kind = peaks()
    achieved = alg_bytes.sum() / (cg_ms.sum() / 1e3) / 1e9
    per_unit = profile_traffic(multigrid)
    units = fluid * (its + refs + 1.0)
    traffic = float(per_unit * units.mean()) if per_unit else None
    phase_share = (phase_ms.sum(axis=0) / phase_ms.sum()).tolist()
    diffusion = diffusion_report(scene, stream, peak, peak_kind) if args.viscosity > 0 else None
    divergence = divergence_report(scene)
    surface = surface_report(scene, n, reference=not args.no_cpu_baseline) if args.surface and rank == 0 else None
    mesh_init = (mesh_init_report(n, local, reference=not args.no_cpu_baseline) if args.mesh_init and rank == 0
                 else None)

    # end to end through the public API with host buffers: H2D particles, one substep, D2H particles
    pin_pos = torch.from_numpy(pos).pin_memory()
    pin_vel = torch.zeros((N, 3), dtype=torch.float32).pin_memory()
    P, V, _ = scene.particles()
    pin_pos.copy_(torch.from_numpy(P))
    pin_vel.copy_(torch.from_numpy(V))
    out_pos = torch.empty((N, 3), dtype=torch.float32).pin_memory()
    out_vel = torch.empty((N, 3), dtype=torch.float32).pin_memory()
    L = fe.lib()
    e2e_steps = max(1, min(args.e2e_steps, args.steps))
    # two pinned buffer sets in turn: each step uploads the previous step's results from the host and reads its own
    # back into the other set (no host-side copy between steps)
    bufs = [(pin_pos, pin_vel), (out_pos, out_vel)]
    barrier()
    t0 = time.perf_counter()
    for k in range(e2e_steps):
        (ip, iv), (op, ov) = bufs[k & 1], bufs[(k + 1) & 1]
        fe._abi.check(L.fe_scene_set_particles(scene.handle, fe._abi.ptr(ip), fe._abi.ptr(iv), None, N))
        fe._abi.check(L.fe_scene_step(scene.handle, DT, 1, None))
        fe._abi.check(L.fe_scene_get_particles(scene.handle, fe._abi.ptr(op), fe._abi.ptr(ov), None, N))
    barrier()
    e2e_s = max_over_ranks(time.perf_counter() - t0, "cuda")
    e2e_value = replica_throughput(world, N, e2e_steps, e2e_s)

    # accuracy beside the result, and the batched / served configurations (one GPU, rank 0 of a single-rank run)
    extras = rank == 0 and world == 1 and not args.no_extras
    oracle64 = None
    if extras and not args.collider and not args.viscosity:
        try:
            oracle64 = oracle_snapshot_report(64, 30, local)
        except Exception as ex:  # reported, never required
            oracle64 = {"error": str(ex)[:200]}
    batched = batched_measure(48, 50, 5, local) if extras else None
    served = None
    if extras:
        res = tuple(int(x) for x in args.trace_res.split(","))
        fr = tuple(int(x) for x in args.trace_frames.split(","))
        served = served_measure(args.trace_rate, args.trace_seconds, res, fr, args.hbm_budget_gb, args.max_batch, local)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            _, _, cpu = reference_sample(n, args.ref_steps, viscosity=args.viscosity, collider=args.collider)
        except Exception as ex:  # the baseline is reported, never required
            cpu = {"value": None, "unit": METRIC, "cores": None, "kind": "unavailable", "sample": str(ex)[:200]}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 (FP64 refinement)", "data": "synthetic (seeded analytic scene)",
            "config": dict(workload_config(n, args.steps, args.warmup, world, N, args.viscosity, args.collider),
                           tuning=tuning),
            "roofline": {"bound": "hbm",
                         "kernel": ("k_mgcg (persistent multigrid-preconditioned FP32 CG + FP64 refinement, one "
                                    "launch/substep)" if multigrid else
                                    "k_cg (persistent FP32 CG + FP64 refinement, one launch/substep)"),
                         "achieved": achieved, "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "algorithmic_bytes_per_launch": float(alg_bytes.mean()),
                         "note": ("algorithmic bytes = FLUID cells x (68 B x inner iterations + 45 B x FP64 residual "
                                  "passes) + 30 B x coarse-level cells x inner iterations; the solve is bound by its "
                                  "grid barriers (about 14 per inner iteration), not by bandwidth: its working set "
                                  "is L2-resident at 128^3" if multigrid else
                                  "algorithmic bytes = fluid cells x (41 B x inner iterations + 45 B x FP64 residual "
                                  "passes); at 128^3 the CG working set is L2-resident")},
            "phases": {"share": {"pre_solve": phase_share[0], "cg_solve": phase_share[1], "post_solve": phase_share[2]},
                       "ms_per_substep": (phase_ms.mean(axis=0)).tolist()},
            "solver": {"cg_iterations_mean": float(its.mean()), "refinements_mean": float(refs.mean()),
                       "rel_residual_max": float(max(s["rel_residual"] for s in stats)),
                       "converged_all": bool(all(s["converged"] for s in stats)),
                       "fluid_cells_mean": float(fluid.mean())},
            "accuracy": {"linear_rel_residual_max": float(max(s["rel_residual"] for s in stats)),
                         "divergence": divergence, "vs_oracle": oracle64,
                         "note": "linear_rel_residual = ||b - A p|| / ||b|| of every timed solve (FP64); divergence = "
                                 "||div u|| over FLUID cells after / before the pressure stage of one more substep of "
                                 "this scene (bounded by the reference's one-sided pressure apply, which the oracle "
                                 "shares: vs_oracle.oracle_div_post_over_pre); vs_oracle = one substep from an "
                                 "identical snapshot against the FP64 oracle"},
            "window": "substeps %d-%d after %d untimed warm-up substeps from rest" % (args.warmup + 1,
                                                                                   args.warmup + args.steps,
                                                                                   args.warmup),
            "e2e": {"value": e2e_value, "unit": METRIC, "h2d_bytes_per_step": int(N * 24),
                    "d2h_bytes_per_step": int(N * 24), "steps": e2e_steps,
                    "path": "fe_scene_set_particles(host) + fe_scene_step(1) + fe_scene_get_particles(host)"},
            "gpu_launches": int(launches),
            "clocks": clocks,
            "cpu_baseline": cpu,
        }
        if batched:
            line["batched"] = batched
        if served:
            line["served"] = served
        if diffusion:
            line["diffusion"] = diffusion
        if surface:
            line["surface"] = surface
        if mesh_init:
            line["mesh_init"] = mesh_init
        print(json.dumps(line), flush=True)
    scene.close()
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
