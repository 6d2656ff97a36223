"""Serving loop: simulation jobs admitted against an HBM budget and advanced with continuous batching.

A job is (scene spec, frames, substeps per frame).  Jobs arrive over time; the server admits waiting jobs
in arrival order whenever a batch slot and enough of the HBM budget are free, keeps every admitted job's
particles and grid resident on the device between frames, and advances all running jobs together: one
fe_batch_step per frame over the current membership (the batch is rebuilt only when a job joins or
leaves, i.e. between frames).  Each job's frame latency is measured from the start of the frame's first
substep to the end of its last; aggregate particle-steps/s counts every running job's particles.

The reference has no serving layer: it runs one simulator per process frame by frame
(SimulationRunner::RunSimulation, simulation_runner.cpp:17-55).
"""
import collections
import heapq
import threading
import time
from dataclasses import dataclass, field

import numpy as np

from . import _abi
from .scene import Batch, Scene


@dataclass
class Job:
    job_id: int
    n: int                      # cells per axis
    solver: int                 # PIC / FLIP / APIC
    regions: list               # fe_seed regions (dicts)
    frames: int
    substeps_per_frame: int
    dt: float
    arrival: float = 0.0        # seconds after the server start
    seed: int = 0
    # filled by the server
    scene: object = None
    particles: int = 0
    admitted_at: float = None
    finished_at: float = None
    frames_done: int = 0
    frame_ms: list = field(default_factory=list)
    seeded: tuple = None        # (pos, vel) once seeded, kept while the job waits for memory
    cancelled: bool = False     # left before its last frame (Server.cancel); its state is not read back


def scene_bytes(n, particles, solver):
    """Device bytes of one scene (allocation plan of fe_scene.cu): grid, solver vectors and particles."""
    cells = n ** 3
    faces = 3 * (n + 1) * n * n
    grid = faces * (5 * 4 + 3) + cells * (1 + 8 + 8 + 9 * 4 + 4 + 4 + 4) + (cells // 512 + 1) * 512 * 8
    grid += cells * 13 // 7  # multigrid levels: mask + residual + correction + scratch per coarse cell (cells / 7)
    per_particle = 2 * (7 + (9 if solver == _abi.APIC else 0)) * 4 + 3 * 4 + 9 * 4 + 4
    return grid + particles * per_particle


class Server:
    """Continuous-batching simulation server on one device.

    Three kinds of work overlap.  Each frame's batched substeps run on a GPU worker thread (the library call
    releases the GIL and blocks only that thread).  A single FIFO I/O thread reads back the jobs that
    finished and prepares the jobs that will join at the next frame boundary (scene taken from the pool and
    reset, or created; particles uploaded).  A small thread pool seeds arrived jobs ahead of time.  The
    serving thread only admits, updates the membership between frames and launches the next frame.
    Finished jobs' scenes go to a pool keyed by (grid, solver) and are reused by later jobs of the same
    shape instead of being freed and allocated again; pooled scenes count against the HBM budget until
    they are evicted (least recently used first) to make room.
    """

    def __init__(self, hbm_budget_bytes, max_batch=32, device=0, cg_rel_tol=1e-6, seed_threads=4,
                 reuse_scenes=True, overlap=False, batch_family=None, flat_max_cells=None):
        self.budget = int(hbm_budget_bytes)
        self.max_batch = min(int(max_batch), 64)
        self.device = device
        self.cg_rel_tol = cg_rel_tol
        self.reuse_scenes = reuse_scenes
        self.overlap = overlap   # batch overlap mode (each job's substep on its own stream, see Batch.set_overlap)
        # solver family of the jobs' scenes inside the batches: None keeps each scene's own choice (the automatic
        # one, or the autotuner's for its grid), "cg" runs the plain CG body for every job (the multi-scene solve
        # overlaps the scenes' barrier latency, which is what the multigrid solver saves a lone scene)
        if batch_family not in (None, "cg"):
            raise ValueError("batch_family is None or 'cg'")
        self.batch_family = batch_family
        # scenes of at most this many cells run in the batches' flat launches (Batch.set_flat); None keeps the
        # library's default
        self.flat_max_cells = flat_max_cells
        self.seed_threads = max(1, int(seed_threads))
        self.used = 0            # bytes of live scenes (running, pooled, being prepared or released)
        self.reserved = 0        # bytes reserved for preparations that need a new scene
        self._releasing = 0      # finished jobs whose read-back / release is still queued
        self._releasing_shapes = collections.Counter()  # (n, solver) of those jobs: scenes about to enter the pool
        self.waiting = []        # heap of (arrival, job_id, job)
        self.running = []
        self.preparing = []
        self.done = []
        self.batch = None
        self.particle_steps = 0
        self.pool = collections.OrderedDict()   # (n, solver, id) -> (scene, bytes), least recently used first
        self._lock = threading.Lock()           # pool, used, reserved
        # seconds by activity: on the serving thread the waits for seeds, for preparations, for the
        # in-flight frame, batch rebuilds and idle waits for arrivals; on the I/O thread scene preparation
        # ("create") and read-back + release ("retire"); "step" is the GPU worker's batched-substep time
        self.timing = collections.defaultdict(float)
        self.rebuilds = 0
        self.reused = 0
        self.cancelled = []      # jobs that left through cancel(), in the order they left
        self._cancel = set()     # ids asked to leave, not matched to a job yet

    def submit(self, job):
        heapq.heappush(self.waiting, (job.arrival, job.job_id, job))

    def cancel(self, job_id):
        """Asks job `job_id` to leave; safe from any thread (an on_frame callback included).  A waiting job
        leaves the queue, a running one leaves at the next frame boundary (no frame of it is cut short: the
        frame in flight completes for every member), and a job being prepared leaves when it is ready.  Its
        scene goes back to the pool without a read-back and its memory is released like a finished job's."""
        with self._lock:
            self._cancel.add(job_id)

    # ---------------------------------------------------------------------------------------- helpers
    def _seed(self, job):
        return _abi.seed_regions(job.regions, (job.n,) * 3, seed=job.seed)

    def _prefetch(self, now, executor):
        """Starts seeding arrived jobs near the head of the queue that are not seeded yet."""
        ahead = 0
        for arrival, _, job in sorted(self.waiting):
            if arrival > now or ahead >= 2 * self.seed_threads:
                break
            if job.seeded is None and getattr(job, "_seed_future", None) is None:
                job._seed_future = executor.submit(self._seed, job)
            ahead += 1

    def _evict_for(self, need):
        """Frees pooled scenes (least recently used first) until `need` more bytes fit; True if they do."""
        while True:
            with self._lock:
                if self.used + self.reserved + need <= self.budget or not self.pool:
                    return self.used + self.reserved + need <= self.budget
                _, (scene, nbytes) = self.pool.popitem(last=False)
                self.used -= nbytes
            scene.close()

    def _claim_pooled(self, n, solver):
        """Takes a pooled scene of this grid and solver out of the pool: (scene, bytes) or None."""
        with self._lock:
            for key in list(self.pool.keys()):
                if key[0] == n and key[1] == solver:
                    return self.pool.pop(key)
        return None

    def _prepare_job(self, job, claimed, need):
        """I/O thread: a scene for the job (the claimed pooled one, reset, or a new one) with its particles."""
        t = time.perf_counter()
        if claimed is not None:
            scene, nbytes = claimed
            scene.reset()
            self.reused += 1
        else:
            with self._lock:
                self.reserved -= need
                self.used += need
            nbytes = need
            scene = Scene((job.n,) * 3, solver=job.solver, max_cfl=1.0, cg_rel_tol=self.cg_rel_tol,
                          device=self.device)
        if self.batch_family == "cg":
            scene.set_tuning(multigrid=0)
        pos, vel = job.seeded
        scene.set_particles(pos, vel)
        job.scene = scene
        job.bytes = nbytes
        job.particles = pos.shape[0]
        job.seeded = None
        self.timing["create"] += time.perf_counter() - t

    def _release_job(self, job, now, read_back=True):
        """I/O thread: reads back a finished job and returns its scene to the pool (or frees it)."""
        t = time.perf_counter()
        job.finished_at = now
        job.final = job.scene.particles() if read_back else None
        scene, job.scene = job.scene, None
        if self.reuse_scenes:
            with self._lock:
                self.pool[(job.n, job.solver, id(scene))] = (scene, job.bytes)
                self._releasing -= 1
                self._releasing_shapes[(job.n, job.solver)] -= 1
        else:
            scene.close()
            with self._lock:
                self.used -= job.bytes
                self._releasing -= 1
                self._releasing_shapes[(job.n, job.solver)] -= 1
        self.timing["retire"] += time.perf_counter() - t

    def _admit(self, now, io):
        """Schedules preparations for waiting jobs (arrival order) while slots and the budget allow."""
        while self.waiting and self.waiting[0][0] <= now and \
                len(self.running) + len(self.preparing) < self.max_batch:
            _, _, job = self.waiting[0]
            if job.seeded is None:
                fut = getattr(job, "_seed_future", None)
                if fut is None:
                    break
                if not fut.done():
                    if self.running or self.preparing:
                        break  # the GPU has work; come back after this frame
                    t = time.perf_counter()
                    fut.result()
                    self.timing["seed_wait"] += time.perf_counter() - t
                job.seeded = fut.result()
                job._seed_future = None
            pos, _ = job.seeded
            need = scene_bytes(job.n, pos.shape[0], job.solver)
            claimed = self._claim_pooled(job.n, job.solver) if self.reuse_scenes else None
            if claimed is None and self.reuse_scenes:
                with self._lock:
                    coming = self._releasing_shapes[(job.n, job.solver)] > 0
                if coming:
                    break  # a scene of this shape is being read back and pooled: take it once it is there
            if claimed is None:
                if not self._evict_for(need):
                    if not (self.running or self.preparing or self._releasing):
                        raise MemoryError("job %d needs %d bytes, more than the whole budget" % (job.job_id, need))
                    break  # wait for running jobs to leave
                with self._lock:
                    self.reserved += need
            heapq.heappop(self.waiting)
            job.admitted_at = now
            job._prep = io.submit(self._prepare_job, job, claimed, need)
            self.preparing.append(job)

    def _frame(self, groups):
        """GPU worker: one frame of every running job (jobs sharing dt and substeps share one batch)."""
        out = []
        for (dt, nsub), jobs in groups:
            f0 = time.perf_counter()
            if len(groups) == 1:
                self.batch.step(dt, nsub, stats=False)
            else:
                b = Batch([j.scene for j in jobs])
                if self.overlap:
                    b.set_overlap(True)
                if self.flat_max_cells is not None:
                    b.set_flat(self.flat_max_cells)
                b.step(dt, nsub, stats=False)
                b.close()
            out.append((jobs, nsub, (time.perf_counter() - f0) * 1e3))
        return out

    # ------------------------------------------------------------------------------------------- loop
    def run(self, on_frame=None):
        """Serves until every submitted job is done; returns (wall seconds, particle-steps)."""
        from concurrent.futures import ThreadPoolExecutor

        t0 = time.perf_counter()
        inflight = None
        releases = []
        with ThreadPoolExecutor(self.seed_threads) as seeders, ThreadPoolExecutor(1) as io, \
                ThreadPoolExecutor(1) as gpu:
            while True:
                now = time.perf_counter() - t0
                self._prefetch(now, seeders)
                self._admit(now, io)
                # preparations that finished join at this frame boundary; with an idle GPU wait for one
                if self.preparing and not self.running and inflight is None:
                    t = time.perf_counter()
                    self.preparing[0]._prep.result()
                    self.timing["prepare_wait"] += time.perf_counter() - t
                ready = [j for j in self.preparing if j._prep.done()]
                for j in ready:
                    j._prep.result()  # re-raises a failed preparation
                    j._prep = None
                self.preparing = [j for j in self.preparing if j._prep is not None]
                finished = []
                if inflight is not None:
                    t = time.perf_counter()
                    results = inflight.result()
                    self.timing["frame_wait"] += time.perf_counter() - t
                    inflight = None
                    for jobs, nsub, ms in results:
                        self.timing["step"] += ms / 1e3
                        for j in jobs:
                            j.frames_done += 1
                            j.frame_ms.append(ms)
                            self.particle_steps += j.particles * nsub
                        if on_frame:
                            on_frame(jobs, ms)
                    finished = [j for j in self.running if j.frames_done >= j.frames]
                    if finished:
                        self.running = [j for j in self.running if j.frames_done < j.frames]
                        done_at = time.perf_counter() - t0
                        for j in finished:
                            with self._lock:
                                self._releasing += 1
                                self._releasing_shapes[(j.n, j.solver)] += 1
                            releases.append(io.submit(self._release_job, j, done_at))
                            self.done.append(j)
                with self._lock:
                    asked = set(self._cancel)
                gone = []
                if asked:
                    # cancelled jobs leave at this frame boundary: waiting ones drop out of the queue, running
                    # and just-prepared ones release their scenes like finished jobs, without a read-back
                    keep = [e for e in self.waiting if e[2].job_id not in asked]
                    gone = [e[2] for e in self.waiting if e[2].job_id in asked]
                    if gone:
                        self.waiting = keep
                        heapq.heapify(self.waiting)
                    leaving = [j for j in self.running + ready if j.job_id in asked]
                    if leaving:
                        self.running = [j for j in self.running if j.job_id not in asked]
                        ready = [j for j in ready if j.job_id not in asked]
                        done_at = time.perf_counter() - t0
                        for j in leaving:
                            with self._lock:
                                self._releasing += 1
                                self._releasing_shapes[(j.n, j.solver)] += 1
                            releases.append(io.submit(self._release_job, j, done_at, False))
                    gone += leaving
                    for j in gone:
                        j.cancelled = True
                        self.cancelled.append(j)
                    with self._lock:
                        self._cancel -= {j.job_id for j in gone}
                changed = bool(finished) or bool(ready) or bool(gone)
                self.running.extend(ready)
                if not self.running:
                    if self.preparing:
                        continue
                    if not self.waiting:
                        break
                    t = time.perf_counter()
                    nxt = self.waiting[0][0] - (time.perf_counter() - t0)
                    time.sleep(min(0.005, nxt) if nxt > 0 else 0.001)  # next arrival, or memory being released
                    self.timing["idle"] += time.perf_counter() - t
                    continue
                if changed or self.batch is None:
                    t = time.perf_counter()
                    if self.batch is None:
                        self.batch = Batch([j.scene for j in self.running])
                        if self.overlap:
                            self.batch.set_overlap(True)
                        if self.flat_max_cells is not None:
                            self.batch.set_flat(self.flat_max_cells)
                    else:
                        self.batch.set_scenes([j.scene for j in self.running])
                    self.rebuilds += 1
                    self.timing["batch_build"] += time.perf_counter() - t
                groups = {}
                for j in self.running:
                    groups.setdefault((j.dt, j.substeps_per_frame), []).append(j)
                inflight = gpu.submit(self._frame, list(groups.items()))
            if self.batch is not None:
                self.batch.close()
                self.batch = None
            for f in releases:
                f.result()
        wall = time.perf_counter() - t0
        with self._lock:
            pooled = list(self.pool.values())
            self.pool.clear()
        for scene, nbytes in pooled:
            scene.close()
            self.used -= nbytes
        return wall, self.particle_steps

    def latency_percentiles(self):
        ms = np.array([m for j in self.done for m in j.frame_ms])
        if ms.size == 0:
            return None, None
        return float(np.percentile(ms, 50)), float(np.percentile(ms, 99))


def poisson_trace(rate_hz, duration_s, seed, resolutions=(32, 48, 64, 96, 128, 192), frames=(24, 240),
                  substeps_per_frame=4, dt=1.0 / 480.0, solver=_abi.APIC):
    """Seeded Poisson arrival trace of pool + falling-sphere jobs (the served configuration's scene family)."""
    rng = np.random.default_rng(seed)
    t, jobs, jid = 0.0, [], 0
    while True:
        t += rng.exponential(1.0 / rate_hz)
        if t > duration_s:
            break
        n = int(rng.choice(resolutions))
        nf = int(rng.integers(frames[0], frames[1] + 1))
        regions = [dict(kind=0, lo=(0.0, 0.0, 0.0), hi=(1.0, 0.3, 1.0)),
                   dict(kind=1, lo=(0.5, 0.7, 0.5), hi=(0.15,), vel=(0.0, -2.0, 0.0))]
        jobs.append(Job(job_id=jid, n=n, solver=solver, regions=regions, frames=nf,
                        substeps_per_frame=substeps_per_frame, dt=dt, arrival=t, seed=int(rng.integers(1 << 30))))
        jid += 1
    return jobs
