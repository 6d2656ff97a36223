"""Serving loop: simulation jobs admitted against an HBM budget and advanced with continuous batching.

A job is (scene spec, frames, substeps per frame).  Jobs arrive over time; the server admits waiting jobs
in arrival order whenever a batch slot and enough of the HBM budget are free, keeps every admitted job's
particles and grid resident on the device between frames, and advances all running jobs together: one
fe_batch_step per substep over the current membership (the batch is rebuilt only when a job joins or
leaves, i.e. between frames).  Each job's frame latency is measured from the start of the frame's first
substep to the end of its last; aggregate particle-steps/s counts every running job's particles.

The reference has no serving layer: it runs one simulator per process frame by frame
(SimulationRunner::RunSimulation, simulation_runner.cpp:17-55).
"""
import collections
import heapq
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


def scene_bytes(n, particles, solver):
    """Device bytes of one scene (allocation plan of fe_scene.cu): grid, solver vectors and particles."""
    cells = n ** 3
    faces = 3 * (n + 1) * n * n
    grid = faces * (5 * 4 + 3) + cells * (1 + 8 + 8 + 8 * 4 + 4 + 4 + 4) + (cells // 512 + 1) * 512 * 8
    per_particle = 2 * (7 + (9 if solver == _abi.APIC else 0)) * 4 + 3 * 4 + 9 * 4 + 4
    return grid + particles * per_particle


class Server:
    """Continuous-batching simulation server on one device."""

    def __init__(self, hbm_budget_bytes, max_batch=32, device=0, cg_rel_tol=1e-6):
        self.budget = int(hbm_budget_bytes)
        self.max_batch = min(int(max_batch), 64)
        self.device = device
        self.cg_rel_tol = cg_rel_tol
        self.used = 0
        self.waiting = []    # heap of (arrival, job_id, job)
        self.running = []
        self.done = []
        self.batch = None
        self.particle_steps = 0
        # wall seconds by activity: seeding, scene creation + upload, batch rebuilds, batched substeps
        # (launch + device time), retirement (read-back + release), idle waits for arrivals
        self.timing = collections.defaultdict(float)
        self.rebuilds = 0

    def submit(self, job):
        heapq.heappush(self.waiting, (job.arrival, job.job_id, job))

    def _admit(self, now):
        changed = False
        while self.waiting and self.waiting[0][0] <= now and len(self.running) < self.max_batch:
            _, _, job = self.waiting[0]
            if job.seeded is None:
                t = time.perf_counter()
                job.seeded = _abi.seed_regions(job.regions, (job.n,) * 3, seed=job.seed)
                self.timing["seed"] += time.perf_counter() - t
            pos, vel = job.seeded
            need = scene_bytes(job.n, pos.shape[0], job.solver)
            if self.used + need > self.budget:
                if not self.running:
                    raise MemoryError("job %d needs %d bytes, more than the whole budget" % (job.job_id, need))
                break  # wait for running jobs to leave
            heapq.heappop(self.waiting)
            t = time.perf_counter()
            job.scene = Scene((job.n,) * 3, solver=job.solver, max_cfl=1.0, cg_rel_tol=self.cg_rel_tol,
                              device=self.device)
            job.scene.set_particles(pos, vel)
            job.seeded = None
            self.timing["create"] += time.perf_counter() - t
            job.particles = pos.shape[0]
            job.admitted_at = now
            job.bytes = need
            self.used += need
            self.running.append(job)
            changed = True
        return changed

    def _retire(self, now):
        keep = []
        changed = False
        t = time.perf_counter()
        for job in self.running:
            if job.frames_done >= job.frames:
                job.finished_at = now
                job.final = job.scene.particles()
                job.scene.close()
                job.scene = None
                self.used -= job.bytes
                self.done.append(job)
                changed = True
            else:
                keep.append(job)
        self.running = keep
        self.timing["retire"] += time.perf_counter() - t
        return changed

    def run(self, on_frame=None):
        """Serves until every submitted job is done; returns (wall seconds, particle-steps)."""
        t0 = time.perf_counter()
        while self.waiting or self.running:
            now = time.perf_counter() - t0
            changed = self._retire(now)
            changed |= self._admit(now)
            if not self.running:
                if not self.waiting:
                    break
                # idle until the next arrival
                t = time.perf_counter()
                time.sleep(max(0.0, min(0.01, self.waiting[0][0] - now)))
                self.timing["idle"] += time.perf_counter() - t
                continue
            if changed or self.batch is None:
                t = time.perf_counter()
                if self.batch is not None:
                    self.batch.close()
                self.batch = Batch([j.scene for j in self.running])
                self.rebuilds += 1
                self.timing["batch_build"] += time.perf_counter() - t
            # one frame of the common substep pattern: jobs share dt and substeps per frame within a batch
            groups = {}
            for j in self.running:
                groups.setdefault((j.dt, j.substeps_per_frame), []).append(j)
            for (dt, nsub), jobs in groups.items():
                f0 = time.perf_counter()
                if len(groups) == 1:
                    self.batch.step(dt, nsub, stats=False)
                else:
                    b = Batch([j.scene for j in jobs])
                    b.step(dt, nsub, stats=False)
                    b.close()
                ms = (time.perf_counter() - f0) * 1e3
                self.timing["step"] += ms / 1e3
                for j in jobs:
                    j.frames_done += 1
                    j.frame_ms.append(ms)
                    self.particle_steps += j.particles * nsub
                if on_frame:
                    on_frame(jobs, ms)
        if self.batch is not None:
            self.batch.close()
            self.batch = None
        self._retire(time.perf_counter() - t0)
        return time.perf_counter() - t0, self.particle_steps

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
