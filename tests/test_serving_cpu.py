"""Host logic of the serving loop (admission against the HBM budget, continuous batching across frame
boundaries, scene reuse, read-back of finished jobs), with the device replaced by stand-ins: a scene
records what it was asked to do and a batch "step" only sleeps, so this runs without a GPU."""
import time

import numpy as np
import pytest

from fluide_engine_b200 import serving


class FakeScene:
    live = 0
    created = 0
    tunings = []

    def __init__(self, n, solver=0, max_cfl=1.0, cg_rel_tol=1e-6, device=0):
        self.n, self.solver = n, solver
        self.steps = 0
        self.resets = 0
        self.np = 0
        self.closed = False
        FakeScene.live += 1
        FakeScene.created += 1

    def set_particles(self, pos, vel=None, C=None):
        self.np = pos.shape[0]
        self.steps = 0
        self.pos = pos.copy()

    def reset(self):
        self.resets += 1

    def set_tuning(self, **kw):
        FakeScene.tunings.append(kw)

    def particles(self):
        return self.pos + self.steps, np.full_like(self.pos, self.steps), np.zeros((self.np, 9), np.float32)

    def close(self):
        assert not self.closed
        self.closed = True
        FakeScene.live -= 1


class FakeBatch:
    def __init__(self, scenes):
        assert len(scenes) == len({id(s) for s in scenes}), "a scene appears twice in a batch"
        assert not any(s.closed for s in scenes)
        self.scenes = scenes

    def set_scenes(self, scenes):
        self.__init__(scenes)

    def set_overlap(self, on=True):
        self.overlap = on

    def step(self, dt, nsub, stats=True):
        time.sleep(0.002)
        for s in self.scenes:
            s.steps += nsub

    def close(self):
        pass


def fake_seed(regions, n, seed=0):
    count = n[0] * 10 + seed % 3
    pos = np.full((count, 3), float(seed), np.float32)
    return pos, np.zeros_like(pos)


@pytest.fixture(autouse=True)
def stand_ins(monkeypatch):
    monkeypatch.setattr(serving, "Scene", FakeScene)
    monkeypatch.setattr(serving, "Batch", FakeBatch)
    monkeypatch.setattr(serving._abi, "seed_regions", fake_seed)
    FakeScene.live = 0
    FakeScene.created = 0
    FakeScene.tunings = []


def jobs(k, n=16, frames=3, spacing=0.0, nsub=2):
    return [serving.Job(job_id=i, n=n if np.isscalar(n) else n[i % len(n)], solver=1, regions=[], frames=frames + i % 2,
                        substeps_per_frame=nsub, dt=0.01, arrival=spacing * i, seed=i) for i in range(k)]


def test_every_job_runs_all_frames_and_is_read_back():
    js = jobs(7, n=(16, 24), spacing=0.001)
    srv = serving.Server(hbm_budget_bytes=1 << 40, max_batch=3)
    for j in js:
        srv.submit(j)
    wall, psteps = srv.run()
    assert len(srv.done) == 7 and not srv.running and not srv.preparing
    for j in js:
        assert j.frames_done == j.frames
        P, V, _ = j.final
        # the read-back happened after the job's last frame: every substep of the job, and nothing more
        assert np.all(V == j.frames * j.substeps_per_frame)
    assert psteps == sum(j.frames * j.substeps_per_frame * (j.n * 10 + j.seed % 3) for j in js)
    assert FakeScene.live == 0  # pooled scenes are freed at the end


def test_budget_and_slots_bound_the_running_set():
    js = jobs(6, n=16)
    one = serving.scene_bytes(16, 160, 1)
    srv = serving.Server(hbm_budget_bytes=int(2.5 * one), max_batch=8)
    seen = []
    srv_ref = srv

    def on_frame(jobs_, ms):
        seen.append((len(jobs_), srv_ref.used + srv_ref.reserved))

    for j in js:
        srv.submit(j)
    srv.run(on_frame=on_frame)
    assert len(srv.done) == 6
    assert max(k for k, _ in seen) <= 2
    assert max(b for _, b in seen) <= 2.5 * one
    assert FakeScene.created <= 2 and srv.reused == 4  # later jobs ran on reset, reused scenes


def test_max_batch_limits_membership():
    js = jobs(9, n=16)
    srv = serving.Server(hbm_budget_bytes=1 << 40, max_batch=4)
    sizes = []
    for j in js:
        srv.submit(j)
    srv.run(on_frame=lambda jobs_, ms: sizes.append(len(jobs_)))
    assert max(sizes) <= 4 and len(srv.done) == 9


def test_without_reuse_every_job_gets_a_new_scene():
    js = jobs(4, n=16)
    srv = serving.Server(hbm_budget_bytes=1 << 40, max_batch=2, reuse_scenes=False)
    for j in js:
        srv.submit(j)
    srv.run()
    assert FakeScene.created == 4 and srv.reused == 0 and FakeScene.live == 0 and srv.used == 0


def test_job_larger_than_budget_raises():
    js = jobs(1, n=64)
    srv = serving.Server(hbm_budget_bytes=1000, max_batch=2)
    srv.submit(js[0])
    with pytest.raises(MemoryError):
        srv.run()


def test_frame_latency_and_arrival_order():
    js = jobs(5, n=16, spacing=0.01)
    srv = serving.Server(hbm_budget_bytes=1 << 40, max_batch=8)
    for j in reversed(js):
        srv.submit(j)
    srv.run()
    p50, p99 = srv.latency_percentiles()
    assert p50 is not None and p99 >= p50 > 0
    admitted = sorted(js, key=lambda j: j.admitted_at)
    assert [j.job_id for j in admitted] == sorted(j.job_id for j in js)


def test_cancelled_jobs_leave_and_release_their_memory():
    """A job cancelled mid-run leaves at the next frame boundary (not read back, scene released); a job cancelled
    while it waits never runs; the others run all their frames."""
    js = jobs(6, n=16, frames=6, spacing=0.0)
    js[5].arrival = 10.0  # still waiting when it is cancelled
    srv = serving.Server(hbm_budget_bytes=1 << 40, max_batch=4, reuse_scenes=False)
    frames = []

    def on_frame(jobs_, ms):
        frames.append({j.job_id for j in jobs_})
        if any(j.job_id == 1 and j.frames_done == 2 for j in jobs_):
            srv.cancel(1)   # running: leaves after this frame
            srv.cancel(5)   # waiting

    for j in js:
        srv.submit(j)
    srv.run(on_frame=on_frame)
    by_id = {j.job_id: j for j in js}
    assert by_id[1].cancelled and by_id[1].frames_done == 2 and by_id[1].final is None
    assert by_id[5].cancelled and by_id[5].frames_done == 0 and by_id[5].admitted_at is None
    assert {j.job_id for j in srv.cancelled} == {1, 5}
    for i in (0, 2, 3, 4):
        j = by_id[i]
        assert not j.cancelled and j.frames_done == j.frames
        assert np.all(j.final[1] == j.frames * j.substeps_per_frame)
    assert sum(1 in f for f in frames) == 2
    assert FakeScene.live == 0 and srv.used == 0


def test_batch_family_cg_puts_every_job_on_the_plain_solver():
    js = jobs(5, n=(16, 24), spacing=0.001)
    srv = serving.Server(hbm_budget_bytes=1 << 40, max_batch=3, batch_family="cg")
    for j in js:
        srv.submit(j)
    srv.run()
    assert len(srv.done) == 5
    # every job's scene (new or reused from the pool) was put on the plain CG before it joined a batch
    assert FakeScene.tunings == [{"multigrid": 0}] * 5
    with pytest.raises(ValueError):
        serving.Server(hbm_budget_bytes=1 << 40, batch_family="mg")
