"""Batched scenes and the serving loop: each scene's result is the same alone and in the mix.

Scenes stepped inside a batch (one batched pressure solve per substep, one CUDA graph) must match the
same scenes stepped alone within the substep tolerance (positions rel-L2 1e-5, velocities 1e-4: the
float atomics of P2G and the order of the dot-product reductions differ between the two runs).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

fe = pytest.importorskip("fluide_engine_b200")
from fluide_engine_b200 import serving  # noqa: E402


def rel_l2(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-300))


SPECS = [((24, 24, 24), fe.PIC, (0.0, 0.0, 0.0, 0.5, 0.4, 0.7)),
         ((32, 32, 32), fe.FLIP, (0.1, 0.0, 0.0, 0.5, 0.6, 1.0)),
         ((20, 16, 12), fe.APIC, (0.0, 0.0, 0.2, 0.6, 0.5, 0.8)),
         ((48, 48, 48), fe.FLIP, (0.0, 0.0, 0.0, 0.3, 0.5, 0.5))]


def make(spec, seed):
    n, solver, box = spec
    pos, _ = fe.seed_regions([dict(kind=0, lo=box[:3], hi=box[3:])], n, seed=seed)
    vel = (np.random.default_rng(seed).standard_normal(pos.shape) * 0.3).astype(np.float32)
    s = fe.Scene(n, solver=solver, max_cfl=1.0, cg_rel_tol=1e-6)
    s.set_particles(pos, vel)
    return s


def test_batch_matches_scenes_alone():
    dt = 1.0 / 240.0
    alone = [make(sp, i) for i, sp in enumerate(SPECS)]
    mixed = [make(sp, i) for i, sp in enumerate(SPECS)]
    batch = fe.Batch(mixed)
    # first substep: both runs mark cells from identical particles, so the marks are bit-identical
    for s in alone:
        s.step(dt, 1)
    stats1 = batch.step(dt, 1)
    for a, m in zip(alone, mixed):
        assert np.array_equal(a.grid()[4], m.grid()[4])
    for s in alone:
        s.step(dt, 3)
    stats = batch.step(dt, 3)
    batch.close()
    for a, m, st1, st in zip(alone, mixed, stats1, stats):
        assert all(x["converged"] == 1 and x["rel_residual"] <= 1e-6 for x in st1 + st), st
        Pa, Va, _ = a.particles()
        Pm, Vm, _ = m.particles()
        assert rel_l2(Pm, Pa) < 1e-5
        assert rel_l2(Vm, Va) < 1e-4
        # later substeps mark from positions that differ in the last bits (the solves' dot products are
        # summed in a different order with a different block split, and P2G flushes with float atomics), so
        # a cell whose nearest particle sits within rounding of the marking radius may flip: at most a
        # handful of cells, never a systematic difference
        ma, mm = a.grid()[4], m.grid()[4]
        differ = int((ma != mm).sum())
        assert differ <= max(2, int(5e-4 * (ma == fe.FLUID).sum())), differ


def test_batch_then_single_steps_continue():
    # a scene leaves a batch and keeps stepping alone (parities and buffers stay consistent)
    dt = 1.0 / 240.0
    s1, s2 = make(SPECS[0], 5), make(SPECS[1], 6)
    ref = make(SPECS[0], 5)
    b = fe.Batch([s1, s2])
    b.step(dt, 3)
    b.close()
    s1.step(dt, 2)
    ref.step(dt, 5)
    assert rel_l2(s1.particles()[0], ref.particles()[0]) < 1e-5


def test_server_results_match_jobs_run_alone():
    jobs = []
    for k, (n, solver, box) in enumerate(SPECS[:3]):
        regions = [dict(kind=0, lo=box[:3], hi=box[3:])]
        jobs.append(serving.Job(job_id=k, n=n[0], solver=solver, regions=regions, frames=2 + k,
                                substeps_per_frame=2, dt=1.0 / 240.0, arrival=0.02 * k, seed=k))
    srv = serving.Server(hbm_budget_bytes=2 << 30, max_batch=8)
    for j in jobs:
        srv.submit(j)
    wall, psteps = srv.run()
    assert len(srv.done) == 3 and psteps > 0
    p50, p99 = srv.latency_percentiles()
    assert p50 is not None and p99 >= p50
    for j in srv.done:
        pos, vel = fe.seed_regions(j.regions, (j.n,) * 3, seed=j.seed)
        s = fe.Scene((j.n,) * 3, solver=j.solver, max_cfl=1.0, cg_rel_tol=1e-6)
        s.set_particles(pos, vel)
        s.step(j.dt, j.frames * j.substeps_per_frame)
        P, V, _ = s.particles()
        assert rel_l2(j.final[0], P) < 1e-5
        assert rel_l2(j.final[1], V) < 1e-4


def test_server_admission_respects_budget():
    regions = [dict(kind=0, lo=(0, 0, 0), hi=(0.5, 0.5, 0.5))]
    jobs = [serving.Job(job_id=k, n=32, solver=fe.FLIP, regions=regions, frames=1, substeps_per_frame=1,
                        dt=1 / 240, arrival=0.0, seed=k) for k in range(4)]
    one = serving.scene_bytes(32, fe.seed_regions(regions, (32,) * 3)[0].shape[0], fe.FLIP)
    srv = serving.Server(hbm_budget_bytes=int(2.5 * one), max_batch=8)
    peak = []
    for j in jobs:
        srv.submit(j)
    srv.run(on_frame=lambda jobs_, ms: peak.append(len(srv.running)))
    assert max(peak) <= 2 and len(srv.done) == 4


def test_scene_reset_matches_fresh_scene():
    """A scene that ran one job, reset and given new particles, steps like a freshly created scene."""
    dt = 1.0 / 240.0
    used = make(SPECS[1], 3)
    used.step(dt, 6)  # leaves pressure (warm start), grid and solver state behind
    used.reset()
    fresh = make(SPECS[1], 9)
    pos, vel, _ = fresh.particles()
    used.set_particles(pos, vel)
    p_used = used.grid()[3]
    assert not np.any(p_used)  # the warm start is gone
    st_u = used.step(dt, 3)
    st_f = fresh.step(dt, 3)
    assert [x["fluid_cells"] for x in st_u] == [x["fluid_cells"] for x in st_f]
    Pu, Vu, _ = used.particles()
    Pf, Vf, _ = fresh.particles()
    assert rel_l2(Pu, Pf) < 1e-5
    assert rel_l2(Vu, Vf) < 1e-4


def test_batch_step_profiled_phases():
    dt = 1.0 / 240.0
    scenes = [make(sp, i) for i, sp in enumerate(SPECS[:3])]
    b = fe.Batch(scenes)
    stats, ms = b.step_profiled(dt, 3)
    b.close()
    assert ms.shape == (3, 3) and np.all(ms > 0)
    assert len(stats) == 3 and all(len(s) == 3 for s in stats)
    assert all(x["converged"] == 1 for s in stats for x in s)


def test_server_reuses_scenes_and_matches_alone():
    """Jobs of one shape served one after another (one slot): later jobs run on reset, reused scenes."""
    regions = [dict(kind=0, lo=(0.0, 0.0, 0.0), hi=(0.4, 0.5, 0.6))]
    jobs = [serving.Job(job_id=k, n=24, solver=fe.APIC, regions=regions, frames=2, substeps_per_frame=2,
                        dt=1.0 / 240.0, arrival=0.0, seed=20 + k) for k in range(3)]
    srv = serving.Server(hbm_budget_bytes=2 << 30, max_batch=1)
    for j in jobs:
        srv.submit(j)
    srv.run()
    assert len(srv.done) == 3 and srv.reused == 2
    for j in srv.done:
        pos, vel = fe.seed_regions(j.regions, (j.n,) * 3, seed=j.seed)
        s = fe.Scene((j.n,) * 3, solver=j.solver, max_cfl=1.0, cg_rel_tol=1e-6)
        s.set_particles(pos, vel)
        s.step(j.dt, j.frames * j.substeps_per_frame)
        P, V, C = s.particles()
        assert rel_l2(j.final[0], P) < 1e-5
        assert rel_l2(j.final[1], V) < 1e-4
        s.close()


def test_batch_membership_change_matches_alone():
    """One batch whose scenes change between substeps (fe_batch_set_scenes): every scene still matches the
    same scene stepped alone for the same number of substeps."""
    dt = 1.0 / 240.0
    a, b, c = (make(SPECS[k], 30 + k) for k in (0, 1, 2))
    ra, rb, rc = (make(SPECS[k], 30 + k) for k in (0, 1, 2))
    batch = fe.Batch([a, b])
    batch.step(dt, 3)
    batch.set_scenes([b, c])       # a leaves, c joins
    batch.step(dt, 10)             # long enough for the batch graph to be captured with the new members
    batch.set_scenes([c, a, b])    # a returns
    batch.step(dt, 2)
    batch.close()
    ra.step(dt, 5)
    rb.step(dt, 15)
    rc.step(dt, 12)
    for m, r in ((a, ra), (b, rb), (c, rc)):
        Pm, Vm, _ = m.particles()
        Pr, Vr, _ = r.particles()
        assert rel_l2(Pm, Pr) < 1e-5
        assert rel_l2(Vm, Vr) < 1e-4


def test_batch_with_multigrid_scenes_matches_alone():
    """Scenes configured for the multigrid-preconditioned solver (used when they step alone; the batched
    launch solves every scene with the plain CG body) match the same scenes stepped alone, within the solve
    tolerance."""
    dt = 1.0 / 240.0
    specs = [((40, 40, 40), fe.FLIP, (0.0, 0.0, 0.0, 0.5, 0.5, 0.8), fe.MGPCG),
             ((24, 24, 24), fe.APIC, (0.0, 0.0, 0.0, 0.6, 0.4, 1.0), fe.CG),
             ((36, 20, 28), fe.PIC, (0.1, 0.0, 0.0, 0.7, 0.6, 0.9), fe.MGPCG)]

    def mk(k):
        n, solver, box, ps = specs[k]
        pos, _ = fe.seed_regions([dict(kind=0, lo=box[:3], hi=box[3:])], n, seed=40 + k)
        vel = (np.random.default_rng(k).standard_normal(pos.shape) * 0.3).astype(np.float32)
        s = fe.Scene(n, solver=solver, max_cfl=1.0, cg_rel_tol=1e-6, pressure_solver=ps)
        s.set_particles(pos, vel)
        return s
    alone = [mk(k) for k in range(3)]
    mixed = [mk(k) for k in range(3)]
    for s in alone:
        s.step(dt, 12)
    b = fe.Batch(mixed)
    stats = b.step(dt, 12)  # past the batch-graph capture
    b.close()
    for a, m, st in zip(alone, mixed, stats):
        assert all(x["converged"] == 1 and x["rel_residual"] <= 1e-6 for x in st), st
        Pa, Va, _ = a.particles()
        Pm, Vm, _ = m.particles()
        assert rel_l2(Pm, Pa) < 1e-5
        assert rel_l2(Vm, Va) < 1e-4


def test_server_job_cancelled_mid_run_leaves_the_others_unchanged():
    """A job cancelled while it runs leaves at the next frame boundary; the jobs it ran beside still match the
    same jobs run alone, and a job cancelled before admission never runs."""
    regions = [dict(kind=0, lo=(0.0, 0.0, 0.0), hi=(0.4, 0.5, 0.6))]
    jobs = [serving.Job(job_id=k, n=24 + 8 * (k % 2), solver=(fe.FLIP, fe.APIC, fe.PIC)[k % 3], regions=regions,
                        frames=5, substeps_per_frame=2, dt=1.0 / 240.0, arrival=0.0 if k < 3 else 30.0, seed=50 + k)
            for k in range(4)]
    srv = serving.Server(hbm_budget_bytes=4 << 30, max_batch=4)

    def on_frame(jobs_, ms):
        if any(j.job_id == 1 and j.frames_done == 2 for j in jobs_):
            srv.cancel(1)
            srv.cancel(3)

    for j in jobs:
        srv.submit(j)
    srv.run(on_frame=on_frame)
    assert jobs[1].cancelled and jobs[1].frames_done == 2 and jobs[1].final is None
    assert jobs[3].cancelled and jobs[3].frames_done == 0
    for j in (jobs[0], jobs[2]):
        assert not j.cancelled and j.frames_done == j.frames
        pos, vel = fe.seed_regions(j.regions, (j.n,) * 3, seed=j.seed)
        s = fe.Scene((j.n,) * 3, solver=j.solver, max_cfl=1.0, cg_rel_tol=1e-6)
        s.set_particles(pos, vel)
        s.step(j.dt, j.frames * j.substeps_per_frame)
        P, V, _ = s.particles()
        assert rel_l2(j.final[0], P) < 1e-5
        assert rel_l2(j.final[1], V) < 1e-4
        s.close()


def test_overlap_mode_matches_alone():
    """Overlap mode (each scene's whole substep on its own stream with its own solve on its share of the solver
    blocks): every scene still matches the same scene stepped alone, through the young substeps, the re-split of
    the shares and the captured batch graph."""
    dt = 1.0 / 240.0
    alone = [make(sp, 60 + i) for i, sp in enumerate(SPECS)]
    mixed = [make(sp, 60 + i) for i, sp in enumerate(SPECS)]
    mixed[1].set_tuning(multigrid=1)  # one scene on the multigrid body
    alone[1].set_tuning(multigrid=1)
    for s in alone:
        s.step(dt, 14)
    b = fe.Batch(mixed)
    b.set_overlap(True)
    stats = b.step(dt, 14)
    b.close()
    for a, m, st in zip(alone, mixed, stats):
        assert all(x["converged"] == 1 and x["rel_residual"] <= 1e-6 for x in st), st
        Pa, Va, _ = a.particles()
        Pm, Vm, _ = m.particles()
        assert rel_l2(Pm, Pa) < 1e-5
        assert rel_l2(Vm, Va) < 1e-4
