"""Viscosity on the GPU (ComputeDiffusion, pic_simulator.cpp:214-222) against the FP64 oracle.

The diffusion stage alone is compared bit for bit: on the same FP32 grid and particles, the face markers, the
Jacobi iteration counts and the diffused velocities (the oracle's FP64 result rounded to FP32) are identical.
Whole viscous substeps are compared with the substep tolerance (particle velocities rel-L2 1e-4), and scenes
in a batch with the same scenes stepped alone (positions 1e-5, velocities 1e-4).
"""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

fe = pytest.importorskip("fluide_engine_b200")


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def pair(n, solver, nu, seed=0, box=(0.0, 0.0, 0.0, 0.4, 0.6, 1.0), origin=(0.0, 0.0, 0.0), vel_scale=0.5,
         max_cfl=1.0):
    lo = tuple(origin[a] + box[a] for a in range(3))
    hi = tuple(origin[a] + box[3 + a] for a in range(3))
    pos, _ = fe.seed_regions([dict(kind=0, lo=lo, hi=hi)], n, origin, (1, 1, 1), seed)
    rng = np.random.default_rng(seed + 20)
    pos = pos[rng.permutation(pos.shape[0])]
    vel = (rng.standard_normal(pos.shape) * vel_scale).astype(np.float32)
    C = (rng.standard_normal((pos.shape[0], 9)) * 0.3).astype(np.float32)
    g = fe.Scene(n, solver=solver, origin=origin, max_cfl=max_cfl, cg_rel_tol=1e-6, viscosity=nu,
                 pressure_solver=fe.CG)
    g.set_particles(pos, vel, C)
    o = oracle.OracleSim(n, solver, origin=origin, max_cfl=max_cfl, cg_rel_tol=1e-10, cg_max_it=20000, viscosity=nu)
    o.set_particles(pos.astype(np.float64), vel.astype(np.float64), C.astype(np.float64))
    return g, o, pos, vel, C


# c = nu dt / h^2 from 0.004 (the solve stops at its first check) through ~0.6 (tens of iterations) to > 10
# (the 1000-iteration cap), on cubic, non-cubic and offset domains
CASES = [((16, 16, 16), fe.FLIP, 0.01, (0.0, 0.0, 0.0)),
         ((20, 12, 9), fe.APIC, 1.0, (0.0, 0.0, 0.0)),
         ((24, 20, 16), fe.PIC, 30.0, (0.0, 0.0, 0.0)),
         ((10, 14, 12), fe.FLIP, 0.5, (-0.5, 0.25, 1.0)),
         ((64, 64, 64), fe.FLIP, 0.2, (0.0, 0.0, 0.0)),
         ((48, 48, 48), fe.FLIP, 0.002, (0.0, 0.0, 0.0))]  # iterates become periodic long before the cap


@pytest.mark.parametrize("n, solver, nu, origin", CASES)
def test_diffusion_stage_bit_exact(n, solver, nu, origin):
    g, o, *_ = pair(n, solver, nu, seed=3, origin=origin)
    dt = 1 / 240
    g.run_stages(dt, fe.STAGE_SORT, fe.STAGE_PRE)
    u, v, w, _, _ = g.grid()
    o.stage("p2g")
    o.stage("sdf")
    o.set_grid(u.astype(np.float64), v.astype(np.float64), w.astype(np.float64))  # identical solver input
    g.run_stages(dt, fe.STAGE_DIFFUSE, fe.STAGE_DIFFUSE)
    o.stage("diffusion", dt)
    its, marks = g.diffusion()
    for a, b in zip(marks, o.diffusion_markers()):
        assert np.array_equal(a, b)
    assert sum(int(m.sum()) for m in marks) > 0
    assert its == o.diffusion_iterations()
    ug, vg, wg, _, _ = g.grid()
    for a, b in zip((ug, vg, wg), o.grid()):
        assert np.array_equal(a, b.astype(np.float32))
    # the solve changed the grid (on the offset domain the velocity grid's origin quirk leaves u all zero)
    assert any(not np.array_equal(a, b) for a, b in zip((ug, vg, wg), (u, v, w)))


def test_diffusion_zero_viscosity_is_a_no_op():
    g, _, *_ = pair((16, 16, 16), fe.FLIP, 0.0, seed=4)
    dt = 1 / 240
    g.run_stages(dt, fe.STAGE_SORT, fe.STAGE_PRE)
    before = g.grid()[:3]
    g.run_stages(dt, fe.STAGE_DIFFUSE, fe.STAGE_DIFFUSE)
    assert all(np.array_equal(a, b) for a, b in zip(g.grid()[:3], before))


@pytest.mark.parametrize("solver", [fe.PIC, fe.FLIP, fe.APIC])
def test_viscous_substeps_track_oracle(solver):
    n = (24, 20, 16)
    g, o, *_ = pair(n, solver, 0.3, seed=5)
    dt = 1 / 240
    for _ in range(2):
        stats = g.step(dt, 1)
        o.substep(dt)
        assert stats[0]["converged"] == 1
    P, V, C = g.particles()
    Po, Vo, Co = o.particles()
    assert rel_l2(P, Po) < 1e-6
    assert rel_l2(V, Vo) < 1e-4
    if solver == fe.APIC:
        assert rel_l2(C, Co) < 1e-4
    for a, b in zip(g.grid()[:3], o.grid()):
        assert rel_l2(a, b) < 1e-4


def test_viscosity_set_after_steps_and_empty_scene():
    n = (16, 16, 16)
    dt = 1 / 240
    g1, _, pos, vel, C = pair(n, fe.FLIP, 0.0, seed=6)
    g2 = fe.Scene(n, solver=fe.FLIP, max_cfl=1.0, viscosity=0.4, pressure_solver=fe.CG)
    g2.set_particles(pos, vel, C)
    g1.step(dt, 1)
    g1.set_viscosity(0.4)  # re-captures the substep graphs with the diffusion stage
    g1.step(dt, 2)
    g2.step(dt, 3)
    V1, V2 = g1.particles()[1], g2.particles()[1]
    assert rel_l2(V1, V2) > 0  # the first substep of g1 had no viscosity
    g3 = fe.Scene(n, solver=fe.FLIP, max_cfl=1.0, viscosity=0.4, pressure_solver=fe.CG)
    g3.set_particles(pos, vel, C)
    g3.step(dt, 1)
    g3.set_viscosity(0.4)
    g3.step(dt, 2)
    assert rel_l2(g3.particles()[1], V2) < 1e-4
    # no particles in the band: every face is AIR, only the walls are zeroed
    e = fe.Scene(n, solver=fe.FLIP, max_cfl=1.0, viscosity=1.0)
    e.set_particles(np.array([[0.5, 0.5, 0.5]], np.float32))
    e.run_stages(dt, fe.STAGE_SORT, fe.STAGE_DIFFUSE)
    its, marks = e.diffusion()
    assert its == (6, 6, 6) or sum(int(m.sum()) for m in marks) > 0


def test_batch_with_viscous_scenes_matches_alone():
    dt = 1.0 / 240.0
    specs = [((24, 24, 24), fe.PIC, 0.2, (0.0, 0.0, 0.0, 0.5, 0.4, 0.7)),
             ((32, 32, 32), fe.FLIP, 0.0, (0.1, 0.0, 0.0, 0.5, 0.6, 1.0)),
             ((20, 16, 12), fe.APIC, 1.5, (0.0, 0.0, 0.2, 0.6, 0.5, 0.8)),
             ((28, 28, 28), fe.FLIP, 0.05, (0.0, 0.0, 0.0, 0.3, 0.5, 0.5))]

    def make(spec, seed):
        n, solver, nu, box = spec
        pos, _ = fe.seed_regions([dict(kind=0, lo=box[:3], hi=box[3:])], n, seed=seed)
        vel = (np.random.default_rng(seed).standard_normal(pos.shape) * 0.3).astype(np.float32)
        s = fe.Scene(n, solver=solver, max_cfl=1.0, cg_rel_tol=1e-6, viscosity=nu)
        s.set_particles(pos, vel)
        return s

    alone = [make(sp, i) for i, sp in enumerate(specs)]
    mixed = [make(sp, i) for i, sp in enumerate(specs)]
    for s in alone:
        s.step(dt, 12)
    batch = fe.Batch(mixed)
    stats = batch.step(dt, 12)  # 8 substeps replaying the scenes' graphs, then the captured batch graph
    batch.close()
    for a, m, st in zip(alone, mixed, stats):
        assert all(x["converged"] == 1 for x in st), st
        Pa, Va, _ = a.particles()
        Pm, Vm, _ = m.particles()
        assert rel_l2(Pm, Pa) < 1e-5
        assert rel_l2(Vm, Va) < 1e-4
