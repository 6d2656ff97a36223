"""Flat batch launches: every pre- and post-solve pass is one launch for all scenes over a (scene, block) work list.

The flat form, the per-scene form (each scene's passes on its own stream, fe_batch_set_flat(0)) and their mix (small
scenes flat, the rest on their own streams, concurrently) run the same algorithm; both must match the scenes stepped alone within the substep tolerance (positions rel-L2 1e-5,
velocities 1e-4), with marks bit-identical after the first substep (identical particles).  Twelve substeps cover
the directly launched young substeps and the captured batch graph (captured after eight).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

fe = pytest.importorskip("fluide_engine_b200")

DT = 1.0 / 240.0

# uneven grids (a non-power-of-two, an anisotropic one), all three transfers, a scene with no particles' worth of
# work in most tiles (a thin block)
SPECS = [((24, 24, 24), fe.PIC, (0.0, 0.0, 0.0, 0.5, 0.4, 0.7)),
         ((32, 32, 32), fe.FLIP, (0.1, 0.0, 0.0, 0.5, 0.6, 1.0)),
         ((20, 16, 12), fe.APIC, (0.0, 0.0, 0.2, 0.6, 0.5, 0.8)),
         ((40, 40, 40), fe.FLIP, (0.0, 0.0, 0.0, 0.3, 0.5, 0.5)),
         ((16, 16, 16), fe.APIC, (0.0, 0.0, 0.0, 1.0, 0.1, 1.0))]


def rel_l2(a, b):
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(np.asarray(a, np.float64) - b)) / max(float(np.linalg.norm(b)), 1e-300)


def make(spec, seed, max_cfl=1.0):
    n, solver, box = spec
    pos, _ = fe.seed_regions([dict(kind=0, lo=box[:3], hi=box[3:])], n, seed=seed)
    vel = (np.random.default_rng(seed).standard_normal(pos.shape) * 0.3).astype(np.float32)
    s = fe.Scene(n, solver=solver, max_cfl=max_cfl, cg_rel_tol=1e-6)
    s.set_particles(pos, vel)
    return s


def check_close(alone, mixed):
    for a, m in zip(alone, mixed):
        Pa, Va, Ca = a.particles()
        Pm, Vm, Cm = m.particles()
        assert rel_l2(Pm, Pa) < 1e-5
        assert rel_l2(Vm, Va) < 1e-4
        if a.solver == fe.APIC:
            assert rel_l2(Cm, Ca) < 1e-4


# every scene flat, none, and a mix (scenes up to 20000 cells flat, the 32^3 and 40^3 scenes on their own streams)
@pytest.mark.parametrize("flat", [-1, 0, 20000])
def test_flat_and_forked_match_alone(flat):
    alone = [make(sp, i) for i, sp in enumerate(SPECS)]
    mixed = [make(sp, i) for i, sp in enumerate(SPECS)]
    batch = fe.Batch(mixed)
    batch.set_flat(flat)
    for s in alone:
        s.step(DT, 1)
    st1 = batch.step(DT, 1)
    for a, m in zip(alone, mixed):
        assert np.array_equal(a.grid()[4], m.grid()[4])
        assert np.array_equal(a.face_markers()[0], m.face_markers()[0])
    for s in alone:
        s.step(DT, 11)
    st = batch.step(DT, 11)
    batch.close()
    for s1, s in zip(st1, st):
        assert all(x["converged"] == 1 and x["rel_residual"] <= 1e-6 for x in s1 + s), s
    check_close(alone, mixed)


def test_flat_first_substep_grid_equals_alone():
    # one substep from identical particles: the flat passes produce the same grid velocities, pressure and marks as
    # the scene's own launches (the pressure to the solve's tolerance)
    alone = [make(sp, 10 + i) for i, sp in enumerate(SPECS)]
    mixed = [make(sp, 10 + i) for i, sp in enumerate(SPECS)]
    batch = fe.Batch(mixed)
    batch.set_flat(-1)
    for s in alone:
        s.step(DT, 1)
    batch.step(DT, 1)
    batch.close()
    for a, m in zip(alone, mixed):
        ga, gm = a.grid(), m.grid()
        assert np.array_equal(ga[4], gm[4])
        for k in range(3):
            assert rel_l2(gm[k], ga[k]) < 1e-5
        assert rel_l2(gm[3], ga[3]) < 1e-4


def test_flat_extrapolation_depths_and_membership_changes():
    # scenes with different extrapolation depths (maxCfl 1, 2.5 and 3) in one batch; the membership changes and a
    # scene is stepped alone between batch steps (its particle parity moves against the batch's)
    cfl = [1.0, 2.5, 3.0, 1.0, 2.5]
    alone = [make(sp, 20 + i, c) for i, (sp, c) in enumerate(zip(SPECS, cfl))]
    mixed = [make(sp, 20 + i, c) for i, (sp, c) in enumerate(zip(SPECS, cfl))]
    batch = fe.Batch(mixed[:3])
    batch.set_flat(-1)
    batch.step(DT, 9)  # past the capture of the batch graph
    for s in alone[:3]:
        s.step(DT, 9)
    mixed[1].step(DT, 1)  # stepped alone: its parity now differs from the batch's plan
    alone[1].step(DT, 1)
    batch.step(DT, 3)
    for s in alone[:3]:
        s.step(DT, 3)
    batch.set_scenes(mixed)
    batch.step(DT, 10)
    for s in alone:
        s.step(DT, 10)
    batch.close()
    check_close(alone, mixed)


def test_flat_profiled_phases():
    mixed = [make(sp, 30 + i) for i, sp in enumerate(SPECS)]
    alone = [make(sp, 30 + i) for i, sp in enumerate(SPECS)]
    batch = fe.Batch(mixed)
    batch.set_flat(20000)  # three scenes flat, two on their own streams
    stats, ms = batch.step_profiled(DT, 3)
    batch.close()
    ms = np.asarray(ms).reshape(3, 3)
    assert np.all(ms > 0.0)
    for s in alone:
        s.step(DT, 3)
    check_close(alone, mixed)
