"""Per-job checkpoint / resume on the device (fe_scene_snapshot / fe_scene_restore).

A scene restored from a snapshot steps as it did from that point on: the same substeps after a restore into the
same scene, or into a fresh scene of the same grid and solver, reach the original's particles within the substep
tolerance (positions rel-L2 1e-5, velocities 1e-4: the solver's dot products are summed in a varying order, so two
runs agree to rounding, not bit for bit).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

fe = pytest.importorskip("fluide_engine_b200")


def rel_l2(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def scene(n, solver, seed):
    pos, _ = fe.seed_regions([dict(kind=0, lo=(0.0, 0.0, 0.0), hi=(0.4, 0.6, 0.8))], n, seed=seed)
    rng = np.random.default_rng(seed)
    vel = (rng.standard_normal(pos.shape) * 0.3).astype(np.float32)
    C = (rng.standard_normal((pos.shape[0], 9)) * 0.1).astype(np.float32)
    s = fe.Scene(n, solver=solver, max_cfl=1.0, cg_rel_tol=1e-7)
    s.set_particles(pos, vel, C)
    return s


@pytest.mark.parametrize("solver", [fe.FLIP, fe.APIC])
def test_restore_resumes_the_same_trajectory(solver):
    n = (32, 32, 32)
    dt = 1.0 / 240.0
    s = scene(n, solver, 3)
    s.step(dt, 5)
    snap = s.checkpoint()
    info = snap.info()
    assert info["particles"] == s.num_particles() and info["bytes"] > 0
    s.step(dt, 6)
    Pa, Va, Ca = s.particles()
    pa = s.grid()[3]
    # back into the same scene
    s.restore(snap)
    s.step(dt, 6)
    Pb, Vb, Cb = s.particles()
    assert rel_l2(Pb, Pa) < 1e-5 and rel_l2(Vb, Va) < 1e-4
    assert rel_l2(s.grid()[3], pa) < 1e-3
    # into a fresh scene of the same grid and solver
    t = fe.Scene(n, solver=solver, max_cfl=1.0, cg_rel_tol=1e-7)
    t.restore(snap)
    t.step(dt, 6)
    Pc, Vc, Cc = t.particles()
    assert rel_l2(Pc, Pa) < 1e-5 and rel_l2(Vc, Va) < 1e-4
    if solver == fe.APIC:
        assert rel_l2(Cb, Ca) < 1e-3 and rel_l2(Cc, Ca) < 1e-3
    snap.close()
    s.close()
    t.close()


def test_restore_rejects_another_grid():
    s = scene((24, 24, 24), fe.FLIP, 1)
    s.step(1.0 / 240.0, 1)
    snap = s.checkpoint()
    other = fe.Scene((32, 32, 32), solver=fe.FLIP)
    with pytest.raises(fe.FluideError):
        other.restore(snap)
    snap.close()
    s.close()
    other.close()
