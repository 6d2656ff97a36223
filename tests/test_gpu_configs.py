"""Full-substep parity with the FP64 oracle on the benchmark scenes themselves, at sizes the oracle runs in
seconds: the FLIP dam break at 64^3 (the 128^3 headline scene's parity size) and the APIC sphere drop into a pool
at 48^3 with the pressure refined to 1e-8 in FP64 (the 256^3 scene's settings).

Each comparison starts from an identical snapshot: the first substep from the seeded particles, and a later
substep after the oracle has been re-seeded with the GPU's particles and pressure (the warm start) -- whole
trajectories diverge chaotically, so per-substep errors are what is compared.  Tolerances (relative L2): particle
positions 1e-6, particle velocities 1e-4, grid velocities 1e-4, pressure 1e-3, APIC matrices 1e-4 of the larger of
their norm and the gradient scale |v| / h; cell marks bit-exact.  The GPU's FP64 relative residual must meet the scene's target.
"""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

fe = pytest.importorskip("fluide_engine_b200")

DAM = [dict(kind=0, lo=(0.0, 0.0, 0.0), hi=(0.4, 0.6, 1.0))]
POOL = [dict(kind=0, lo=(0.0, 0.0, 0.0), hi=(1.0, 0.3, 1.0)),
        dict(kind=1, lo=(0.5, 0.7, 0.5), hi=(0.15, 0.0, 0.0), vel=(0.0, -2.0, 0.0))]


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def compare_substep(g, o, dt, solver, rel_tol):
    st = g.step(dt, 1)
    o.substep(dt)
    assert st[0]["converged"] == 1 and st[0]["rel_residual"] <= rel_tol, st
    u, v, w, p, m = g.grid()
    assert np.array_equal(m, o.marks())
    P, V, C = g.particles()
    Po, Vo, Co = o.particles()
    # the three face arrays as one vector: from rest, u and w hold only rounding noise, so their own relative
    # norms say nothing
    ug = np.concatenate([np.ravel(a) for a in (u, v, w)])
    uo = np.concatenate([np.ravel(a) for a in o.grid()])
    err = dict(P=rel_l2(P, Po), V=rel_l2(V, Vo), p=rel_l2(p, o.pressure()), grid=rel_l2(ug, uo))
    if solver == fe.APIC:
        # C is a velocity gradient: where the flow is uniform (a falling sphere, a pool at rest) the oracle's C is
        # FP64 rounding noise, so its error is taken relative to the larger of |C| and the gradient scale |v| / h
        scale = max(np.linalg.norm(Co), np.linalg.norm(Vo) * max(g.n))
        err["C"] = float(np.linalg.norm(C.astype(np.float64) - Co) / scale)
    assert err["P"] < 1e-6, err
    assert err["V"] < 1e-4, err
    assert err["grid"] < 1e-4, err
    assert err["p"] < 1e-3, err
    if solver == fe.APIC:
        assert err["C"] < 1e-4, err
    return err


def run_scene(n, solver, regions, seed, dt, rel_tol, later, pressure_solver=fe.AUTO):
    pos, vel = fe.seed_regions(regions, n, seed=seed)
    C = np.zeros((pos.shape[0], 9), np.float32)
    g = fe.Scene(n, solver=solver, max_cfl=1.0, cg_rel_tol=rel_tol, cg_max_it=4000, pressure_solver=pressure_solver)
    g.set_particles(pos, vel, C)
    o = oracle.OracleSim(n, solver, max_cfl=1.0, cg_rel_tol=min(rel_tol * 1e-3, 1e-10), cg_max_it=20000)
    o.set_particles(pos.astype(np.float64), vel.astype(np.float64), C.astype(np.float64))
    first = compare_substep(g, o, dt, solver, rel_tol)
    g.step(dt, later - 2)
    # re-seed the oracle with the GPU's state at substep `later - 1` (particles and the pressure warm start)
    P, V, Cg = g.particles()
    o.set_particles(P.astype(np.float64), V.astype(np.float64), Cg.astype(np.float64))
    o.set_pressure(g.grid()[3])
    again = compare_substep(g, o, dt, solver, rel_tol)
    g.close()
    return first, again


def test_flip_dam_break_64_tracks_oracle():
    """The 128^3 FLIP dam break's scene at 64^3 (503,367 particles, seed 0, FLIP 0.95, dt 1/240, rel 1e-6): the
    first substep and substep 30."""
    first, again = run_scene((64, 64, 64), fe.FLIP, DAM, 0, 1.0 / 240.0, 1e-6, 30)
    assert first["V"] < 1e-4 and again["V"] < 1e-4


@pytest.mark.parametrize("psolver", [fe.CG, fe.MGPCG])
def test_apic_pool_sphere_48_tracks_oracle(psolver):
    """The APIC sphere drop into a pool (pool y < 0.3, sphere r 0.15 at (0.5, 0.7, 0.5) moving at (0, -2, 0),
    seed 1, dt 1/480) at 48^3 with the pressure refined in FP64 to a relative residual of 1e-8: the first substep
    and substep 80 (the sphere has entered the pool), with the plain and the multigrid-preconditioned inner
    solver."""
    first, again = run_scene((48, 48, 48), fe.APIC, POOL, 1, 1.0 / 480.0, 1e-8, 80, pressure_solver=psolver)
    assert first["C"] < 1e-4 and again["C"] < 1e-4


def test_time_extrapolated_warm_start_reaches_the_oracle():
    """With the solve warm-started from 2 p(n-1) - p(n-2) (a tuning choice; the reference starts from p(n-1)) every
    solve still meets its residual target, and a substep from an identical snapshot matches the oracle, which keeps
    the reference's warm start, within the same tolerances."""
    n = (40, 40, 40)
    pos, vel = fe.seed_regions(DAM, n, seed=5)
    g = fe.Scene(n, solver=fe.FLIP, max_cfl=1.0, cg_rel_tol=1e-6)
    g.set_tuning(pressure_extrapolation=1)
    assert g.tuning()["pressure_extrapolation"] == 1
    g.set_particles(pos, vel)
    st = g.step(1.0 / 240.0, 12)
    assert all(x["converged"] == 1 and x["rel_residual"] <= 1e-6 for x in st), st
    P, V, _ = g.particles()
    o = oracle.OracleSim(n, fe.FLIP, max_cfl=1.0, cg_rel_tol=1e-10, cg_max_it=20000)
    o.set_particles(P.astype(np.float64), V.astype(np.float64))
    o.set_pressure(g.grid()[3])
    compare_substep(g, o, 1.0 / 240.0, fe.FLIP, 1e-6)
    g.close()
