"""Position-dependent external forces on the GPU (PointField, SwirlField, VolumeField after gravity in
ComputeExternalForces, pic_simulator.cpp:203-212) against the oracle, which equals the reference bit for bit
(tests/test_oracle_vs_reference.py).

Exact: the VolumeField node vectors, and the force pass itself -- on the same FP32 grid the GPU's faces equal the
oracle's FP64 sums rounded to FP32.  Whole substeps with forces are compared with the substep tolerance
(positions rel-L2 1e-6, velocities 1e-4).
"""
import numpy as np
import pytest

import oracle
from meshes import box, icosphere

pytestmark = pytest.mark.gpu

fe = pytest.importorskip("fluide_engine_b200")


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


SPHERE = icosphere((0.55, 0.45, 0.5), 0.2, 1)
# no VolumeField node on a mesh surface: there the node vector is 0 and the reference's Sample divides 0 by 0
BOX = box((0.11, 0.61, 0.21), (0.41, 0.91, 0.53))

FORCES = {
    "point": [("point", ((0.3, 0.7, 0.4), 2.5))],
    "swirl": [("swirl", ((0.5, 0.4, 0.6), (0.2, 1.0, -0.3), 4.0))],
    "volume": [("volume", (SPHERE, (10, 9, 8), (0.0, 0.0, 0.0), (1.0, 1.0, 1.0), -6.0))],
    "all": [("swirl", ((0.6, 0.5, 0.5), (0.0, 1.0, 0.0), -3.0)), ("point", ((0.2, 0.3, 0.6), 1.5)),
            ("volume", (BOX, (8, 8, 8), (0.0, 0.0, 0.0), (1.0, 1.0, 1.0), 2.0))],
}


def add_forces(sim, forces):
    for kind, args in forces:
        if kind == "point":
            sim.add_point_field(*args)
        elif kind == "swirl":
            sim.add_swirl_field(*args)
        else:
            (V, T), n, o, size, strength = args
            sim.add_volume_field(V, T, n, o, size, strength)


def pair(n, solver, forces, seed=0, gravity=(0.0, -9.81, 0.0), origin=(0.0, 0.0, 0.0), max_cfl=1.0):
    pos, _ = fe.seed_regions([dict(kind=0, lo=(0.0, 0.0, 0.0), hi=(0.5, 0.6, 1.0))], n, origin, (1, 1, 1), seed)
    rng = np.random.default_rng(seed + 30)
    pos = pos[rng.permutation(pos.shape[0])]
    vel = (rng.standard_normal(pos.shape) * 0.4).astype(np.float32)
    C = (rng.standard_normal((pos.shape[0], 9)) * 0.2).astype(np.float32)
    g = fe.Scene(n, solver=solver, origin=origin, max_cfl=max_cfl, cg_rel_tol=1e-6, gravity=gravity,
                 pressure_solver=fe.CG)
    g.set_particles(pos, vel, C)
    add_forces(g, forces)
    o = oracle.OracleSim(n, solver, origin=origin, max_cfl=max_cfl, cg_rel_tol=1e-10, cg_max_it=20000,
                         gravity=gravity)
    o.set_particles(pos.astype(np.float64), vel.astype(np.float64), C.astype(np.float64))
    add_forces(o, forces)
    return g, o


@pytest.mark.parametrize("mesh", ["sphere", "box"])
def test_volume_field_vectors_bit_exact(mesh):
    V, T = SPHERE if mesh == "sphere" else BOX
    for n, o, h in (((10, 9, 8), (0.0, 0.0, 0.0), (0.1, 0.1111, 0.125)), ((7, 12, 5), (-0.3, 0.2, 0.1), (0.2, 0.09, 0.3))):
        assert np.array_equal(fe.volume_field_vectors(V, T, n, o, h), oracle.volume_field_vectors(V, T, n, o, h))


@pytest.mark.parametrize("which", list(FORCES))
def test_force_pass_bit_exact(which):
    """The force pass alone: with gravity 0 the pre-solve pass leaves the faces it extrapolated, and the forces add
    to exactly those values; the GPU's result equals the oracle's FP64 sum (same FP32 input) rounded to FP32."""
    n = (16, 14, 12)
    dt = 1 / 240
    g0, _ = pair(n, fe.FLIP, [], seed=2, gravity=(0.0, 0.0, 0.0))
    g1, o = pair(n, fe.FLIP, FORCES[which], seed=2, gravity=(0.0, 0.0, 0.0))
    g0.run_stages(dt, fe.STAGE_SORT, fe.STAGE_MARK)
    g1.run_stages(dt, fe.STAGE_SORT, fe.STAGE_MARK)
    g1.set_grid(*g0.grid()[:3])  # identical input (P2G's float atomics may order sums differently between runs)
    g0.run_stages(dt, fe.STAGE_PRE, fe.STAGE_PRE)
    g1.run_stages(dt, fe.STAGE_PRE, fe.STAGE_PRE)
    base = g0.grid()[:3]
    o.set_grid(*[a.astype(np.float64) for a in base])
    o.stage("forces", dt)
    got = g1.grid()[:3]
    for a, b, c in zip(got, o.grid(), base):
        assert np.array_equal(a, b.astype(np.float32))
        assert np.isfinite(a).all()
    assert any(not np.array_equal(a, c) for a, c in zip(got, base))


@pytest.mark.parametrize("solver", [fe.FLIP, fe.APIC])
@pytest.mark.parametrize("which", ["swirl", "all"])
def test_substeps_with_forces_track_oracle(solver, which):
    n = (24, 20, 16)
    g, o = pair(n, solver, FORCES[which], seed=4)
    dt = 1 / 240
    for _ in range(3):
        st = g.step(dt, 1)
        o.substep(dt)
        assert st[0]["converged"] == 1
    P, V, C = g.particles()
    Po, Vo, Co = o.particles()
    assert rel_l2(P, Po) < 1e-6
    assert rel_l2(V, Vo) < 1e-4
    if solver == fe.APIC:
        assert rel_l2(C, Co) < 1e-4


def test_forces_change_the_captured_substep():
    """Adding or clearing forces re-captures the substep graphs: a scene given its force after a step matches one
    that had it from the start only after that step, and clearing returns to the gravity-only trajectory."""
    n = (16, 16, 16)
    dt = 1 / 240
    f = FORCES["point"]
    a, _ = pair(n, fe.FLIP, f, seed=6)
    b, _ = pair(n, fe.FLIP, [], seed=6)
    c, _ = pair(n, fe.FLIP, [], seed=6)
    a.step(dt, 2)
    b.step(dt, 2)
    c.step(dt, 2)
    assert rel_l2(a.particles()[1], b.particles()[1]) > 1e-3  # the force acted
    add_forces(b, f)
    a.clear_forces()
    a.step(dt, 2)
    b.step(dt, 2)
    c.step(dt, 2)
    assert rel_l2(b.particles()[1], c.particles()[1]) > 1e-3
    with pytest.raises(fe.FluideError):
        for _ in range(9):
            add_forces(c, f)  # at most 8 per scene
