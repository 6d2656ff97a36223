"""Scene initialisation from meshes on the GPU (Mesh2SDF, InitializeFromTriangleMesh, VolumeEmitter) against the
oracle, which is pinned to the reference (tests/test_oracle_vs_reference.py).

Exact: the mesh SDF (distances and signs), the seeded cells and counts (16 particles per cell inside the mesh),
the emitted counts per substep.  The positions inside a cell come from this library's counter-based generator
(the reference's std::rand() in a parallel loop is not reproducible): checked to lie in their cell.
"""
import numpy as np
import pytest

import oracle
from meshes import box, icosphere

pytestmark = pytest.mark.gpu

fe = pytest.importorskip("fluide_engine_b200")

MESHES = [("box", box((0.1, 0.05, 0.2), (0.55, 0.6, 0.8)), (16, 16, 16), (0.0, 0.0, 0.0)),
          ("sphere", icosphere((0.5, 0.45, 0.5), 0.3, 2), (20, 18, 16), (0.0, 0.0, 0.0)),
          ("sphere_offset", icosphere((0.2, 1.4, 0.3), 0.25, 1), (12, 12, 12), (-0.2, 1.0, -0.1))]


@pytest.mark.parametrize("case", range(3))
def test_mesh_to_sdf_bit_exact(case):
    _, (V, T), n, origin = MESHES[case]
    h = [1.0 / n[a] for a in range(3)]
    for org, hh in (([origin[a] + h[a] / 2.0 for a in range(3)], h), (origin, [0.05, 0.055, 0.0625])):
        g = fe.mesh_to_sdf(V, T, n, org, hh)
        o = oracle.mesh_to_sdf(V, T, n, org, hh)
        assert np.array_equal(g, o)


@pytest.mark.parametrize("case", range(3))
@pytest.mark.parametrize("solver", [fe.FLIP, fe.APIC])
def test_init_from_mesh(case, solver):
    _, (V, T), n, origin = MESHES[case]
    h = [1.0 / n[a] for a in range(3)]
    g = fe.Scene(n, solver=solver, origin=origin, max_cfl=1.0)
    g.init_from_mesh(V, T, seed=5)
    sdf = oracle.mesh_to_sdf(V, T, n, [origin[a] + h[a] / 2.0 for a in range(3)], h)
    assert np.array_equal(g.fluid_sdf(), sdf)  # Fluid3::sdf holds the mesh SDF until the next substep
    o = oracle.OracleSim(n, oracle.FLIP, origin=origin)
    o.set_sdf(sdf)
    mask = o.seed_cells()
    P, Vel, _ = g.particles()
    assert P.shape[0] == 16 * int(mask.sum()) > 0 and not Vel.any()
    rel = (P.astype(np.float64) - np.array(origin)) / np.array(h)
    cells = np.minimum(np.floor(rel).astype(int), np.array(n) - 1)
    occ = np.zeros_like(mask)
    np.add.at(occ, (cells[:, 2], cells[:, 1], cells[:, 0]), 1)
    assert np.array_equal(occ, mask * 16)
    # the surface before any substep is the mesh SDF's (PICSimulator::GetSurface of Fluid3::sdf)
    Vs, Ns, Ts = g.surface()
    Vo, No, To = oracle.build_surface(sdf, n, [origin[a] + h[a] / 2.0 for a in range(3)], h)
    assert np.array_equal(Vs, Vo) and np.array_equal(Ts, To)
    # a substep afterwards runs on the seeded particles and replaces the mesh SDF by the particles' own
    g.step(1 / 240, 1)
    assert g.num_particles() == P.shape[0]
    assert not np.array_equal(g.fluid_sdf(), sdf)
    # seeding again appends (ParticleSystem::AddParticles)
    g.init_from_mesh(V, T, particles_per_cell=2, seed=6)
    assert g.num_particles() == P.shape[0] + 2 * int(mask.sum())


def test_volume_emitter_counts_per_substep():
    n = (16, 16, 16)
    h = 1.0 / 16
    V, T = box((0.3, 0.6, 0.3), (0.7, 0.9, 0.7))
    g = fe.Scene(n, solver=fe.FLIP, max_cfl=1.0)
    pos, _ = fe.seed_regions([dict(kind=0, lo=(0, 0, 0), hi=(1.0, 0.2, 1.0))], n)
    g.set_particles(pos)
    eid = g.add_volume_emitter(V, T, n, (0, 0, 0), (1, 1, 1), particles_per_block=8, velocity=(0.0, 6.0, 0.0), seed=3)
    assert eid == 0
    esdf = oracle.mesh_to_sdf(V, T, n, (0, 0, 0), (h, h, h))
    # first substep: the collider SDF still holds its initial 0, which fails the emitter's > 0 test everywhere
    np0 = g.num_particles()
    g.step(1 / 240, 1)
    assert g.num_particles() == np0
    # second substep: every node inside the emitter where the first substep's fluid SDF is >= 0 emits
    fluid = g.fluid_sdf()
    g.step(1 / 240, 1)
    np1 = g.num_particles()
    assert np1 - np0 == 8 * int(((esdf <= 0) & (fluid >= 0)).sum()) > 0
    P, Vel, _ = g.particles()
    new_p = P[np0:].astype(np.float64)
    # emitted inside the emitter's nodes (box [0.3, 0.7] x [0.6, 0.9] x [0.3, 0.7] plus one cell of node extent),
    # then advected by one substep (|v| dt well under a cell)
    lo, hi = np.array([0.3, 0.6, 0.3]) - 2 * h, np.array([0.7, 0.9, 0.7]) + 2 * h
    assert ((new_p >= lo) & (new_p <= hi)).all()
    assert Vel[np0:, 1].mean() > 1.0  # they start at (0, 6, 0)
    # third substep: where the emitted particles now make the fluid SDF negative, nothing more is emitted
    fluid = g.fluid_sdf()
    g.step(1 / 240, 1)
    assert g.num_particles() - np1 == 8 * int(((esdf <= 0) & (fluid >= 0)).sum())
    g.clear_emitters()
    np2 = g.num_particles()
    g.step(1 / 240, 1)
    assert g.num_particles() == np2


def test_emitter_scene_without_particles():
    """A scene with an emitter and no particles steps (the reference's main.cpp scene): the first substep emits
    first; an emitter that never emits leaves every substep empty (skipped, reported as converged empty solves)."""
    n = (16, 16, 16)
    h = 1.0 / 16
    V, T = box((0.3, 0.6, 0.3), (0.7, 0.9, 0.7))
    esdf = oracle.mesh_to_sdf(V, T, n, (0, 0, 0), (h, h, h))
    g = fe.Scene(n, solver=fe.APIC, max_cfl=1.0)
    g.add_volume_emitter(V, T, n, (0, 0, 0), (1, 1, 1), particles_per_block=3, velocity=(0.0, -1.0, 0.0), seed=1)
    assert g.num_particles() == 0
    assert g.advance_frame(1 / 60) == 1  # CFL of no particles: one substep of the whole frame, emitting nothing
    assert g.num_particles() == 0
    assert g.advance_frame(1 / 60) == 1  # the collider SDF is built now: every node inside the emitter emits
    assert g.num_particles() == 3 * int((esdf <= 0).sum())
    P, Vel, _ = g.particles()
    assert np.isfinite(P).all() and (Vel[:, 1] < 0).mean() > 0.5
    # an emitter outside the grid's nodes never emits
    e = fe.Scene(n, solver=fe.FLIP, max_cfl=1.0)
    Vo, To = box((3.0, 3.0, 3.0), (3.5, 3.5, 3.5))
    e.add_volume_emitter(Vo, To, n, (0, 0, 0), (1, 1, 1), particles_per_block=4)
    stats = e.step(1 / 240, 3)
    assert e.num_particles() == 0
    assert [s["converged"] for s in stats] == [1, 1, 1] and all(s["fluid_cells"] == 0 for s in stats)
    assert e.advance_frame(1 / 60) == 1 and e.num_particles() == 0
    # without particles or emitters a scene still refuses to step
    with pytest.raises(fe.FluideError):
        fe.Scene(n, solver=fe.FLIP).step(1 / 240, 1)


def test_emitter_sdf_and_fluid_sdf_setters():
    n = (12, 10, 8)
    h = (1.0 / 12, 1.0 / 10, 1.0 / 8)
    V, T = box((0.2, 0.2, 0.2), (0.8, 0.8, 0.8))
    g = fe.Scene(n, solver=fe.FLIP, max_cfl=1.0)
    eid = g.add_volume_emitter(V, T, (6, 5, 4), (0, 0, 0), (0.5, 0.5, 0.5), particles_per_block=2)
    sdf = np.ones((4, 5, 6))
    sdf[1:3, 2, 1:5] = -1.0  # 2 * 1 * 4 nodes (VolumeEmitter::InitializeFromSdf)
    g.set_emitter_sdf(eid, sdf)
    g.step(1 / 240, 1)  # the first substep emits nothing (and, without particles, is skipped)
    assert g.num_particles() == 0
    # Fluid3::sdf set by the caller: negative (fluid) at one of those nodes, so it does not emit
    fluid = np.full((n[2], n[1], n[0]), 0.5)
    fluid[1, 2, 1] = -0.5
    g.set_fluid_sdf(fluid)
    assert np.array_equal(g.fluid_sdf(), fluid)
    g.step(1 / 240, 1)
    assert g.num_particles() == 2 * (8 - 1)
    P = g.particles()[0].astype(np.float64)
    assert (P >= 0).all() and (P[:, 0] < 5 * 0.5 / 6 + 0.05).all()
    with pytest.raises(fe.FluideError):
        g.set_emitter_sdf(eid + 1, sdf)


def test_advance_frame_emits_every_substep():
    """PhysicsAnimation::AdvanceTimeStep takes each substep's count from the particles before the emitter runs
    (physics_animation.cpp:76-86, pic_simulator.cpp:160-163); every substep of the frame emits."""
    n = (16, 16, 16)
    h = 1.0 / 16
    V, T = box((0.3, 0.6, 0.3), (0.7, 0.9, 0.7))
    esdf = oracle.mesh_to_sdf(V, T, n, (0, 0, 0), (h, h, h))
    g = fe.Scene(n, solver=fe.FLIP, max_cfl=1.0)
    pos, _ = fe.seed_regions([dict(kind=0, lo=(0, 0, 0), hi=(1.0, 0.2, 1.0))], n)
    g.set_particles(pos)
    g.add_volume_emitter(V, T, n, (0, 0, 0), (1, 1, 1), particles_per_block=2, velocity=(0.0, 3.0, 0.0))
    np0 = g.num_particles()
    assert g.advance_frame(1 / 60) == 1  # particles at rest: CFL 0, one substep, the scene's first: no emission
    assert g.num_particles() == np0
    fluid = g.fluid_sdf()
    nsub = g.advance_frame(1 / 60)  # its first substep emits where the previous substep's fluid SDF is >= 0
    assert nsub >= 1
    first = 2 * int(((esdf <= 0) & (fluid >= 0)).sum())
    assert first > 0 and g.num_particles() - np0 >= first
