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
    # first substep: Fluid3::sdf is still its initial 0 everywhere, so every emitter node with sdf <= 0 emits
    np0 = g.num_particles()
    g.step(1 / 240, 1)
    np1 = g.num_particles()
    assert np1 - np0 == 8 * int((esdf <= 0).sum()) > 0
    P, Vel, _ = g.particles()
    new_p = P[np0:].astype(np.float64)
    # emitted inside the emitter's nodes (box [0.3, 0.7] x [0.6, 0.9] x [0.3, 0.7] plus one cell of node extent),
    # then advected by one substep (|v| dt well under a cell)
    lo, hi = np.array([0.3, 0.6, 0.3]) - 2 * h, np.array([0.7, 0.9, 0.7]) + 2 * h
    assert ((new_p >= lo) & (new_p <= hi)).all()
    assert Vel[np0:, 1].mean() > 1.0  # they start at (0, 6, 0)
    # second substep: emission where the fluid SDF of the previous substep is >= 0
    fluid = g.fluid_sdf()
    g.step(1 / 240, 1)
    assert g.num_particles() - np1 == 8 * int(((esdf <= 0) & (fluid >= 0)).sum())
    g.clear_emitters()
    np2 = g.num_particles()
    g.step(1 / 240, 1)
    assert g.num_particles() == np2
