"""Solid colliders on the GPU (TriangleMeshCollider: ColliderCollection::BuildSdf, ExtrapolateIntoCollider, BOUNDRY
cells, BlockedBoundryConditionSolver's collider branches, ResolveCollision in MoveParticles) against the oracle,
which equals the reference bit for bit (tests/test_oracle_vs_reference.py).

Exact: the collider SDF, the fluid SDF after ExtrapolateIntoCollider, the cell marks and the surface mesh.  Grid
stages and whole substeps are compared with the tolerances of the collider-free path (grid rel-L2 1e-5; particle
positions 1e-5 and velocities 1e-4 after several substeps).  The collision response moves particle c onto collider
c's surface and keeps or reflects its velocity by TriangleMesh::IsInside of the previous resolution's closest point,
which lies on the mesh: that test turns on the last bits of the point (the winding term of the triangle holding it
is +pi or -pi by the sign of a zero determinant), so from FP32 particle positions those few velocities can take the
other branch.  Their positions are compared; their velocities are left out of the velocity norm, and where the
response runs every substep (fluid seeded through the obstacle) the velocities they hand to the grid reach their
neighbours, so that scene's velocity tolerance is 1e-3.
"""
import numpy as np
import pytest

import oracle
from meshes import box, icosphere, with_face_normals

pytestmark = pytest.mark.gpu

fe = pytest.importorskip("fluide_engine_b200")

COLLIDERS = [with_face_normals(*box((0.45, 0.0, 0.3), (0.7, 0.35, 0.7))),
             with_face_normals(*icosphere((0.3, 0.25, 0.6), 0.15, 1))]


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def pair(n, solver, ncoll, scene="approach", seed=11, max_cfl=1.0):
    if scene == "approach":
        pos, _ = fe.seed_regions([dict(kind=0, lo=(0.0, 0.0, 0.0), hi=(0.4, 0.6, 1.0))], n, (0, 0, 0), (1, 1, 1), seed)
    else:  # seeded through the obstacle: particles end inside it and the collision response runs
        pos, _ = fe.seed_regions([dict(kind=0, lo=(0.35, 0.0, 0.2), hi=(0.65, 0.5, 0.8))], n, (0, 0, 0), (1, 1, 1), seed)
    rng = np.random.default_rng(seed)
    vel = (rng.standard_normal(pos.shape) * 0.4).astype(np.float32)
    if scene == "approach":
        vel[:, 0] += 1.5
    C = (rng.standard_normal((pos.shape[0], 9)) * 0.1).astype(np.float32)
    g = fe.Scene(n, solver=solver, max_cfl=max_cfl, cg_rel_tol=1e-8)
    o = oracle.OracleSim(n, solver, max_cfl=max_cfl, cg_rel_tol=1e-10, cg_max_it=20000)
    h = tuple(1.0 / n[a] for a in range(3))
    for V, T, N in COLLIDERS[:ncoll]:
        g.add_mesh_collider(V, T, N, n, (0.0, 0.0, 0.0), h)
        o.add_mesh_collider(V, T, N, n, (0.0, 0.0, 0.0), h)
    g.set_particles(pos, vel, C)
    o.set_particles(pos.astype(np.float64), vel.astype(np.float64), C.astype(np.float64))
    return g, o


@pytest.mark.parametrize("ncoll", [1, 2])
def test_collider_sdf_marks_and_fluid_sdf_exact(ncoll):
    n = (16, 16, 16)
    g, o = pair(n, fe.FLIP, ncoll, scene="overlap")
    assert not g.collider_sdf().any()  # the reference's collider SDF holds its initial 0 until the first substep
    o.build_collider()
    g.run_stages(1 / 120, fe.STAGE_SORT, fe.STAGE_MARK)
    assert np.array_equal(g.collider_sdf(), o.collider_sdf())
    o.stage("p2g")
    o.stage("sdf")  # BuildSignedDistanceField + ExtrapolateIntoCollider
    o.stage("markers")
    assert np.array_equal(g.fluid_sdf(), o.sdf())
    marks = g.grid()[4]
    assert np.array_equal(marks, o.marks())
    assert (marks == fe.FLUID).sum() > 0 and (marks == 2).sum() > 0  # FLUID and BOUNDRY cells


@pytest.mark.parametrize("solver", [fe.PIC, fe.FLIP, fe.APIC])
def test_pre_stage_with_colliders(solver):
    n = (16, 16, 16)
    g, o = pair(n, solver, 2)
    dt = 1 / 120
    o.build_collider()
    g.run_stages(dt, fe.STAGE_SORT, fe.STAGE_PRE)
    for st in ("p2g", "sdf", "extrapolate", "bc"):
        o.stage(st)
    o.stage("forces", dt)
    for a, b in zip(g.grid()[:3], o.grid()):
        assert rel_l2(a, b) < 1e-5


@pytest.mark.parametrize("solver", [fe.PIC, fe.FLIP, fe.APIC])
@pytest.mark.parametrize("ncoll", [1, 2])
@pytest.mark.parametrize("scene", ["approach", "overlap"])
def test_substeps_with_colliders_track_oracle(solver, ncoll, scene):
    n = (16, 16, 16)
    g, o = pair(n, solver, ncoll, scene=scene)
    dt = 1 / 120
    for _ in range(4):
        st = g.step(dt, 1)
        o.substep(dt)
        assert st[0]["converged"] == 1
        assert np.array_equal(g.grid()[4], o.marks())
    P, V, C = g.particles()
    Po, Vo, Co = o.particles()
    assert rel_l2(P, Po) < 1e-5
    assert rel_l2(V[ncoll:], Vo[ncoll:]) < (1e-4 if scene == "approach" else 1e-3)  # see the module docstring
    if solver == fe.APIC:
        assert rel_l2(C, Co) < 1e-4
    if scene == "overlap":  # particle 0 sits on the first collider's surface, as in the reference
        assert np.abs(P[0].astype(np.float64) - Po[0]).max() < 1e-5
        Vc, Tc, _ = COLLIDERS[0]
        lo, hi = Vc.min(axis=0), Vc.max(axis=0)
        on_face = np.isclose(Po[0], lo, atol=1e-12) | np.isclose(Po[0], hi, atol=1e-12)
        assert on_face.any()


def test_surface_with_colliders_exact():
    """MarchingCubesSolver::BuildSurface with the collider SDF: nodes inside fluid and collider take -collider."""
    n = (16, 16, 16)
    g, o = pair(n, fe.FLIP, 1, scene="overlap")
    g.step(1 / 120, 1)
    o.substep(1 / 120)
    sdf, csdf = o.sdf(), o.collider_sdf()
    assert np.array_equal(g.fluid_sdf(), sdf)
    mod = np.where((sdf < 0) & (csdf < 0), -csdf, sdf)
    h = 1.0 / 16
    Vs, Ns, Ts = g.surface()
    Vo, No, To = oracle.build_surface(mod, n, (h / 2, h / 2, h / 2), (h, h, h))
    assert np.array_equal(Vs, Vo) and np.array_equal(Ns, No) and np.array_equal(Ts, To)
    assert Ts.shape[0] > 0


def test_collider_scene_rules():
    n = (16, 16, 16)
    g, _ = pair(n, fe.FLIP, 1)
    with pytest.raises(fe.FluideError):
        g.set_viscosity(0.1)  # BackwardEulerDiffusionSolver's BOUNDRY faces are not on this path
    with pytest.raises(fe.FluideError):
        fe.Batch([g])
    V, T, N = COLLIDERS[0]
    bad = T.copy()
    bad[0, 3] = N.shape[0]  # normal id out of range
    with pytest.raises(fe.FluideError):
        g.add_mesh_collider(V, bad, N, n, (0, 0, 0), (1 / 16,) * 3)
    # emitter nodes inside the collider do not emit (colliderSdf(i, j, k) > 0 fails there)
    e = fe.Scene(n, solver=fe.FLIP, max_cfl=1.0)
    e.add_mesh_collider(V, T, N, n, (0.0, 0.0, 0.0), (1 / 16,) * 3)
    Ve, Te = box((0.4, 0.1, 0.35), (0.8, 0.3, 0.65))
    e.add_volume_emitter(Ve, Te, n, (0, 0, 0), (1, 1, 1), particles_per_block=2)
    e.step(1 / 240, 2)
    o = oracle.OracleSim(n, oracle.FLIP)
    o.add_mesh_collider(V, T, N, n, (0.0, 0.0, 0.0), (1 / 16,) * 3)
    o.build_collider()
    esdf = oracle.mesh_to_sdf(Ve, Te, n, (0, 0, 0), (1 / 16,) * 3)
    expect = 2 * int(((esdf <= 0) & (o.collider_sdf() > 0)).sum())
    assert 0 < expect < 2 * int((esdf <= 0).sum())
    assert e.num_particles() == expect
    e.clear_colliders()
    e.set_viscosity(0.1)


def test_collider_outside_the_domain_tracks_oracle():
    """A collider with no face inside the domain: its fixed face lists are empty (no boundary-condition passes run)
    and the substeps still track the oracle."""
    n = (16, 16, 16)
    V, T, N = with_face_normals(*box((1.3, 1.2, 1.25), (1.6, 1.7, 1.5)))
    pos, _ = fe.seed_regions([dict(kind=0, lo=(0.0, 0.0, 0.0), hi=(0.4, 0.6, 1.0))], n, (0, 0, 0), (1, 1, 1), 5)
    rng = np.random.default_rng(5)
    vel = (rng.standard_normal(pos.shape) * 0.3).astype(np.float32)
    C = np.zeros((pos.shape[0], 9), dtype=np.float32)
    g = fe.Scene(n, solver=fe.FLIP, max_cfl=1.0, cg_rel_tol=1e-8)
    o = oracle.OracleSim(n, fe.FLIP, max_cfl=1.0, cg_rel_tol=1e-10, cg_max_it=20000)
    h = (1.0 / 16,) * 3
    g.add_mesh_collider(V, T, N, n, (0.0, 0.0, 0.0), h)
    o.add_mesh_collider(V, T, N, n, (0.0, 0.0, 0.0), h)
    g.set_particles(pos, vel, C)
    o.set_particles(pos.astype(np.float64), vel.astype(np.float64), C.astype(np.float64))
    dt = 1 / 120
    for _ in range(3):
        st = g.step(dt, 1)
        o.substep(dt)
        assert st[0]["converged"] == 1
        assert np.array_equal(g.grid()[4], o.marks())
    assert (g.collider_sdf() > 0).all()  # nothing of the domain is inside the collider
    P, V1, _ = g.particles()
    Po, Vo, _ = o.particles()
    assert rel_l2(P, Po) < 1e-5
    assert rel_l2(V1, Vo) < 1e-4


# A collider slab wider than the domain with a full pool under it: the FLUID cells below the slab touch only
# BOUNDRY cells and walls, a component without AIR neighbours (a pure-Neumann block), next to fluid above it.
LID = with_face_normals(*box((-0.1, 0.25, -0.1), (1.1, 0.4, 1.1)))
LID_REGIONS = [dict(kind=0, lo=(0, 0, 0), hi=(1, 0.22, 1)), dict(kind=0, lo=(0, 0.45, 0), hi=(0.4, 0.8, 1.0))]


def enclosed_cells(marks):
    """FLUID cells of 6-connected FLUID components with no AIR neighbour."""
    from scipy import ndimage

    fl = marks == fe.FLUID
    lab, nl = ndimage.label(fl)
    touch = ndimage.binary_dilation(marks == 0, ndimage.generate_binary_structure(3, 1)) & fl
    open_labels = set(np.unique(lab[touch]).tolist()) - {0}
    return np.isin(lab, [l for l in range(1, nl + 1) if l not in open_labels])


def lid_inputs(n, seed=1):
    pos, _ = fe.seed_regions(LID_REGIONS, n, (0, 0, 0), (1, 1, 1), seed)
    rng = np.random.default_rng(seed)
    vel = (rng.standard_normal(pos.shape) * 0.3).astype(np.float32)
    C = (rng.standard_normal((pos.shape[0], 9)) * 0.1).astype(np.float32)
    return pos, vel, C


def lid_oracle(n, solver, projection=True, max_it=20000, seed=1):
    pos, vel, C = lid_inputs(n, seed)
    o = oracle.OracleSim(n, solver, max_cfl=1.0, cg_rel_tol=1e-10, cg_max_it=max_it)
    o.set_enclosed_projection(projection)
    V, T, N = LID
    o.add_mesh_collider(V, T, N, n, (0.0, 0.0, 0.0), tuple(1.0 / n[a] for a in range(3)))
    o.set_particles(pos.astype(np.float64), vel.astype(np.float64), C.astype(np.float64))
    return o


def lid_pair(n, solver, seed=1):
    pos, vel, C = lid_inputs(n, seed)
    g = fe.Scene(n, solver=solver, max_cfl=1.0, cg_rel_tol=1e-8)
    V, T, N = LID
    g.add_mesh_collider(V, T, N, n, (0.0, 0.0, 0.0), tuple(1.0 / n[a] for a in range(3)))
    g.set_particles(pos, vel, C)
    return g, lid_oracle(n, solver, seed=seed)


def test_enclosed_component_inconsistent_rhs_matches_oracle():
    """A velocity field with a net flux into the enclosed block makes its right-hand side inconsistent: the
    reference's system has no solution there (its CG stalls), the GPU removes the block's right-hand-side mean,
    and so does the oracle's restatement of that step; pressures and projected velocities agree."""
    n = (24, 24, 24)
    dt = 1 / 240
    g, o = lid_pair(n, fe.FLIP)
    ref = lid_oracle(n, fe.FLIP, projection=False, max_it=1500)
    g.run_stages(dt, fe.STAGE_SORT, fe.STAGE_PRE)
    u, v, w, _, _ = g.grid()
    rng = np.random.default_rng(5)
    noisy = [(a + rng.standard_normal(a.shape).astype(np.float32) * 0.05).astype(np.float32) for a in (u, v, w)]
    g.set_grid(*noisy)
    for sim in (o, ref):
        sim.build_collider()
        for st in ("p2g", "sdf"):
            sim.stage(st)
        sim.set_grid(*[a.astype(np.float64) for a in noisy])
    g.run_stages(dt, fe.STAGE_PRESSURE, fe.STAGE_PRESSURE)
    o.stage("pressure", dt)
    ref.stage("pressure", dt)
    ug, vg, wg, pg, mg = g.grid()
    assert np.array_equal(mg, o.marks())
    enc = enclosed_cells(mg)
    assert enc.sum() > 1000  # the block under the slab
    assert ref.cg_rel_residual() > 1e-4  # the reference's system is inconsistent there
    assert o.cg_rel_residual() < 1e-9
    assert rel_l2(g.rhs(), o.rhs()) < 1e-12
    assert abs(g.rhs()[enc].sum()) < 1e-9 * np.abs(g.rhs()[enc]).sum()
    # the enclosed block's pressure is defined up to a constant (a pure-Neumann block): the solvers may drift
    # apart along that constant by rounding, which changes no velocity, so it is removed before comparing
    po = o.pressure()
    pg = pg.copy()
    pg[enc] -= (pg[enc] - po[enc]).mean()
    assert rel_l2(pg, po) < 1e-4
    for a, b in zip((ug, vg, wg), o.grid()):
        assert rel_l2(a, b) < 1e-5


@pytest.mark.parametrize("solver", [fe.FLIP, fe.APIC])
def test_enclosed_component_substeps_track_oracle(solver):
    n = (24, 24, 24)
    g, o = lid_pair(n, solver)
    dt = 1 / 240
    for _ in range(4):
        st = g.step(dt, 1)
        o.substep(dt)
        assert st[0]["converged"] == 1 and st[0]["rel_residual"] <= 1e-8
        m = g.grid()[4]
        assert np.array_equal(m, o.marks())
        assert enclosed_cells(m).sum() > 1000
    P, V, C = g.particles()
    Po, Vo, Co = o.particles()
    assert rel_l2(P, Po) < 1e-5
    assert rel_l2(V, Vo) < 1e-4
    if solver == fe.APIC:
        assert rel_l2(C, Co) < 1e-4
