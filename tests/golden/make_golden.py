"""Generates the golden fixtures in this directory from the reference's own CPU simulator.

Run from the repository root with the reference built (python oracle/build_ref.py):

    python tests/golden/make_golden.py

It writes the fixtures that are missing (--force rewrites all of them).  Each fixture is one substep of a
small seeded scene (dam-break block, 8 particles per cell) run by
the serial build of the reference (PICSimulator / FLIPSimulator / APICSimulator::OnAdvanceTimeStep
behind oracle/ref_harness.cpp): the inputs (FP32 positions widened to FP64, velocities, APIC C,
warm-start pressure) and the outputs after P2G, after the particle SDF, and after the whole substep.
The fixtures travel with the repository, so the oracle restatement can be re-pinned on machines
that do not have the reference sources.
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
import oracle  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))

CASES = [
    # name, n, solver, region, seed, max_cfl, origin
    ("flip_12", (12, 12, 12), oracle.FLIP, (0.0, 0.0, 0.0, 0.4, 0.6, 1.0), 0, 1.0, (0.0, 0.0, 0.0)),
    ("pic_12x10x8", (12, 10, 8), oracle.PIC, (0.0, 0.0, 0.0, 0.5, 0.5, 0.7), 1, 2.0, (0.0, 0.0, 0.0)),
    ("apic_10", (10, 10, 10), oracle.APIC, (0.2, 0.0, 0.1, 0.7, 0.5, 0.9), 2, 1.0, (0.0, 0.0, 0.0)),
    ("flip_16_cfl3", (16, 16, 16), oracle.FLIP, (0.0, 0.0, 0.0, 0.4, 0.6, 1.0), 3, 3.0, (0.0, 0.0, 0.0)),
    # viscous scenes (BackwardEulerDiffusionSolver with the CPU Jacobi solver): c = nu dt / h^2 of 0.006 (the
    # Jacobi solve stops at its first checks), 0.6 (about 80 iterations) and 12.5 (the 1000-iteration cap)
    ("flip_12_visc", (12, 12, 12), oracle.FLIP, (0.0, 0.0, 0.0, 0.4, 0.6, 1.0), 4, 1.0, (0.0, 0.0, 0.0), 0.01),
    ("apic_12x10x9_visc", (12, 10, 9), oracle.APIC, (0.1, 0.0, 0.0, 0.6, 0.5, 0.8), 5, 1.0, (0.0, 0.0, 0.0), 1.0),
    ("pic_10_visc_cap", (10, 10, 10), oracle.PIC, (0.0, 0.0, 0.2, 0.5, 0.6, 0.9), 6, 2.0, (0.0, 0.0, 0.0), 30.0),
    # position-dependent forces after gravity (PointField, SwirlField, VolumeField of an icosphere)
    ("flip_12_forces", (12, 12, 12), oracle.FLIP, (0.0, 0.0, 0.0, 0.5, 0.6, 1.0), 7, 1.0, (0.0, 0.0, 0.0), 0.0,
     "forces"),
    # a TriangleMeshCollider through the seeded block (BOUNDRY cells, collider boundary conditions, the collision
    # response with the reference's shadowed particle index)
    ("apic_16_collider", (16, 16, 16), oracle.APIC, (0.35, 0.0, 0.2, 0.65, 0.5, 0.8), 8, 1.0, (0.0, 0.0, 0.0), 0.0,
     "collider"),
]


def extras_of(kind):
    """The forces or collider of a case, as the arrays stored in its fixture."""
    sys.path.insert(0, os.path.dirname(OUT))
    from meshes import box, icosphere, with_face_normals

    if kind == "forces":
        V, T = icosphere((0.6, 0.5, 0.5), 0.2, 1)
        return dict(force_kind=np.array([1, 2, 3]), force_origin=np.array([[0.3, 0.7, 0.4], [0.5, 0.4, 0.6], [0, 0, 0]]),
                    force_axis=np.array([[0, 1, 0], [0.2, 1.0, -0.3], [0, 1, 0]], dtype=np.float64),
                    force_strength=np.array([2.5, 4.0, -6.0]), fv_V=V, fv_T=T, fv_n=np.array([8, 8, 8]),
                    fv_o=np.zeros(3), fv_size=np.ones(3))
    if kind == "collider":
        V, T, N = with_face_normals(*box((0.45, 0.0, 0.3), (0.7, 0.35, 0.7)))
        return dict(coll_V=V, coll_T=T, coll_N=N)
    return {}


def apply_extras(sim, g, n):
    """Adds a fixture's forces and collider to a simulator (OracleSim or RefSim)."""
    if "force_kind" in g:
        for k, o, a, st in zip(g["force_kind"], g["force_origin"], g["force_axis"], g["force_strength"]):
            if k == 1:
                sim.add_point_field(tuple(o), float(st))
            elif k == 2:
                sim.add_swirl_field(tuple(o), tuple(a), float(st))
            else:
                sim.add_volume_field(g["fv_V"], g["fv_T"], tuple(int(x) for x in g["fv_n"]), tuple(g["fv_o"]),
                                     tuple(g["fv_size"]), float(st))
    if "coll_V" in g:
        sim.add_mesh_collider(g["coll_V"], g["coll_T"], g["coll_N"], n, (0.0, 0.0, 0.0), tuple(1.0 / x for x in n))


def scene(n, region, seed, origin):
    lo = tuple(origin[a] + region[a] for a in range(3))
    hi = tuple(origin[a] + region[3 + a] for a in range(3))
    pos, _ = oracle.seed_regions([dict(kind=0, lo=lo, hi=hi)], n, origin, (1, 1, 1), seed)
    rng = np.random.default_rng(100 + seed)
    vel = (rng.standard_normal(pos.shape) * 0.5).astype(np.float32)
    C = (rng.standard_normal((pos.shape[0], 9)) * 0.2).astype(np.float32)
    p0 = rng.standard_normal((n[2], n[1], n[0])) * 1e-3
    return pos.astype(np.float64), vel.astype(np.float64), C.astype(np.float64), p0


def make(name, n, solver, region, seed, max_cfl, origin, viscosity=0.0, extras=None, dt=1.0 / 240.0):
    pos, vel, C, p0 = scene(n, region, seed, origin)
    kw = dict(origin=origin, max_cfl=max_cfl, cg_rel_tol=1e-6, cg_max_it=500, viscosity=viscosity)
    ex = extras_of(extras)
    r = oracle.RefSim(n, solver, **kw)
    apply_extras(r, ex, n)
    r.set_particles(pos, vel, C)
    r.set_pressure(p0)
    r.stage("p2g")
    p2g = r.grid()
    r.stage("sdf")
    sdf = r.sdf()
    r = oracle.RefSim(n, solver, **kw)
    apply_extras(r, ex, n)
    r.set_particles(pos, vel, C)
    r.set_pressure(p0)
    r.substep(dt)
    u, v, w = r.grid()
    P, V, CC = r.particles()
    np.savez_compressed(
        os.path.join(OUT, name + ".npz"), n=np.array(n), solver=solver, max_cfl=max_cfl, dt=dt, viscosity=viscosity,
        origin=np.array(origin), pos=pos, vel=vel, C=C, p0=p0, p2g_u=p2g[0], p2g_v=p2g[1], p2g_w=p2g[2], sdf=sdf,
        out_u=u, out_v=v, out_w=w, out_p=r.pressure(), out_marks=r.marks(), out_pos=P, out_vel=V, out_C=CC, **ex)


SURFACE_CASES = [
    # name, n, region, seed, origin: the reference's GetSurface (marching cubes + caps) of the particle SDF
    ("surface_16", (16, 16, 16), (0.0, 0.0, 0.0, 0.4, 0.6, 1.0), 0, (0.0, 0.0, 0.0)),
    ("surface_12x20x9", (12, 20, 9), (0.1, 0.0, 0.2, 0.7, 0.5, 0.8), 1, (0.0, 0.0, 0.0)),
]


def make_surface(name, n, region, seed, origin):
    lo = tuple(origin[a] + region[a] for a in range(3))
    hi = tuple(origin[a] + region[3 + a] for a in range(3))
    pos, _ = oracle.seed_regions([dict(kind=0, lo=lo, hi=hi)], n, origin, (1, 1, 1), seed)
    r = oracle.RefSim(n, oracle.FLIP, origin=origin)
    r.set_particles(pos.astype(np.float64))
    r.stage("sdf")
    V, N, T = r.surface()
    np.savez_compressed(os.path.join(OUT, name + ".npz"), n=np.array(n), origin=np.array(origin), sdf=r.sdf(), V=V, N=N,
                        T=T)


if __name__ == "__main__":
    if not oracle.ref_available("serial"):
        sys.exit("build the reference first: python oracle/build_ref.py")
    force = "--force" in sys.argv
    for c in CASES:
        if not force and os.path.exists(os.path.join(OUT, c[0] + ".npz")):
            continue
        make(*c)
        print("wrote", c[0])
    for c in SURFACE_CASES:
        if not force and os.path.exists(os.path.join(OUT, c[0] + ".npz")):
            continue
        make_surface(*c)
        print("wrote", c[0])
