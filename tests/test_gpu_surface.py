"""Fluid surface on the GPU (GetSurface: marching cubes + face caps, OBJ output) against the oracle.

The mesh is compared exactly: the same vertices and normals (FP64) in the same order, the same triangles with the
reference's normal index, and byte-identical OBJ files.  The oracle's mesh and OBJ are themselves pinned to the
compiled reference (tests/test_oracle_vs_reference.py).
"""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

fe = pytest.importorskip("fluide_engine_b200")


def scene_pair(n, solver, seed, box, origin=(0.0, 0.0, 0.0)):
    lo = tuple(origin[a] + box[a] for a in range(3))
    hi = tuple(origin[a] + box[3 + a] for a in range(3))
    pos, _ = fe.seed_regions([dict(kind=0, lo=lo, hi=hi)], n, origin, (1, 1, 1), seed)
    rng = np.random.default_rng(seed + 30)
    pos = pos[rng.permutation(pos.shape[0])]
    vel = (rng.standard_normal(pos.shape) * 0.5).astype(np.float32)
    g = fe.Scene(n, solver=solver, origin=origin, max_cfl=1.0)
    g.set_particles(pos, vel)
    return g, pos, vel


def oracle_mesh(pos, n, origin):
    o = oracle.OracleSim(n, oracle.FLIP, origin=origin)
    o.set_particles(np.asarray(pos, dtype=np.float64))
    o.stage("sdf")
    h = [1.0 / n[a] for a in range(3)]
    return o.sdf(), oracle.build_surface(o.sdf(), n, [origin[a] + h[a] / 2.0 for a in range(3)], h)


CASES = [((16, 16, 16), (0.0, 0.0, 0.0, 0.4, 0.6, 1.0), (0.0, 0.0, 0.0)),
         ((24, 20, 16), (0.05, 0.0, 0.1, 0.55, 0.63, 0.9), (0.0, 0.0, 0.0)),
         ((10, 14, 12), (0.0, 0.0, 0.0, 0.4, 0.55, 0.9), (-0.5, 0.25, 1.0)),
         ((2, 5, 3), (0.0, 0.0, 0.0, 1.0, 0.5, 1.0), (0.0, 0.0, 0.0)),
         ((64, 64, 64), (0.0, 0.0, 0.0, 0.4, 0.6, 1.0), (0.0, 0.0, 0.0))]


@pytest.mark.parametrize("n, box, origin", CASES)
def test_surface_bit_exact(n, box, origin, tmp_path):
    g, pos, _ = scene_pair(n, fe.FLIP, 1, box, origin)
    sdf, (V, N, T) = oracle_mesh(pos, n, origin)
    assert np.array_equal(g.fluid_sdf(), sdf)
    Vg, Ng, Tg = g.surface()
    assert Vg.shape == V.shape and Tg.shape == T.shape and T.shape[0] > 0
    assert np.array_equal(Vg, V) and np.array_equal(Ng, N) and np.array_equal(Tg, T)
    g.write_surface_obj(tmp_path / "g.obj", "fluid")
    oracle.write_obj(str(tmp_path / "o.obj"), "fluid", V, N, T)
    assert (tmp_path / "g.obj").read_bytes() == (tmp_path / "o.obj").read_bytes()


@pytest.mark.parametrize("solver", [fe.PIC, fe.FLIP, fe.APIC])
def test_surface_after_substeps_uses_last_substep_sdf(solver):
    """Fluid3::sdf is built at the start of a substep, so after a step the surface is that of the particles as the
    last substep found them (here: the seeded positions), not of the advected ones."""
    n = (20, 16, 12)
    g, pos, vel = scene_pair(n, solver, 2, (0.0, 0.0, 0.0, 0.5, 0.5, 0.7))
    g.step(1 / 240, 1)
    _, (V, N, T) = oracle_mesh(pos, n, (0.0, 0.0, 0.0))
    Vg, Ng, Tg = g.surface()
    assert np.array_equal(Vg, V) and np.array_equal(Ng, N) and np.array_equal(Tg, T)
    # one more substep: the surface follows the particles of the start of that substep
    P1 = g.particles()[0]
    g.step(1 / 240, 1)
    _, (V1, N1, T1) = oracle_mesh(P1, n, (0.0, 0.0, 0.0))
    Vg, Ng, Tg = g.surface()
    assert np.array_equal(Vg, V1) and np.array_equal(Ng, N1) and np.array_equal(Tg, T1)


def test_surface_of_batched_scene_and_write_obj_api(tmp_path):
    n = (16, 16, 16)
    g, pos, _ = scene_pair(n, fe.FLIP, 3, (0.0, 0.0, 0.0, 0.4, 0.6, 1.0))
    b = fe.Batch([g])
    b.step(1 / 240, 1)
    b.close()
    _, (V, N, T) = oracle_mesh(pos, n, (0.0, 0.0, 0.0))
    Vg, Ng, Tg = g.surface()
    assert np.array_equal(Vg, V) and np.array_equal(Tg, T)
    # fe_write_obj on a caller's mesh equals the oracle's writer
    L = fe.lib()
    fe._abi.check(L.fe_write_obj(str(tmp_path / "w.obj").encode(), b"m", fe._abi.ptr(np.ascontiguousarray(V)),
                                 fe._abi.ptr(np.ascontiguousarray(N)), V.shape[0], fe._abi.ptr(np.ascontiguousarray(T)),
                                 T.shape[0]))
    oracle.write_obj(str(tmp_path / "o.obj"), "m", V, N, T)
    assert (tmp_path / "w.obj").read_bytes() == (tmp_path / "o.obj").read_bytes()
