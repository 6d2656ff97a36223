"""The oracle's restatement of the GPU's enclosed-component step (CPU only; not the reference).

With colliders, FLUID cells walled in by BOUNDRY cells and domain walls form a pure-Neumann block whose system the
reference leaves singular.  The GPU removes each such block's right-hand-side mean (and leaves all-zero rows out of
the solve); the oracle restates that behind OracleSim.set_enclosed_projection.  These tests pin the restatement:
on a consistent block it changes nothing beyond rounding (the reference's own result stands), and on an
inconsistent block it turns a diverging solve into a converged one.
"""
import os
import sys

import numpy as np

import oracle

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from meshes import box, with_face_normals  # noqa: E402

LID = with_face_normals(*box((-0.1, 0.25, -0.1), (1.1, 0.4, 1.1)))
REGIONS = [dict(kind=0, lo=(0, 0, 0), hi=(1, 0.22, 1)), dict(kind=0, lo=(0, 0.45, 0), hi=(0.4, 0.8, 1.0))]


def lid_oracle(n, projection, max_it=20000):
    pos, _ = oracle.seed_regions(REGIONS, n, (0, 0, 0), (1, 1, 1), 1)
    vel = np.random.default_rng(1).standard_normal(pos.shape) * 0.3
    o = oracle.OracleSim(n, oracle.FLIP, max_cfl=1.0, cg_rel_tol=1e-10, cg_max_it=max_it)
    o.set_enclosed_projection(projection)
    V, T, N = LID
    o.add_mesh_collider(V, T, N, n, (0, 0, 0), tuple(1.0 / x for x in n))
    o.set_particles(pos.astype(np.float64), vel)
    return o


def rel(a, b):
    return np.linalg.norm(np.ravel(a) - np.ravel(b)) / np.linalg.norm(np.ravel(b))


def enclosed_count(marks):
    """FLUID cells in 6-connected FLUID components with no AIR neighbour."""
    from scipy import ndimage

    fl = marks == 1
    lab, nl = ndimage.label(fl)
    touch = ndimage.binary_dilation(marks == 0, ndimage.generate_binary_structure(3, 1)) & fl
    open_labels = set(np.unique(lab[touch]).tolist()) - {0}
    return int(np.isin(lab, [l for l in range(1, nl + 1) if l not in open_labels]).sum())


def test_consistent_enclosed_block_is_unchanged():
    n = (24, 24, 24)
    a, b = lid_oracle(n, False), lid_oracle(n, True)
    for _ in range(2):
        a.substep(1 / 240)
        b.substep(1 / 240)
    assert np.array_equal(a.marks(), b.marks())
    assert enclosed_count(b.marks()) > 1000  # the block under the slab
    assert rel(b.particles()[1], a.particles()[1]) < 1e-8
    assert a.cg_rel_residual() < 1e-9 and b.cg_rel_residual() < 1e-9


def test_inconsistent_enclosed_block_becomes_solvable():
    n = (24, 24, 24)
    sims = [lid_oracle(n, False, max_it=1000), lid_oracle(n, True)]
    for o in sims:
        o.build_collider()
        o.stage("p2g")
        o.stage("sdf")
    rng = np.random.default_rng(5)
    noisy = [g + rng.standard_normal(g.shape) * 0.05 for g in sims[0].grid()]
    for o in sims:
        o.set_grid(*noisy)
        o.stage("pressure", 1 / 240)
    assert sims[0].cg_rel_residual() > 1e-4  # the reference's system: no solution in the enclosed block
    assert sims[1].cg_rel_residual() < 1e-9
    # the projected right-hand side differs only in the enclosed block, by a constant per block
    marks = sims[1].marks()
    d = sims[1].rhs() - sims[0].rhs()
    changed = d != 0
    assert changed.any() and (marks[changed] == 1).all()
    assert np.ptp(d[changed]) < 1e-9 * np.abs(d[changed]).max()
