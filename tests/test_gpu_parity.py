"""Parity of the CUDA path (through the C ABI) with the FP64 C oracle, stage by stage and per substep.

Bit-exact: cell keys, the stable particle sort, P2G face markers, FLUID/AIR marks.  Floating point
(FP32 state on the GPU vs the FP64 oracle on identical inputs): relative L2 <= 1e-5 for grid stages,
1e-4 for pressure and particle velocities (the stated substep tolerance).
"""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

fe = pytest.importorskip("fluide_engine_b200")


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def make_scene_pair(n, solver, seed=0, box=(0.0, 0.0, 0.0, 0.4, 0.6, 1.0), vel_scale=0.5, max_cfl=1.0,
                    origin=(0.0, 0.0, 0.0), cg_rel_tol=1e-6, oracle_tol=None, shuffle=True, pressure_solver=None):
    lo = tuple(origin[a] + box[a] for a in range(3))
    hi = tuple(origin[a] + box[3 + a] for a in range(3))
    pos, _ = fe.seed_regions([dict(kind=0, lo=lo, hi=hi)], n, origin, (1, 1, 1), seed)
    rng = np.random.default_rng(seed + 10)
    if shuffle:
        pos = pos[rng.permutation(pos.shape[0])]
    vel = (rng.standard_normal(pos.shape) * vel_scale).astype(np.float32)
    C = (rng.standard_normal((pos.shape[0], 9)) * 0.3).astype(np.float32)
    g = fe.Scene(n, solver=solver, origin=origin, max_cfl=max_cfl, cg_rel_tol=cg_rel_tol,
                 pressure_solver=fe.AUTO if pressure_solver is None else pressure_solver)
    g.set_particles(pos, vel, C)
    o = oracle.OracleSim(n, solver, origin=origin, max_cfl=max_cfl, cg_rel_tol=oracle_tol or cg_rel_tol,
                         cg_max_it=20000)
    o.set_particles(pos.astype(np.float64), vel.astype(np.float64), C.astype(np.float64))
    return g, o, pos, vel, C


@pytest.mark.parametrize("n", [(16, 16, 16), (20, 12, 9), (64, 64, 64)])
def test_sort_bit_exact(n):
    g, o, pos, vel, C = make_scene_pair(n, fe.FLIP, seed=3)
    g.run_stages(1 / 240, fe.STAGE_SORT, fe.STAGE_SORT)
    keys, perm = g.sort_result()
    k_ref, p_ref = oracle.sort_keys(pos, n, (0, 0, 0), (1, 1, 1))
    assert np.array_equal(keys, k_ref)
    assert np.array_equal(perm, p_ref)
    # the particles themselves are unchanged by the sort (returned in the order they were set)
    P, V, _ = g.particles()
    assert np.array_equal(P, pos) and np.array_equal(V, vel)


@pytest.mark.parametrize("pile", [(0, 40), (1500, 5), (5000, 2), (70000, 1)])
def test_sort_bit_exact_piled_cells(pile):
    """Cells holding hundreds to tens of thousands of particles (particles clamped onto a wall corner pile up
    at one point): runs below and above the long-run threshold, next to ordinary cells."""
    count, groups = pile
    n = (16, 16, 16)
    rng = np.random.default_rng(11 + count)
    base = rng.uniform(0.0, 1.0, (20000, 3)).astype(np.float32)
    corners = np.array([[0.0, 0.0, 0.0], [1.0, 1.0, 1.0], [0.5, 0.0, 0.25], [0.999, 0.03, 0.5],
                        [0.31, 0.77, 0.0]], dtype=np.float32)
    piles = [np.repeat(corners[k % len(corners)][None], count + 37 * k, axis=0) for k in range(groups)]
    pos = np.concatenate([base] + piles)
    pos = pos[rng.permutation(pos.shape[0])]  # piles interleaved with the rest in particle order
    g = fe.Scene(n, solver=fe.FLIP, max_cfl=1.0)
    g.set_particles(pos, np.zeros_like(pos))
    g.run_stages(1 / 240, fe.STAGE_SORT, fe.STAGE_SORT)
    keys, perm = g.sort_result()
    k_ref, p_ref = oracle.sort_keys(pos, n, (0, 0, 0), (1, 1, 1))
    assert np.array_equal(keys, k_ref)
    assert np.array_equal(perm, p_ref)
    g.close()


@pytest.mark.parametrize("solver", [fe.PIC, fe.FLIP, fe.APIC])
@pytest.mark.parametrize("n", [(16, 16, 16), (20, 12, 9)])
def test_p2g(solver, n):
    g, o, *_ = make_scene_pair(n, solver, seed=1)
    g.run_stages(1 / 240, fe.STAGE_SORT, fe.STAGE_P2G)
    o.stage("p2g")
    u, v, w, _, _ = g.grid()
    for a, b in zip((u, v, w), o.grid()):
        assert rel_l2(a, b) < 1e-5
    for a, b in zip(g.face_markers(), o.face_markers()):
        assert np.array_equal(a, b)
    if solver == fe.FLIP:
        for a, b in zip(g.snapshot(), (u, v, w)):
            assert np.array_equal(a, b)


@pytest.mark.parametrize("n", [(32, 32, 32), (24, 20, 16), (48, 48, 48), (12, 30, 10)])
def test_marks_bit_exact(n):
    g, o, *_ = make_scene_pair(n, fe.FLIP, seed=2, box=(0.05, 0.0, 0.1, 0.55, 0.63, 0.9))
    g.run_stages(1 / 240, fe.STAGE_SORT, fe.STAGE_MARK)
    o.stage("sdf")
    o.stage("markers")
    marks = g.grid()[4]
    assert np.array_equal(marks, o.marks())
    assert marks.sum() > 0


def test_fluid_sdf_bit_exact():
    n = (24, 20, 16)
    g, o, *_ = make_scene_pair(n, fe.FLIP, seed=4)
    o.stage("sdf")
    assert np.array_equal(g.fluid_sdf(), o.sdf())


@pytest.mark.parametrize("solver", [fe.PIC, fe.FLIP, fe.APIC])
@pytest.mark.parametrize("max_cfl", [1.0, 2.5])
def test_pre_stage(solver, max_cfl):
    n = (16, 16, 16)
    g, o, *_ = make_scene_pair(n, solver, seed=5, max_cfl=max_cfl)
    dt = 1 / 240
    g.run_stages(dt, fe.STAGE_SORT, fe.STAGE_PRE)
    for st in ("p2g", "sdf", "extrapolate", "bc"):
        o.stage(st)
    o.stage("forces", dt)
    u, v, w, _, _ = g.grid()
    for a, b in zip((u, v, w), o.grid()):
        assert rel_l2(a, b) < 1e-5


@pytest.mark.parametrize("solver", [fe.FLIP, fe.APIC])
@pytest.mark.parametrize("psolver", [fe.CG, fe.MGPCG])
def test_pressure_stage(solver, psolver):
    n = (32, 32, 32)
    g, o, *_ = make_scene_pair(n, solver, seed=6, cg_rel_tol=1e-8, oracle_tol=1e-12, pressure_solver=psolver)
    dt = 1 / 240
    g.run_stages(dt, fe.STAGE_SORT, fe.STAGE_PRE)
    u, v, w, _, _ = g.grid()
    for st in ("p2g", "sdf"):
        o.stage(st)
    o.set_grid(u.astype(np.float64), v.astype(np.float64), w.astype(np.float64))  # identical solver input
    g.run_stages(dt, fe.STAGE_PRESSURE, fe.STAGE_PRESSURE)
    o.stage("pressure", dt)
    ug, vg, wg, pg, mg = g.grid()
    assert np.array_equal(mg, o.marks())
    assert rel_l2(g.rhs(), o.rhs()) < 1e-12
    assert rel_l2(pg, o.pressure()) < 1e-4
    for a, b in zip((ug, vg, wg), o.grid()):
        assert rel_l2(a, b) < 1e-5


@pytest.mark.parametrize("psolver", [fe.CG, fe.MGPCG])
@pytest.mark.parametrize("solver", [fe.PIC, fe.FLIP, fe.APIC])
@pytest.mark.parametrize("n", [(32, 32, 32), (24, 20, 16)])
def test_full_substep(solver, n, psolver):
    g, o, *_ = make_scene_pair(n, solver, seed=7, cg_rel_tol=1e-6, oracle_tol=1e-10, pressure_solver=psolver)
    dt = 1 / 240
    stats = g.step(dt, 1)
    o.substep(dt)
    assert stats[0]["converged"] == 1 and stats[0]["rel_residual"] <= 1e-6
    P, V, C = g.particles()
    Po, Vo, Co = o.particles()
    assert rel_l2(P, Po) < 1e-6
    assert rel_l2(V, Vo) < 1e-4
    if solver == fe.APIC:
        assert rel_l2(C, Co) < 1e-4
    u, v, w, p, m = g.grid()
    assert np.array_equal(m, o.marks())
    for a, b in zip((u, v, w), o.grid()):
        assert rel_l2(a, b) < 1e-4
    assert rel_l2(p, o.pressure()) < 1e-3


def test_graph_and_stage_paths_agree():
    n = (24, 24, 24)
    g1, _, pos, vel, C = make_scene_pair(n, fe.FLIP, seed=8)
    g2 = fe.Scene(n, solver=fe.FLIP, max_cfl=1.0)
    g2.set_particles(pos, vel, C)
    dt = 1 / 240
    for _ in range(3):
        g1.step(dt, 1)
        g2.run_stages(dt, fe.STAGE_SORT, fe.STAGE_MOVE)
    P1, V1, _ = g1.particles()
    P2, V2, _ = g2.particles()
    assert rel_l2(P1, P2) < 1e-6 and rel_l2(V1, V2) < 1e-4


def test_projection_known_answer():
    # test/single_phase_pressuer_solver_test.cpp:61-133 through the C ABI: 4^3 all-FLUID, h = 1.
    n = (4, 4, 4)
    g = fe.Scene(n, solver=fe.FLIP, size=(4.0, 4.0, 4.0), cg_rel_tol=1e-10, max_cfl=1.0)
    pos, _ = fe.seed_regions([dict(kind=0, lo=(0, 0, 0), hi=(4, 4, 4))], n, (0, 0, 0), (4, 4, 4), 0)
    g.set_particles(pos)
    g.run_stages(1.0, fe.STAGE_SORT, fe.STAGE_MARK)
    assert (g.grid()[4] == fe.FLUID).all()
    u = np.zeros((4, 4, 5), np.float32); v = np.zeros((4, 5, 4), np.float32); w = np.zeros((5, 4, 4), np.float32)
    for j in range(4):
        v[:, j, :] = 0.0 if j in (0, 3) else 1.0
    g.set_grid(u, v, w)
    g.run_stages(1.0, fe.STAGE_PRESSURE, fe.STAGE_PRESSURE)
    ug, vg, wg, p, _ = g.grid()
    assert np.abs(ug[:3, :3, :4]).max() < 1e-6
    assert np.abs(vg[:3, :4, :3]).max() < 1e-6
    assert np.abs(wg[:4, :3, :3]).max() < 1e-6
    np.testing.assert_allclose(p[:3, 1:3, :3] - p[:3, 0:2, :3], -1.0, atol=1e-6)


def test_multi_substep_aggregates_track_oracle():
    n = (32, 32, 32)
    g, o, *_ = make_scene_pair(n, fe.FLIP, seed=9, vel_scale=0.0, shuffle=False, oracle_tol=1e-6)
    dt = 1 / 240
    g.step(dt, 20)
    for _ in range(20):
        o.substep(dt)
    P, V, _ = g.particles()
    Po, Vo, _ = o.particles()
    np.testing.assert_allclose(P.mean(axis=0), Po.mean(axis=0), atol=1e-4)
    ke, keo = (V.astype(np.float64) ** 2).sum(), (Vo ** 2).sum()
    assert abs(ke - keo) / keo < 1e-3


def test_adaptive_frame_matches_oracle():
    n = (16, 16, 16)
    g, o, *_ = make_scene_pair(n, fe.FLIP, seed=11, vel_scale=3.0, max_cfl=1.0, oracle_tol=1e-8,
                               cg_rel_tol=1e-8)
    assert abs(g.cfl(1 / 24) - o.cfl(1 / 24)) < 1e-12  # grid is zero before the first substep
    ns = g.advance_frame(1 / 24)
    no = o.advance_time(1 / 24)
    assert ns == no
    P, V, _ = g.particles()
    Po, Vo, _ = o.particles()
    assert rel_l2(P, Po) < 1e-4


def test_error_statuses():
    with pytest.raises(fe.FluideError) as e:
        fe.Scene((1, 8, 8))
    assert e.value.status == 2
    s = fe.Scene((8, 8, 8))
    with pytest.raises(fe.FluideError) as e:
        s.step(1 / 240, 1)
    assert e.value.status == 6  # FE_ERR_STATE: no particles yet
    s.set_particles(np.full((10, 3), 0.5, np.float32))
    with pytest.raises(fe.FluideError) as e:
        s.step(-1.0, 1)
    assert e.value.status == 2


@pytest.mark.parametrize("n", [(40, 24, 18), (33, 17, 50), (70, 9, 12)])
def test_multigrid_pressure_odd_grids(n):
    """The multigrid-preconditioned solve on grids whose axes halve unevenly (odd sizes, very flat levels)
    reaches the same FP64 residual target and the oracle's pressure."""
    g, o, *_ = make_scene_pair(n, fe.FLIP, seed=12, cg_rel_tol=1e-8, oracle_tol=1e-12, pressure_solver=fe.MGPCG,
                               box=(0.1, 0.0, 0.05, 0.8, 0.7, 0.9))
    dt = 1 / 240
    g.run_stages(dt, fe.STAGE_SORT, fe.STAGE_PRE)
    u, v, w, _, _ = g.grid()
    for st in ("p2g", "sdf"):
        o.stage(st)
    o.set_grid(u.astype(np.float64), v.astype(np.float64), w.astype(np.float64))
    g.run_stages(dt, fe.STAGE_PRESSURE, fe.STAGE_PRESSURE)
    o.stage("pressure", dt)
    ug, vg, wg, pg, mg = g.grid()
    assert np.array_equal(mg, o.marks())
    assert rel_l2(pg, o.pressure()) < 1e-4
    for a, b in zip((ug, vg, wg), o.grid()):
        assert rel_l2(a, b) < 1e-5


def test_multigrid_iterations_bounded():
    """The multigrid preconditioner keeps the inner iteration count small (the reason it exists): a 64^3 dam
    break needs under 40 inner iterations per substep where the plain CG needs over 200."""
    stats = {}
    for ps in (fe.CG, fe.MGPCG):
        g, _, *_ = make_scene_pair((64, 64, 64), fe.FLIP, seed=3, pressure_solver=ps)
        st = g.step(1 / 240, 3)
        assert all(x["converged"] == 1 and x["rel_residual"] <= 1e-6 for x in st)
        stats[ps] = max(x["cg_iterations"] for x in st)
        g.close()
    assert stats[fe.MGPCG] < 40 < 200 < stats[fe.CG], stats


@pytest.mark.parametrize("tuning", [dict(multigrid=0, cg_block_threads=1024, cg_cluster=1),
                                    dict(multigrid=0, cg_block_threads=512, cg_cluster=1),
                                    dict(multigrid=0, cg_block_threads=256, cg_cluster=1),
                                    dict(multigrid=0, cg_block_threads=1024, cg_cluster=2),
                                    dict(multigrid=0, cg_block_threads=512, cg_cluster=4),
                                    dict(multigrid=1, cg_block_threads=1024, mg_block_level_cells=4096, cg_cluster=1),
                                    dict(multigrid=1, cg_block_threads=512, mg_block_level_cells=2048, cg_cluster=1),
                                    dict(multigrid=1, cg_block_threads=1024, mg_block_level_cells=4096, cg_cluster=2)])
def test_tuning_choices_reach_the_oracle(tuning):
    """Every launch choice the autotuner can make (fe_scene_set_tuning) solves to the same FP64 residual and the
    oracle's pressure; only the speed differs."""
    n = (40, 40, 40)
    g, o, *_ = make_scene_pair(n, fe.FLIP, seed=13, cg_rel_tol=1e-8, oracle_tol=1e-12)
    g.set_tuning(**tuning)
    got = g.tuning()
    for k, val in tuning.items():
        assert got[k] == val, (k, got)
    dt = 1 / 240
    g.run_stages(dt, fe.STAGE_SORT, fe.STAGE_PRE)
    u, v, w, _, _ = g.grid()
    for st in ("p2g", "sdf"):
        o.stage(st)
    o.set_grid(u.astype(np.float64), v.astype(np.float64), w.astype(np.float64))
    g.run_stages(dt, fe.STAGE_PRESSURE, fe.STAGE_PRESSURE)
    o.stage("pressure", dt)
    ug, vg, wg, pg, mg = g.grid()
    assert np.array_equal(mg, o.marks())
    assert rel_l2(pg, o.pressure()) < 1e-4
    for a, b in zip((ug, vg, wg), o.grid()):
        assert rel_l2(a, b) < 1e-5
    # and whole substeps through the captured graphs
    st = g.step(dt, 3)
    assert all(x["converged"] == 1 and x["rel_residual"] <= 1e-8 for x in st), st
    g.close()


@pytest.mark.gpu
def test_launch_shape_changes_between_solves_keep_the_barrier_state():
    """The solvers' grid barrier counts arrivals over a whole launch and the last block to leave puts the count and
    the reduction totals back to zero; consecutive solves of one scene with different block counts, block sizes,
    clusters and solver families (each launch expects a different number of arrivals) must all start from a clean
    state: every solve converges to the FP64 tolerance, and the final pressure matches the oracle's stage solve."""
    n = (40, 40, 40)
    g, o, *_ = make_scene_pair(n, fe.FLIP, seed=21, cg_rel_tol=1e-8, oracle_tol=1e-12)
    dt = 1 / 240
    shapes = [dict(multigrid=0, cg_block_threads=1024, cg_cluster=1),
              dict(multigrid=0, cg_block_threads=256, cg_cluster=1),
              dict(multigrid=1, cg_block_threads=512, mg_block_level_cells=2048, cg_cluster=1),
              dict(multigrid=0, cg_block_threads=512, cg_cluster=2),
              dict(multigrid=1, cg_block_threads=1024, mg_block_level_cells=4096, cg_cluster=1),
              dict(multigrid=0, cg_block_threads=1024, cg_cluster=1)]
    for shape in shapes:
        g.set_tuning(**shape)
        st = g.step(dt, 2)
        assert all(x["converged"] == 1 and x["rel_residual"] <= 1e-8 for x in st), (shape, st)
    # one more pressure stage against the oracle from the GPU's state
    g.run_stages(dt, fe.STAGE_SORT, fe.STAGE_PRE)
    P, V, _ = g.particles()
    o.set_particles(P.astype(np.float64), V.astype(np.float64))
    u, v, w, _, _ = g.grid()
    for stg in ("p2g", "sdf"):
        o.stage(stg)
    o.set_grid(u.astype(np.float64), v.astype(np.float64), w.astype(np.float64))
    g.run_stages(dt, fe.STAGE_PRESSURE, fe.STAGE_PRESSURE)
    o.stage("pressure", dt)
    _, _, _, pg, mg = g.grid()
    assert np.array_equal(mg, o.marks())
    assert rel_l2(pg, o.pressure()) < 1e-4
    g.close()
