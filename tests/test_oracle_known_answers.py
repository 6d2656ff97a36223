"""Known-answer tests of the reference, restated against the C oracle (CPU only).

Each test carries the inputs and expected values of a reference gtest case; together they pin the
oracle's sampling, interpolation, BLAS-free projection and clamping arithmetic without needing the
reference sources.
"""
import numpy as np
import pytest

import oracle


def test_lerp_bilerp_trilerp():
    # test/math_utils_test.cpp:5-30
    L = oracle.lib()
    assert L.or_lerp(0.0, 2.0, 0.5) == 1.0
    c = np.array([0, 2, 0, 2, 0, 2, 0, 2], dtype=np.float64)
    assert L.or_trilerp(oracle.dptr(c), 0.5, 0.5, 0.5) == 1.0
    # LerpVector3_Test: (0,1,2)->(2,3,3) at 0.5 = (1,2,2.5)
    assert [L.or_lerp(a, b, 0.5) for a, b in zip((0, 1, 2), (2, 3, 3))] == [1, 2, 2.5]


def test_face_centered_sample():
    # test/face_centered_grid3d_test.cpp:65-81: 3^3 grid, spacing 0.5, origin 0.
    L = oracle.lib()
    n = 3
    u = np.ones((n, n, n + 1)); v = np.full((n, n + 1, n), 2.0); w = np.full((n + 1, n, n), 3.0)
    u[0, 0, 1] = 3  # x(1,0,0)
    v[0, 1, 0] = 4  # y(0,1,0)
    w[1, 0, 0] = 6  # z(0,0,1)
    h = np.array([0.5, 0.5, 0.5]); pos = np.array([0.25, 0.25, 0.25])
    res = []
    for arr, size, o in ((u, (n + 1, n, n), (0, 0.25, 0.25)), (v, (n, n + 1, n), (0.25, 0, 0.25)),
                         (w, (n, n, n + 1), (0.25, 0.25, 0))):
        res.append(L.or_sample_face_array(oracle.dptr(np.ascontiguousarray(arr)), oracle.iptr(np.array(size, dtype=np.int32)),
                                          oracle.dptr(np.array(o, dtype=np.float64)), oracle.dptr(h), oracle.dptr(pos)))
    assert res == [2.0, 3.0, 4.5]


def test_scalar_grid_sample():
    # test/scalar_grid3d_test.cpp:41-70
    L = oracle.lib()
    g = np.zeros((3, 3, 3))  # [k, j, i]
    for (i, j, k) in [(0, 1, 0), (1, 1, 0), (0, 1, 1), (1, 1, 1), (2, 1, 1), (1, 1, 2), (2, 1, 2), (0, 1, 2), (2, 1, 0)]:
        g[k, j, i] = 1
    for (i, j, k) in [(0, 2, 0), (1, 2, 0), (0, 2, 1), (1, 2, 1), (2, 2, 1), (1, 2, 2), (2, 2, 2), (0, 2, 2), (2, 2, 0)]:
        g[k, j, i] = 4
    size = oracle.iptr(np.array([3, 3, 3], dtype=np.int32))
    o = oracle.dptr(np.zeros(3)); h = oracle.dptr(np.ones(3))
    for y, want in [(0, 0), (0.5, 0.5), (0.75, 0.75), (1, 1), (1.25, 1.75), (1.5, 2.5), (2, 4)]:
        assert L.or_scalar_sample(oracle.dptr(g), size, o, h, oracle.dptr(np.array([1.0, y, 1.0]))) == want
    # Sample2_test (:72-86): origin 0.5, value 1 except (1,1,1)=4, sampled at grid nodes.
    g2 = np.ones((3, 3, 3)); g2[1, 1, 1] = 4
    o2 = np.full(3, 0.5)
    for (i, j, k), want in [((0, 0, 0), 1), ((1, 0, 0), 1), ((0, 1, 0), 1), ((1, 1, 0), 1), ((0, 0, 1), 1), ((1, 1, 1), 4)]:
        p = np.array([0.5 + i, 0.5 + j, 0.5 + k])
        assert L.or_scalar_sample(oracle.dptr(g2), size, oracle.dptr(o2), h, oracle.dptr(p)) == want


def test_single_phase_projection_known_answer():
    # test/single_phase_pressuer_solver_test.cpp:61-133: 4^3 all-FLUID grid, h = 1, v = 1 inside and 0 on
    # the j=0 and j=3 layers; after projection |u|,|v|,|w| < 1e-6 and p(j+1)-p(j) = -1.
    n = (4, 4, 4)
    u = np.zeros((4, 4, 5)); v = np.zeros((4, 5, 4)); w = np.zeros((5, 4, 4))
    for j in range(4):
        v[:, j, :] = 0.0 if j in (0, 3) else 1.0
    marks = np.ones((4, 4, 4), dtype=np.uint8)
    p = np.zeros((4, 4, 4))
    it, res = oracle.project(n, (1, 1, 1), marks, u, v, w, p, rel_tol=1e-12, max_it=1000)
    assert it > 0 and res < 1e-9
    assert np.abs(u[:3, :3, :4]).max() < 1e-6
    assert np.abs(v[:3, :4, :3]).max() < 1e-6
    assert np.abs(w[:4, :3, :3]).max() < 1e-6
    dp = p[:3, 1:3, :3] - p[:3, 0:2, :3]
    np.testing.assert_allclose(dp, -1.0, atol=1e-6)


def test_seed_counts():
    # Dam-break block [0,0.4]x[0,0.6]x[0,1] on 32^3: 26*38*64 subcells have their centre inside.
    pos, vel = oracle.seed_regions([dict(kind=0, lo=(0, 0, 0), hi=(0.4, 0.6, 1.0))], (32, 32, 32), (0, 0, 0), (1, 1, 1), 0)
    assert pos.shape == (26 * 38 * 64, 3) and pos.dtype == np.float32
    assert (pos >= 0).all() and (pos[:, 0] <= 0.4 + 1 / 64).all()
    pos2, _ = oracle.seed_regions([dict(kind=0, lo=(0, 0, 0), hi=(0.4, 0.6, 1.0))], (32, 32, 32), (0, 0, 0), (1, 1, 1), 0)
    assert np.array_equal(pos, pos2)


def test_sort_keys_is_stable_counting_sort():
    rng = np.random.default_rng(5)
    pos = rng.random((5000, 3)).astype(np.float32)
    pos[:100] = pos[0]  # a crowded cell
    keys, perm = oracle.sort_keys(pos, (20, 12, 9), (0, 0, 0), (1, 1, 1))
    assert (np.diff(keys.astype(np.int64)) >= 0).all()
    # stability: within a key, original indices increase
    same = keys[1:] == keys[:-1]
    assert (perm[1:][same] > perm[:-1][same]).all()
    assert np.array_equal(np.sort(perm), np.arange(5000))
