"""The autotuner on the GPU (fe_scene_autotune): it leaves the scene's state as it found it, applies a choice that
solves to the scene's residual target, and scenes created afterwards with the automatic solver choice start from
that choice."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

fe = pytest.importorskip("fluide_engine_b200")
from fluide_engine_b200 import autotune  # noqa: E402


def test_autotune_restores_state_and_seeds_new_scenes(tmp_path):
    n = (40, 40, 40)
    pos, _ = fe.seed_regions([dict(kind=0, lo=(0.0, 0.0, 0.0), hi=(0.4, 0.6, 1.0))], n, seed=4)
    vel = (np.random.default_rng(4).standard_normal(pos.shape) * 0.3).astype(np.float32)
    s = fe.Scene(n, solver=fe.FLIP, max_cfl=1.0, cg_rel_tol=1e-6)
    s.set_particles(pos, vel)
    s.step(1 / 240, 3)
    P0, V0, _ = s.particles()
    p0 = s.grid()[3]
    choice, ms = autotune.tune(s, 1 / 240, substeps=2, path=str(tmp_path / "t.json"))
    assert ms > 0 and choice["cg_block_threads"] in (256, 512, 1024)
    assert s.tuning() == choice
    P1, V1, _ = s.particles()
    assert np.array_equal(P0, P1) and np.array_equal(V0, V1)      # the state the search found
    assert np.array_equal(p0, s.grid()[3])
    st = s.step(1 / 240, 3)
    assert all(x["converged"] == 1 and x["rel_residual"] <= 1e-6 for x in st)
    # a scene created later with the automatic solver choice starts from the stored choice
    t = fe.Scene(n, solver=fe.FLIP, max_cfl=1.0)
    assert t.tuning() == choice
    # and a new process would: the file holds it
    assert autotune.read_file(str(tmp_path / "t.json"))[(n, fe.FLIP)] == choice
    s.close()
    t.close()
