"""Failure detection on the GPU without faulting it: every device-side wait is bounded and a wait that runs out
surfaces as a status with the context still usable; non-finite inputs end in a status, not a hang.

The bounded waits are made to run out through a test hook (fe_debug_set_barrier_limits): the pressure solvers'
grid barrier is told to expect one arrival more than the blocks launched, so no barrier can complete, and its
poll limit is cut to a few thousand polls.  Each waiting block then gives up, records FE_ERR_TIMEOUT and leaves
the kernel; the step returns that status, the host resets the barrier words, and after the limits are restored
the same scene steps normally.  Nothing here traps, asserts on the device or reads out of bounds.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

fe = pytest.importorskip("fluide_engine_b200")
from fluide_engine_b200 import _abi  # noqa: E402


def dam(n, solver=fe.FLIP, pressure_solver=fe.AUTO, seed=0):
    pos, vel = fe.seed_regions([dict(kind=0, lo=(0.0, 0.0, 0.0), hi=(0.4, 0.6, 1.0))], n, seed=seed)
    s = fe.Scene(n, solver=solver, max_cfl=1.0, cg_rel_tol=1e-6, pressure_solver=pressure_solver)
    s.set_particles(pos, vel)
    return s


@pytest.fixture
def restore_limits():
    yield
    _abi.set_barrier_limits(0, 0)


@pytest.mark.parametrize("psolver,cluster", [(fe.CG, 1), (fe.MGPCG, 1), (fe.CG, 2)])
def test_barrier_wait_runs_out_and_the_scene_recovers(psolver, cluster, restore_limits):
    n = (32, 32, 32)
    s = dam(n, pressure_solver=psolver)
    s.set_tuning(cg_cluster=cluster)
    st = s.step(1 / 240, 2)  # graphs captured, solver warm
    assert all(x["converged"] == 1 for x in st)
    _abi.set_barrier_limits(spin_limit=1 << 12, extra_arrivals=1)
    with pytest.raises(fe.FluideError) as e:
        s.step(1 / 240, 1)
    assert e.value.status == _abi.FE_ERR_TIMEOUT
    _abi.set_barrier_limits(0, 0)
    st = s.step(1 / 240, 3)  # same scene, same captured graphs: barrier words were reset by the host
    assert all(x["converged"] == 1 and x["rel_residual"] <= 1e-6 for x in st), st
    # a fresh scene on the same context is unaffected
    t = dam(n, pressure_solver=psolver, seed=1)
    st = t.step(1 / 240, 2)
    assert all(x["converged"] == 1 for x in st)
    s.close()
    t.close()


def test_non_finite_velocities_end_in_a_status(restore_limits):
    n = (24, 24, 24)
    pos, vel = fe.seed_regions([dict(kind=0, lo=(0.0, 0.0, 0.0), hi=(0.4, 0.6, 1.0))], n, seed=2)
    bad = vel.copy()
    bad[::97, 1] = np.nan
    s = fe.Scene(n, solver=fe.FLIP, max_cfl=1.0, cg_rel_tol=1e-6, cg_max_it=500)
    s.set_particles(pos, bad)
    st = s.step(1 / 240, 1)  # returns: the solve cannot converge on a NaN right-hand side
    assert st[0]["converged"] == 0
    # the scene is reusable after a reset (the NaN pressure warm start is cleared)
    s.reset()
    s.set_particles(pos, vel)
    st = s.step(1 / 240, 2)
    assert all(x["converged"] == 1 for x in st), st
    P, V, _ = s.particles()
    assert np.isfinite(P).all() and np.isfinite(V).all()
    s.close()
