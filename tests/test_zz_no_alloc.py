"""The allocation-free pressure projection (fe_project_noalloc) against the scene path's pressure stage.

fe_project_noalloc serves callers that cannot allocate device memory on the path where they project a
velocity field (a per-frame or real-time callback where cudaMalloc would stall the device, or memory
owned by another allocator).  They pass their own device buffers; the solver's scratch is a static
device array.  This test hands it device buffers holding exactly the input of a scene's pressure stage
and checks, on two calls in a row (the second one sees the first one's leftover scratch), that its
pressure and projected velocities match the scene path within the tolerance used by the other parity
tests, and that repeated calls leave the device's free memory unchanged.  It lives in its own file so
that it runs last.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

fe = pytest.importorskip("fluide_engine_b200")
torch = pytest.importorskip("torch")


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def test_noalloc_projection_matches_scene_pressure_stage():
    from fluide_engine_b200 import _abi

    n = (32, 32, 32)
    dt = 1.0 / 240.0
    pos, _ = fe.seed_regions([dict(kind=0, lo=(0.0, 0.0, 0.0), hi=(0.4, 0.6, 1.0))], n)
    vel = (np.random.default_rng(3).standard_normal(pos.shape) * 0.5).astype(np.float32)
    # fe_project_noalloc runs the plain CG solver: compare with the scene path configured the same way
    scene = fe.Scene(n, solver=fe.FLIP, max_cfl=1.0, cg_rel_tol=1e-6, cg_max_it=2000, pressure_solver=fe.CG)
    scene.set_particles(pos, vel)
    scene.run_stages(dt, fe.STAGE_SORT, fe.STAGE_PRE)
    u0, v0, w0, p0, marks = scene.grid()  # exactly what the pressure stage consumes
    scene.run_stages(dt, fe.STAGE_PRESSURE, fe.STAGE_PRESSURE)
    u1, v1, w1, p1, _ = scene.grid()
    scene.close()
    assert (marks == fe.FLUID).sum() > 1000

    L = fe.lib()
    n3 = (ctypes.c_int32 * 3)(*n)
    h3 = (ctypes.c_double * 3)(1.0 / n[0], 1.0 / n[1], 1.0 / n[2])
    host = [np.ascontiguousarray(a) for a in (marks, u0, v0, w0, p0)]
    dev = [torch.from_numpy(a).cuda() for a in host]
    src = [torch.from_numpy(a).cuda() for a in host]  # pristine inputs, copied in before every call
    torch.cuda.synchronize()
    free_after_first = None
    for call in range(6):
        for d, s0 in zip(dev, src):
            d.copy_(s0)  # device-to-device copy into the existing buffers: no allocation
        torch.cuda.synchronize()
        stats = _abi.StepStats()
        st = L.fe_project_noalloc(n3, h3, *[ctypes.c_void_p(t.data_ptr()) for t in dev], 1e-6, 2000, None,
                                  ctypes.byref(stats))
        assert st == 0, L.fe_last_error()
        assert stats.converged == 1 and stats.rel_residual <= 1e-6
        torch.cuda.synchronize()
        free_now = torch.cuda.mem_get_info()[0]
        if call == 0:
            free_after_first = free_now
        else:
            # the calls after the first allocate nothing on the device
            assert free_now == free_after_first, (call, free_after_first - free_now)
        if call < 2:
            _, du, dv, dw, dp = (t.cpu().numpy() for t in dev)
            assert rel_l2(dp, p1) < 1e-6, call
            for a, b in zip((du, dv, dw), (u1, v1, w1)):
                assert rel_l2(a, b) < 1e-6, call


def test_noalloc_rejects_grids_beyond_its_scratch():
    L = fe.lib()
    n3 = (ctypes.c_int32 * 3)(128, 128, 128)
    h3 = (ctypes.c_double * 3)(1.0, 1.0, 1.0)
    dummy = torch.zeros(16, device="cuda")
    ptr = ctypes.c_void_p(dummy.data_ptr())
    st = L.fe_project_noalloc(n3, h3, ptr, ptr, ptr, ptr, ptr, 1e-6, 100, None, None)
    assert st == 2  # FE_ERR_BAD_ARG
    assert b"at most" in L.fe_last_error()
