"""CPU-side checks of the C ABI library: it loads, exports every entry point include/fluide_b200.h
declares, and rejects bad descriptors without touching a device."""
import ctypes
import os
import re

import numpy as np
import pytest

import fluide_engine_b200 as fe
from fluide_engine_b200 import _abi

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "fluide_b200.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(fe_[a-z_0-9]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    L = fe.lib()
    names = declared_functions()
    assert len(names) >= 20
    for name in names:
        assert hasattr(L, name), name
    assert sorted(names) == sorted(_abi.EXPORTS)


def test_abi_version_and_error_string():
    L = fe.lib()
    assert L.fe_abi_version() == 10600
    assert isinstance(L.fe_last_error(), bytes)


@pytest.mark.parametrize("field,value", [("n", (1, 8, 8)), ("size", (0.0, 1.0, 1.0)), ("solver", 7),
                                         ("max_cfl", 0.0), ("cg_rel_tol", -1.0)])
def test_create_rejects_bad_descriptor(field, value):
    L = fe.lib()
    d = _abi.SceneDesc()
    assert L.fe_scene_desc_default(ctypes.byref(d)) == 0
    if isinstance(value, tuple):
        for a in range(3):
            getattr(d, field)[a] = value[a]
    else:
        setattr(d, field, value)
    h = ctypes.c_void_p()
    assert L.fe_scene_create(ctypes.byref(d), ctypes.byref(h)) == _abi.FE_ERR_BAD_ARG
    assert not h.value


def test_null_arguments_are_rejected():
    L = fe.lib()
    assert L.fe_scene_destroy(None) == _abi.FE_ERR_BAD_ARG
    assert L.fe_scene_step(None, 0.01, 1, None) == _abi.FE_ERR_BAD_ARG
    assert L.fe_scene_create(None, None) == _abi.FE_ERR_BAD_ARG


def test_seed_regions_matches_oracle_seeding():
    import oracle

    regions = [dict(kind=0, lo=(0, 0, 0), hi=(1, 0.3, 1)), dict(kind=1, lo=(0.5, 0.7, 0.5), hi=(0.15,), vel=(0, -2, 0))]
    p1, v1 = fe.seed_regions(regions, (24, 24, 24))
    p2, v2 = oracle.seed_regions(regions, (24, 24, 24), (0, 0, 0), (1, 1, 1), 0)
    assert np.array_equal(p1, p2) and np.array_equal(v1, v2)
    d = np.linalg.norm(p1 - np.array([0.5, 0.7, 0.5]), axis=1)
    assert (v1[d < 0.11][:, 1] == -2).all() and (v1[d > 0.2][:, 1] == 0).all()
    assert (d < 0.11).sum() > 0


def test_python_mirror_api_without_device():
    sim = fe.FLIPSimulator(fe.Vector3S(16, 16, 16), fe.BoundingBox3D(fe.Vector3D(0.0), fe.Vector3D(1.0)))
    assert sim.GetBlendingFactor() == 0.05 and sim.MaxCfl() == 3.0
    sim.SetMaxClf(1.0)
    sim.AddExternalForce(fe.DirectionalField(fe.Vector3D(0.0, -9.81, 0.0)))
    n = sim.InitializeFromRegions([dict(kind=0, lo=(0, 0, 0), hi=(0.4, 0.6, 1.0))])
    assert sim.GetNumberOfParticles() == n == 13 * 19 * 32
    assert tuple(sim.GetGridSpacing()) == (1 / 16, 1 / 16, 1 / 16)
    with pytest.raises(TypeError):
        sim.AddCollider(object())  # a TriangleMeshCollider is expected
    sim.SetViscosity(0.1)  # kept until the scene exists (no device here)
    assert sim.GetViscosity() == 0.1
    with pytest.raises(ValueError):
        sim.SetViscosity(-1.0)


def test_write_obj_matches_oracle_writer(tmp_path):
    """fe_write_obj (host code, formatted by several threads) writes the same bytes as the oracle's serial restatement
    of OBJManager::Save, which is pinned to the reference; no device needed."""
    import numpy as np

    import oracle
    from fluide_engine_b200 import _abi

    rng = np.random.default_rng(3)
    nv, nt = 70001, 120003  # several formatting threads, uneven ranges
    V = rng.standard_normal((nv, 3)) * 10.0
    V[5] = [-0.0, 1e-7, -5e-7]  # signed zero and values that round to zero in "%f"
    N = rng.standard_normal((nv, 3))
    T = rng.integers(0, nv, (nt, 4)).astype(np.int64)
    T[0, 3] = -1  # the reference's size_t(-1) normal index prints as 0
    L = _abi.lib()
    _abi.check(L.fe_write_obj(str(tmp_path / "a.obj").encode(), b"fluid", _abi.ptr(V), _abi.ptr(N), nv, _abi.ptr(T), nt))
    oracle.write_obj(str(tmp_path / "b.obj"), "fluid", V, N, T)
    assert (tmp_path / "a.obj").read_bytes() == (tmp_path / "b.obj").read_bytes()
