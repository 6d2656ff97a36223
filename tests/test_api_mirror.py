"""The reference-facing APIs: the PyFluidEngine pybind11 module and the C++ header API.

CPU: the module imports, exposes the reference's class and method names, accepts the reference's
construction sequence and reports a missing device as a Python exception; the C++ API compiles and links.
GPU: frames advanced through PyFluidEngine and through the C++ API match the oracle.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "fluide_engine_b200")


def pyf():
    from fluide_engine_b200 import build

    build.build()
    if PKG not in sys.path:
        sys.path.insert(0, PKG)
    import PyFluidEngine

    return PyFluidEngine


# Names bound by the reference (python_wrapper/simulators_wrapper.cu:38-84, frame/vector3/bounding box/forces).
REFERENCE_SIMULATOR_METHODS = ["AdvanceSingleFrame", "InitializeFromTriangleMesh", "AddExternalForce", "AddCollider",
                               "AddEmitter", "SetCurrentFrame", "SetViscosity", "SetMaxClf", "GetSurface"]
REFERENCE_HYBRID_METHODS = ["MaxCfl", "GetViscosity", "GetParticlesPerBlock", "GetOrigin", "GetResolution",
                            "GetGridSpacing", "GetNumberOfParticles"]


def test_module_names_match_reference():
    m = pyf()
    for cls in ("Vector3D", "Vector3S", "Frame", "BoundingBox3D", "DirectionalField", "PointField", "SwirlField",
                "VolumeField", "PICSimulator", "FLIPSimulator", "APICSimulator", "HybridSimulator"):
        assert hasattr(m, cls), cls
    for cls in ("PICSimulator", "FLIPSimulator", "APICSimulator"):
        for name in REFERENCE_SIMULATOR_METHODS + REFERENCE_HYBRID_METHODS:
            assert hasattr(getattr(m, cls), name), (cls, name)
    assert hasattr(m.FLIPSimulator, "SetBlendingFactor")
    # triangle_mesh_wrapper.cpp / obj_manager_wrapper.cpp
    assert hasattr(m.TriangleMesh, "Clear") and hasattr(m.OBJManager, "Save") and hasattr(m.OBJManager, "Load")
    # emitters_wrapper.cpp / scalar_grid_3d_wrapper.cpp
    assert hasattr(m, "Emitter") and issubclass(m.VolumeEmitter, m.Emitter)
    for name in ("InitializeFromTriangleMesh", "InitializeFromSdf"):
        assert hasattr(m.VolumeEmitter, name)
    assert hasattr(m.ScalarGrid3D, "GetElement") and hasattr(m.ScalarGrid3D, "SetElement")


def test_reference_construction_sequence_without_device():
    m = pyf()
    domain = m.BoundingBox3D(m.Vector3D(0.0, 0.0, 0.0), m.Vector3D(1.0, 1.0, 1.0))
    sim = m.APICSimulator(m.Vector3S(16, 16, 16), domain)
    sim.AddExternalForce(m.DirectionalField(m.Vector3D(0.0, -9.81, 0.0)))
    sim.SetMaxClf(2.0)
    assert sim.MaxCfl() == 2.0
    assert sim.InitializeFromRegions([dict(kind=0, lo=(0, 0, 0), hi=(0.4, 0.6, 1.0))]) == 13 * 19 * 32
    g = sim.GetGridSpacing()
    assert (g.x, g.y, g.z) == (1 / 16, 1 / 16, 1 / 16)
    sim.SetViscosity(0.5)  # HybridSimulator::SetViscosity; the scene is created on the first step
    assert sim.GetViscosity() == 0.5
    with pytest.raises((ValueError, RuntimeError)):
        sim.SetViscosity(-0.5)
    with pytest.raises((ValueError, TypeError, RuntimeError)):
        sim.AddCollider(None)
    # emitters are kept until the first step registers them with the scene
    em = m.VolumeEmitter(m.TriangleMesh(), m.Vector3S(16, 16, 16), domain, 8, m.Vector3D(0.0, 6.0, 0.0), m.Vector3D(0.0))
    grid = m.ScalarGrid3D(m.Vector3S(16, 16, 16), 1.0, m.Vector3D(0.0), m.Vector3D(1.0 / 16))
    grid.SetElement(3, 4, 5, -2.0)
    assert grid.GetElement(3, 4, 5) == -2.0 and grid.GetElement(4, 4, 5) == 1.0
    em.InitializeFromSdf(grid)
    sim.AddEmitter(em)
    with pytest.raises(TypeError):
        sim.AddEmitter(grid)


def test_python_mirror_obj_load_and_emitter_without_device(tmp_path):
    import fluide_engine_b200 as m
    from meshes import box, write_obj

    V, T = box((0.1, 0.2, 0.3), (0.4, 0.5, 0.6))
    write_obj(tmp_path / "b.obj", V, T, name="emitter")
    mesh = m.TriangleMesh()
    m.OBJManager().Load(str(tmp_path / "b.obj"), mesh)
    assert mesh.GetObjectName() == "emitter"
    assert np.array_equal(mesh.vertices, V) and np.array_equal(mesh.triangles[:, :3], T[:, :3])
    m.OBJManager().Load(str(tmp_path / "missing.obj"), mesh)  # reported, mesh unchanged
    assert mesh.vertices.shape[0] == 8
    domain = m.BoundingBox3D(m.Vector3D(0.0), m.Vector3D(1.0))
    em = m.VolumeEmitter(mesh, m.Vector3S(8, 8, 8), domain, 4, m.Vector3D(0.0, 1.0, 0.0), m.Vector3D(0.0))
    grid = m.ScalarGrid3D(m.Vector3S(4, 4, 4), 1.0)
    with pytest.raises(ValueError):
        em.InitializeFromSdf(grid)  # smaller than the emitter's grid
    sim = m.FLIPSimulator(m.Vector3S(8, 8, 8), domain)
    sim.AddEmitter(em)
    with pytest.raises(TypeError):
        sim.AddEmitter(grid)


def build_cpp_api_binary(name="api_dam_break"):
    from fluide_engine_b200 import build

    build.build()
    out = os.path.join(PKG, "_build", name)
    src = os.path.join(ROOT, "tests", "cpp", name + ".cpp")
    cmd = ["/usr/bin/g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"), src, "-o", out, "-L", PKG,
           "-l:libfluide_b200.so", "-Wl,-rpath," + PKG]
    subprocess.run(cmd, check=True)
    return out


def test_cpp_api_compiles_and_links():
    assert os.path.exists(build_cpp_api_binary())
    assert os.path.exists(build_cpp_api_binary("api_emitter"))
    assert os.path.exists(build_cpp_api_binary("api_collider"))


def mesh_scene_expectations(Vf, Tf, Ve, Te, n, size, ppc=16):
    """Oracle values for InitializeFromTriangleMesh on an n-cell domain [0, size]^3: the particle count (ppc per
    seeded cell), the fluid mesh's SDF and the emitter mesh's SDF on the emitter grid."""
    import oracle

    h = [size / n[a] for a in range(3)]
    sdf = oracle.mesh_to_sdf(Vf, Tf, n, [h[a] / 2.0 for a in range(3)], h)
    o = oracle.OracleSim(n, oracle.FLIP, size=(size,) * 3)
    o.set_sdf(sdf)
    init = ppc * int(o.seed_cells().sum())
    esdf = oracle.mesh_to_sdf(Ve, Te, n, (0.0, 0.0, 0.0), h)
    return init, sdf, esdf


@pytest.mark.gpu
def test_cpp_api_emitter_scene(tmp_path):
    """The reference's main.cpp sequence (fluid mesh, VolumeEmitter, viscosity, SetMaxClf, frames) through the C++
    API: seeded and emitted counts equal the oracle's."""
    from meshes import box, write_obj

    Vf, Tf = box((0.2, 0.2, 0.2), (2.6, 2.0, 5.8))
    Ve, Te = box((1.9, 1.5, 1.9), (3.1, 2.5, 3.1))  # overlaps the fluid: nodes inside it do not emit
    write_obj(tmp_path / "emitter.obj", Ve, Te)
    write_obj(tmp_path / "fluid.obj", Vf, Tf)
    sdf_path = tmp_path / "fluid_sdf.bin"
    out = subprocess.run([build_cpp_api_binary("api_emitter"), str(tmp_path / "emitter.obj"), str(tmp_path / "fluid.obj"),
                          str(sdf_path)], capture_output=True, text=True, check=True).stdout
    fields = {k: int(v) for k, v in (kv.split("=") for kv in out.split())}
    init, _, esdf = mesh_scene_expectations(Vf, Tf, Ve, Te, (30, 30, 30), 6.0)
    fluid = np.fromfile(sdf_path, dtype=np.float64).reshape(30, 30, 30)  # after the first substep
    emit = 12 * int(((esdf <= 0) & (fluid >= 0)).sum())
    assert fields["sdf_kept"] == 1  # the mesh's fluid SDF survived SetMaxClf's scene rebuild
    assert fields["init"] == init > 0
    assert fields["none"] == init  # the first substep emits nothing: the collider SDF is still its initial 0
    assert 0 < emit < 12 * int((esdf <= 0).sum())  # the emitter overlaps the fluid: nodes inside it do not emit
    assert fields["first"] == init + emit
    assert fields["frames"] == 3 and fields["final"] >= fields["first"]
    assert fields["emit_only_first"] == 0  # no particles: one substep of the whole frame, emitting nothing
    assert fields["emit_only_frame"] == 12 * int((esdf <= 0).sum())
    assert fields["sdf_emitter"] == 5 * 3 * 2 * 4


@pytest.mark.gpu
@pytest.mark.parametrize("which", ["pybind", "python"])
def test_mesh_init_and_emitter_through_mirrors(tmp_path, which):
    from meshes import box, write_obj

    if which == "pybind":
        m = pyf()
    else:
        import fluide_engine_b200 as m
    Vf, Tf = box((0.05, 0.05, 0.05), (0.45, 0.5, 0.95))
    Ve, Te = box((0.35, 0.4, 0.35), (0.65, 0.7, 0.65))
    write_obj(tmp_path / "fluid.obj", Vf, Tf)
    write_obj(tmp_path / "emitter.obj", Ve, Te)
    fluid, emitter = m.TriangleMesh(), m.TriangleMesh()
    m.OBJManager().Load(str(tmp_path / "fluid.obj"), fluid)
    m.OBJManager().Load(str(tmp_path / "emitter.obj"), emitter)
    n = 16
    domain = m.BoundingBox3D(m.Vector3D(0.0, 0.0, 0.0), m.Vector3D(1.0, 1.0, 1.0))
    sim = m.FLIPSimulator(m.Vector3S(n, n, n), domain)
    sim.AddExternalForce(m.DirectionalField(m.Vector3D(0.0, -9.81, 0.0)))
    sim.InitializeFromTriangleMesh(fluid)
    init, mesh_sdf, esdf = mesh_scene_expectations(Vf, Tf, Ve, Te, (n, n, n), 1.0)
    assert sim.GetNumberOfParticles() == init > 0
    em = m.VolumeEmitter(emitter, m.Vector3S(n, n, n), domain, 12, m.Vector3D(0.0, 6.0, 0.0), m.Vector3D(0.0))
    sim.AddEmitter(em)
    sim.SetMaxClf(1.0)  # rebuilds the scene, keeping the particles and the mesh's fluid SDF
    assert np.array_equal(sim.GetFluidSdf(), mesh_sdf)
    sim.AdvanceFixedSubsteps(1.0 / 240.0, 1)
    assert sim.GetNumberOfParticles() == init  # the scene's first substep emits nothing
    fl = sim.GetFluidSdf()
    sim.AdvanceFixedSubsteps(1.0 / 240.0, 1)
    emit = 12 * int(((esdf <= 0) & (fl >= 0)).sum())
    assert 0 < emit < 12 * int((esdf <= 0).sum())
    assert sim.GetNumberOfParticles() == init + emit
    # an emitter changed after AddEmitter is re-registered at the next step: an all-positive SDF emits nothing
    em.InitializeFromSdf(m.ScalarGrid3D(m.Vector3S(n, n, n), 1.0, m.Vector3D(0.0), m.Vector3D(1.0 / n)))
    before = sim.GetNumberOfParticles()
    sim.AdvanceFixedSubsteps(1.0 / 240.0, 2)
    assert sim.GetNumberOfParticles() == before
    sim.SetCurrentFrame(m.Frame(1.0 / 60.0))
    sim.AdvanceSingleFrame()
    assert sim.GetNumberOfParticles() == before


@pytest.mark.gpu
def test_pyfluidengine_frames_match_oracle():
    import oracle

    m = pyf()
    sim = m.FLIPSimulator(m.Vector3S(16, 16, 16), m.BoundingBox3D(m.Vector3D(0.0, 0.0, 0.0), m.Vector3D(1.0, 1.0, 1.0)))
    sim.AddExternalForce(m.DirectionalField(m.Vector3D(0.0, -9.81, 0.0)))
    sim.SetMaxClf(1.0)
    sim.SetPressureSolverTolerance(1e-8, 4000)
    sim.InitializeFromRegions([dict(kind=0, lo=(0, 0, 0), hi=(0.4, 0.6, 1.0))])
    P0, V0, _ = sim.GetParticles()
    o = oracle.OracleSim((16, 16, 16), oracle.FLIP, max_cfl=1.0, cg_rel_tol=1e-10, cg_max_it=5000)
    o.set_particles(P0.astype(np.float64), V0.astype(np.float64))
    sim.SetCurrentFrame(m.Frame(1.0 / 60.0))
    for _ in range(2):
        sim.AdvanceSingleFrame()
        n_o = o.advance_time(1.0 / 60.0)
        assert sim.GetNumberOfSubTimeSteps() == n_o
    P, V, _ = sim.GetParticles()
    Po, Vo, _ = o.particles()
    assert np.linalg.norm(P - Po) / np.linalg.norm(Po) < 1e-4
    assert sim.GetCurrentFrame().GetIndex() == 2


@pytest.mark.gpu
def test_cpp_api_binary_runs(tmp_path):
    obj = tmp_path / "frame.obj"
    out = subprocess.run([build_cpp_api_binary(), str(obj)], capture_output=True, text=True, check=True).stdout
    fields = dict(kv.split("=") for kv in out.split())
    assert fields["frames"] == "3" and int(fields["particles"]) == 13 * 19 * 32
    assert int(fields["substeps"]) >= 3
    assert 0.0 < float(fields["mean_y"]) < 0.3  # the block's centre (0.3) falls under gravity
    nv, nt = int(fields["surface_v"]), int(fields["surface_t"])
    assert nv > 0 and nt > 0
    text = obj.read_text().splitlines()
    assert text[:2] == ["mtllib test.mtl", "o fluid"]
    assert sum(l.startswith("v ") for l in text) == nv and sum(l.startswith("f ") for l in text) == nt


@pytest.mark.gpu
def test_pyfluidengine_surface_obj_round_trip(tmp_path):
    """The SimulationRunner sequence through PyFluidEngine: AdvanceSingleFrame, GetSurface into a TriangleMesh,
    OBJManager.Save; OBJManager.Load reads the file back (to the file's 6 decimals)."""
    m = pyf()
    sim = m.APICSimulator(m.Vector3S(16, 16, 16), m.BoundingBox3D(m.Vector3D(0.0, 0.0, 0.0), m.Vector3D(1.0, 1.0, 1.0)))
    sim.AddExternalForce(m.DirectionalField(m.Vector3D(0.0, -9.81, 0.0)))
    sim.SetMaxClf(1.0)
    sim.SetViscosity(0.01)
    sim.InitializeFromRegions([dict(kind=0, lo=(0, 0, 0), hi=(0.4, 0.6, 1.0))])
    sim.SetCurrentFrame(m.Frame(1.0 / 60.0))
    sim.AdvanceSingleFrame()
    mesh = m.TriangleMesh()
    sim.GetSurface(mesh)
    mesh.SetObjectName("fluid")
    V, N, T = mesh.GetVertices(), mesh.GetNormals(), mesh.GetTriangles()
    assert V.shape[0] > 0 and T.shape[0] > 0 and N.shape == V.shape
    path = str(tmp_path / "f.obj")
    m.OBJManager().Save(path, mesh)
    back = m.TriangleMesh()
    m.OBJManager().Load(path, back)
    assert back.GetObjectName() == "fluid"
    np.testing.assert_allclose(back.GetVertices(), V, atol=5e-7)
    np.testing.assert_allclose(back.GetNormals(), N, atol=5e-7)
    assert np.array_equal(back.GetTriangles(), T)
    # GetSurface appends: a second call doubles the mesh, ids continuing after the first copy
    sim.GetSurface(mesh)
    T2 = mesh.GetTriangles()
    assert T2.shape[0] == 2 * T.shape[0] and np.array_equal(T2[T.shape[0]:], T + V.shape[0])


@pytest.mark.gpu
@pytest.mark.parametrize("which", ["pybind", "python"])
def test_simulation_runner_writes_frames(tmp_path, which):
    """SimulationRunner.RunSimulation (simulation_runner.cpp:16-56) as the reference's Python example and Blender
    add-on call it: one OBJ per frame under <cache>/simulated_frames, log.txt with the stats, GetStats."""
    if which == "pybind":
        m = pyf()
        V3, V3S, BB = m.Vector3D, m.Vector3S, m.BoundingBox3D
        sim = m.FLIPSimulator(V3S(16, 16, 16), BB(V3(0.0, 0.0, 0.0), V3(1.0, 1.0, 1.0)))
        sim.AddExternalForce(m.DirectionalField(V3(0.0, -9.81, 0.0)))
        runner = m.SimulationRunner()
    else:
        import fluide_engine_b200 as m

        sim = m.FLIPSimulator(m.Vector3S(16, 16, 16), m.BoundingBox3D(m.Vector3D(0.0), m.Vector3D(1.0)))
        sim.AddExternalForce(m.DirectionalField(m.Vector3D(0.0, -9.81, 0.0)))
        runner = m.SimulationRunner()
    sim.SetMaxClf(1.0)
    sim.InitializeFromRegions([dict(kind=0, lo=(0, 0, 0), hi=(0.4, 0.6, 1.0))])
    runner.RunSimulation(sim, 1.0 / 60.0, 3, "dam", str(tmp_path))
    frames = sorted((tmp_path / "simulated_frames").glob("dam_*.obj"))
    assert [f.name for f in frames] == ["dam_0.obj", "dam_1.obj", "dam_2.obj"]
    for f in frames:
        lines = f.read_text().splitlines()
        assert lines[0] == "mtllib test.mtl" and any(l.startswith("f ") for l in lines)
    log = (tmp_path / "log.txt").read_text()
    assert "Iteration: 2" in log and "SIMULATION STATS" in log
    st = runner.GetStats()
    assert st.numberOfIterations == 3 and len(st.iterationTimeInSeconds) == 3 and len(st.cflPerIteration) == 3
    assert st.numberOfParticles == 13 * 19 * 32 and st.gridSize.x == 16


@pytest.mark.gpu
@pytest.mark.parametrize("which", ["pybind", "python"])
def test_field_forces_through_mirrors_match_oracle(tmp_path, which):
    """AddExternalForce with DirectionalField, PointField, SwirlField and VolumeField (a mesh loaded by OBJManager)
    through PyFluidEngine and the Python mirror: frames match the oracle with the same forces."""
    import oracle
    from meshes import icosphere, write_obj

    V, T = icosphere((0.6, 0.5, 0.5), 0.2, 1)
    write_obj(tmp_path / "field.obj", V, T)
    if which == "pybind":
        m = pyf()
    else:
        import fluide_engine_b200 as m
    mesh = m.TriangleMesh()
    m.OBJManager().Load(str(tmp_path / "field.obj"), mesh)
    domain = m.BoundingBox3D(m.Vector3D(0.0, 0.0, 0.0), m.Vector3D(1.0, 1.0, 1.0))
    sim = m.FLIPSimulator(m.Vector3S(16, 16, 16), domain)
    sim.AddExternalForce(m.DirectionalField(m.Vector3D(0.0, -9.81, 0.0)))
    sim.AddExternalForce(m.SwirlField(m.Vector3D(0.5, 0.3, 0.5), m.Vector3D(0.0, 2.0, 0.0), 3.0, 1.0))
    sim.SetMaxClf(1.0)
    sim.InitializeFromRegions([dict(kind=0, lo=(0, 0, 0), hi=(0.4, 0.6, 1.0))])
    sim.AddExternalForce(m.VolumeField(mesh, m.Vector3S(8, 8, 8), domain, -4.0))  # after the scene exists
    sim.AddExternalForce(m.PointField(m.Vector3D(0.2, 0.8, 0.3), 2.0, 1.0))
    if which == "pybind":
        sim.SetPressureSolverTolerance(1e-8, 4000)
    else:
        sim.SetPressureSolverSettings(cg_rel_tol=1e-8, cg_max_it=4000)
    P0, V0, _ = sim.GetParticles()
    o = oracle.OracleSim((16, 16, 16), oracle.FLIP, max_cfl=1.0, cg_rel_tol=1e-10, cg_max_it=5000)
    o.add_swirl_field((0.5, 0.3, 0.5), (0.0, 2.0, 0.0), 3.0)
    o.add_volume_field(V, T, (8, 8, 8), (0.0, 0.0, 0.0), (1.0, 1.0, 1.0), -4.0)
    o.add_point_field((0.2, 0.8, 0.3), 2.0)
    o.set_particles(P0.astype(np.float64), V0.astype(np.float64))
    sim.SetCurrentFrame(m.Frame(1.0 / 60.0))
    for _ in range(2):
        sim.AdvanceSingleFrame()
        assert o.advance_time(1.0 / 60.0) >= 1
    P, Vel, _ = sim.GetParticles()
    Po, Vo, _ = o.particles()
    assert np.linalg.norm(P - Po) / np.linalg.norm(Po) < 1e-4
    assert np.linalg.norm(Vel - Vo) / np.linalg.norm(Vo) < 1e-3


def collider_scene_meshes(tmp_path):
    from meshes import box, with_face_normals, write_obj

    Vf, Tf = box((0.05, 0.05, 0.05), (0.45, 0.6, 0.95))
    Vc, Tc, Nc = with_face_normals(*box((0.5, 0.0, 0.3), (0.75, 0.4, 0.7)))
    write_obj(tmp_path / "fluid.obj", Vf, Tf)
    write_obj(tmp_path / "collider.obj", Vc, Tc, N=Nc)
    return (Vf, Tf), (Vc, Tc, Nc)


def oracle_frames_with_collider(pos, vel, coll, frames, max_cfl):
    import oracle

    o = oracle.OracleSim((16, 16, 16), oracle.PIC, max_cfl=max_cfl, cg_rel_tol=1e-10, cg_max_it=5000)
    o.add_mesh_collider(*coll, (16, 16, 16), (0.0, 0.0, 0.0), (1 / 16,) * 3)
    o.set_particles(pos.astype(np.float64), vel.astype(np.float64))
    subs = [o.advance_time(1 / 60) for _ in range(frames)]
    return o, subs


@pytest.mark.gpu
def test_cpp_api_collider_scene(tmp_path):
    """test/pic_simulator_test.cpp's collider sequence through the C++ API tracks the oracle over two frames."""
    _, coll = collider_scene_meshes(tmp_path)
    a, b = tmp_path / "init.bin", tmp_path / "final.bin"
    out = subprocess.run([build_cpp_api_binary("api_collider"), str(tmp_path / "fluid.obj"),
                          str(tmp_path / "collider.obj"), str(a), str(b)], capture_output=True, text=True,
                         check=True).stdout
    fields = {k: int(v) for k, v in (kv.split("=") for kv in out.split())}
    init = np.fromfile(a, dtype=np.float32).reshape(-1, 6)
    final = np.fromfile(b, dtype=np.float32).reshape(-1, 6)
    assert fields["particles"] == init.shape[0] == final.shape[0] > 0 and fields["inside"] == 1
    o, subs = oracle_frames_with_collider(init[:, :3], init[:, 3:], coll, 2, 2.0)
    assert fields["substeps"] == sum(subs)
    Po, Vo, _ = o.particles()
    assert np.linalg.norm(final[:, :3] - Po) / np.linalg.norm(Po) < 1e-4
    assert np.linalg.norm(final[1:, 3:] - Vo[1:]) / np.linalg.norm(Vo[1:]) < 1e-3


@pytest.mark.gpu
@pytest.mark.parametrize("which", ["pybind", "python"])
def test_colliders_through_mirrors_track_oracle(tmp_path, which):
    _, coll = collider_scene_meshes(tmp_path)
    if which == "pybind":
        m = pyf()
    else:
        import fluide_engine_b200 as m
    fluid, cmesh = m.TriangleMesh(), m.TriangleMesh()
    m.OBJManager().Load(str(tmp_path / "fluid.obj"), fluid)
    m.OBJManager().Load(str(tmp_path / "collider.obj"), cmesh)
    domain = m.BoundingBox3D(m.Vector3D(0.0, 0.0, 0.0), m.Vector3D(1.0, 1.0, 1.0))
    sim = m.PICSimulator(m.Vector3S(16, 16, 16), domain)
    sim.AddExternalForce(m.DirectionalField(m.Vector3D(0.0, -9.81, 0.0)))
    sim.InitializeFromTriangleMesh(fluid)
    col = m.TriangleMeshCollider(m.Vector3S(16, 16, 16), m.Vector3D(0.0, 0.0, 0.0), m.Vector3D(1 / 16, 1 / 16, 1 / 16),
                                 cmesh)
    assert col.IsInside(m.Vector3D(0.6, 0.2, 0.5)) and not col.IsInside(m.Vector3D(0.2, 0.2, 0.5))
    collection = m.ColliderCollection(m.Vector3S(16, 16, 16), m.Vector3D(1 / 16, 1 / 16, 1 / 16), m.Vector3D(0.0, 0.0, 0.0))
    collection.AddCollider(col)
    sim.SetColliders(collection)
    sim.SetMaxClf(2.0)
    if which == "pybind":
        sim.SetPressureSolverTolerance(1e-8, 4000)
    else:
        sim.SetPressureSolverSettings(cg_rel_tol=1e-8, cg_max_it=4000)
    P0, V0, _ = sim.GetParticles()
    o, subs = oracle_frames_with_collider(P0, V0, coll, 2, 2.0)
    sim.SetCurrentFrame(m.Frame(1.0 / 60.0))
    n = 0
    for _ in range(2):
        sim.AdvanceSingleFrame()
        n += sim.GetNumberOfSubTimeSteps()
    assert n == sum(subs)
    P, V, _ = sim.GetParticles()
    Po, Vo, _ = o.particles()
    assert np.linalg.norm(P - Po) / np.linalg.norm(Po) < 1e-4
    assert np.linalg.norm(V[1:] - Vo[1:]) / np.linalg.norm(Vo[1:]) < 1e-3
    with pytest.raises((ValueError, TypeError, RuntimeError, m.FluideError if hasattr(m, "FluideError") else RuntimeError)):
        sim.SetViscosity(0.1)  # colliders with viscosity are not on this path
