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
    for cls in ("Vector3D", "Vector3S", "Frame", "BoundingBox3D", "DirectionalField", "PICSimulator", "FLIPSimulator",
                "APICSimulator", "HybridSimulator"):
        assert hasattr(m, cls), cls
    for cls in ("PICSimulator", "FLIPSimulator", "APICSimulator"):
        for name in REFERENCE_SIMULATOR_METHODS + REFERENCE_HYBRID_METHODS:
            assert hasattr(getattr(m, cls), name), (cls, name)
    assert hasattr(m.FLIPSimulator, "SetBlendingFactor")
    # triangle_mesh_wrapper.cpp / obj_manager_wrapper.cpp
    assert hasattr(m.TriangleMesh, "Clear") and hasattr(m.OBJManager, "Save") and hasattr(m.OBJManager, "Load")


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
    with pytest.raises(RuntimeError):
        sim.AddCollider(None)


def build_cpp_api_binary():
    from fluide_engine_b200 import build

    build.build()
    out = os.path.join(PKG, "_build", "api_dam_break")
    src = os.path.join(ROOT, "tests", "cpp", "api_dam_break.cpp")
    cmd = ["/usr/bin/g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"), src, "-o", out, "-L", PKG,
           "-l:libfluide_b200.so", "-Wl,-rpath," + PKG]
    subprocess.run(cmd, check=True)
    return out


def test_cpp_api_compiles_and_links():
    assert os.path.exists(build_cpp_api_binary())


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
