// pyfluidengine.cpp -- the PyFluidEngine pybind11 module over include/fluide_engine.hpp.
//
// Same module name, class names and method names as the reference's binding
// (python_wrapper/main.cpp:20-33, simulators_wrapper.cu:36-85, vector3_wrapper.cpp, frame_wrapper.cpp,
// bounding_box_3d_wrapper.cpp, exteranl_forces_wrapper.cpp, triangle_mesh_wrapper.cpp, obj_manager_wrapper.cpp,
// scalar_grid_3d_wrapper.cpp, emitters_wrapper.cpp) for the substep path, its surface output and scene
// initialisation, so
// `import PyFluidEngine as pyf` keeps working for a caller of the simulators.  The GIL is released while
// a frame or a batch of substeps runs.  Extensions for seeding and reading particles take and return
// numpy arrays.
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include "../../../include/fluide_engine.hpp"

namespace py = pybind11;

namespace {

using FArr = py::array_t<float, py::array::c_style | py::array::forcecast>;

std::vector<float> to_vec(const FArr& a) { return std::vector<float>(a.data(), a.data() + a.size()); }

py::array_t<float> to_arr(const std::vector<float>& v, size_t cols)
{
    py::array_t<float> out({(py::ssize_t)(v.size() / cols), (py::ssize_t)cols});
    std::copy(v.begin(), v.end(), out.mutable_data());
    return out;
}

}  // namespace

PYBIND11_MODULE(PyFluidEngine, m)
{
    m.doc() = "B200-native hybrid particle-grid substep (PIC / FLIP / APIC) behind the reference's Python API";

    py::register_exception<fluide::Error>(m, "FluideError", PyExc_RuntimeError);

    py::class_<Vector3<double>>(m, "Vector3D")
        .def(py::init<double>())
        .def(py::init<double, double, double>())
        .def_readwrite("x", &Vector3<double>::x)
        .def_readwrite("y", &Vector3<double>::y)
        .def_readwrite("z", &Vector3<double>::z);
    py::class_<Vector3<size_t>>(m, "Vector3S")
        .def(py::init<size_t>())
        .def(py::init<size_t, size_t, size_t>())
        .def_readwrite("x", &Vector3<size_t>::x)
        .def_readwrite("y", &Vector3<size_t>::y)
        .def_readwrite("z", &Vector3<size_t>::z);
    py::class_<Frame>(m, "Frame")
        .def(py::init<>())
        .def(py::init<double>())
        .def("Advance", &Frame::Advance)
        .def("GetIndex", &Frame::GetIndex)
        .def("GetTimeIntervalInSeconds", &Frame::GetTimeIntervalInSeconds)
        .def("GetTimeInSeconds", &Frame::GetTimeInSeconds);
    // TriangleMesh / OBJManager (triangle_mesh_wrapper.cpp, obj_manager_wrapper.cpp); the mesh's arrays are also
    // readable as numpy (vertices (V,3), normals (V,3), triangles (T,4): vertex ids, normal id).
    py::class_<TriangleMesh>(m, "TriangleMesh")
        .def(py::init<>())
        .def("Clear", &TriangleMesh::Clear)
        .def("GetObjectName", &TriangleMesh::GetObjectName)
        .def("SetObjectName", &TriangleMesh::SetObjectName)
        .def("GetVertices", [](const TriangleMesh& mesh) {
            const auto& V = mesh.GetVerticies();
            py::array_t<double> out({(py::ssize_t)V.size(), (py::ssize_t)3});
            for (size_t i = 0; i < V.size(); ++i) {
                out.mutable_at(i, 0) = V[i].x; out.mutable_at(i, 1) = V[i].y; out.mutable_at(i, 2) = V[i].z;
            }
            return out;
        })
        .def("GetNormals", [](const TriangleMesh& mesh) {
            const auto& N = mesh.GetNormals();
            py::array_t<double> out({(py::ssize_t)N.size(), (py::ssize_t)3});
            for (size_t i = 0; i < N.size(); ++i) {
                out.mutable_at(i, 0) = N[i].x; out.mutable_at(i, 1) = N[i].y; out.mutable_at(i, 2) = N[i].z;
            }
            return out;
        })
        .def("GetTriangles", [](const TriangleMesh& mesh) {
            const auto& T = mesh.GetTriangles();
            py::array_t<int64_t> out({(py::ssize_t)T.size(), (py::ssize_t)4});
            for (size_t i = 0; i < T.size(); ++i) {
                out.mutable_at(i, 0) = (int64_t)T[i].point1Idx; out.mutable_at(i, 1) = (int64_t)T[i].point2Idx;
                out.mutable_at(i, 2) = (int64_t)T[i].point3Idx; out.mutable_at(i, 3) = (int64_t)T[i].normalIdx;
            }
            return out;
        });
    py::class_<OBJManager>(m, "OBJManager")
        .def(py::init<>())
        .def("Save", &OBJManager::Save)
        .def("Load", &OBJManager::Load);
    py::class_<BoundingBox3D>(m, "BoundingBox3D")
        .def(py::init<Vector3<double>, Vector3<double>>())
        .def("GetOrigin", &BoundingBox3D::GetOrigin)
        .def("GetSize", &BoundingBox3D::GetSize);
    py::class_<ExternalForce, std::shared_ptr<ExternalForce>>(m, "ExternalForce");
    py::class_<DirectionalField, std::shared_ptr<DirectionalField>, ExternalForce>(m, "DirectionalField")
        .def(py::init<Vector3<double>>())
        .def("Sample", &DirectionalField::Sample)
        .def("SetStrength", &DirectionalField::SetStrength);
    py::class_<PointField, std::shared_ptr<PointField>, ExternalForce>(m, "PointField")
        .def(py::init<Vector3<double>, double, double>())
        .def("Sample", &PointField::Sample)
        .def("GetStrength", &PointField::GetStrength)
        .def("SetStrength", &PointField::SetStrength);
    py::class_<SwirlField, std::shared_ptr<SwirlField>, ExternalForce>(m, "SwirlField")
        .def(py::init<Vector3<double>, Vector3<double>, double, double>())
        .def("Sample", &SwirlField::Sample)
        .def("GetStrength", &SwirlField::GetStrength)
        .def("SetStrength", &SwirlField::SetStrength);
    py::class_<VolumeField, std::shared_ptr<VolumeField>, ExternalForce>(m, "VolumeField")
        .def(py::init<const TriangleMesh&, Vector3<size_t>, BoundingBox3D, double>())
        .def("Sample", &VolumeField::Sample)
        .def("GetStrength", &VolumeField::GetStrength)
        .def("SetStrength", &VolumeField::SetStrength);

    py::class_<HybridSimulator, std::shared_ptr<HybridSimulator>>(m, "HybridSimulator")
        .def("MaxCfl", &HybridSimulator::MaxCfl)
        .def("GetViscosity", &HybridSimulator::GetViscosity)
        .def("GetParticlesPerBlock", &HybridSimulator::GetParticlesPerBlock)
        .def("GetOrigin", &HybridSimulator::GetOrigin)
        .def("GetResolution", &HybridSimulator::GetResolution)
        .def("GetGridSpacing", &HybridSimulator::GetGridSpacing)
        .def("GetNumberOfParticles", &HybridSimulator::GetNumberOfParticles)
        .def("GetCurrentFrame", &HybridSimulator::GetCurrentFrame)
        .def("GetCurrentTimeInSeconds", &HybridSimulator::GetCurrentTimeInSeconds)
        .def("GetNumberOfSubTimeSteps", &HybridSimulator::GetNumberOfSubTimeSteps)
        .def("Cfl", &HybridSimulator::Cfl)
        .def("SetDensity", &HybridSimulator::SetDensity)
        .def("GetDensity", &HybridSimulator::GetDensity)
        .def("SetParticlesPerBlock", &HybridSimulator::SetParticlesPerBlock)
        .def("SetPressureSolverTolerance", &HybridSimulator::SetPressureSolverTolerance)
        .def("SetPressureSolverKind", [](HybridSimulator& s, int kind) { s.SetPressureSolverKind((fe_pressure_solver)kind); })
        // extensions: deterministic seeding and numpy particle access
        .def("InitializeFromRegions",
             [](HybridSimulator& s, const py::list& regions, uint64_t seed) {
                 std::vector<fe_region_desc> r;
                 for (auto item : regions) {
                     py::dict d = item.cast<py::dict>();
                     fe_region_desc g{};
                     g.kind = d.contains("kind") ? d["kind"].cast<int>() : 0;
                     auto lo = d["lo"].cast<std::vector<double>>();
                     auto hi = d["hi"].cast<std::vector<double>>();
                     std::vector<double> vel = d.contains("vel") ? d["vel"].cast<std::vector<double>>()
                                                                 : std::vector<double>{0, 0, 0};
                     for (int a = 0; a < 3; ++a) {
                         g.lo[a] = lo[a];
                         g.hi[a] = a < (int)hi.size() ? hi[a] : 0.0;
                         g.vel[a] = vel[a];
                     }
                     r.push_back(g);
                 }
                 return s.InitializeFromRegions(r, seed);
             },
             py::arg("regions"), py::arg("seed") = 0)
        .def("SetParticles",
             [](HybridSimulator& s, FArr pos, py::object vel, py::object C) {
                 std::vector<float> v = vel.is_none() ? std::vector<float>() : to_vec(vel.cast<FArr>());
                 std::vector<float> c = C.is_none() ? std::vector<float>() : to_vec(C.cast<FArr>());
                 s.SetParticles(to_vec(pos), v, c);
             },
             py::arg("pos"), py::arg("vel") = py::none(), py::arg("C") = py::none())
        .def("GetParticles",
             [](HybridSimulator& s) {
                 std::vector<float> p, v, c;
                 s.GetParticles(p, v, &c);
                 if (c.size() != p.size() * 3) c.assign(p.size() * 3, 0.f);
                 return py::make_tuple(to_arr(p, 3), to_arr(v, 3), to_arr(c, 9));
             })
        .def("GetFluidSdf",
             [](HybridSimulator& s) {
                 const ScalarGrid3D g = s.GetFluidSdf();
                 const Vector3<size_t> n = g.GetSize();
                 py::array_t<double> out({(py::ssize_t)n.z, (py::ssize_t)n.y, (py::ssize_t)n.x});
                 std::copy(g.GetRawData().begin(), g.GetRawData().end(), out.mutable_data());
                 return out;
             })
        .def("AdvanceFixedSubsteps",
             [](HybridSimulator& s, double dt, int nsub) {
                 std::vector<fe_step_stats> st((size_t)std::max(nsub, 1));
                 {
                     py::gil_scoped_release rel;
                     s.AdvanceFixedSubsteps(dt, nsub, st.data());
                 }
                 py::list out;
                 for (int i = 0; i < nsub; ++i) {
                     py::dict d;
                     d["cg_iterations"] = st[i].cg_iterations;
                     d["refinements"] = st[i].refinements;
                     d["converged"] = st[i].converged;
                     d["fluid_cells"] = st[i].fluid_cells;
                     d["rel_residual"] = st[i].rel_residual;
                     d["b_norm"] = st[i].b_norm;
                     out.append(d);
                 }
                 return out;
             });

    // SimulationStats / SimulationRunner (simulator_runner_wrapper.cpp)
    py::class_<SimulationStats>(m, "SimulationStats")
        .def(py::init<>())
        .def("PrintStats", [](const SimulationStats& st) { st.PrintStats(); })
        .def("Clear", &SimulationStats::Clear)
        .def_readwrite("simulatorType", &SimulationStats::simulatorType)
        .def_readwrite("numberOfIterations", &SimulationStats::numberOfIterations)
        .def_readwrite("gridSize", &SimulationStats::gridSize)
        .def_readwrite("numberOfParticles", &SimulationStats::numberOfParticles)
        .def_readwrite("timeIntervalInSeconds", &SimulationStats::timeIntervalInSeconds)
        .def_readwrite("simulationTimeInSeconds", &SimulationStats::simulationTimeInSeconds)
        .def_readwrite("iterationTimeInSeconds", &SimulationStats::iterationTimeInSeconds)
        .def_readwrite("cflPerIteration", &SimulationStats::cflPerIteration);
    py::class_<ScalarGrid3D>(m, "ScalarGrid3D")
        .def(py::init<const Vector3<size_t>&, const double&, Vector3<double>, Vector3<double>>())
        .def("GetElement", [](const ScalarGrid3D& g, size_t i, size_t j, size_t k) { return g.GetElement(i, j, k); })
        .def("SetElement", &ScalarGrid3D::SetElement);
    // colliders_wrapper.cpp
    py::class_<Collider, std::shared_ptr<Collider>>(m, "Collider")
        .def("IsInside", &Collider::IsInside)
        .def("GetClosestDistanceAt", &Collider::GetClosestDistanceAt);
    py::class_<TriangleMeshCollider, std::shared_ptr<TriangleMeshCollider>, Collider>(m, "TriangleMeshCollider")
        .def(py::init<const Vector3<size_t>&, const Vector3<double>&, const Vector3<double>&, const TriangleMesh&>());
    py::class_<ColliderCollection, std::shared_ptr<ColliderCollection>>(m, "ColliderCollection")
        .def(py::init<const Vector3<size_t>&, const Vector3<double>&, const Vector3<double>&>())
        .def("AddCollider", &ColliderCollection::AddCollider)
        .def("IsInside", &ColliderCollection::IsInside);
    py::class_<Emitter, std::shared_ptr<Emitter>>(m, "Emitter");
    py::class_<VolumeEmitter, std::shared_ptr<VolumeEmitter>, Emitter>(m, "VolumeEmitter")
        .def(py::init<const TriangleMesh&, Vector3<size_t>, BoundingBox3D, const size_t&, const Vector3<double>&,
                      const Vector3<double>&>())
        .def("InitializeFromTriangleMesh", &VolumeEmitter::InitializeFromTriangleMesh)
        .def("InitializeFromSdf", &VolumeEmitter::InitializeFromSdf);
    py::class_<SimulationRunner>(m, "SimulationRunner")
        .def(py::init<>())
        .def("RunSimulation", &SimulationRunner::RunSimulation, py::call_guard<py::gil_scoped_release>())
        .def("GetStats", &SimulationRunner::GetStats);

    py::class_<PICSimulator, std::shared_ptr<PICSimulator>, HybridSimulator> pic(m, "PICSimulator");
    pic.def(py::init<Vector3<size_t>, BoundingBox3D>())
        .def("AdvanceSingleFrame", &PICSimulator::AdvanceSingleFrame, py::call_guard<py::gil_scoped_release>())
        .def("InitializeFromTriangleMesh", &PICSimulator::InitializeFromTriangleMesh)
        .def("AddExternalForce", [](PICSimulator& s, std::shared_ptr<ExternalForce> f) { s.AddExternalForce(f); })
        .def("AddCollider", &PICSimulator::AddCollider)
        .def("SetColliders", &PICSimulator::SetColliders)
        .def("AddEmitter", &PICSimulator::AddEmitter)
        .def("SetCurrentFrame", &PICSimulator::SetCurrentFrame)
        .def("SetViscosity", &PICSimulator::SetViscosity)
        .def("SetMaxClf", &PICSimulator::SetMaxClf)
        .def("GetSurface", &PICSimulator::GetSurface, py::call_guard<py::gil_scoped_release>());
    py::class_<APICSimulator, std::shared_ptr<APICSimulator>, PICSimulator>(m, "APICSimulator")
        .def(py::init<Vector3<size_t>, BoundingBox3D>());
    py::class_<FLIPSimulator, std::shared_ptr<FLIPSimulator>, PICSimulator>(m, "FLIPSimulator")
        .def(py::init<Vector3<size_t>, BoundingBox3D>())
        .def("SetBlendingFactor", &FLIPSimulator::SetBlendingFactor)
        .def("GetBlendingFactor", &FLIPSimulator::GetBlendingFactor);
}
