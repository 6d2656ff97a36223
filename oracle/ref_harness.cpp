// ref_harness.cpp -- TEST INFRASTRUCTURE ONLY.
//
// A C-ABI driver around the reference's own CPU simulators (PICSimulator / FLIPSimulator /
// APICSimulator of AleksanderSiwek/Fluide_Engine), compiled from the reference sources by
// oracle/build_ref.py into oracle/_ref/.  It pins the C restatement (fe_oracle.c) and serves as the
// timed CPU baseline.  It seeds particles directly (the public API only seeds through std::rand in
// PICSimulator::InitializeParticles, pic_simulator.cpp:521-548), swaps in a relative-tolerance CG
// (the reference CG stops on an absolute r.r, conjugate_gradient_solver.cpp:26), and exposes the
// protected substep stages so single stages can be compared.
//
// Private members are reached with the usual test-only access trick; layout is unchanged.
// The mesh writer is used through its public interface; its standard-library headers must not see the access
// trick below, so it comes first.
#include <fstream>
#include <sstream>
#include "3d/obj_manager.hpp"
#include "3d/triangle_mesh.hpp"

#define private public
#define protected public
#include "pic_simulator.hpp"
#include "flip_simulator.hpp"
#include "apic_simulator.hpp"
#include "fluid_solvers/single_phase_pressure_solver.hpp"
#include "linear_system/conjugate_gradient_solver.hpp"
#include "linear_system/blas.hpp"
#include "linear_system/cuda_jacobi_iteration_solver.hpp"
#include "linear_system/jacobi_iteration_solver.hpp"
#include "3d/mesh_2_sdf.hpp"
#include "fluid_solvers/backward_euler_diffusion_solver.hpp"
#include "forces/directional_field.hpp"
#include "forces/point_field.hpp"
#include "forces/swirl_field.hpp"
#include "forces/volume_field.hpp"
#include "3d/triangle_mesh_collider.hpp"
#undef private
#undef protected

#include <cstdint>
#include <cstring>
#include <memory>
#include <iostream>
#include <sstream>

// The reference constructs CudaJacobiIterationSolver as its default pressure solver
// (fluid_solvers/single_phase_pressure_solver.cpp:11); the harness replaces it before any solve, so
// the CPU build only needs the class to exist.  These definitions are the harness's own.
CudaJacobiIterationSolver::CudaJacobiIterationSolver(size_t maxNumberOfIterations, size_t residualCheckInterval,
                                                     double tolerance)
    : _maxNumberOfIterations(maxNumberOfIterations), _toleranceCheckInterval(residualCheckInterval),
      _tolerance(tolerance), _iteration(0), _wasMemoryAllocatedOnDevice(false)
{
}
CudaJacobiIterationSolver::~CudaJacobiIterationSolver() {}
void CudaJacobiIterationSolver::Solve(LinearSystem*) { throw std::runtime_error("CUDA Jacobi is not built on the CPU"); }

namespace {

// ConjugateGradientSolver with tol = rel * ||b||_2: the benchmark scenes' "CG to relative residual".
struct RelTolCG : public LinearSystemSolver {
    double rel;
    size_t maxIt;
    size_t lastIterations = 0;
    RelTolCG(double r, size_t m) : rel(r), maxIt(m) {}
    void Solve(LinearSystem* system) override
    {
        double tol = rel * BLAS::L2Norm(system->b);
        ConjugateGradientSolver cg(maxIt, tol);
        cg.Solve(system);
    }
};

struct Handle {
    TriangleMesh mesh;  // the last GetSurface result
    int solver;
    std::shared_ptr<PICSimulator> sim;
    std::shared_ptr<SinglePhasePressureSolver> pressure;
    std::shared_ptr<RelTolCG> cg;
    std::streambuf* saved = nullptr;
    std::ostringstream sink;
};

void quiet(Handle* h, bool on)
{
    if (on) h->saved = std::cout.rdbuf(h->sink.rdbuf());
    else if (h->saved) { std::cout.rdbuf(h->saved); h->sink.str(""); }
}

template <class F>
void each3(const Array3<double>& a, F f)
{
    const auto& s = a.GetSize();
    for (size_t k = 0; k < s.z; ++k)
        for (size_t j = 0; j < s.y; ++j)
            for (size_t i = 0; i < s.x; ++i) f(i, j, k, i + s.x * (j + s.y * k));
}

}  // namespace

extern "C" {

void* ref_create(int solver, int nx, int ny, int nz, const double* origin, const double* size, double blend,
                 const double* gravity, double max_cfl, double cg_rel_tol, int cg_max_it)
{
    Handle* h = new Handle();
    h->solver = solver;
    Vector3<size_t> n(nx, ny, nz);
    BoundingBox3D domain(Vector3<double>(origin[0], origin[1], origin[2]), Vector3<double>(size[0], size[1], size[2]));
    quiet(h, true);
    if (solver == 0) h->sim = std::make_shared<PICSimulator>(n, domain);
    else if (solver == 1) {
        auto f = std::make_shared<FLIPSimulator>(n, domain);
        f->SetBlendingFactor(blend);
        h->sim = f;
    } else h->sim = std::make_shared<APICSimulator>(n, domain);
    h->pressure = std::make_shared<SinglePhasePressureSolver>();
    h->cg = std::make_shared<RelTolCG>(cg_rel_tol, (size_t)cg_max_it);
    h->pressure->SetLinearSystemSolver(h->cg);
    h->sim->SetPressureSolver(h->pressure);
    h->sim->SetMaxClf(max_cfl);
    h->sim->AddExternalForce(std::make_shared<DirectionalField>(Vector3<double>(gravity[0], gravity[1], gravity[2])));
    quiet(h, false);
    return h;
}

void ref_destroy(void* p) { delete (Handle*)p; }

// HybridSimulator::SetViscosity (hybrid_simulator.cpp:97-100).  The diffusion solver's default linear solver is
// CudaJacobiIterationSolver(1000, 5, 1e-14) (fluid_solvers/backward_euler_diffusion_solver.cpp:10); on the CPU
// the reference's own JacobiIterationSolver with the same settings takes its place (same relaxation and check
// schedule, linear_system/jacobi_iteration_solver.cpp:14-76).
void ref_set_viscosity(void* p, double viscosity)
{
    Handle* h = (Handle*)p;
    auto diffusion = std::make_shared<BackwardEulerDiffusionSolver>();
    diffusion->_systemSolver = std::make_shared<JacobiIterationSolver>(1000, 5, 0.00000000000001);
    h->sim->SetDiffusionSolver(diffusion);
    h->sim->SetViscosity(viscosity);
}

void ref_set_particles(void* p, size_t n, const double* pos, const double* vel, const double* C)
{
    Handle* h = (Handle*)p;
    auto& ps = h->sim->_fluid.particleSystem;
    std::vector<Vector3<double>> P(n), V(n);
    for (size_t i = 0; i < n; ++i) {
        P[i] = Vector3<double>(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]);
        V[i] = vel ? Vector3<double>(vel[3 * i], vel[3 * i + 1], vel[3 * i + 2]) : Vector3<double>(0, 0, 0);
    }
    if (ps.GetParticleNumber() == 0) ps.AddParticles(n, P, h->sim->PARTICLE_POSITION_KEY);
    ps.Resize(n);
    ps.SetVectorValues(h->sim->PARTICLE_POSITION_KEY, P);
    ps.SetVectorValues(h->sim->PARTICLE_VELOCITY_KEY, V);
    if (h->solver == 2) {
        auto* a = (APICSimulator*)h->sim.get();
        a->_cX.assign(n, Vector3<double>(0, 0, 0));
        a->_cY.assign(n, Vector3<double>(0, 0, 0));
        a->_cZ.assign(n, Vector3<double>(0, 0, 0));
        if (C)
            for (size_t i = 0; i < n; ++i) {
                a->_cX[i] = Vector3<double>(C[9 * i + 0], C[9 * i + 1], C[9 * i + 2]);
                a->_cY[i] = Vector3<double>(C[9 * i + 3], C[9 * i + 4], C[9 * i + 5]);
                a->_cZ[i] = Vector3<double>(C[9 * i + 6], C[9 * i + 7], C[9 * i + 8]);
            }
    }
}

size_t ref_num_particles(void* p) { return ((Handle*)p)->sim->GetNumberOfParticles(); }

void ref_get_particles(void* p, double* pos, double* vel, double* C)
{
    Handle* h = (Handle*)p;
    auto& ps = h->sim->_fluid.particleSystem;
    const auto& P = ps.GetVectorValues(h->sim->PARTICLE_POSITION_KEY);
    const auto& V = ps.GetVectorValues(h->sim->PARTICLE_VELOCITY_KEY);
    for (size_t i = 0; i < P.size(); ++i) {
        if (pos) { pos[3 * i] = P[i].x; pos[3 * i + 1] = P[i].y; pos[3 * i + 2] = P[i].z; }
        if (vel) { vel[3 * i] = V[i].x; vel[3 * i + 1] = V[i].y; vel[3 * i + 2] = V[i].z; }
    }
    if (C && h->solver == 2) {
        auto* a = (APICSimulator*)h->sim.get();
        for (size_t i = 0; i < a->_cX.size(); ++i) {
            const Vector3<double>* r[3] = {&a->_cX[i], &a->_cY[i], &a->_cZ[i]};
            for (int t = 0; t < 3; ++t) { C[9 * i + 3 * t] = r[t]->x; C[9 * i + 3 * t + 1] = r[t]->y; C[9 * i + 3 * t + 2] = r[t]->z; }
        }
    }
}

void ref_get_grid(void* p, double* u, double* v, double* w)
{
    Handle* h = (Handle*)p;
    auto& g = h->sim->_fluid.velocityGrid;
    each3(g.GetDataXRef(), [&](size_t i, size_t j, size_t k, size_t f) { u[f] = g.x(i, j, k); });
    each3(g.GetDataYRef(), [&](size_t i, size_t j, size_t k, size_t f) { v[f] = g.y(i, j, k); });
    each3(g.GetDataZRef(), [&](size_t i, size_t j, size_t k, size_t f) { w[f] = g.z(i, j, k); });
}

void ref_set_grid(void* p, const double* u, const double* v, const double* w)
{
    Handle* h = (Handle*)p;
    auto& g = h->sim->_fluid.velocityGrid;
    each3(g.GetDataXRef(), [&](size_t i, size_t j, size_t k, size_t f) { g.x(i, j, k) = u[f]; });
    each3(g.GetDataYRef(), [&](size_t i, size_t j, size_t k, size_t f) { g.y(i, j, k) = v[f]; });
    each3(g.GetDataZRef(), [&](size_t i, size_t j, size_t k, size_t f) { g.z(i, j, k) = w[f]; });
}

void ref_get_pressure(void* p, double* out)
{
    Handle* h = (Handle*)p;
    const auto& x = h->pressure->_system.x;
    if (x.GetSize().x == 0) return;
    each3(x, [&](size_t i, size_t j, size_t k, size_t f) { out[f] = x(i, j, k); });
}

void ref_set_pressure(void* p, const double* in)
{
    Handle* h = (Handle*)p;
    auto& x = h->pressure->_system.x;
    x.Resize(h->sim->GetResolution());
    each3(x, [&](size_t i, size_t j, size_t k, size_t f) { x(i, j, k) = in[f]; });
}

void ref_get_marks(void* p, uint8_t* out)
{
    Handle* h = (Handle*)p;
    const auto& m = h->pressure->_fluidMarkers;
    const auto& s = m.GetSize();
    for (size_t k = 0; k < s.z; ++k)
        for (size_t j = 0; j < s.y; ++j)
            for (size_t i = 0; i < s.x; ++i) out[i + s.x * (j + s.y * k)] = (uint8_t)m(i, j, k);
}

void ref_get_sdf(void* p, double* out)
{
    Handle* h = (Handle*)p;
    const auto& s = h->sim->_fluid.sdf;
    each3(s, [&](size_t i, size_t j, size_t k, size_t f) { out[f] = s(i, j, k); });
}

void ref_get_face_markers(void* p, uint8_t* mu, uint8_t* mv, uint8_t* mw)
{
    Handle* h = (Handle*)p;
    auto& f = h->sim->_fluid;
    const Array3<int>* arr[3] = {&f.xMarkers, &f.yMarkers, &f.zMarkers};
    uint8_t* out[3] = {mu, mv, mw};
    for (int a = 0; a < 3; ++a) {
        const auto& s = arr[a]->GetSize();
        for (size_t k = 0; k < s.z; ++k)
            for (size_t j = 0; j < s.y; ++j)
                for (size_t i = 0; i < s.x; ++i) out[a][i + s.x * (j + s.y * k)] = (uint8_t)(*arr[a])(i, j, k);
    }
}

// Stage entry points (protected hooks of PICSimulator, pic_simulator.hpp:55-80).
void ref_stage_p2g(void* p) { Handle* h = (Handle*)p; quiet(h, true); h->sim->TransferParticles2Grid(); quiet(h, false); }
void ref_stage_sdf(void* p) { Handle* h = (Handle*)p; quiet(h, true); h->sim->BuildSignedDistanceField(); quiet(h, false); }
void ref_stage_begin(void* p, double dt) { Handle* h = (Handle*)p; quiet(h, true); h->sim->BeginAdvanceTimeStep(dt); quiet(h, false); }
void ref_stage_forces(void* p, double dt) { Handle* h = (Handle*)p; quiet(h, true); h->sim->ComputeExternalForces(dt); quiet(h, false); }
// Overwrites Fluid3::sdf (x-fastest node values), the input of GetSurface.
void ref_set_sdf(void* p, const double* values)
{
    Handle* h = (Handle*)p;
    auto& sdf = h->sim->_fluid.sdf;
    each3(sdf, [&](size_t i, size_t j, size_t k, size_t c) { sdf(i, j, k) = values[c]; });
}

// PICSimulator::GetSurface (pic_simulator.cpp:71-78) into a fresh mesh; copies up to the given capacities.
void ref_get_surface(void* p, double* v, double* n, int64_t* t, size_t cap_v, size_t cap_t, size_t* nv, size_t* nt)
{
    Handle* h = (Handle*)p;
    quiet(h, true);
    h->mesh.Clear();
    h->sim->GetSurface(h->mesh);
    quiet(h, false);
    const auto& V = h->mesh.GetVerticies();
    const auto& N = h->mesh.GetNormals();
    const auto& T = h->mesh.GetTriangles();
    *nv = V.size();
    *nt = T.size();
    for (size_t i = 0; v && i < V.size() && i < cap_v; ++i) {
        v[3 * i] = V[i].x; v[3 * i + 1] = V[i].y; v[3 * i + 2] = V[i].z;
        n[3 * i] = N[i].x; n[3 * i + 1] = N[i].y; n[3 * i + 2] = N[i].z;
    }
    for (size_t i = 0; t && i < T.size() && i < cap_t; ++i) {
        t[4 * i] = (int64_t)T[i].point1Idx; t[4 * i + 1] = (int64_t)T[i].point2Idx;
        t[4 * i + 2] = (int64_t)T[i].point3Idx; t[4 * i + 3] = (int64_t)T[i].normalIdx;
    }
}

static TriangleMesh make_mesh(const double* v, size_t nv, const int64_t* t, size_t nt)
{
    TriangleMesh mesh;
    for (size_t i = 0; i < nv; ++i) mesh.AddVertex(Vector3<double>(v[3 * i], v[3 * i + 1], v[3 * i + 2]));
    for (size_t i = 0; i < nt; ++i)
        mesh.AddTriangle(Triangle3D_t((size_t)t[4 * i], (size_t)t[4 * i + 1], (size_t)t[4 * i + 2], (size_t)t[4 * i + 3]));
    return mesh;
}

// Mesh2SDF::Build (3d/mesh_2_sdf.cpp:14-18) onto a ScalarGrid3D of the given size, origin and spacing.
void ref_mesh_to_sdf(const double* v, size_t nv, const int64_t* t, size_t nt, const int* n, const double* origin,
                     const double* h, double* out)
{
    TriangleMesh mesh = make_mesh(v, nv, t, nt);
    ScalarGrid3D sdf(Vector3<size_t>(n[0], n[1], n[2]), 0.0, Vector3<double>(origin[0], origin[1], origin[2]),
                     Vector3<double>(h[0], h[1], h[2]));
    Mesh2SDF().Build(mesh, sdf);
    each3(sdf, [&](size_t i, size_t j, size_t k, size_t c) { out[c] = sdf(i, j, k); });
}

// PICSimulator::InitializeFromTriangleMesh (pic_simulator.cpp:33-39).
void ref_init_from_mesh(void* p, const double* v, size_t nv, const int64_t* t, size_t nt)
{
    Handle* h = (Handle*)p;
    TriangleMesh mesh = make_mesh(v, nv, t, nt);
    quiet(h, true);
    h->sim->InitializeFromTriangleMesh(mesh);
    quiet(h, false);
}

// OBJManager::Save of the last GetSurface mesh under the given object name.
void ref_save_obj(void* p, const char* path, const char* name)
{
    Handle* h = (Handle*)p;
    h->mesh.SetObjectName(name);
    OBJManager obj;
    quiet(h, true);
    obj.Save(path, h->mesh);
    quiet(h, false);
}

// PICSimulator::AddExternalForce (pic_simulator.cpp:41-44) of the reference's position-dependent fields, after the
// DirectionalField that ref_create adds.
void ref_add_point_field(void* p, const double* origin, double strength, double falloff)
{
    Handle* h = (Handle*)p;
    h->sim->AddExternalForce(std::make_shared<PointField>(Vector3<double>(origin[0], origin[1], origin[2]), strength, falloff));
}

void ref_add_swirl_field(void* p, const double* origin, const double* axis, double strength, double falloff)
{
    Handle* h = (Handle*)p;
    h->sim->AddExternalForce(std::make_shared<SwirlField>(Vector3<double>(origin[0], origin[1], origin[2]),
                                                          Vector3<double>(axis[0], axis[1], axis[2]), strength, falloff));
}

void ref_add_volume_field(void* p, const double* v, size_t nv, const int64_t* t, size_t nt, const int* n,
                          const double* domain_origin, const double* domain_size, double strength)
{
    Handle* h = (Handle*)p;
    TriangleMesh mesh = make_mesh(v, nv, t, nt);
    BoundingBox3D domain(Vector3<double>(domain_origin[0], domain_origin[1], domain_origin[2]),
                         Vector3<double>(domain_size[0], domain_size[1], domain_size[2]));
    quiet(h, true);
    h->sim->AddExternalForce(std::make_shared<VolumeField>(mesh, Vector3<size_t>(n[0], n[1], n[2]), domain, strength));
    quiet(h, false);
}

// PICSimulator::AddCollider (pic_simulator.cpp:66-69) of a TriangleMeshCollider on its own node grid; the mesh
// carries normals n (3 doubles each), indexed by the triangles' normal ids.
void ref_add_mesh_collider(void* p, const double* v, size_t nv, const int64_t* t, size_t nt, const double* nrm,
                           size_t nn, const int* n, const double* origin, const double* h)
{
    Handle* hd = (Handle*)p;
    TriangleMesh mesh = make_mesh(v, nv, t, nt);
    for (size_t i = 0; i < nn; ++i) mesh.AddNormal(Vector3<double>(nrm[3 * i], nrm[3 * i + 1], nrm[3 * i + 2]));
    quiet(hd, true);
    hd->sim->AddCollider(std::make_shared<TriangleMeshCollider>(Vector3<size_t>(n[0], n[1], n[2]),
                                                                Vector3<double>(origin[0], origin[1], origin[2]),
                                                                Vector3<double>(h[0], h[1], h[2]), mesh));
    quiet(hd, false);
}

void ref_get_collider_sdf(void* p, double* out)
{
    Handle* hd = (Handle*)p;
    const ScalarGrid3D& g = hd->sim->_boundryConditionSolver->GetColliderSdf();
    each3(g, [&](size_t i, size_t j, size_t k, size_t c) { out[c] = g(i, j, k); });
}

void ref_stage_diffusion(void* p, double dt) { Handle* h = (Handle*)p; quiet(h, true); h->sim->ComputeDiffusion(dt); quiet(h, false); }
void ref_stage_pressure(void* p, double dt) { Handle* h = (Handle*)p; quiet(h, true); h->sim->ComputePressure(dt); quiet(h, false); }
void ref_stage_advection(void* p, double dt) { Handle* h = (Handle*)p; quiet(h, true); h->sim->ComputeAdvection(dt); quiet(h, false); }
void ref_substep(void* p, double dt) { Handle* h = (Handle*)p; quiet(h, true); h->sim->OnAdvanceTimeStep(dt); quiet(h, false); }
double ref_cfl(void* p, double dt) { Handle* h = (Handle*)p; return h->sim->Cfl(dt); }

// PhysicsAnimation::AdvanceSingleFrame (physics_animation.cpp:17-21) with a Frame of interval dt.
void ref_advance_frame(void* p, double dt)
{
    Handle* h = (Handle*)p;
    quiet(h, true);
    h->sim->SetCurrentFrame(Frame(dt)); /* index 0: AdvanceSingleFrame advances exactly one frame of dt */
    h->sim->AdvanceSingleFrame();
    quiet(h, false);
}

}  // extern "C"
