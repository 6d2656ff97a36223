/*
 * fe_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU, FP64, single-threaded restatement of the reference's hybrid particle-grid substep
 * (AleksanderSiwek/Fluide_Engine, src/pic_simulator.cpp, flip_simulator.cpp, apic_simulator.cpp
 * and the solvers they call).  It is the checker for the CUDA path: only the tests, the smoke
 * check and the CPU-baseline leg of the benchmark may load it.  Nothing in the product links it.
 *
 * Every function keeps the reference's floating-point operation order, so on identical inputs
 * it reproduces the serial reference build bit for bit (pinned by tests/test_oracle_vs_reference.py
 * against the reference compiled from its own sources, and by the reference's known-answer tests
 * restated in tests/test_oracle_known_answers.py).
 *
 * Scope: the no-collider, no-emitter scenes of the benchmark configurations, with or without viscosity.  With
 * no colliders the collider SDF is 1.7976931348623157e30 everywhere (3d/collider_collection.cpp:3,38),
 * which makes the collider branches of BlockedBoundryConditionSolver::ConstrainVelocity, the
 * BOUNDRY marker and ExtrapolateIntoCollider provable no-ops; they are restated as such.
 */
#ifndef FE_ORACLE_H
#define FE_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { OR_PIC = 0, OR_FLIP = 1, OR_APIC = 2 };
enum { OR_AIR = 0, OR_FLUID = 1, OR_BOUNDRY = 2 };

typedef struct {
    int n[3];            /* cells per axis */
    double origin[3];    /* domain origin (BoundingBox3D::GetOrigin) */
    double size[3];      /* domain extents (BoundingBox3D::GetSize) */
    int solver;          /* OR_PIC / OR_FLIP / OR_APIC */
    double blend;        /* FLIPSimulator::_blendingFactor, reference default 0.05 */
    double gravity[3];   /* DirectionalField strength */
    double max_cfl;      /* HybridSimulator::_maxCfl */
    double cg_rel_tol;   /* CG stops when r.r <= (rel * ||b||_2)^2 */
    int cg_max_it;       /* ConjugateGradientSolver::_maxNumberOfIterations */
    double viscosity;    /* Fluid3::viscosity (HybridSimulator::SetViscosity); 0 skips ComputeDiffusion */
} or_desc;

typedef struct or_sim or_sim;

or_sim* or_create(const or_desc* d);
void or_destroy(or_sim* s);

int or_set_particles(or_sim* s, size_t n, const double* pos, const double* vel, const double* C);
size_t or_num_particles(const or_sim* s);
void or_get_particles(const or_sim* s, double* pos, double* vel, double* C);

/* Grid state: u (nx+1)*ny*nz, v nx*(ny+1)*nz, w nx*ny*(nz+1), x-fastest; p, sdf, marks nx*ny*nz. */
void or_get_grid(const or_sim* s, double* u, double* v, double* w);
void or_set_grid(or_sim* s, const double* u, const double* v, const double* w);
void or_get_pressure(const or_sim* s, double* p);
void or_set_pressure(or_sim* s, const double* p);
/* Not the reference: with colliders, give enclosed FLUID components (no AIR neighbour) a solvable system the
 * way the GPU does (all-zero rows -> identity, right-hand-side mean removed per enclosed component). */
void or_set_enclosed_projection(or_sim* s, int on);
void or_get_marks(const or_sim* s, uint8_t* marks);
void or_get_sdf(const or_sim* s, double* sdf);
void or_get_face_markers(const or_sim* s, uint8_t* mu, uint8_t* mv, uint8_t* mw);
void or_get_snapshot(const or_sim* s, double* u, double* v, double* w);
void or_get_rhs(const or_sim* s, double* b);

/* Substep stages, in the order PICSimulator::OnAdvanceTimeStep runs them. */
void or_stage_p2g(or_sim* s);                       /* TransferParticles2Grid (virtual per solver) */
void or_stage_sdf(or_sim* s);                       /* BuildSignedDistanceField */
void or_stage_extrapolate(or_sim* s);               /* ExtrapolateVelocityToAir */
void or_stage_bc(or_sim* s);                        /* ApplyBoundryCondition */
void or_stage_forces(or_sim* s, double dt);         /* ComputeExternalForces (forces + BC) */
void or_stage_pressure(or_sim* s, double dt);       /* ComputePressure (markers, system, CG, apply, BC) */
void or_stage_advection(or_sim* s, double dt);      /* ComputeAdvection (extrap, BC, G2P, move) */
void or_stage_g2p(or_sim* s);                       /* TransferGrid2Particles only */
void or_stage_move(or_sim* s, double dt);           /* MoveParticles only */
void or_build_markers(or_sim* s);                   /* SinglePhasePressureSolver::BuildMarkers only */
void or_stage_diffusion(or_sim* s, double dt);      /* ComputeDiffusion (3 Jacobi solves + BC; no-op at viscosity 0) */

/* Position-dependent external forces, applied by or_stage_forces after the DirectionalField of or_desc::gravity
 * in the order added (at most 8); 0 on success.  PointField (forces/point_field.cpp), SwirlField
 * (forces/swirlf_field.cpp), VolumeField (forces/volume_field.cpp, mesh as in or_mesh_to_sdf). */
enum { OR_FORCE_POINT = 1, OR_FORCE_SWIRL = 2, OR_FORCE_VOLUME = 3 };
int or_add_point_field(or_sim* s, const double origin[3], double strength);
int or_add_swirl_field(or_sim* s, const double origin[3], const double axis[3], double strength);
int or_add_volume_field(or_sim* s, const double* V, const int64_t* T, size_t nt, const int n[3],
                        const double domain_origin[3], const double domain_size[3], double strength);
/* Colliders (at most 8): TriangleMeshCollider(gridSize, gridOrigin, gridSpacing, mesh) (3d/triangle_mesh_collider.cpp)
 * with its mesh normals N (3 doubles each; triangle t's normal id is T[4t + 3]); 0 on success.  With colliders the
 * stages run the reference's collider branches: BuildCollider (or_build_collider, first in or_substep),
 * ExtrapolateIntoCollider (in or_stage_sdf), BOUNDRY markers, ConstrainVelocity's blocking, extrapolation and
 * friction projection (or_stage_bc), and ResolveCollision in MoveParticles. */
int or_add_mesh_collider(or_sim* s, const double* V, size_t nv, const int64_t* T, size_t nt, const double* N,
                         size_t nn, const int n[3], const double origin[3], const double h[3]);
void or_build_collider(or_sim* s);                  /* ColliderCollection::BuildSdf */
void or_get_collider_sdf(const or_sim* s, double* out); /* the collider SDF on the n nodes at the domain origin */

/* VolumeField::Initialize's closest-point vectors on a node grid (3 doubles per node, x-fastest). */
void or_volume_field_vectors(const double* V, const int64_t* T, size_t nt, const int n[3], const double o[3],
                             const double h[3], double* out);

void or_substep(or_sim* s, double dt);              /* PICSimulator::OnAdvanceTimeStep */
double or_cfl(const or_sim* s, double dt);          /* PICSimulator::Cfl */
unsigned or_number_of_substeps(const or_sim* s, double dt); /* PICSimulator::NumberOfSubTimeSteps */
int or_advance_time(or_sim* s, double frame_dt);    /* PhysicsAnimation::AdvanceTimeStep; returns substeps */

int or_cg_iterations(const or_sim* s);              /* iterations of the last solve */
int or_diffusion_iterations(const or_sim* s, int component); /* Jacobi iterations of the last diffusion solve */
/* Face markers of the last diffusion solve (BackwardEulerDiffusionSolver::_fluidMarkers per component). */
void or_get_diffusion_markers(const or_sim* s, uint8_t* mu, uint8_t* mv, uint8_t* mw);
double or_cg_rel_residual(const or_sim* s);         /* true ||b - A p|| / ||b|| after the last solve */
double or_divergence_l2(const or_sim* s);           /* ||div u||_2 over FLUID cells of the current grid */

/* Reference known-answer helpers (common/math_utils.hpp, grid_systems/face_centered_grid3d.cpp). */
double or_lerp(double a, double b, double f);
double or_trilerp(const double c[8], double fx, double fy, double fz);
double or_sample_face_array(const double* arr, const int size[3], const double origin[3], const double h[3],
                            const double pos[3]);
double or_scalar_sample(const double* arr, const int size[3], const double origin[3], const double h[3],
                        const double pos[3]);

/* Standalone pressure projection on a caller-supplied grid with caller-supplied markers
 * (SinglePhasePressureSolver::Solve with the CG of conjugate_gradient_solver.cpp). */
int or_project(const int n[3], const double h[3], const uint8_t* marks, double* u, double* v, double* w,
               double* p, double rel_tol, int max_it, double* rel_residual);

/* MarchingCubesSolver::BuildSurface (3d/marching_cubes_solver.cpp:25-50) with iso value 0 and no colliders, on a
 * node grid of n[0]*n[1]*n[2] values (x-fastest) with the given origin and spacing.  Fills up to cap_v vertices and
 * normals (3 doubles each) and cap_t triangles (4 int64 each: vertex ids, normal id) in the reference's order and
 * returns the full counts in *nv, *nt (call with NULL buffers to size them). */
int or_build_surface(const double* sdf, const int n[3], const double origin[3], const double h[3], double* vertices,
                     double* normals, int64_t* tris, size_t cap_v, size_t cap_t, size_t* nv, size_t* nt);
/* OBJManager::Save of such a mesh (3d/obj_manager.cpp:14-90). */
int or_write_obj(const char* path, const char* name, const double* v, const double* vn, size_t nv, const int64_t* t,
                 size_t nt);

/* Mesh2SDF::Build (3d/mesh_2_sdf.cpp:14-82) of a triangle mesh (V: 3 doubles per vertex, T: 4 int64 per triangle,
 * the last unused) onto a node grid n[3] with origin and spacing; sdf receives n[0]*n[1]*n[2] values, x-fastest. */
void or_mesh_to_sdf(const double* V, size_t nv, const int64_t* T, size_t nt, const int n[3], const double origin[3],
                    const double h[3], double* sdf);
double or_distance_to_triangle(const double pt[3], const double p0[3], const double p1[3], const double p2[3]);
int or_mesh_is_inside(const double* V, const int64_t* T, size_t nt, const double pt[3]);
/* InitializeParticles' cell test on the simulator's current fluid SDF (1 where particles would be seeded). */
void or_seed_cells(const or_sim* s, uint8_t* mask);
void or_set_sdf(or_sim* s, const double* sdf);

/* Stable counting sort of FP32 particle positions by fe_keys.h cell key; writes keys and perm. */
void or_sort_keys(const float* pos, size_t n, const int dims[3], const float origin[3], const float inv_h[3],
                  uint32_t* keys_sorted, uint32_t* perm);

/* Seeding of the analytic scenes (fe_seed.h), for CPU-only tests. */
size_t or_seed_regions(const void* regions, int nreg, const int n[3], const double origin[3], const double h[3],
                       uint64_t seed, float* pos, float* vel, size_t cap);

#ifdef __cplusplus
}
#endif

#endif /* FE_ORACLE_H */
