/*
 * fluide_b200.h -- C ABI of the B200-native hybrid particle-grid (PIC / FLIP / APIC) substep.
 *
 * One fe_scene owns one simulation's state resident in HBM: FP32 particles (struct of arrays,
 * kept sorted by cell key), the FP32 staggered MAC grid, FP64 pressure and the solver scratch.
 * All entry points return an fe_status; no entry point throws or aborts.  Pointers passed for
 * particle / grid data may be host or device pointers (they are copied with cudaMemcpyDefault).
 * Layouts match the reference: face arrays u (nx+1)*ny*nz, v nx*(ny+1)*nz, w nx*ny*(nz+1) and cell
 * arrays nx*ny*nz, all x-fastest (common/array3.hpp:65-85); particle arrays are xyz-interleaved.
 *
 * Reference citations are relative to AleksanderSiwek/Fluide_Engine's src/ directory.
 */
#ifndef FLUIDE_B200_H
#define FLUIDE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    FE_OK = 0,
    FE_ERR_CUDA = 1,           /* a CUDA runtime call failed; fe_last_error() has the message */
    FE_ERR_BAD_ARG = 2,        /* invalid argument (null handle, size mismatch, bad descriptor) */
    FE_ERR_OOM = 3,            /* device allocation failed */
    FE_ERR_NOT_CONVERGED = 4,  /* pressure solve hit its iteration cap (state is still advanced) */
    FE_ERR_TIMEOUT = 5,        /* a bounded device-side wait gave up; the context stays usable */
    FE_ERR_STATE = 6,          /* call out of order (e.g. step before particles are set) */
    FE_ERR_NO_DEVICE = 7       /* no CUDA device / the library was built without device code */
} fe_status;

typedef enum { FE_SOLVER_PIC = 0, FE_SOLVER_FLIP = 1, FE_SOLVER_APIC = 2 } fe_solver_kind;

typedef enum { FE_CELL_AIR = 0, FE_CELL_FLUID = 1, FE_CELL_BOUNDRY = 2 } fe_cell_mark;

/* Scene description.  Mirrors the state the reference constructors fix:
 * PICSimulator(gridSize, domain) (pic_simulator.cpp:17-26, hybrid_simulator.cpp:4-25),
 * FLIPSimulator::SetBlendingFactor (flip_simulator.cpp:15-18), HybridSimulator::SetMaxClf
 * (hybrid_simulator.cpp:92-95), DirectionalField gravity (forces/directional_field.cpp:3-16) and the
 * pressure solver settings (linear_system/conjugate_gradient_solver.cpp:3-7). */
typedef struct {
    int32_t n[3];            /* cells per axis (gridSize) */
    double origin[3];        /* BoundingBox3D origin */
    double size[3];          /* BoundingBox3D size; grid spacing h = size / n */
    int32_t solver;          /* fe_solver_kind */
    double flip_blend;       /* v = (1 - blend) * flip + blend * pic; reference default 0.05 */
    double gravity[3];       /* external acceleration added to every face each substep */
    double max_cfl;          /* extrapolation depth ceil(max_cfl), RK2 sub-steps max(max_cfl,1) */
    double cg_rel_tol;       /* stop when ||b - A p||_2 <= cg_rel_tol * ||b||_2 (FP64 test) */
    int32_t cg_max_it;       /* cap on inner FP32 CG iterations per pressure solve */
    double cg_inner_tol;     /* relative residual reduction asked of each FP32 inner solve; 0 (default): 1e-4 for the
                                plain CG; for the multigrid-preconditioned CG cg_rel_tol split evenly over the fewest
                                refinements that 1e-4 per inner solve allows (1e-3 at 1e-6, 1e-4 at 1e-8) */
    int32_t max_refine;      /* cap on FP64 outer refinement steps per pressure solve */
    int32_t device;          /* CUDA device ordinal */
    uint64_t max_particles;  /* capacity; 0 = sized by the first fe_scene_set_particles */
    int32_t pressure_solver; /* fe_pressure_solver: how the inner FP32 solve runs (same system, same FP64 test) */
    double viscosity;        /* kinematic viscosity (HybridSimulator::SetViscosity); 0 = none, the reference default */
} fe_scene_desc;

/* Inner solver of the pressure projection.  Both solve the reference's system
 * (single_phase_pressure_solver.cpp:99-164) to the same FP64 relative-residual target inside the same FP64
 * refinement; they differ in how many inner iterations that takes.  The reference uses unpreconditioned CG
 * (linear_system/conjugate_gradient_solver.cpp:14-55). */
typedef enum {
    FE_PRESSURE_AUTO = 0,    /* default: MGPCG for grids of 2^15 cells (32^3) or more, CG below (faster there) */
    FE_PRESSURE_MGPCG = 1,   /* CG preconditioned by one multigrid V-cycle: 10-25 inner iterations, 4 L - 2 barriers each */
    FE_PRESSURE_CG = 2       /* unpreconditioned CG: one grid barrier per iteration, 130-1100 iterations */
} fe_pressure_solver;

/* Per-substep statistics. */
typedef struct {
    int32_t cg_iterations;     /* inner FP32 CG iterations */
    int32_t refinements;       /* FP64 outer refinement steps */
    int32_t converged;         /* 1 if ||b - A p|| <= tol * ||b|| */
    int32_t fluid_cells;       /* number of FLUID-marked cells */
    double rel_residual;       /* final FP64 ||b - A p|| / ||b|| */
    double b_norm;             /* ||b||_2 (divergence before projection over FLUID cells) */
} fe_step_stats;

typedef struct fe_scene fe_scene;

/* Stages of one substep, in PICSimulator::OnAdvanceTimeStep order (pic_simulator.cpp:111-196). */
typedef enum {
    FE_STAGE_SORT = 0,       /* cell keys + stable counting sort (no reference counterpart) */
    FE_STAGE_P2G = 1,        /* TransferParticles2Grid (pic :356-437, flip :25-119, apic :15-118) */
    FE_STAGE_MARK = 2,       /* BuildSignedDistanceField + BuildMarkers (pic :452-475, single_phase :30-48) */
    FE_STAGE_PRE = 3,        /* ExtrapolateVelocityToAir + BC + gravity + BC (pic :186-212) */
    FE_STAGE_DIFFUSE = 4,    /* ComputeDiffusion: backward Euler viscosity + BC (pic :214-222); no-op at viscosity 0 */
    FE_STAGE_PRESSURE = 5,   /* BuildSystem + CG + ApplyPressure + BC (pic :224-229) */
    FE_STAGE_POST = 6,       /* ExtrapolateVelocityToAir + BC (pic :233-234) */
    FE_STAGE_G2P = 7,        /* TransferGrid2Particles (pic :439-450, flip :121-161, apic :120-176) */
    FE_STAGE_MOVE = 8,       /* MoveParticles (pic :239-312) */
    FE_STAGE_COUNT = 9
} fe_stage;

/* Fills *d with the reference defaults (maxCfl 3 from hybrid_simulator.cpp:21, blend 0.05 from
 * flip_simulator.cpp:5, gravity (0,-9.81,0), CG rel 1e-6 / 500 iterations). */
fe_status fe_scene_desc_default(fe_scene_desc* d);

/* Creates a scene on desc->device.  Replaces PICSimulator/FLIPSimulator/APICSimulator construction
 * (pic_simulator.cpp:17-26, flip_simulator.cpp:4-8, apic_simulator.cpp:4-7). */
fe_status fe_scene_create(const fe_scene_desc* desc, fe_scene** out);

/* Releases the scene.  Its device memory returns to the library's stream-ordered pool for the device, which
 * keeps freed memory cached for later scenes (creating and destroying scenes then costs no driver allocation
 * and no device-wide synchronisation); the pool's memory is returned to the driver when the process exits. */
fe_status fe_scene_destroy(fe_scene* s);

/* Sets the particles: pos and vel are n*3 floats (xyz interleaved), C is n*9 floats (rows cX, cY, cZ
 * of apic_simulator.hpp:21-23) or NULL for zero.  Replaces ParticleSystem::AddParticles /
 * SetVectorValues (particle_systems/particle_system.cpp:36-44,97-107) and APICSimulator::_cX.. */
fe_status fe_scene_set_particles(fe_scene* s, const float* pos, const float* vel, const float* C, uint64_t n);

/* Returns the scene to the state fe_scene_create leaves it in -- velocity buffers, FLIP snapshot, face and
 * cell markers, pressure (the next solve's warm start, linear_system.cpp:13-18), right-hand side and solver
 * scratch zeroed -- while keeping its allocations, particles and captured graphs, so a server can reuse the
 * scene for a new job of the same grid and solver without allocating.  No reference counterpart (a
 * reference simulator lives for one run). */
fe_status fe_scene_reset(fe_scene* s);

/* Copies the particles out in the order they were set (ParticleSystem::GetVectorValues,
 * particle_systems/particle_system.cpp:133-141).  Any pointer may be NULL. */
fe_status fe_scene_get_particles(fe_scene* s, float* pos, float* vel, float* C, uint64_t n);

/* Number of particles (HybridSimulator::GetNumberOfParticles, hybrid_simulator.cpp:87-90). */
fe_status fe_scene_num_particles(const fe_scene* s, uint64_t* n);

/* Runs nsub substeps of fixed length dt (PICSimulator::OnAdvanceTimeStep, pic_simulator.cpp:111-154),
 * replayed as three captured CUDA graphs per substep.  stats may be NULL (no host synchronisation then); else it
 * receives nsub entries and the call synchronises the scene's stream. */
fe_status fe_scene_step(fe_scene* s, double dt, int32_t nsub, fe_step_stats* stats);

/* fe_scene_step with per-substep device timing: CUDA events recorded on the scene's stream before, between
 * and after the three phase graphs of each substep (pre-solve: SORT..PRE + rhs; solve: the CG kernel;
 * post-solve: apply..MOVE).  phase_ms receives nsub * 3 floats; the call synchronises. */
fe_status fe_scene_step_profiled(fe_scene* s, double dt, int32_t nsub, fe_step_stats* stats, float* phase_ms);

/* Advances one frame of length frame_dt with the reference's CFL-adaptive substepping
 * (PhysicsAnimation::AdvanceSingleFrame / AdvanceTimeStep, physics_animation.cpp:17-21,64-92, with
 * PICSimulator::NumberOfSubTimeSteps, pic_simulator.cpp:349-354).  *substeps receives the count. */
fe_status fe_scene_advance_frame(fe_scene* s, double frame_dt, int32_t* substeps);

/* CFL number of the current grid for interval dt (PICSimulator::Cfl, pic_simulator.cpp:80-97). */
fe_status fe_scene_cfl(fe_scene* s, double dt, double* cfl);

/* Runs stages [first, last] of one substep of length dt (for stage-by-stage parity checks). */
fe_status fe_scene_run_stages(fe_scene* s, double dt, int32_t first, int32_t last);

/* Grid access (Fluid3 velocityGrid / SinglePhasePressureSolver::GetPressure / _fluidMarkers,
 * fluid3.hpp:10-26, single_phase_pressure_solver.cpp:50-53).  Any pointer may be NULL. */
fe_status fe_scene_get_grid(fe_scene* s, float* u, float* v, float* w, double* p, uint8_t* marks);
fe_status fe_scene_set_grid(fe_scene* s, const float* u, const float* v, const float* w);
fe_status fe_scene_set_pressure(fe_scene* s, const double* p);
/* P2G face markers (Fluid3 xMarkers/yMarkers/zMarkers) and the FLIP snapshot (FLIPSimulator::
 * _velocityResiduals right after P2G, flip_simulator.cpp:107-118). */
fe_status fe_scene_get_face_markers(fe_scene* s, uint8_t* mu, uint8_t* mv, uint8_t* mw);
fe_status fe_scene_get_snapshot(fe_scene* s, float* u, float* v, float* w);
/* Right-hand side b = div u of the last pressure solve (SinglePhasePressureSolver::BuildSystem b). */
fe_status fe_scene_get_rhs(fe_scene* s, double* b);
/* Band-limited particle SDF on the cell-centred grid (HybridSimulator::GetFluidSdf, hybrid_simulator.cpp:82-85,
 * as built by PICSimulator::BuildSignedDistanceField, pic_simulator.cpp:452-475), FP64: the one built at the
 * start of the last substep (from the current particles before any substep). */
fe_status fe_scene_get_fluid_sdf(fe_scene* s, double* sdf);
/* Fluid surface (PICSimulator::GetSurface, pic_simulator.cpp:71-78: MarchingCubesSolver::BuildSurface,
 * 3d/marching_cubes_solver.cpp:25-583, iso value 0, no colliders) of the band particle SDF the reference holds in
 * Fluid3::sdf: the one built at the start of the last substep (from the current particles before any substep).
 * The mesh equals the reference's: vertices and normals in its creation order (FP64), triangles as 4 int64 each
 * (three vertex ids, then the normal id the reference stores: the last vertex created so far).  Built on the
 * device; fe_scene_build_surface returns the counts, fe_scene_get_surface copies the mesh out (host or device
 * pointers; any may be NULL), fe_scene_write_surface_obj writes it as OBJManager::Save does. */
fe_status fe_scene_build_surface(fe_scene* s, uint64_t* n_vertices, uint64_t* n_triangles);
fe_status fe_scene_get_surface(fe_scene* s, double* vertices, double* normals, int64_t* triangles);
fe_status fe_scene_write_surface_obj(fe_scene* s, const char* path, const char* object_name);
/* OBJManager::Save (3d/obj_manager.cpp:14-90, 3d/mesh_file_manager.cpp) of a mesh in the layout above (host
 * pointers): the reference's header, "v" / "vn" lines in "%f" format, "s off", "f a//n b//n c//n" lines. */
fe_status fe_write_obj(const char* path, const char* object_name, const double* vertices, const double* normals,
                       uint64_t n_vertices, const int64_t* triangles, uint64_t n_triangles);

/* Scene initialisation from triangle meshes.  Meshes are given as vertices (3 doubles each) and triangles (4 int64
 * each: three vertex ids, then a normal id that is not used), host or device pointers.
 *
 * fe_mesh_to_sdf: Mesh2SDF::Build (3d/mesh_2_sdf.cpp:14-82) onto a node grid of n[0]*n[1]*n[2] values (x-fastest)
 * with the given origin and spacing: exact distances within the band of every triangle's index box (box from the
 * vertex coordinates times 1 / spacing[0], without the origin, as the reference computes it), the fill value
 * max(spacing) * (n[0] + n[1] + n[2]) elsewhere, negated inside the mesh (winding number, TriangleMesh::IsInside
 * with abs on the double as on the reference's platform).  Distances equal the reference's bit for bit.
 *
 * fe_scene_init_from_mesh: PICSimulator::InitializeFromTriangleMesh (pic_simulator.cpp:33-39): the mesh SDF
 * becomes the scene's Fluid3::sdf (returned by fe_scene_get_fluid_sdf and used by the surface until the next
 * substep), and every cell whose velocity-grid position (domain origin + h * index) samples it below 0 receives
 * particles_per_cell particles (0: the reference default 16) at position + h * U[0,1]^3, velocity 0, appended to
 * the scene's particles.  The reference draws the offsets from the unseeded std::rand() in a parallel loop; here
 * they come from a counter-based generator started at `seed`, so the cells and counts equal the reference's and
 * the positions are reproducible.
 *
 * fe_scene_add_volume_emitter: VolumeEmitter (emmiter/volume_emmiter.cpp:8-86) with the mesh SDF on its own grid
 * (resolution, domain; resolution within the scene's grid): at the start of every substep each emitter node
 * with SDF <= 0 whose fluid SDF value (same index; the SDF of the previous substep) is >= 0 receives
 * particles_per_block particles at position + h * U[0,1]^3 with `velocity` (PICSimulator::OnBeginAdvanceTimeStep,
 * pic_simulator.cpp:160-163), except in the scene's first substep: the reference's emitters also require the
 * collider SDF > 0 and run before the first BuildCollider, while that SDF still holds its initial 0, so the first
 * substep emits nothing (fe_scene_reset starts over).  A scene with emitters steps without graphs (its particle count changes) and cannot
 * join a batch; it may start without particles (fe_scene_step and fe_scene_advance_frame then emit first; a
 * substep that still has none is skipped and reports a converged empty solve).  fe_scene_clear_emitters removes
 * them (fe_scene_reset does too). */
fe_status fe_mesh_to_sdf(const double* vertices, uint64_t n_vertices, const int64_t* triangles, uint64_t n_triangles,
                         const int32_t n[3], const double origin[3], const double spacing[3], double* sdf, int32_t device);
fe_status fe_scene_init_from_mesh(fe_scene* s, const double* vertices, uint64_t n_vertices, const int64_t* triangles,
                                  uint64_t n_triangles, uint32_t particles_per_cell, uint64_t seed);
fe_status fe_scene_add_volume_emitter(fe_scene* s, const double* vertices, uint64_t n_vertices, const int64_t* triangles,
                                      uint64_t n_triangles, const int32_t resolution[3], const double domain_origin[3],
                                      const double domain_size[3], uint32_t particles_per_block, const double velocity[3],
                                      uint64_t seed, int32_t* emitter_id);
fe_status fe_scene_clear_emitters(fe_scene* s);
/* VolumeEmitter::InitializeFromSdf (emmiter/volume_emmiter.cpp:50-56): replaces emitter `id`'s SDF with node values
 * on its grid (resolution[0] * resolution[1] * resolution[2] doubles, x-fastest; host or device pointer). */
fe_status fe_scene_set_emitter_sdf(fe_scene* s, int32_t id, const double* sdf);
/* Fluid3::sdf (fluid3.hpp:22, a public member of the reference's fluid) set to node values on the scene's SDF grid
 * (n[0] * n[1] * n[2] doubles, x-fastest, host or device pointer); held, like the mesh SDF of
 * fe_scene_init_from_mesh, until the next substep builds the particles' SDF.  Lets a caller that rebuilds a scene
 * between seeding and the first substep (e.g. to change its settings) carry the fluid SDF over. */
fe_status fe_scene_set_fluid_sdf(fe_scene* s, const double* sdf);

/* Position-dependent external forces (PICSimulator::AddExternalForce, pic_simulator.cpp:41-44, of a PointField,
 * SwirlField or VolumeField; a DirectionalField is fe_scene_desc::gravity).  Every substep, after gravity,
 * ComputeExternalForces (pic_simulator.cpp:203-212) adds dt * each force's component at every face position
 * (ExternalForce::ApplyExternalForce, forces/external_force.cpp:3-29) in the order added, then re-zeroes the
 * walls.  At most 8 per scene; kept by fe_scene_reset, removed by fe_scene_clear_forces.
 *   FE_FORCE_POINT  PointField(origin, strength, falloff) (forces/point_field.cpp:3-56)
 *   FE_FORCE_SWIRL  SwirlField(origin, axis, strength, falloff) (forces/swirlf_field.cpp:5-23; the axis is
 *                   normalised as its constructor does)
 *   FE_FORCE_VOLUME VolumeField(mesh, resolution, domain, strength) (forces/volume_field.cpp:5-89): node vectors
 *                   from `field` (3 doubles per node, x-fastest, host or device) when non-null, else computed
 *                   from the mesh (closest point on the first nearest triangle minus the node, on the GPU)
 * falloff is stored by the reference and unused by its samples. */
typedef enum { FE_FORCE_POINT = 1, FE_FORCE_SWIRL = 2, FE_FORCE_VOLUME = 3 } fe_force_kind;
typedef struct fe_force_desc {
    int32_t kind;
    double origin[3];
    double axis[3];
    double strength;
    double falloff;
    const double* vertices;   /* volume: mesh, 3 doubles per vertex */
    uint64_t n_vertices;
    const int64_t* triangles; /* volume: 4 int64 per triangle (vertex ids, unused normal id) */
    uint64_t n_triangles;
    int32_t resolution[3];    /* volume: nodes per axis */
    double domain_origin[3];  /* volume: grid origin; spacing = domain_size / resolution */
    double domain_size[3];
    const double* field;      /* volume: precomputed node vectors, or NULL */
} fe_force_desc;
fe_status fe_scene_add_force(fe_scene* s, const fe_force_desc* force, int32_t* id);
fe_status fe_scene_clear_forces(fe_scene* s);
/* VolumeField::Initialize's node vectors (forces/volume_field.cpp:72-89) on a grid of n nodes with the given
 * origin and spacing: 3 doubles per node, x-fastest, written to `out` (host or device). */
fe_status fe_volume_field_vectors(const double* vertices, uint64_t n_vertices, const int64_t* triangles,
                                  uint64_t n_triangles, const int32_t n[3], const double origin[3],
                                  const double spacing[3], double* out, int32_t device);

/* Solid colliders: PICSimulator::AddCollider (pic_simulator.cpp:66-69) of a TriangleMeshCollider(gridSize,
 * gridOrigin, gridSpacing, mesh) (3d/triangle_mesh_collider.cpp:4-100): the mesh's Mesh2SDF on the collider's own
 * node grid (resolution, grid_origin, grid_spacing), and the mesh itself with normals (3 doubles each; each
 * triangle's 4th id indexes them) for the collision response.  With colliders every substep runs the reference's
 * collider branches: the collider SDF (ColliderCollection::BuildSdf on the scene's n nodes at the domain origin),
 * ExtrapolateIntoCollider of the fluid SDF, BOUNDRY cells in the pressure system, BlockedBoundryConditionSolver's
 * blocking, extrapolation and tangential projection at every ApplyBoundryCondition, and ResolveCollision in
 * MoveParticles with the reference's indexing (a particle ending inside the collider SDF moves particle number c
 * onto collider c's surface; pic_simulator.cpp:296-305).  At most 8; kept by fe_scene_reset.  A scene with
 * colliders uses the plain CG pressure solver, cannot join a batch and cannot have a viscosity > 0.
 * fe_scene_get_collider_sdf returns the collider SDF as the reference holds it (0 before the first substep). */
fe_status fe_scene_add_mesh_collider(fe_scene* s, const double* vertices, uint64_t n_vertices, const int64_t* triangles,
                                     uint64_t n_triangles, const double* normals, uint64_t n_normals,
                                     const int32_t resolution[3], const double grid_origin[3],
                                     const double grid_spacing[3], int32_t* id);
fe_status fe_scene_clear_colliders(fe_scene* s);
fe_status fe_scene_get_collider_sdf(fe_scene* s, double* sdf);

/* Viscosity (HybridSimulator::SetViscosity, hybrid_simulator.cpp:97-100), settable at any time.  When it is > 0
 * every substep runs ComputeDiffusion (pic_simulator.cpp:214-222) after the external forces: the reference's
 * BackwardEulerDiffusionSolver (fluid_solvers/backward_euler_diffusion_solver.cpp:20-242) -- per component, faces
 * whose fluid-SDF sample is < 0 are FLUID and (1 + sum c) u' - c sum u'_nbr = u with c = viscosity dt / h^2 is
 * relaxed by the Jacobi iteration of CudaJacobiIterationSolver(1000, 5, 1e-14) -- in FP64 with the reference's
 * operation order, then the wall layers are zeroed.  The first call with a viscosity > 0 allocates the solve's
 * buffers (about 48 bytes per cell). */
fe_status fe_scene_set_viscosity(fe_scene* s, double viscosity);
/* Last viscosity solve: iterations[0..2] = the reference's Jacobi iterations per component (1000 = the cap),
 * iterations[3] = relaxation passes the GPU ran (fewer than 1000 when every component's iterates became
 * periodic, after which iterate 1000 is known without running to it); and the FLUID face markers of each
 * component (BackwardEulerDiffusionSolver::_fluidMarkers, face-array layout).  Any pointer may be NULL;
 * FE_ERR_STATE if the scene never had a viscosity > 0. */
fe_status fe_scene_get_diffusion(fe_scene* s, int32_t* iterations, uint8_t* mu, uint8_t* mv, uint8_t* mw);
/* Sorted cell keys and the permutation of the last sort (slot -> particle id), n entries each. */
fe_status fe_scene_get_sort(fe_scene* s, uint32_t* keys, uint32_t* perm, uint64_t n);
/* Post-projection ||div u||_2 over FLUID cells of the current grid (FP64). */
fe_status fe_scene_divergence(fe_scene* s, double* l2);

/* Pressure projection of a caller-owned MAC grid that allocates no device memory.  No counterpart in
 * the reference: it exists for callers that cannot call cudaMalloc/cudaFree on this path (a per-frame or
 * real-time callback where an allocation's implicit device synchronisation would stall, or memory owned by
 * another allocator).  All pointers except n, h and stats are device pointers: marks (nx*ny*nz, FE_CELL_*),
 * u/v/w (face arrays, updated in place), p (pressure, warm start in, solution out).  Runs the scene path's
 * pressure stage (rhs, CG in FP64 refinement to rel_tol, apply) on `stream` (NULL = legacy default stream),
 * then reads the status back and synchronises that stream.  Scratch lives in one static device array of
 * about 11.6 MB per device (held until the process exits), so grids are limited to 2^18 cells (e.g. 64^3);
 * larger grids return FE_ERR_BAD_ARG.  The first call on a device (and the first after its context was
 * replaced, e.g. by cudaDeviceReset) resolves the array's address (cudaGetSymbolAddress); make it before any
 * stream capture begins.  Calls share the array and it keeps the last call's contents: calls that overlap on
 * the GPU race, so issue them on one stream.  stats (host) may be NULL. */
fe_status fe_project_noalloc(const int32_t n[3], const double h[3], const uint8_t* marks, float* u, float* v,
                             float* w, double* p, double rel_tol, int32_t max_it, void* stream,
                             fe_step_stats* stats);

/* Launch choices of a scene's pressure solve that change its speed, not its result (every choice reaches the same
 * FP64 relative residual).  No reference counterpart: they are what the autotuner (fe_scene_autotune) searches.
 * In fe_scene_set_tuning a negative or zero field keeps the current choice. */
typedef struct fe_tuning {
    int32_t multigrid;            /* 1: multigrid-preconditioned CG, 0: plain CG (grids too small for a hierarchy stay plain) */
    int32_t cg_block_threads;     /* threads per persistent solver block: 256, 512 or 1024 (1024 threads per SM in total) */
    int32_t mg_block_level_cells; /* multigrid levels of at most this many cells are processed by one block */
    int32_t cg_cluster;           /* thread-block cluster size of the persistent solve (1, 2, 4, 8, 16): the blocks of a
                                     cluster pre-reduce their sums in distributed shared memory and one block per
                                     cluster arrives at the grid barrier */
    int32_t pressure_extrapolation; /* 1: warm-start each solve from 2 p(n-1) - p(n-2) where a cell held pressure in
                                     both earlier substeps, instead of the reference's p(n-1) (linear_system.cpp:13-18);
                                     the solve still stops at the same relative residual */
} fe_tuning;
/* Applies `t` (the scene's captured substeps are captured again on the next step); multigrid = 1 allocates the
 * hierarchy on first use. */
fe_status fe_scene_set_tuning(fe_scene* s, const fe_tuning* t);
fe_status fe_scene_get_tuning(fe_scene* s, fe_tuning* t);
/* Search scope of the autotuner: every candidate, or only the launch shapes of the scene's current solver family
 * (plain or multigrid CG).  The family's iteration count can change over a run (the multigrid solver's grows as the
 * free surface gets ragged), so a family picked from the first substeps need not stay the faster one; the shape of
 * a given family does not depend on that. */
enum { FE_TUNE_ALL = 0, FE_TUNE_SHAPE = 1 };
/* The autotuner: times every candidate launch choice of the scene's pressure solve -- the plain CG at 256 / 512 /
 * 1024 threads per block, alone or in clusters of 2 blocks, and (grids with a multigrid hierarchy, no colliders)
 * the multigrid-preconditioned CG at 512 / 1024 threads with one-block levels up to 2048 or 4096 cells; with
 * FE_TUNE_SHAPE only the current family's --
 * over `substeps` substeps of dt each from the scene's current state (CUDA events on the scene's stream,
 * after one untimed substep that captures the choice's graphs), keeps the fastest whose solves all converged,
 * restores the scene's state and applies the choice.  The choice is also stored for (device, grid, transfer):
 * scenes created later with FE_PRESSURE_AUTO start from it.  best / best_ms (ms per substep) may be NULL. */
fe_status fe_scene_autotune(fe_scene* s, double dt, int32_t substeps, int32_t scope, fe_tuning* best,
                            float* best_ms);
/* The autotuner's per-process store (e.g. filled from a file a previous process wrote): */
fe_status fe_tuning_store(int32_t device, const int32_t n[3], int32_t solver, const fe_tuning* t);
fe_status fe_tuning_lookup(int32_t device, const int32_t n[3], int32_t solver, fe_tuning* t);  /* FE_ERR_STATE: none */

/* Per-job checkpoint / resume (no reference counterpart: FileSystem::SaveFrame, file_systems/file_system.cpp:14-17,
 * is empty).  fe_scene_snapshot copies the scene's state at a substep boundary on the device -- its particles in
 * slot order, the positions at the start of the last substep, the pressure warm start, the current velocity grid and
 * the counters that steer the next substeps -- into memory from the scene's device pool; fe_scene_restore puts it
 * back into a scene of the same grid, solver and device (the one it came from, or a fresh one), after which the scene
 * steps as the original did from that point (within the solve tolerance: the solver's reduction order varies). */
typedef struct fe_snapshot fe_snapshot;
fe_status fe_scene_snapshot(fe_scene* s, fe_snapshot** out);
fe_status fe_scene_restore(fe_scene* s, const fe_snapshot* snap);
fe_status fe_snapshot_info(const fe_snapshot* snap, uint64_t* particles, uint64_t* bytes);
fe_status fe_snapshot_destroy(fe_snapshot* snap);

/* Stream the scene's work is issued on (a cudaStream_t); NULL selects the scene's own stream. */
fe_status fe_scene_set_stream(fe_scene* s, void* stream);
fe_status fe_scene_synchronize(fe_scene* s);

/* Batches: many independent scenes (up to 64, one device) advanced together.  Per substep ONE cooperative
 * launch solves all scenes' pressure systems (each scene on its own block range, sized by its measured solve work,
 * with its own grid barrier, so the scenes iterate independently and concurrently).  Around it, each scene runs its
 * pre- and post-solve passes on its own stream, concurrently with the others; scenes selected by fe_batch_set_flat
 * instead run every pre- and post-solve pass (clears, sort, gather, P2G, marking, extrapolation + boundary
 * conditions + gravity, right-hand side; pressure apply, extrapolation + boundary conditions, transfer + move) as
 * ONE launch for all of them over a flat (scene, block) work list on the batch stream.  The batch substep is one
 * captured CUDA graph.  Scenes with viscosity or external forces always run their passes on their own streams.
 * Results equal each scene stepped alone (same algorithm, each scene's own tolerances).  No reference counterpart:
 * the reference runs one simulator per process (PhysicsAnimation::AdvanceSingleFrame, physics_animation.cpp:17-21). */
typedef struct fe_batch fe_batch;
fe_status fe_batch_create(fe_scene* const* scenes, int32_t count, fe_batch** out);
fe_status fe_batch_destroy(fe_batch* b);
/* Replaces the batch's scenes (same rules as fe_batch_create) without allocating or freeing device memory:
 * a server whose running set changes between frames keeps one batch; the batch graph is captured again
 * once the new membership has run a few substeps.  Waits for the batch's earlier work to finish. */
fe_status fe_batch_set_scenes(fe_batch* b, fe_scene* const* scenes, int32_t count);
/* Overlap mode (on != 0): instead of all scenes' pre-solve, then one multi-scene solve, then all post-solve, every
 * scene runs its whole substep on its own stream -- pre-solve, its own cooperative solve on its share of the
 * co-resident solver blocks (split by each scene's measured solve work; the shares add up to the device's
 * capacity, so every solve in flight fits at once), post-solve -- so one scene's latency-bound solve overlaps other
 * scenes' transfer kernels.  Same results; ignored while any scene has viscosity (its cooperative Jacobi solve
 * stays alone).  fe_batch_step_profiled always runs the phase-separated form. */
fe_status fe_batch_set_overlap(fe_batch* b, int32_t on);
/* Which scenes run in the flat launches: those of at most max_cells cells; 0 (the default) puts every scene on its
 * own stream, a negative value puts every scene (without viscosity or forces) in the flat launches.  Same results
 * either way; which is faster depends on the mix (fluide_engine_b200.autotune.tune_batch times the choices on the
 * batch's own substeps).  Waits for the batch's earlier work.  No reference counterpart. */
fe_status fe_batch_set_flat(fe_batch* b, int64_t max_cells);
/* nsub substeps of dt for every scene; stats (NULL or count * nsub entries, scene-major) as fe_scene_step. */
fe_status fe_batch_step(fe_batch* b, double dt, int32_t nsub, fe_step_stats* stats);
/* fe_batch_step with per-substep device timing of the batch's three phases (all scenes' pre-solve, the
 * multi-scene solve, all scenes' post-solve; events on the batch stream between them), launching the flat passes
 * directly (or, when the batch is not flat, replaying the scenes' own phase graphs around the solve launch);
 * phase_ms receives nsub * 3 floats; synchronises. */
fe_status fe_batch_step_profiled(fe_batch* b, double dt, int32_t nsub, fe_step_stats* stats, float* phase_ms);

/* Number of kernels the library launched since load (counts graph-launched kernels too). */
uint64_t fe_kernel_launch_count(void);

/* Failure-detection test hook (no reference counterpart: the reference has no error handling).  Sets, for the
 * current device, the bounded wait of the pressure solvers' grid barrier: spin_limit polls before a block gives
 * up (0 restores the default, a few seconds of polling), and extra_arrivals, arrivals the barrier waits for
 * beyond the launched blocks (0 in normal operation).  With extra_arrivals = 1 no barrier can complete: every
 * waiting block gives up after spin_limit polls, the solve ends, and the step returns FE_ERR_TIMEOUT with the
 * context usable; the scene's barrier words are reset, so once the limits are restored it steps normally.
 * Applies to launches (and graph replays) issued after the call. */
fe_status fe_debug_set_barrier_limits(uint64_t spin_limit, uint32_t extra_arrivals);

/* Deterministic seeding of analytic box / sphere regions (subcell-centre rule).  Region layout:
 * {int32 kind (0 box, 1 sphere); double lo[3]; double hi[3] (sphere: hi[0] = radius); double vel[3]}.
 * Returns the particle count; pos/vel (n*3 floats) are written when non-NULL, at most cap particles.
 * Replaces PICSimulator::InitializeParticles' std::rand() seeding (pic_simulator.cpp:521-548). */
uint64_t fe_seed_regions(const void* regions, int32_t nregions, const int32_t n[3], const double origin[3],
                         const double size[3], uint64_t seed, float* pos, float* vel, uint64_t cap);

/* Message of the last error on the calling thread ("" if none). */
const char* fe_last_error(void);

/* ABI version: major * 10000 + minor * 100 + patch. */
int32_t fe_abi_version(void);

#ifdef __cplusplus
}
#endif

#endif /* FLUIDE_B200_H */
