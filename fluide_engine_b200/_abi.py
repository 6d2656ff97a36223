"""ctypes binding of the C ABI declared in include/fluide_b200.h.

The product path is the sm_100a library libfluide_b200.so built in-tree by build.py; importing this
module never falls back to anything else: if the library is missing it raises.
"""
import ctypes
import os

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libfluide_b200.so")

FE_OK = 0
TUNE_ALL, TUNE_SHAPE = 0, 1
FE_ERR_CUDA, FE_ERR_BAD_ARG, FE_ERR_OOM, FE_ERR_NOT_CONVERGED, FE_ERR_TIMEOUT, FE_ERR_STATE, FE_ERR_NO_DEVICE = range(1, 8)
PIC, FLIP, APIC = 0, 1, 2
AUTO, MGPCG, CG = 0, 1, 2  # fe_pressure_solver
AIR, FLUID, BOUNDRY = 0, 1, 2
(STAGE_SORT, STAGE_P2G, STAGE_MARK, STAGE_PRE, STAGE_DIFFUSE, STAGE_PRESSURE, STAGE_POST, STAGE_G2P,
 STAGE_MOVE) = range(9)

STATUS_NAMES = {0: "FE_OK", 1: "FE_ERR_CUDA", 2: "FE_ERR_BAD_ARG", 3: "FE_ERR_OOM", 4: "FE_ERR_NOT_CONVERGED",
                5: "FE_ERR_TIMEOUT", 6: "FE_ERR_STATE", 7: "FE_ERR_NO_DEVICE"}

# Every symbol include/fluide_b200.h declares (checked by the CPU test suite).
EXPORTS = [
    "fe_scene_desc_default", "fe_scene_create", "fe_scene_destroy", "fe_scene_set_particles", "fe_scene_reset",
    "fe_scene_get_particles",
    "fe_scene_num_particles", "fe_scene_step", "fe_scene_step_profiled", "fe_scene_advance_frame", "fe_scene_cfl", "fe_scene_run_stages",
    "fe_scene_get_grid", "fe_scene_set_grid", "fe_scene_set_pressure", "fe_scene_get_face_markers",
    "fe_scene_get_snapshot", "fe_scene_get_rhs", "fe_scene_get_fluid_sdf", "fe_scene_set_viscosity",
    "fe_scene_get_diffusion", "fe_scene_build_surface", "fe_scene_get_surface", "fe_scene_write_surface_obj",
    "fe_write_obj", "fe_mesh_to_sdf", "fe_scene_init_from_mesh", "fe_scene_add_volume_emitter", "fe_scene_clear_emitters",
    "fe_scene_set_emitter_sdf", "fe_scene_set_fluid_sdf", "fe_scene_add_force", "fe_scene_clear_forces",
    "fe_volume_field_vectors", "fe_scene_add_mesh_collider", "fe_scene_clear_colliders", "fe_scene_get_collider_sdf",
    "fe_scene_get_sort", "fe_scene_divergence",
    "fe_scene_set_stream", "fe_scene_synchronize", "fe_project_noalloc", "fe_batch_create", "fe_batch_destroy", "fe_batch_set_scenes",
    "fe_batch_step", "fe_batch_step_profiled", "fe_kernel_launch_count", "fe_seed_regions", "fe_last_error",
    "fe_abi_version", "fe_debug_set_barrier_limits", "fe_scene_set_tuning", "fe_scene_get_tuning",
    "fe_scene_snapshot", "fe_scene_restore", "fe_snapshot_info", "fe_snapshot_destroy",
    "fe_scene_autotune", "fe_tuning_store", "fe_tuning_lookup", "fe_batch_set_overlap",
    "fe_batch_set_flat",
]


class FluideError(RuntimeError):
    def __init__(self, status, message):
        super().__init__("%s: %s" % (STATUS_NAMES.get(status, status), message))
        self.status = status


class SceneDesc(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int32 * 3), ("origin", ctypes.c_double * 3), ("size", ctypes.c_double * 3),
                ("solver", ctypes.c_int32), ("flip_blend", ctypes.c_double), ("gravity", ctypes.c_double * 3),
                ("max_cfl", ctypes.c_double), ("cg_rel_tol", ctypes.c_double), ("cg_max_it", ctypes.c_int32),
                ("cg_inner_tol", ctypes.c_double), ("max_refine", ctypes.c_int32), ("device", ctypes.c_int32),
                ("max_particles", ctypes.c_uint64), ("pressure_solver", ctypes.c_int32), ("viscosity", ctypes.c_double)]


class Tuning(ctypes.Structure):
    _fields_ = [("multigrid", ctypes.c_int32), ("cg_block_threads", ctypes.c_int32),
                ("mg_block_level_cells", ctypes.c_int32), ("cg_cluster", ctypes.c_int32),
                ("pressure_extrapolation", ctypes.c_int32)]


class StepStats(ctypes.Structure):
    _fields_ = [("cg_iterations", ctypes.c_int32), ("refinements", ctypes.c_int32), ("converged", ctypes.c_int32),
                ("fluid_cells", ctypes.c_int32), ("rel_residual", ctypes.c_double), ("b_norm", ctypes.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


FORCE_POINT, FORCE_SWIRL, FORCE_VOLUME = 1, 2, 3


class ForceDesc(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("origin", ctypes.c_double * 3), ("axis", ctypes.c_double * 3),
                ("strength", ctypes.c_double), ("falloff", ctypes.c_double),
                ("vertices", ctypes.c_void_p), ("n_vertices", ctypes.c_uint64),
                ("triangles", ctypes.c_void_p), ("n_triangles", ctypes.c_uint64),
                ("resolution", ctypes.c_int32 * 3), ("domain_origin", ctypes.c_double * 3),
                ("domain_size", ctypes.c_double * 3), ("field", ctypes.c_void_p)]


class Region(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("lo", ctypes.c_double * 3), ("hi", ctypes.c_double * 3),
                ("vel", ctypes.c_double * 3)]


_lib = None


def lib():
    """Loads libfluide_b200.so (building it first when nvcc is available and the library is stale)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH) and os.path.exists("/usr/local/cuda/bin/nvcc"):
        from . import build as _build
        _build.build()
    if not os.path.exists(LIB_PATH):
        raise ImportError("libfluide_b200.so is not built (run python fluide_engine_b200/build.py)")
    L = ctypes.CDLL(LIB_PATH)
    P = ctypes.c_void_p
    F = ctypes.POINTER(ctypes.c_float)
    D = ctypes.POINTER(ctypes.c_double)
    U8 = ctypes.POINTER(ctypes.c_uint8)
    U32 = ctypes.POINTER(ctypes.c_uint32)
    I = ctypes.c_int
    L.fe_scene_desc_default.argtypes = [ctypes.POINTER(SceneDesc)]
    L.fe_scene_create.argtypes = [ctypes.POINTER(SceneDesc), ctypes.POINTER(P)]
    L.fe_scene_destroy.argtypes = [P]
    L.fe_scene_set_particles.argtypes = [P, P, P, P, ctypes.c_uint64]
    L.fe_scene_reset.argtypes = [P]
    L.fe_scene_get_particles.argtypes = [P, P, P, P, ctypes.c_uint64]
    L.fe_scene_num_particles.argtypes = [P, ctypes.POINTER(ctypes.c_uint64)]
    L.fe_scene_step.argtypes = [P, ctypes.c_double, ctypes.c_int32, ctypes.POINTER(StepStats)]
    L.fe_scene_step_profiled.argtypes = [P, ctypes.c_double, ctypes.c_int32, ctypes.POINTER(StepStats),
                                         ctypes.POINTER(ctypes.c_float)]
    L.fe_scene_advance_frame.argtypes = [P, ctypes.c_double, ctypes.POINTER(ctypes.c_int32)]
    L.fe_scene_cfl.argtypes = [P, ctypes.c_double, D]
    L.fe_scene_run_stages.argtypes = [P, ctypes.c_double, ctypes.c_int32, ctypes.c_int32]
    L.fe_scene_get_grid.argtypes = [P, P, P, P, P, P]
    L.fe_scene_set_grid.argtypes = [P, P, P, P]
    L.fe_scene_set_pressure.argtypes = [P, P]
    L.fe_scene_get_face_markers.argtypes = [P, P, P, P]
    L.fe_scene_get_snapshot.argtypes = [P, P, P, P]
    L.fe_scene_get_rhs.argtypes = [P, P]
    L.fe_scene_get_fluid_sdf.argtypes = [P, P]
    L.fe_scene_set_viscosity.argtypes = [P, ctypes.c_double]
    L.fe_scene_get_diffusion.argtypes = [P, P, P, P, P]
    L.fe_scene_build_surface.argtypes = [P, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64)]
    L.fe_scene_get_surface.argtypes = [P, P, P, P]
    L.fe_scene_write_surface_obj.argtypes = [P, ctypes.c_char_p, ctypes.c_char_p]
    L.fe_write_obj.argtypes = [ctypes.c_char_p, ctypes.c_char_p, P, P, ctypes.c_uint64, P, ctypes.c_uint64]
    L.fe_mesh_to_sdf.argtypes = [P, ctypes.c_uint64, P, ctypes.c_uint64, P, P, P, P, ctypes.c_int32]
    L.fe_scene_init_from_mesh.argtypes = [P, P, ctypes.c_uint64, P, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint64]
    L.fe_scene_add_volume_emitter.argtypes = [P, P, ctypes.c_uint64, P, ctypes.c_uint64, P, P, P, ctypes.c_uint32, P,
                                              ctypes.c_uint64, ctypes.POINTER(ctypes.c_int32)]
    L.fe_scene_clear_emitters.argtypes = [P]
    L.fe_scene_set_emitter_sdf.argtypes = [P, ctypes.c_int32, P]
    L.fe_scene_set_fluid_sdf.argtypes = [P, P]
    L.fe_scene_add_force.argtypes = [P, ctypes.POINTER(ForceDesc), ctypes.POINTER(ctypes.c_int32)]
    L.fe_scene_clear_forces.argtypes = [P]
    L.fe_scene_add_mesh_collider.argtypes = [P, P, ctypes.c_uint64, P, ctypes.c_uint64, P, ctypes.c_uint64, P, P, P,
                                             ctypes.POINTER(ctypes.c_int32)]
    L.fe_scene_clear_colliders.argtypes = [P]
    L.fe_scene_get_collider_sdf.argtypes = [P, P]
    L.fe_volume_field_vectors.argtypes = [P, ctypes.c_uint64, P, ctypes.c_uint64, P, P, P, P, ctypes.c_int32]
    L.fe_scene_get_sort.argtypes = [P, P, P, ctypes.c_uint64]
    L.fe_scene_divergence.argtypes = [P, D]
    L.fe_scene_set_stream.argtypes = [P, P]
    L.fe_project_noalloc.argtypes = [P, P, P, P, P, P, P, ctypes.c_double, ctypes.c_int32, P,
                                     ctypes.POINTER(StepStats)]
    L.fe_scene_synchronize.argtypes = [P]
    L.fe_batch_create.argtypes = [ctypes.POINTER(P), ctypes.c_int32, ctypes.POINTER(P)]
    L.fe_batch_set_scenes.argtypes = [P, ctypes.POINTER(P), ctypes.c_int32]
    L.fe_batch_destroy.argtypes = [P]
    L.fe_batch_set_overlap.argtypes = [P, ctypes.c_int32]
    L.fe_batch_set_flat.argtypes = [P, ctypes.c_int64]
    L.fe_batch_step.argtypes = [P, ctypes.c_double, ctypes.c_int32, ctypes.POINTER(StepStats)]
    L.fe_batch_step_profiled.argtypes = [P, ctypes.c_double, ctypes.c_int32, ctypes.POINTER(StepStats),
                                         ctypes.POINTER(ctypes.c_float)]
    L.fe_kernel_launch_count.restype = ctypes.c_uint64
    L.fe_debug_set_barrier_limits.argtypes = [ctypes.c_uint64, ctypes.c_uint32]
    L.fe_scene_set_tuning.argtypes = [P, ctypes.POINTER(Tuning)]
    L.fe_scene_get_tuning.argtypes = [P, ctypes.POINTER(Tuning)]
    L.fe_scene_snapshot.argtypes = [P, ctypes.POINTER(P)]
    L.fe_scene_restore.argtypes = [P, P]
    L.fe_snapshot_info.argtypes = [P, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64)]
    L.fe_snapshot_destroy.argtypes = [P]
    L.fe_scene_autotune.argtypes = [P, ctypes.c_double, ctypes.c_int32, ctypes.c_int32, ctypes.POINTER(Tuning),
                                    ctypes.POINTER(ctypes.c_float)]
    L.fe_tuning_store.argtypes = [ctypes.c_int32, P, ctypes.c_int32, ctypes.POINTER(Tuning)]
    L.fe_tuning_lookup.argtypes = [ctypes.c_int32, P, ctypes.c_int32, ctypes.POINTER(Tuning)]
    L.fe_seed_regions.restype = ctypes.c_uint64
    L.fe_seed_regions.argtypes = [P, ctypes.c_int32, P, P, P, ctypes.c_uint64, P, P, ctypes.c_uint64]
    L.fe_last_error.restype = ctypes.c_char_p
    L.fe_abi_version.restype = ctypes.c_int32
    for name in EXPORTS:
        fn = getattr(L, name)
        if fn.restype is ctypes.c_int or fn.restype is None:
            fn.restype = ctypes.c_int
    L.fe_kernel_launch_count.restype = ctypes.c_uint64
    L.fe_seed_regions.restype = ctypes.c_uint64
    L.fe_last_error.restype = ctypes.c_char_p
    _lib = L
    return L


def check(status):
    if status != FE_OK:
        raise FluideError(status, lib().fe_last_error().decode(errors="replace"))


def ptr(a):
    """Raw pointer of a numpy array, a torch tensor (host or device) or None."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        assert a.flags["C_CONTIGUOUS"]
        return ctypes.c_void_p(a.ctypes.data)
    if hasattr(a, "data_ptr"):
        assert a.is_contiguous()
        return ctypes.c_void_p(a.data_ptr())
    if isinstance(a, int):
        return ctypes.c_void_p(a)
    raise TypeError("unsupported buffer type %r" % type(a))


def kernel_launch_count():
    return int(lib().fe_kernel_launch_count())


def set_barrier_limits(spin_limit=0, extra_arrivals=0):
    """Failure-detection test hook: the pressure solvers' bounded barrier wait on the current device
    (fe_debug_set_barrier_limits; spin_limit 0 and extra_arrivals 0 restore normal operation)."""
    check(lib().fe_debug_set_barrier_limits(int(spin_limit), int(extra_arrivals)))


def seed_regions(regions, n, origin=(0.0, 0.0, 0.0), size=(1.0, 1.0, 1.0), seed=0):
    """Seeds particles with the library's subcell rule.  regions: dicts {kind 0 box/1 sphere, lo, hi, vel}."""
    L = lib()
    arr = (Region * len(regions))()
    for i, r in enumerate(regions):
        arr[i].kind = r.get("kind", 0)
        for a in range(3):
            arr[i].lo[a] = r["lo"][a]
            arr[i].hi[a] = r["hi"][a] if a < len(r["hi"]) else 0.0
            arr[i].vel[a] = r.get("vel", (0.0, 0.0, 0.0))[a]
    n3 = (ctypes.c_int32 * 3)(*n)
    o = (ctypes.c_double * 3)(*origin)
    s = (ctypes.c_double * 3)(*size)
    cnt = L.fe_seed_regions(ctypes.cast(arr, ctypes.c_void_p), len(regions), n3, o, s, seed, None, None, 0)
    pos = np.zeros((cnt, 3), dtype=np.float32)
    vel = np.zeros((cnt, 3), dtype=np.float32)
    L.fe_seed_regions(ctypes.cast(arr, ctypes.c_void_p), len(regions), n3, o, s, seed, ptr(pos), ptr(vel), cnt)
    return pos, vel


def volume_field_vectors(vertices, triangles, n, origin, spacing, device=0):
    """VolumeField::Initialize's closest-point vectors on the GPU (fe_volume_field_vectors): (nz, ny, nx, 3)."""
    L = lib()
    V = np.ascontiguousarray(vertices, dtype=np.float64)
    T = np.ascontiguousarray(triangles, dtype=np.int64)
    if T.ndim == 2 and T.shape[1] == 3:
        T = np.ascontiguousarray(np.concatenate([T, np.zeros((T.shape[0], 1), np.int64)], axis=1))
    out = np.zeros((n[2], n[1], n[0], 3))
    check(L.fe_volume_field_vectors(ptr(V), V.shape[0], ptr(T), T.shape[0], (ctypes.c_int32 * 3)(*n),
                                    (ctypes.c_double * 3)(*origin), (ctypes.c_double * 3)(*spacing), ptr(out), device))
    return out


def force_desc(kind, origin=(0.0, 0.0, 0.0), axis=(0.0, 1.0, 0.0), strength=0.0, falloff=1.0, vertices=None,
               triangles=None, resolution=(1, 1, 1), domain_origin=(0.0, 0.0, 0.0), domain_size=(1.0, 1.0, 1.0),
               field=None):
    """An fe_force_desc; the arrays it points to are returned alongside and must outlive the call."""
    d = ForceDesc()
    d.kind = kind
    d.origin[:] = origin
    d.axis[:] = axis
    d.strength = strength
    d.falloff = falloff
    keep = []
    if vertices is not None:
        V = np.ascontiguousarray(vertices, dtype=np.float64)
        T = np.asarray(triangles, dtype=np.int64)
        if T.ndim == 2 and T.shape[1] == 3:
            T = np.concatenate([T, np.zeros((T.shape[0], 1), np.int64)], axis=1)
        T = np.ascontiguousarray(T)
        keep += [V, T]
        d.vertices, d.n_vertices = V.ctypes.data, V.shape[0]
        d.triangles, d.n_triangles = T.ctypes.data, T.shape[0]
    d.resolution[:] = resolution
    d.domain_origin[:] = domain_origin
    d.domain_size[:] = domain_size
    if field is not None:
        F = np.ascontiguousarray(field, dtype=np.float64)
        keep.append(F)
        d.field = F.ctypes.data
    return d, keep


def mesh_to_sdf(vertices, triangles, n, origin, spacing, device=0):
    """Mesh2SDF::Build on the GPU (fe_mesh_to_sdf): node values (nz, ny, nx) float64."""
    L = lib()
    V = np.ascontiguousarray(vertices, dtype=np.float64)
    T = np.ascontiguousarray(triangles, dtype=np.int64)
    if T.ndim == 2 and T.shape[1] == 3:
        T = np.ascontiguousarray(np.concatenate([T, np.zeros((T.shape[0], 1), np.int64)], axis=1))
    out = np.zeros((n[2], n[1], n[0]))
    n3 = (ctypes.c_int32 * 3)(*n)
    o = (ctypes.c_double * 3)(*origin)
    h = (ctypes.c_double * 3)(*spacing)
    check(L.fe_mesh_to_sdf(ptr(V), V.shape[0], ptr(T), T.shape[0], n3, o, h, ptr(out), device))
    return out
