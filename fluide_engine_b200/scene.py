"""Scene: one device-resident simulation behind the C ABI (include/fluide_b200.h)."""
import ctypes

import numpy as np

from . import _abi
from ._abi import check, ptr


def _tri4(triangles):
    """Triangles as (T, 4) int64 (three vertex ids and an unused normal id), from (T, 3) or (T, 4)."""
    T = np.asarray(triangles, dtype=np.int64)
    if T.ndim == 2 and T.shape[1] == 3:
        T = np.concatenate([T, np.zeros((T.shape[0], 1), np.int64)], axis=1)
    return np.ascontiguousarray(T)


def face_shapes(n):
    """numpy shapes (z, y, x) of the u, v, w face arrays; memory is x-fastest like the reference's Array3."""
    nx, ny, nz = n
    return (nz, ny, nx + 1), (nz, ny + 1, nx), (nz + 1, ny, nx)


class Scene:
    """Owns an fe_scene.  All arrays exchanged are numpy (host) unless a torch CUDA tensor is passed."""

    def __init__(self, n, solver=_abi.FLIP, origin=(0.0, 0.0, 0.0), size=(1.0, 1.0, 1.0), flip_blend=0.05,
                 gravity=(0.0, -9.81, 0.0), max_cfl=1.0, cg_rel_tol=1e-6, cg_max_it=2000, cg_inner_tol=0.0,
                 max_refine=12, device=0, max_particles=0, pressure_solver=_abi.AUTO, viscosity=0.0):
        L = _abi.lib()
        d = _abi.SceneDesc()
        check(L.fe_scene_desc_default(ctypes.byref(d)))
        for a in range(3):
            d.n[a] = int(n[a])
            d.origin[a] = origin[a]
            d.size[a] = size[a]
            d.gravity[a] = gravity[a]
        d.solver, d.flip_blend, d.max_cfl = solver, flip_blend, max_cfl
        d.cg_rel_tol, d.cg_max_it, d.cg_inner_tol, d.max_refine = cg_rel_tol, cg_max_it, cg_inner_tol, max_refine
        d.device, d.max_particles, d.pressure_solver = device, max_particles, pressure_solver
        d.viscosity = viscosity
        h = ctypes.c_void_p()
        check(L.fe_scene_create(ctypes.byref(d), ctypes.byref(h)))
        self._h = h
        self._L = L
        self.n = tuple(int(x) for x in n)
        self.solver = solver
        self.desc = d

    def close(self):
        if getattr(self, "_h", None):
            self._L.fe_scene_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    # particles -----------------------------------------------------------------------------------
    def set_particles(self, pos, vel=None, C=None):
        pos = np.ascontiguousarray(pos, dtype=np.float32) if isinstance(pos, np.ndarray) else pos
        vel = np.ascontiguousarray(vel, dtype=np.float32) if isinstance(vel, np.ndarray) else vel
        C = np.ascontiguousarray(C, dtype=np.float32) if isinstance(C, np.ndarray) else C
        check(self._L.fe_scene_set_particles(self._h, ptr(pos), ptr(vel), ptr(C), int(pos.shape[0])))

    def reset(self):
        """Back to the freshly created state (grid, pressure warm start, solver scratch), keeping allocations."""
        check(self._L.fe_scene_reset(self._h))

    def num_particles(self):
        n = ctypes.c_uint64()
        check(self._L.fe_scene_num_particles(self._h, ctypes.byref(n)))
        return n.value

    def particles(self):
        N = self.num_particles()
        pos = np.zeros((N, 3), dtype=np.float32)
        vel = np.zeros((N, 3), dtype=np.float32)
        C = np.zeros((N, 9), dtype=np.float32)
        check(self._L.fe_scene_get_particles(self._h, ptr(pos), ptr(vel), ptr(C), N))
        return pos, vel, C

    # stepping ------------------------------------------------------------------------------------
    def step(self, dt, nsub=1, stats=True):
        if stats:
            arr = (_abi.StepStats * max(nsub, 1))()
            check(self._L.fe_scene_step(self._h, dt, nsub, arr))
            return [arr[i].as_dict() for i in range(nsub)]
        check(self._L.fe_scene_step(self._h, dt, nsub, None))
        return None

    def step_profiled(self, dt, nsub):
        """Like step(), plus per-substep phase times in ms: array [nsub, 3] = (pre-solve, CG solve, post-solve)."""
        arr = (_abi.StepStats * max(nsub, 1))()
        ms = np.zeros((max(nsub, 1), 3), dtype=np.float32)
        check(self._L.fe_scene_step_profiled(self._h, dt, nsub, arr, ms.ctypes.data_as(ctypes.POINTER(ctypes.c_float))))
        return [arr[i].as_dict() for i in range(nsub)], ms[:nsub]

    def checkpoint(self):
        """The scene's state at this substep boundary, on the device (fe_scene_snapshot): a Snapshot to restore
        into this scene or another one of the same grid and solver."""
        h = ctypes.c_void_p()
        check(self._L.fe_scene_snapshot(self._h, ctypes.byref(h)))
        return Snapshot(h, self._L)

    def restore(self, snap):
        check(self._L.fe_scene_restore(self._h, snap.handle))

    def set_tuning(self, multigrid=-1, cg_block_threads=0, mg_block_level_cells=0, cg_cluster=0,
                   pressure_extrapolation=-1):
        """Launch choices of the pressure solve (fe_scene_set_tuning); -1 / 0 keeps a field's current choice."""
        t = _abi.Tuning(int(multigrid), int(cg_block_threads), int(mg_block_level_cells), int(cg_cluster),
                        int(pressure_extrapolation))
        check(self._L.fe_scene_set_tuning(self._h, ctypes.byref(t)))

    def tuning(self):
        t = _abi.Tuning()
        check(self._L.fe_scene_get_tuning(self._h, ctypes.byref(t)))
        return {"multigrid": t.multigrid, "cg_block_threads": t.cg_block_threads,
                "mg_block_level_cells": t.mg_block_level_cells, "cg_cluster": t.cg_cluster,
                "pressure_extrapolation": t.pressure_extrapolation}

    def set_stream(self, stream_handle):
        """Issues the scene's work on an external cudaStream_t (an int handle, e.g. torch stream.cuda_stream)."""
        check(self._L.fe_scene_set_stream(self._h, ctypes.c_void_p(stream_handle) if stream_handle else None))

    def advance_frame(self, frame_dt):
        n = ctypes.c_int32()
        check(self._L.fe_scene_advance_frame(self._h, frame_dt, ctypes.byref(n)))
        return n.value

    def run_stages(self, dt, first, last):
        check(self._L.fe_scene_run_stages(self._h, dt, first, last))

    def cfl(self, dt):
        c = ctypes.c_double()
        check(self._L.fe_scene_cfl(self._h, dt, ctypes.byref(c)))
        return c.value

    def synchronize(self):
        check(self._L.fe_scene_synchronize(self._h))

    # grid ----------------------------------------------------------------------------------------
    def grid(self):
        su, sv, sw = face_shapes(self.n)
        u, v, w = (np.zeros(s, dtype=np.float32) for s in (su, sv, sw))
        nx, ny, nz = self.n
        p = np.zeros((nz, ny, nx), dtype=np.float64)
        m = np.zeros((nz, ny, nx), dtype=np.uint8)
        check(self._L.fe_scene_get_grid(self._h, ptr(u), ptr(v), ptr(w), ptr(p), ptr(m)))
        return u, v, w, p, m

    def set_grid(self, u, v, w):
        u, v, w = (np.ascontiguousarray(a, dtype=np.float32) for a in (u, v, w))
        check(self._L.fe_scene_set_grid(self._h, ptr(u), ptr(v), ptr(w)))

    def set_pressure(self, p):
        p = np.ascontiguousarray(p, dtype=np.float64)
        check(self._L.fe_scene_set_pressure(self._h, ptr(p)))

    def face_markers(self):
        su, sv, sw = face_shapes(self.n)
        a, b, c = (np.zeros(s, dtype=np.uint8) for s in (su, sv, sw))
        check(self._L.fe_scene_get_face_markers(self._h, ptr(a), ptr(b), ptr(c)))
        return a, b, c

    def snapshot(self):
        su, sv, sw = face_shapes(self.n)
        a, b, c = (np.zeros(s, dtype=np.float32) for s in (su, sv, sw))
        check(self._L.fe_scene_get_snapshot(self._h, ptr(a), ptr(b), ptr(c)))
        return a, b, c

    def rhs(self):
        nx, ny, nz = self.n
        b = np.zeros((nz, ny, nx), dtype=np.float64)
        check(self._L.fe_scene_get_rhs(self._h, ptr(b)))
        return b

    def fluid_sdf(self):
        nx, ny, nz = self.n
        s = np.zeros((nz, ny, nx), dtype=np.float64)
        check(self._L.fe_scene_get_fluid_sdf(self._h, ptr(s)))
        return s

    def init_from_mesh(self, vertices, triangles, particles_per_cell=0, seed=0):
        """InitializeFromTriangleMesh: mesh SDF as the fluid SDF, particles appended in the cells inside it."""
        V = np.ascontiguousarray(vertices, dtype=np.float64)
        T = _tri4(triangles)
        check(self._L.fe_scene_init_from_mesh(self._h, ptr(V), V.shape[0], ptr(T), T.shape[0], particles_per_cell, seed))

    def add_volume_emitter(self, vertices, triangles, resolution, domain_origin, domain_size, particles_per_block=8,
                           velocity=(0.0, 0.0, 0.0), seed=0):
        """VolumeEmitter: emits at the start of every substep; returns its id."""
        V = np.ascontiguousarray(vertices, dtype=np.float64)
        T = _tri4(triangles)
        eid = ctypes.c_int32()
        check(self._L.fe_scene_add_volume_emitter(
            self._h, ptr(V), V.shape[0], ptr(T), T.shape[0], (ctypes.c_int32 * 3)(*resolution),
            (ctypes.c_double * 3)(*domain_origin), (ctypes.c_double * 3)(*domain_size), particles_per_block,
            (ctypes.c_double * 3)(*velocity), seed, ctypes.byref(eid)))
        return eid.value

    def set_emitter_sdf(self, emitter_id, sdf):
        """VolumeEmitter::InitializeFromSdf: node values on the emitter's grid, shape (nz, ny, nx)."""
        S = np.ascontiguousarray(sdf, dtype=np.float64)
        check(self._L.fe_scene_set_emitter_sdf(self._h, emitter_id, ptr(S)))

    def add_point_field(self, origin, strength, falloff=1.0):
        """PointField after gravity in the force list (fe_scene_add_force); returns its index."""
        return self._add_force(_abi.force_desc(_abi.FORCE_POINT, origin=origin, strength=strength, falloff=falloff))

    def add_swirl_field(self, origin, axis, strength, falloff=1.0):
        """SwirlField (the axis is normalised as the reference's constructor does)."""
        return self._add_force(_abi.force_desc(_abi.FORCE_SWIRL, origin=origin, axis=axis, strength=strength,
                                               falloff=falloff))

    def add_volume_field(self, vertices, triangles, resolution, domain_origin, domain_size, strength, field=None):
        """VolumeField of a mesh on its own node grid (vectors computed on the GPU unless `field` is given)."""
        return self._add_force(_abi.force_desc(_abi.FORCE_VOLUME, strength=strength, vertices=vertices,
                                               triangles=triangles, resolution=resolution,
                                               domain_origin=domain_origin, domain_size=domain_size, field=field))

    def _add_force(self, desc_keep):
        desc, _keep = desc_keep
        fid = ctypes.c_int32()
        check(self._L.fe_scene_add_force(self._h, ctypes.byref(desc), ctypes.byref(fid)))
        return fid.value

    def add_mesh_collider(self, vertices, triangles, normals, resolution, grid_origin, grid_spacing):
        """TriangleMeshCollider on its own node grid (triangles (T, 4): vertex ids and a normal id into normals)."""
        V = np.ascontiguousarray(vertices, dtype=np.float64)
        T = np.ascontiguousarray(triangles, dtype=np.int64)
        N = np.ascontiguousarray(normals, dtype=np.float64)
        cid = ctypes.c_int32()
        check(self._L.fe_scene_add_mesh_collider(self._h, ptr(V), V.shape[0], ptr(T), T.shape[0], ptr(N), N.shape[0],
                                                 (ctypes.c_int32 * 3)(*resolution), (ctypes.c_double * 3)(*grid_origin),
                                                 (ctypes.c_double * 3)(*grid_spacing), ctypes.byref(cid)))
        return cid.value

    def clear_colliders(self):
        check(self._L.fe_scene_clear_colliders(self._h))

    def collider_sdf(self):
        nx, ny, nz = self.n
        out = np.zeros((nz, ny, nx))
        check(self._L.fe_scene_get_collider_sdf(self._h, ptr(out)))
        return out

    def clear_forces(self):
        check(self._L.fe_scene_clear_forces(self._h))

    def set_fluid_sdf(self, sdf):
        """Fluid3::sdf until the next substep (as after init_from_mesh), shape (nz, ny, nx)."""
        S = np.ascontiguousarray(sdf, dtype=np.float64)
        check(self._L.fe_scene_set_fluid_sdf(self._h, ptr(S)))

    def clear_emitters(self):
        check(self._L.fe_scene_clear_emitters(self._h))

    def surface(self):
        """GetSurface: (vertices (V,3) f64, normals (V,3) f64, triangles (T,4) int64: vertex ids, normal id)."""
        nv, nt = ctypes.c_uint64(), ctypes.c_uint64()
        check(self._L.fe_scene_build_surface(self._h, ctypes.byref(nv), ctypes.byref(nt)))
        V = np.zeros((nv.value, 3)); N = np.zeros((nv.value, 3)); T = np.zeros((nt.value, 4), dtype=np.int64)
        check(self._L.fe_scene_get_surface(self._h, ptr(V), ptr(N), ptr(T)))
        return V, N, T

    def write_surface_obj(self, path, name=""):
        """Builds the surface and writes it as OBJManager::Save does."""
        check(self._L.fe_scene_build_surface(self._h, None, None))
        check(self._L.fe_scene_write_surface_obj(self._h, str(path).encode(), name.encode()))

    def set_viscosity(self, viscosity):
        check(self._L.fe_scene_set_viscosity(self._h, float(viscosity)))
        self.desc.viscosity = float(viscosity)

    def diffusion(self):
        """(Jacobi iterations per component, (mu, mv, mw) FLUID face markers) of the last viscosity solve."""
        return self.diffusion_info()[:2]

    def diffusion_info(self):
        """As diffusion(), plus the relaxation passes the GPU ran."""
        its = np.zeros(4, dtype=np.int32)
        su, sv, sw = face_shapes(self.n)
        a, b, c = (np.zeros(s, dtype=np.uint8) for s in (su, sv, sw))
        check(self._L.fe_scene_get_diffusion(self._h, ptr(its), ptr(a), ptr(b), ptr(c)))
        return tuple(int(x) for x in its[:3]), (a, b, c), int(its[3])

    def sort_result(self):
        N = self.num_particles()
        keys = np.zeros(N, dtype=np.uint32)
        perm = np.zeros(N, dtype=np.uint32)
        check(self._L.fe_scene_get_sort(self._h, ptr(keys), ptr(perm), N))
        return keys, perm

    def divergence(self):
        d = ctypes.c_double()
        check(self._L.fe_scene_divergence(self._h, ctypes.byref(d)))
        return d.value


class Snapshot:
    """A device-side checkpoint of a scene (fe_snapshot); freed by close() or when collected."""

    def __init__(self, handle, L):
        self._h = handle
        self._L = L

    @property
    def handle(self):
        if self._h is None:
            raise ValueError("snapshot is closed")
        return self._h

    def info(self):
        n, b = ctypes.c_uint64(), ctypes.c_uint64()
        check(self._L.fe_snapshot_info(self.handle, ctypes.byref(n), ctypes.byref(b)))
        return {"particles": int(n.value), "bytes": int(b.value)}

    def close(self):
        if self._h is not None:
            self._L.fe_snapshot_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Many scenes advanced together (fe_batch_*): one batched pressure solve per substep; the small scenes' transfer
    and grid passes as one launch per pass for all of them, the larger scenes' on their own streams; one CUDA
    graph per substep."""

    def __init__(self, scenes):
        self.scenes = list(scenes)
        self._L = _abi.lib()
        arr = (ctypes.c_void_p * len(self.scenes))(*[s.handle.value for s in self.scenes])
        h = ctypes.c_void_p()
        check(self._L.fe_batch_create(arr, len(self.scenes), ctypes.byref(h)))
        self._h = h

    def set_overlap(self, on=True):
        """Overlap mode (fe_batch_set_overlap): each scene's whole substep on its own stream, its solve on its
        share of the solver blocks, so solves overlap other scenes' transfer kernels."""
        check(self._L.fe_batch_set_overlap(self._h, 1 if on else 0))

    def set_flat(self, max_cells=-1):
        """Scenes of at most max_cells cells run every pre- and post-solve pass as one launch for all of them over a
        (scene, block) work list (fe_batch_set_flat); larger scenes run their passes on their own streams.  0 (the
        library's default): no scene in the flat launches; -1: every scene.  True / False select -1 / 0.
        autotune.tune_batch picks the threshold by timing."""
        if max_cells is True:
            max_cells = -1
        elif max_cells is False:
            max_cells = 0
        check(self._L.fe_batch_set_flat(self._h, int(max_cells)))

    def set_scenes(self, scenes):
        """Changes the batch's scenes in place (no device allocation)."""
        scenes = list(scenes)
        arr = (ctypes.c_void_p * len(scenes))(*[s.handle.value for s in scenes])
        check(self._L.fe_batch_set_scenes(self._h, arr, len(scenes)))
        self.scenes = scenes

    def step(self, dt, nsub=1, stats=True):
        S = len(self.scenes)
        if stats:
            arr = (_abi.StepStats * max(1, S * nsub))()
            check(self._L.fe_batch_step(self._h, dt, nsub, arr))
            return [[arr[i * nsub + k].as_dict() for k in range(nsub)] for i in range(S)]
        check(self._L.fe_batch_step(self._h, dt, nsub, None))
        return None

    def step_profiled(self, dt, nsub):
        """Like step(), plus per-substep phase times in ms: array [nsub, 3] = (all pre-solve, multi-scene solve,
        all post-solve); returns (stats per scene per substep, times)."""
        S = len(self.scenes)
        arr = (_abi.StepStats * max(1, S * nsub))()
        ms = np.zeros((max(nsub, 1), 3), dtype=np.float32)
        check(self._L.fe_batch_step_profiled(self._h, dt, nsub, arr,
                                             ms.ctypes.data_as(ctypes.POINTER(ctypes.c_float))))
        return [[arr[i * nsub + k].as_dict() for k in range(nsub)] for i in range(S)], ms[:nsub]

    def close(self):
        if getattr(self, "_h", None):
            self._L.fe_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
