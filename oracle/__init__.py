"""Oracle package -- TEST INFRASTRUCTURE ONLY.

Loads (and, when missing or stale, compiles with gcc) the CPU FP64 restatement of the reference
substep in fe_oracle.c, and wraps the reference's own CPU simulator built by build_ref.py.  Only the
tests, the smoke check and bench.py's CPU-baseline leg may import this package; the product path
never does.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")

PIC, FLIP, APIC = 0, 1, 2
AIR, FLUID, BOUNDRY = 0, 1, 2

_lib = None


def build_oracle(force=False):
    """Compiles fe_oracle.c into liboracle.so (FP64, no FMA contraction)."""
    srcs = [os.path.join(HERE, "fe_oracle.c"), os.path.join(HERE, "fe_oracle.h"),
            os.path.join(HERE, "..", "fluide_engine_b200", "csrc", "fe_keys.h"),
            os.path.join(HERE, "..", "fluide_engine_b200", "csrc", "fe_seed.h"),
            os.path.join(HERE, "..", "fluide_engine_b200", "csrc", "fe_mc_tables.h")]
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= max(os.path.getmtime(s) for s in srcs):
        return LIB
    cmd = ["gcc", "-O2", "-std=c11", "-ffp-contract=off", "-fPIC", "-shared", "-o", LIB,
           os.path.join(HERE, "fe_oracle.c"), "-lm"]
    subprocess.run(cmd, check=True)
    return LIB


class _Desc(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int * 3), ("origin", ctypes.c_double * 3), ("size", ctypes.c_double * 3),
                ("solver", ctypes.c_int), ("blend", ctypes.c_double), ("gravity", ctypes.c_double * 3),
                ("max_cfl", ctypes.c_double), ("cg_rel_tol", ctypes.c_double), ("cg_max_it", ctypes.c_int),
                ("viscosity", ctypes.c_double)]


class Region(ctypes.Structure):
    """Mirror of fe_region (fluide_engine_b200/csrc/fe_seed.h)."""
    _fields_ = [("kind", ctypes.c_int), ("lo", ctypes.c_double * 3), ("hi", ctypes.c_double * 3),
                ("vel", ctypes.c_double * 3)]


def lib():
    global _lib
    if _lib is None:
        build_oracle()
        L = ctypes.CDLL(LIB)
        P = ctypes.c_void_p
        D = ctypes.POINTER(ctypes.c_double)
        L.or_create.restype = P
        L.or_create.argtypes = [ctypes.POINTER(_Desc)]
        L.or_destroy.argtypes = [P]
        L.or_set_particles.argtypes = [P, ctypes.c_size_t, D, D, D]
        L.or_num_particles.restype = ctypes.c_size_t
        L.or_num_particles.argtypes = [P]
        L.or_get_particles.argtypes = [P, D, D, D]
        for name in ("or_get_grid", "or_set_grid", "or_get_snapshot"):
            getattr(L, name).argtypes = [P, D, D, D]
        for name in ("or_get_pressure", "or_set_pressure", "or_get_sdf", "or_get_rhs"):
            getattr(L, name).argtypes = [P, D]
        U8 = ctypes.POINTER(ctypes.c_uint8)
        L.or_get_marks.argtypes = [P, U8]
        L.or_get_face_markers.argtypes = [P, U8, U8, U8]
        L.or_get_diffusion_markers.argtypes = [P, U8, U8, U8]
        L.or_diffusion_iterations.restype = ctypes.c_int
        L.or_diffusion_iterations.argtypes = [P, ctypes.c_int]
        for name in ("or_stage_p2g", "or_stage_sdf", "or_stage_extrapolate", "or_stage_bc", "or_stage_g2p",
                     "or_build_markers"):
            getattr(L, name).argtypes = [P]
        for name in ("or_stage_forces", "or_stage_diffusion", "or_stage_pressure", "or_stage_advection",
                     "or_stage_move", "or_substep"):
            getattr(L, name).argtypes = [P, ctypes.c_double]
        L.or_cfl.restype = ctypes.c_double
        L.or_cfl.argtypes = [P, ctypes.c_double]
        L.or_number_of_substeps.restype = ctypes.c_uint
        L.or_number_of_substeps.argtypes = [P, ctypes.c_double]
        L.or_advance_time.restype = ctypes.c_int
        L.or_advance_time.argtypes = [P, ctypes.c_double]
        L.or_cg_iterations.restype = ctypes.c_int
        L.or_cg_iterations.argtypes = [P]
        L.or_cg_rel_residual.restype = ctypes.c_double
        L.or_cg_rel_residual.argtypes = [P]
        L.or_divergence_l2.restype = ctypes.c_double
        L.or_divergence_l2.argtypes = [P]
        L.or_lerp.restype = ctypes.c_double
        L.or_lerp.argtypes = [ctypes.c_double] * 3
        L.or_trilerp.restype = ctypes.c_double
        L.or_trilerp.argtypes = [D, ctypes.c_double, ctypes.c_double, ctypes.c_double]
        I3 = ctypes.POINTER(ctypes.c_int)
        L.or_sample_face_array.restype = ctypes.c_double
        L.or_sample_face_array.argtypes = [D, I3, D, D, D]
        L.or_scalar_sample.restype = ctypes.c_double
        L.or_scalar_sample.argtypes = [D, I3, D, D, D]
        L.or_project.restype = ctypes.c_int
        L.or_project.argtypes = [I3, D, U8, D, D, D, D, ctypes.c_double, ctypes.c_int, D]
        F = ctypes.POINTER(ctypes.c_float)
        U32 = ctypes.POINTER(ctypes.c_uint32)
        L.or_sort_keys.argtypes = [F, ctypes.c_size_t, I3, F, F, U32, U32]
        I64 = ctypes.POINTER(ctypes.c_int64)
        SZ = ctypes.POINTER(ctypes.c_size_t)
        L.or_build_surface.restype = ctypes.c_int
        L.or_build_surface.argtypes = [D, I3, D, D, D, D, I64, ctypes.c_size_t, ctypes.c_size_t, SZ, SZ]
        L.or_write_obj.restype = ctypes.c_int
        L.or_write_obj.argtypes = [ctypes.c_char_p, ctypes.c_char_p, D, D, ctypes.c_size_t, I64, ctypes.c_size_t]
        L.or_mesh_to_sdf.argtypes = [D, ctypes.c_size_t, I64, ctypes.c_size_t, I3, D, D, D]
        L.or_distance_to_triangle.restype = ctypes.c_double
        L.or_distance_to_triangle.argtypes = [D, D, D, D]
        L.or_mesh_is_inside.restype = ctypes.c_int
        L.or_mesh_is_inside.argtypes = [D, I64, ctypes.c_size_t, D]
        L.or_seed_cells.argtypes = [P, U8]
        L.or_set_sdf.argtypes = [P, D]
        L.or_seed_regions.restype = ctypes.c_size_t
        L.or_seed_regions.argtypes = [ctypes.c_void_p, ctypes.c_int, I3, D, D, ctypes.c_uint64, F, F, ctypes.c_size_t]
        for name in ("or_add_point_field", "or_add_swirl_field", "or_add_volume_field"):
            getattr(L, name).restype = ctypes.c_int
        L.or_add_point_field.argtypes = [P, D, ctypes.c_double]
        L.or_add_swirl_field.argtypes = [P, D, D, ctypes.c_double]
        L.or_add_volume_field.argtypes = [P, D, I64, ctypes.c_size_t, I3, D, D, ctypes.c_double]
        L.or_volume_field_vectors.argtypes = [D, I64, ctypes.c_size_t, I3, D, D, D]
        L.or_add_mesh_collider.restype = ctypes.c_int
        L.or_add_mesh_collider.argtypes = [P, D, ctypes.c_size_t, I64, ctypes.c_size_t, D, ctypes.c_size_t, I3, D, D]
        L.or_build_collider.argtypes = [P]
        L.or_get_collider_sdf.argtypes = [P, D]
        L.or_set_enclosed_projection.argtypes = [P, ctypes.c_int]
        _lib = L
    return _lib


def dptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) if a is not None else None


def fptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float)) if a is not None else None


def u8ptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)) if a is not None else None


def u32ptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))


def iptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


def face_shapes(n):
    """(nz, ny, nx)-ordered numpy shapes of the u, v, w face arrays (x fastest in memory)."""
    nx, ny, nz = n
    return (nz, ny, nx + 1), (nz, ny + 1, nx), (nz + 1, ny, nx)


def seed_regions(regions, n, origin, size, seed):
    """Seeds particles with the shared subcell rule; returns (pos float32 [N,3], vel float32 [N,3])."""
    L = lib()
    arr = (Region * len(regions))()
    for i, r in enumerate(regions):
        arr[i].kind = r["kind"]
        for a in range(3):
            arr[i].lo[a] = r["lo"][a]
            arr[i].hi[a] = r["hi"][a] if a < len(r["hi"]) else 0.0
            arr[i].vel[a] = r.get("vel", (0, 0, 0))[a]
    n3 = np.array(n, dtype=np.int32)
    o = np.array(origin, dtype=np.float64)
    h = np.array([size[a] / n[a] for a in range(3)], dtype=np.float64)
    cnt = L.or_seed_regions(ctypes.cast(arr, ctypes.c_void_p), len(regions), iptr(n3), dptr(o), dptr(h), seed, None, None, 0)
    pos = np.zeros((cnt, 3), dtype=np.float32)
    vel = np.zeros((cnt, 3), dtype=np.float32)
    L.or_seed_regions(ctypes.cast(arr, ctypes.c_void_p), len(regions), iptr(n3), dptr(o), dptr(h), seed, fptr(pos), fptr(vel), cnt)
    return pos, vel


def sort_keys(pos32, n, origin, size):
    """Stable counting sort by fe_keys.h cell key; returns (sorted keys, permutation)."""
    L = lib()
    pos32 = np.ascontiguousarray(pos32, dtype=np.float32)
    N = pos32.shape[0]
    dims = np.array(n, dtype=np.int32)
    o = np.array(origin, dtype=np.float32)
    ih = np.array([np.float32(n[a] / size[a]) for a in range(3)], dtype=np.float32)
    keys = np.zeros(N, dtype=np.uint32)
    perm = np.zeros(N, dtype=np.uint32)
    L.or_sort_keys(fptr(pos32), N, iptr(dims), fptr(o), fptr(ih), u32ptr(keys), u32ptr(perm))
    return keys, perm


class OracleSim:
    """FP64 restatement of one simulator (PIC/FLIP/APIC) over the C oracle."""

    def __init__(self, n, solver, origin=(0, 0, 0), size=(1, 1, 1), blend=0.05, gravity=(0, -9.81, 0), max_cfl=1.0,
                 cg_rel_tol=1e-6, cg_max_it=500, viscosity=0.0):
        L = lib()
        d = _Desc()
        for a in range(3):
            d.n[a] = n[a]
            d.origin[a] = origin[a]
            d.size[a] = size[a]
            d.gravity[a] = gravity[a]
        d.solver, d.blend, d.max_cfl, d.cg_rel_tol, d.cg_max_it = solver, blend, max_cfl, cg_rel_tol, cg_max_it
        d.viscosity = viscosity
        self.n, self.solver = tuple(n), solver
        self.h = L.or_create(ctypes.byref(d))
        if not self.h:
            raise ValueError("bad oracle descriptor")
        self.L = L

    def __del__(self):
        if getattr(self, "h", None):
            self.L.or_destroy(self.h)
            self.h = None

    def set_particles(self, pos, vel=None, C=None):
        pos = np.ascontiguousarray(pos, dtype=np.float64)
        vel = None if vel is None else np.ascontiguousarray(vel, dtype=np.float64)
        C = None if C is None else np.ascontiguousarray(C, dtype=np.float64)
        self.L.or_set_particles(self.h, pos.shape[0], dptr(pos), dptr(vel), dptr(C))

    def particles(self):
        N = self.L.or_num_particles(self.h)
        pos = np.zeros((N, 3)); vel = np.zeros((N, 3)); C = np.zeros((N, 9))
        self.L.or_get_particles(self.h, dptr(pos), dptr(vel), dptr(C))
        return pos, vel, C

    def grid(self):
        su, sv, sw = face_shapes(self.n)
        u, v, w = np.zeros(su), np.zeros(sv), np.zeros(sw)
        self.L.or_get_grid(self.h, dptr(u), dptr(v), dptr(w))
        return u, v, w

    def set_grid(self, u, v, w):
        u, v, w = (np.ascontiguousarray(a, dtype=np.float64) for a in (u, v, w))
        self.L.or_set_grid(self.h, dptr(u), dptr(v), dptr(w))

    def snapshot(self):
        su, sv, sw = face_shapes(self.n)
        u, v, w = np.zeros(su), np.zeros(sv), np.zeros(sw)
        self.L.or_get_snapshot(self.h, dptr(u), dptr(v), dptr(w))
        return u, v, w

    def face_markers(self):
        su, sv, sw = face_shapes(self.n)
        a, b, c = (np.zeros(s, dtype=np.uint8) for s in (su, sv, sw))
        self.L.or_get_face_markers(self.h, u8ptr(a), u8ptr(b), u8ptr(c))
        return a, b, c

    def seed_cells(self):
        """InitializeParticles' cell mask (1: the cell receives particles) from the current fluid SDF."""
        m = self._cells(np.uint8); self.L.or_seed_cells(self.h, u8ptr(m)); return m

    def set_sdf(self, sdf):
        sdf = np.ascontiguousarray(sdf, dtype=np.float64); self.L.or_set_sdf(self.h, dptr(sdf))

    def diffusion_markers(self):
        su, sv, sw = face_shapes(self.n)
        a, b, c = (np.zeros(s, dtype=np.uint8) for s in (su, sv, sw))
        self.L.or_get_diffusion_markers(self.h, u8ptr(a), u8ptr(b), u8ptr(c))
        return a, b, c

    def diffusion_iterations(self):
        return tuple(self.L.or_diffusion_iterations(self.h, c) for c in range(3))

    def _cells(self, dtype):
        nx, ny, nz = self.n
        return np.zeros((nz, ny, nx), dtype=dtype)

    def pressure(self):
        p = self._cells(np.float64); self.L.or_get_pressure(self.h, dptr(p)); return p

    def set_pressure(self, p):
        p = np.ascontiguousarray(p, dtype=np.float64); self.L.or_set_pressure(self.h, dptr(p))

    def marks(self):
        m = self._cells(np.uint8); self.L.or_get_marks(self.h, u8ptr(m)); return m

    def sdf(self):
        s = self._cells(np.float64); self.L.or_get_sdf(self.h, dptr(s)); return s

    def rhs(self):
        b = self._cells(np.float64); self.L.or_get_rhs(self.h, dptr(b)); return b

    def set_enclosed_projection(self, on=True):
        """Not the reference: with colliders, solve enclosed FLUID components the way the GPU does (all-zero
        rows become identity rows, each component without an AIR neighbour loses its right-hand-side mean)."""
        self.L.or_set_enclosed_projection(self.h, 1 if on else 0)

    def add_mesh_collider(self, V, T, N, n, origin, h):
        """TriangleMeshCollider of a mesh (V (nv,3), T (nt,4) int64 with normal ids into N (nn,3)) on its own grid."""
        V = np.ascontiguousarray(V, dtype=np.float64)
        T = np.ascontiguousarray(T, dtype=np.int64)
        N = np.ascontiguousarray(N, dtype=np.float64)
        assert self.L.or_add_mesh_collider(self.h, dptr(V), V.shape[0], T.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                                           T.shape[0], dptr(N), N.shape[0], iptr(np.array(n, dtype=np.int32)),
                                           dptr(np.array(origin, dtype=np.float64)),
                                           dptr(np.array(h, dtype=np.float64))) == 0

    def build_collider(self):
        self.L.or_build_collider(self.h)

    def collider_sdf(self):
        out = np.zeros((self.n[2], self.n[1], self.n[0]))
        self.L.or_get_collider_sdf(self.h, dptr(out))
        return out

    def add_point_field(self, origin, strength):
        """PointField (forces/point_field.cpp) after gravity in the force list."""
        assert self.L.or_add_point_field(self.h, dptr(np.array(origin, dtype=np.float64)), strength) == 0

    def add_swirl_field(self, origin, axis, strength):
        """SwirlField (forces/swirlf_field.cpp)."""
        assert self.L.or_add_swirl_field(self.h, dptr(np.array(origin, dtype=np.float64)),
                                         dptr(np.array(axis, dtype=np.float64)), strength) == 0

    def add_volume_field(self, V, T, n, domain_origin, domain_size, strength):
        """VolumeField (forces/volume_field.cpp) of a mesh (V (nv,3), T (nt,4) int64)."""
        V = np.ascontiguousarray(V, dtype=np.float64)
        T = np.ascontiguousarray(T, dtype=np.int64)
        assert self.L.or_add_volume_field(self.h, dptr(V), T.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), T.shape[0],
                                          iptr(np.array(n, dtype=np.int32)),
                                          dptr(np.array(domain_origin, dtype=np.float64)),
                                          dptr(np.array(domain_size, dtype=np.float64)), strength) == 0

    def stage(self, name, dt=None):
        fn = getattr(self.L, "or_stage_" + name) if name != "markers" else self.L.or_build_markers
        return fn(self.h) if dt is None else fn(self.h, dt)

    def substep(self, dt):
        self.L.or_substep(self.h, dt)

    def cfl(self, dt):
        return self.L.or_cfl(self.h, dt)

    def advance_time(self, dt):
        return self.L.or_advance_time(self.h, dt)

    def cg_iterations(self):
        return self.L.or_cg_iterations(self.h)

    def cg_rel_residual(self):
        return self.L.or_cg_rel_residual(self.h)

    def divergence_l2(self):
        return self.L.or_divergence_l2(self.h)


def build_surface(sdf, n, origin, h):
    """MarchingCubesSolver::BuildSurface on a node grid (numpy (nz, ny, nx)); returns (vertices (V,3), normals (V,3),
    triangles (T,4) int64: vertex ids and normal id)."""
    L = lib()
    sdf = np.ascontiguousarray(sdf, dtype=np.float64)
    n3 = np.array(n, dtype=np.int32)
    o = np.array(origin, dtype=np.float64)
    hh = np.array(h, dtype=np.float64)
    nv, nt = ctypes.c_size_t(), ctypes.c_size_t()
    I64 = ctypes.POINTER(ctypes.c_int64)
    assert L.or_build_surface(dptr(sdf), iptr(n3), dptr(o), dptr(hh), None, None, None, 0, 0, ctypes.byref(nv),
                              ctypes.byref(nt)) == 0
    V = np.zeros((nv.value, 3)); N = np.zeros((nv.value, 3)); T = np.zeros((nt.value, 4), dtype=np.int64)
    assert L.or_build_surface(dptr(sdf), iptr(n3), dptr(o), dptr(hh), dptr(V), dptr(N), T.ctypes.data_as(I64),
                              nv.value, nt.value, ctypes.byref(nv), ctypes.byref(nt)) == 0
    return V, N, T


def volume_field_vectors(V, T, n, origin, h):
    """VolumeField::Initialize's closest-point vectors: (nz, ny, nx, 3)."""
    L = lib()
    V = np.ascontiguousarray(V, dtype=np.float64)
    T = np.ascontiguousarray(T, dtype=np.int64)
    out = np.zeros((n[2], n[1], n[0], 3))
    L.or_volume_field_vectors(dptr(V), T.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), T.shape[0],
                              iptr(np.array(n, dtype=np.int32)), dptr(np.array(origin, dtype=np.float64)),
                              dptr(np.array(h, dtype=np.float64)), dptr(out))
    return out


def mesh_to_sdf(V, T, n, origin, h):
    """Mesh2SDF::Build of a mesh (V (nv,3), T (nt,4) int64) onto a node grid; returns (nz, ny, nx) values."""
    L = lib()
    V = np.ascontiguousarray(V, dtype=np.float64)
    T = np.ascontiguousarray(T, dtype=np.int64)
    n3 = np.array(n, dtype=np.int32)
    o = np.array(origin, dtype=np.float64)
    hh = np.array(h, dtype=np.float64)
    out = np.zeros((n[2], n[1], n[0]))
    L.or_mesh_to_sdf(dptr(V), V.shape[0], T.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), T.shape[0], iptr(n3), dptr(o),
                     dptr(hh), dptr(out))
    return out


def write_obj(path, name, V, N, T):
    """OBJManager::Save of a mesh from build_surface."""
    V, N = (np.ascontiguousarray(a, dtype=np.float64) for a in (V, N))
    T = np.ascontiguousarray(T, dtype=np.int64)
    assert lib().or_write_obj(path.encode(), name.encode(), dptr(V), dptr(N), V.shape[0],
                              T.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), T.shape[0]) == 0


def project(n, h, marks, u, v, w, p, rel_tol=1e-6, max_it=500):
    """Standalone pressure projection (SinglePhasePressureSolver::Solve with CG); returns (its, rel residual)."""
    L = lib()
    n3 = np.array(n, dtype=np.int32)
    hh = np.array(h, dtype=np.float64)
    res = np.zeros(1)
    it = L.or_project(iptr(n3), dptr(hh), u8ptr(np.ascontiguousarray(marks, dtype=np.uint8)), dptr(u), dptr(v),
                      dptr(w), dptr(p), rel_tol, max_it, dptr(res))
    return it, float(res[0])


# ---------------------------------------------------------------------------------------- reference


def ref_mesh_to_sdf(V, T, n, origin, h, variant="serial"):
    """The reference's own Mesh2SDF::Build."""
    L = ref_lib(variant)
    V = np.ascontiguousarray(V, dtype=np.float64)
    T = np.ascontiguousarray(T, dtype=np.int64)
    n3 = (ctypes.c_int * 3)(*n)
    o = np.array(origin, dtype=np.float64)
    hh = np.array(h, dtype=np.float64)
    out = np.zeros((n[2], n[1], n[0]))
    L.ref_mesh_to_sdf(dptr(V), V.shape[0], T.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), T.shape[0], n3, dptr(o),
                      dptr(hh), dptr(out))
    return out


def ref_available(variant="serial"):
    return os.path.exists(os.path.join(REF_DIR, "libfe_ref_%s.so" % variant))


_ref_libs = {}


def ref_lib(variant="serial"):
    if variant not in _ref_libs:
        path = os.path.join(REF_DIR, "libfe_ref_%s.so" % variant)
        L = ctypes.CDLL(path)
        P = ctypes.c_void_p
        D = ctypes.POINTER(ctypes.c_double)
        U8 = ctypes.POINTER(ctypes.c_uint8)
        L.ref_create.restype = P
        L.ref_create.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, D, D, ctypes.c_double, D,
                                 ctypes.c_double, ctypes.c_double, ctypes.c_int]
        L.ref_destroy.argtypes = [P]
        L.ref_set_particles.argtypes = [P, ctypes.c_size_t, D, D, D]
        L.ref_num_particles.restype = ctypes.c_size_t
        L.ref_num_particles.argtypes = [P]
        L.ref_get_particles.argtypes = [P, D, D, D]
        L.ref_get_grid.argtypes = [P, D, D, D]
        L.ref_set_grid.argtypes = [P, D, D, D]
        L.ref_get_pressure.argtypes = [P, D]
        L.ref_set_pressure.argtypes = [P, D]
        L.ref_get_sdf.argtypes = [P, D]
        L.ref_get_marks.argtypes = [P, U8]
        L.ref_get_face_markers.argtypes = [P, U8, U8, U8]
        for name in ("ref_stage_p2g", "ref_stage_sdf"):
            getattr(L, name).argtypes = [P]
        for name in ("ref_stage_begin", "ref_stage_forces", "ref_stage_diffusion", "ref_stage_pressure",
                     "ref_stage_advection", "ref_substep", "ref_advance_frame", "ref_set_viscosity"):
            getattr(L, name).argtypes = [P, ctypes.c_double]
        L.ref_cfl.restype = ctypes.c_double
        L.ref_cfl.argtypes = [P, ctypes.c_double]
        L.ref_set_sdf.argtypes = [P, D]
        I64 = ctypes.POINTER(ctypes.c_int64)
        SZ = ctypes.POINTER(ctypes.c_size_t)
        L.ref_get_surface.argtypes = [P, D, D, I64, ctypes.c_size_t, ctypes.c_size_t, SZ, SZ]
        L.ref_save_obj.argtypes = [P, ctypes.c_char_p, ctypes.c_char_p]
        L.ref_mesh_to_sdf.argtypes = [D, ctypes.c_size_t, I64, ctypes.c_size_t, ctypes.POINTER(ctypes.c_int), D, D, D]
        L.ref_init_from_mesh.argtypes = [P, D, ctypes.c_size_t, I64, ctypes.c_size_t]
        L.ref_add_point_field.argtypes = [P, D, ctypes.c_double, ctypes.c_double]
        L.ref_add_mesh_collider.argtypes = [P, D, ctypes.c_size_t, I64, ctypes.c_size_t, D, ctypes.c_size_t,
                                            ctypes.POINTER(ctypes.c_int), D, D]
        L.ref_get_collider_sdf.argtypes = [P, D]
        L.ref_add_swirl_field.argtypes = [P, D, D, ctypes.c_double, ctypes.c_double]
        L.ref_add_volume_field.argtypes = [P, D, ctypes.c_size_t, I64, ctypes.c_size_t, ctypes.POINTER(ctypes.c_int), D,
                                           D, ctypes.c_double]
        _ref_libs[variant] = L
    return _ref_libs[variant]


class RefSim:
    """The reference's own CPU simulator (serial or threaded build) behind oracle/ref_harness.cpp."""

    def __init__(self, n, solver, origin=(0, 0, 0), size=(1, 1, 1), blend=0.05, gravity=(0, -9.81, 0), max_cfl=1.0,
                 cg_rel_tol=1e-6, cg_max_it=500, variant="serial", viscosity=0.0):
        self.L = ref_lib(variant)
        o = np.array(origin, dtype=np.float64); s = np.array(size, dtype=np.float64)
        g = np.array(gravity, dtype=np.float64)
        self.n, self.solver = tuple(n), solver
        self.h = self.L.ref_create(solver, n[0], n[1], n[2], dptr(o), dptr(s), blend, dptr(g), max_cfl, cg_rel_tol,
                                   cg_max_it)
        if viscosity > 0:
            self.L.ref_set_viscosity(self.h, viscosity)

    def __del__(self):
        if getattr(self, "h", None):
            self.L.ref_destroy(self.h)
            self.h = None

    def set_particles(self, pos, vel=None, C=None):
        pos = np.ascontiguousarray(pos, dtype=np.float64)
        vel = None if vel is None else np.ascontiguousarray(vel, dtype=np.float64)
        C = None if C is None else np.ascontiguousarray(C, dtype=np.float64)
        self.L.ref_set_particles(self.h, pos.shape[0], dptr(pos), dptr(vel), dptr(C))

    def particles(self):
        N = self.L.ref_num_particles(self.h)
        pos = np.zeros((N, 3)); vel = np.zeros((N, 3)); C = np.zeros((N, 9))
        self.L.ref_get_particles(self.h, dptr(pos), dptr(vel), dptr(C))
        return pos, vel, C

    def grid(self):
        su, sv, sw = face_shapes(self.n)
        u, v, w = np.zeros(su), np.zeros(sv), np.zeros(sw)
        self.L.ref_get_grid(self.h, dptr(u), dptr(v), dptr(w))
        return u, v, w

    def set_grid(self, u, v, w):
        u, v, w = (np.ascontiguousarray(a, dtype=np.float64) for a in (u, v, w))
        self.L.ref_set_grid(self.h, dptr(u), dptr(v), dptr(w))

    def pressure(self):
        nx, ny, nz = self.n
        p = np.zeros((nz, ny, nx)); self.L.ref_get_pressure(self.h, dptr(p)); return p

    def set_pressure(self, p):
        p = np.ascontiguousarray(p, dtype=np.float64); self.L.ref_set_pressure(self.h, dptr(p))

    def sdf(self):
        nx, ny, nz = self.n
        s = np.zeros((nz, ny, nx)); self.L.ref_get_sdf(self.h, dptr(s)); return s

    def marks(self):
        nx, ny, nz = self.n
        m = np.zeros((nz, ny, nx), dtype=np.uint8); self.L.ref_get_marks(self.h, u8ptr(m)); return m

    def face_markers(self):
        su, sv, sw = face_shapes(self.n)
        a, b, c = (np.zeros(s, dtype=np.uint8) for s in (su, sv, sw))
        self.L.ref_get_face_markers(self.h, u8ptr(a), u8ptr(b), u8ptr(c))
        return a, b, c

    def add_mesh_collider(self, V, T, N, n, origin, h):
        V = np.ascontiguousarray(V, dtype=np.float64)
        T = np.ascontiguousarray(T, dtype=np.int64)
        N = np.ascontiguousarray(N, dtype=np.float64)
        self.L.ref_add_mesh_collider(self.h, dptr(V), V.shape[0], T.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                                     T.shape[0], dptr(N), N.shape[0], (ctypes.c_int * 3)(*n),
                                     dptr(np.array(origin, dtype=np.float64)), dptr(np.array(h, dtype=np.float64)))

    def collider_sdf(self):
        out = np.zeros((self.n[2], self.n[1], self.n[0]))
        self.L.ref_get_collider_sdf(self.h, dptr(out))
        return out

    def add_point_field(self, origin, strength, falloff=1.0):
        self.L.ref_add_point_field(self.h, dptr(np.array(origin, dtype=np.float64)), strength, falloff)

    def add_swirl_field(self, origin, axis, strength, falloff=1.0):
        self.L.ref_add_swirl_field(self.h, dptr(np.array(origin, dtype=np.float64)),
                                   dptr(np.array(axis, dtype=np.float64)), strength, falloff)

    def add_volume_field(self, V, T, n, domain_origin, domain_size, strength):
        V = np.ascontiguousarray(V, dtype=np.float64)
        T = np.ascontiguousarray(T, dtype=np.int64)
        self.L.ref_add_volume_field(self.h, dptr(V), V.shape[0], T.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                                    T.shape[0], (ctypes.c_int * 3)(*n), dptr(np.array(domain_origin, dtype=np.float64)),
                                    dptr(np.array(domain_size, dtype=np.float64)), strength)

    def stage(self, name, dt=None):
        fn = getattr(self.L, "ref_stage_" + name)
        return fn(self.h) if dt is None else fn(self.h, dt)

    def substep(self, dt):
        self.L.ref_substep(self.h, dt)

    def cfl(self, dt):
        return self.L.ref_cfl(self.h, dt)

    def advance_frame(self, dt):
        self.L.ref_advance_frame(self.h, dt)

    def set_sdf(self, sdf):
        sdf = np.ascontiguousarray(sdf, dtype=np.float64); self.L.ref_set_sdf(self.h, dptr(sdf))

    def surface(self):
        """PICSimulator::GetSurface into a fresh TriangleMesh: (vertices, normals, triangles (T,4) int64)."""
        nv, nt = ctypes.c_size_t(), ctypes.c_size_t()
        I64 = ctypes.POINTER(ctypes.c_int64)
        self.L.ref_get_surface(self.h, None, None, None, 0, 0, ctypes.byref(nv), ctypes.byref(nt))
        V = np.zeros((nv.value, 3)); N = np.zeros((nv.value, 3)); T = np.zeros((nt.value, 4), dtype=np.int64)
        self.L.ref_get_surface(self.h, dptr(V), dptr(N), T.ctypes.data_as(I64), nv.value, nt.value, ctypes.byref(nv),
                               ctypes.byref(nt))
        return V, N, T

    def init_from_mesh(self, V, T):
        """PICSimulator::InitializeFromTriangleMesh (Mesh2SDF into Fluid3::sdf, then InitializeParticles)."""
        V = np.ascontiguousarray(V, dtype=np.float64)
        T = np.ascontiguousarray(T, dtype=np.int64)
        self.L.ref_init_from_mesh(self.h, dptr(V), V.shape[0], T.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                                  T.shape[0])

    def save_obj(self, path, name):
        """OBJManager::Save of the last surface()."""
        self.L.ref_save_obj(self.h, path.encode(), name.encode())
