"""Python mirror of the reference's simulator API for the substep path.

Same class and method names as the reference's pybind11 module PyFluidEngine
(python_wrapper/simulators_wrapper.cu:36-85, frame_wrapper.cpp, vector3_wrapper.cpp,
bounding_box_3d_wrapper.cpp, exteranl_forces_wrapper.cpp) and C++ classes (pic_simulator.hpp:27-43,
hybrid_simulator.hpp:10-41, physics_animation.hpp:8-19, flip_simulator.hpp:9-16), backed by one
device-resident Scene: the substep, mesh initialisation, emitters, external forces, triangle-mesh
colliders, viscosity and the fluid surface.  Invalid arguments raise ValueError / TypeError with the
reason, and library errors raise FluideError carrying the C ABI status.
"""
import numpy as np

from . import _abi
from .scene import Scene


class Vector3D:
    """Vector3<double> (common/vector3.hpp)."""

    def __init__(self, x=0.0, y=None, z=None):
        if y is None:
            y = z = x
        self.x, self.y, self.z = float(x), float(y), float(z)

    def __iter__(self):
        return iter((self.x, self.y, self.z))

    def __repr__(self):
        return "Vector3D(%g, %g, %g)" % (self.x, self.y, self.z)


class Vector3S(Vector3D):
    """Vector3<size_t>."""

    def __init__(self, x=0, y=None, z=None):
        if y is None:
            y = z = x
        self.x, self.y, self.z = int(x), int(y), int(z)


class BoundingBox3D:
    """BoundingBox3D(origin, size) (3d/bounding_box_3d.cpp:4-8)."""

    def __init__(self, origin=Vector3D(0.0), size=Vector3D(1.0)):
        self._origin, self._size = Vector3D(*origin), Vector3D(*size)

    def GetOrigin(self):
        return self._origin

    def GetSize(self):
        return self._size


class Frame:
    """Frame(timeIntervalInSeconds) with an index (common/frame.cpp:3-49)."""

    def __init__(self, timeIntervalInSeconds=1.0 / 60.0):
        self._dt = float(timeIntervalInSeconds)
        self._index = 0

    def GetIndex(self):
        return self._index

    def GetTimeIntervalInSeconds(self):
        return self._dt

    def GetTimeInSeconds(self):
        return self._index * self._dt

    def Advance(self):
        self._index += 1


class ExternalForce:
    pass


class DirectionalField(ExternalForce):
    """Uniform force field (forces/directional_field.cpp:3-21)."""

    def __init__(self, strength=Vector3D(0.0, -9.81, 0.0)):
        self._strength = Vector3D(*strength)

    def Sample(self, position=None):
        return self._strength

    def SetStrength(self, strength):
        self._strength = Vector3D(*strength)


class PointField(ExternalForce):
    """PointField (forces/point_field.cpp:3-56): strength / max(|p - origin|, 1) toward the origin; applied on the
    GPU after gravity."""

    def __init__(self, origin=Vector3D(0.0), strength=0.0, strengthFallOff=1.0):
        self._origin, self._strength, self._falloff = Vector3D(*origin), float(strength), float(strengthFallOff)

    def GetOrigin(self):
        return self._origin

    def GetStrength(self):
        return self._strength

    def SetStrength(self, strength):
        self._strength = float(strength)

    def _add_to(self, scene):
        scene.add_point_field(tuple(self._origin), self._strength, self._falloff)


class SwirlField(ExternalForce):
    """SwirlField (forces/swirlf_field.cpp:5-23); the axis is normalised as the reference's constructor does."""

    def __init__(self, origin=Vector3D(0.0), axisDirection=Vector3D(0.0, 1.0, 0.0), strength=0.0,
                 strengthFallOff=1.0):
        a = np.array(tuple(axisDirection), dtype=np.float64)
        l = np.sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2])
        self._origin, self._axis, self._axisGiven = Vector3D(*origin), Vector3D(*(a / l)), tuple(a)
        self._strength, self._falloff = float(strength), float(strengthFallOff)

    def GetOrigin(self):
        return self._origin

    def GetAxisDirection(self):
        return self._axis

    def GetStrength(self):
        return self._strength

    def SetStrength(self, strength):
        self._strength = float(strength)

    def _add_to(self, scene):
        scene.add_swirl_field(tuple(self._origin), self._axisGiven, self._strength, self._falloff)  # normalised there


class VolumeField(ExternalForce):
    """VolumeField (forces/volume_field.cpp:5-89) of a TriangleMesh on its own node grid; the closest-point
    vectors are computed on the GPU the first time the field is registered with a scene."""

    def __init__(self, mesh, resolution, domain, strength):
        self._V = np.array(mesh.vertices, dtype=np.float64)
        self._T = np.array(mesh.triangles, dtype=np.int64)
        self._res = (int(resolution.x), int(resolution.y), int(resolution.z))
        o, sz = domain.GetOrigin(), domain.GetSize()
        self._origin, self._size = (o.x, o.y, o.z), (sz.x, sz.y, sz.z)
        self._strength = float(strength)
        self._field = None

    def GetStrength(self):
        return self._strength

    def SetStrength(self, strength):
        self._strength = float(strength)

    def _add_to(self, scene):
        if self._field is None:
            h = tuple(self._size[a] / self._res[a] for a in range(3))
            self._field = _abi.volume_field_vectors(self._V, self._T, self._res, self._origin, h)
        scene.add_volume_field(self._V, self._T, self._res, self._origin, self._size, self._strength,
                               field=self._field)


class TriangleMesh:
    """TriangleMesh (3d/triangle_mesh.hpp): vertices (V,3), normals (V,3) and triangles (T,4: three vertex ids and
    the normal id) as numpy arrays, appended to by GetSurface."""

    def __init__(self):
        self.Clear()
        self._name = ""

    def Clear(self):
        self.vertices = np.zeros((0, 3))
        self.normals = np.zeros((0, 3))
        self.triangles = np.zeros((0, 4), dtype=np.int64)

    def GetObjectName(self):
        return self._name

    def SetObjectName(self, name):
        self._name = str(name)

    def _append(self, V, N, T):
        base = self.vertices.shape[0]
        self.vertices = np.concatenate([self.vertices, V])
        self.normals = np.concatenate([self.normals, N])
        self.triangles = np.concatenate([self.triangles, T + base])


class OBJManager:
    """OBJManager::Save (3d/obj_manager.cpp:14-90) through the library's writer; Load reads "o", "v", "vn" and
    three-vertex "f" lines as OBJManager::ParseLine does (:92-161)."""

    def Load(self, name, obj):
        try:
            f = open(name, "rb")
        except OSError:
            return  # the reference reports the error on stdout and leaves the mesh unchanged
        V, N, T = [], [], []
        with f:
            for raw in f.read().decode().split("\n"):
                w = raw.split(" ")
                if w[-1] == "" and len(w) > 1:
                    w = w[:-1]  # std::getline keeps no trailing empty field
                if not w or w == [""]:
                    continue
                if w[0] == "o" and len(w) > 1:
                    obj.SetObjectName(w[1])
                elif w[0] == "v" and len(w) > 3:
                    V.append([float(w[1]), float(w[2]), float(w[3])])
                elif w[0] == "vn" and len(w) > 3:
                    N.append([float(w[1]), float(w[2]), float(w[3])])
                elif w[0] == "f" and len(w) == 4:
                    fv = [x.split("/") for x in w[1:]]
                    vs = [int(x[0]) for x in fv if len(x) > 1]
                    T.append([vs[0] - 1, vs[1] - 1, vs[2] - 1, int(fv[-1][-1]) - 1])
        obj.vertices = np.concatenate([obj.vertices, np.asarray(V, dtype=np.float64).reshape(-1, 3)])
        obj.normals = np.concatenate([obj.normals, np.asarray(N, dtype=np.float64).reshape(-1, 3)])
        obj.triangles = np.concatenate([obj.triangles, np.asarray(T, dtype=np.int64).reshape(-1, 4)])

    def Save(self, name, obj):
        V = np.ascontiguousarray(obj.vertices, dtype=np.float64)
        N = np.ascontiguousarray(obj.normals, dtype=np.float64)
        T = np.ascontiguousarray(obj.triangles, dtype=np.int64)
        L = _abi.lib()
        _abi.check(L.fe_write_obj(str(name).encode(), obj.GetObjectName().encode(), _abi.ptr(V), _abi.ptr(N),
                                  V.shape[0], _abi.ptr(T), T.shape[0]))


class ScalarGrid3D:
    """ScalarGrid3D (3d/scalar_grid3d.hpp), the node-value subset: element (i, j, k) at i + nx * (j + ny * k)."""

    def __init__(self, size=None, initialValue=0.0, origin=None, gridSpacing=None):
        size = Vector3S(1) if size is None else size
        self._size = (int(size.x), int(size.y), int(size.z))
        self._origin = Vector3D(0.0) if origin is None else origin
        self._spacing = Vector3D(1.0) if gridSpacing is None else gridSpacing
        self.values = np.full((self._size[2], self._size[1], self._size[0]), float(initialValue))

    def GetSize(self):
        return Vector3S(*self._size)

    def GetOrigin(self):
        return self._origin

    def GetGridSpacing(self):
        return self._spacing

    def GetElement(self, i, j, k):
        return float(self.values[k, j, i])

    def SetElement(self, i, j, k, value):
        self.values[k, j, i] = value


class Collider:
    """Collider (3d/collider.hpp)."""


class TriangleMeshCollider(Collider):
    """TriangleMeshCollider (3d/triangle_mesh_collider.cpp:4-100) of a TriangleMesh with normals on its own node grid;
    the simulators run its boundary condition and collision response on the GPU."""

    def __init__(self, gridSize, gridOrigin, gridSpacing, mesh):
        self._n = (int(gridSize.x), int(gridSize.y), int(gridSize.z))
        self._origin = (gridOrigin.x, gridOrigin.y, gridOrigin.z)
        self._spacing = (gridSpacing.x, gridSpacing.y, gridSpacing.z)
        self._V = np.array(mesh.vertices, dtype=np.float64)
        self._T = np.array(mesh.triangles, dtype=np.int64)
        self._N = np.array(mesh.normals, dtype=np.float64)
        self._sdf = None

    def GetClosestDistanceAt(self, position):
        """ScalarGrid3D::Sample of the collider's SDF (computed on the GPU the first time)."""
        if self._sdf is None:
            self._sdf = _abi.mesh_to_sdf(self._V, self._T, self._n, self._origin, self._spacing)
        p = np.array(tuple(position), dtype=np.float64)
        n = self._n
        i0, i1, fr = [], [], []
        for a in range(3):
            x = (p[a] - self._origin[a]) / self._spacing[a]
            hi = n[a] - 1
            fl = np.floor(x)
            ii = int(fl)
            if hi == 0 or ii < 0:
                ii, f = 0, 0.0
            elif ii > hi - 1:
                ii, f = hi - 1, 1.0
            else:
                f = x - fl
            i0.append(ii)
            i1.append(min(ii + 1, n[a] - 1))
            fr.append(f)
        at = lambda i, j, k: self._sdf[k, j, i]  # noqa: E731
        lerp = lambda a, b, t: (1 - t) * a + t * b  # noqa: E731
        b0 = lerp(lerp(at(i0[0], i0[1], i0[2]), at(i1[0], i0[1], i0[2]), fr[0]),
                  lerp(at(i0[0], i1[1], i0[2]), at(i1[0], i1[1], i0[2]), fr[0]), fr[1])
        b1 = lerp(lerp(at(i0[0], i0[1], i1[2]), at(i1[0], i0[1], i1[2]), fr[0]),
                  lerp(at(i0[0], i1[1], i1[2]), at(i1[0], i1[1], i1[2]), fr[0]), fr[1])
        return float(lerp(b0, b1, fr[2]))

    def IsInside(self, position):
        return self.GetClosestDistanceAt(position) < 0

    def _add_to(self, scene):
        scene.add_mesh_collider(self._V, self._T, self._N, self._n, self._origin, self._spacing)


class ColliderCollection:
    """ColliderCollection (3d/collider_collection.hpp): the colliders of SetColliders."""

    def __init__(self, size=None, gridSpacing=None, origin=None):
        self._colliders = []

    def AddCollider(self, collider):
        self._colliders.append(collider)

    def GetColliders(self):
        return self._colliders

    def IsInside(self, position):
        return any(c.IsInside(position) for c in self._colliders)


class Emitter:
    """Emitter (emmiter/emmiter.hpp)."""


class VolumeEmitter(Emitter):
    """VolumeEmitter (emmiter/volume_emmiter.cpp:8-86): at the start of every substep each node of its grid with
    SDF <= 0 where the previous substep's fluid SDF is >= 0 receives particlesPerBlock particles (node + spacing *
    U[0,1]^3) with `velocity`; the SDF is the mesh's (built on the GPU at registration) or InitializeFromSdf's.
    velocityVariance is kept and unused, as in the reference.  Changes after AddEmitter apply at the next step."""

    def __init__(self, mesh, resolution, domain, particlesPerBlock, velocity, velocityVariance):
        self._res = (int(resolution.x), int(resolution.y), int(resolution.z))
        o, sz = domain.GetOrigin(), domain.GetSize()
        self._origin = (o.x, o.y, o.z)
        self._size = (sz.x, sz.y, sz.z)
        self._ppb = int(particlesPerBlock)
        self._velocity = (velocity.x, velocity.y, velocity.z)
        self._velocityVariance = velocityVariance
        self._version = 0
        self.InitializeFromTriangleMesh(mesh)

    def InitializeFromTriangleMesh(self, mesh):
        self._V = np.array(mesh.vertices, dtype=np.float64)
        self._T = np.array(mesh.triangles, dtype=np.int64)
        self._sdf = None
        self._version += 1

    def InitializeFromSdf(self, sdf):
        """VolumeEmitter::InitializeFromSdf (:50-56): the emitter's node (i, j, k) takes sdf(i, j, k)."""
        nx, ny, nz = self._res
        if sdf.values.shape[0] < nz or sdf.values.shape[1] < ny or sdf.values.shape[2] < nx:
            raise ValueError("InitializeFromSdf: the grid must cover the emitter's resolution")
        self._sdf = np.ascontiguousarray(sdf.values[:nz, :ny, :nx], dtype=np.float64)
        self._version += 1

    def _add_to(self, scene, seed):
        eid = scene.add_volume_emitter(self._V, self._T, self._res, self._origin, self._size,
                                       particles_per_block=self._ppb, velocity=self._velocity, seed=seed)
        if self._sdf is not None:
            scene.set_emitter_sdf(eid, self._sdf)
        return eid


class HybridSimulator:
    """HybridSimulator (hybrid_simulator.cpp:4-110) over a device Scene."""

    _solver = _abi.PIC

    def __init__(self, gridSize, domain, device=0):
        self._n = (int(gridSize.x), int(gridSize.y), int(gridSize.z))
        self._domain = domain
        o, s = domain.GetOrigin(), domain.GetSize()
        self._origin = (o.x, o.y, o.z)
        self._size = (s.x, s.y, s.z)
        self._h = tuple(self._size[a] / self._n[a] for a in range(3))
        self._maxCfl = 3.0              # hybrid_simulator.cpp:21
        self._particlesPerBlok = 16     # hybrid_simulator.cpp:22
        self._viscosity = 0.0
        self._density = 1.0
        self._blend = 0.05
        self._forces = []
        self._fieldForces = []
        self._colliders = []
        self._emitters = []
        self._registered = None         # (scene, emitter versions) the scene's emitters were built from
        self._meshSeed = 0
        self._meshSdfLive = False       # InitializeFromTriangleMesh ran and no substep since
        self._device = device
        self._scene = None
        self._pending = None            # (pos, vel, C) until the scene exists
        self._currentFrame = Frame()
        self._currentTime = 0.0
        self._numberOfTimeSteps = 0
        self._cg = dict(cg_rel_tol=1e-6, cg_max_it=2000, cg_inner_tol=0.0, max_refine=12)
        self.last_stats = []

    # settings -------------------------------------------------------------------------------------
    def MaxCfl(self):
        return self._maxCfl

    def SetMaxClf(self, maxCfl):
        self._rebuild(lambda: setattr(self, "_maxCfl", float(maxCfl)))

    SetMaxCfl = SetMaxClf  # the name the reference's Python example calls (python_example.py:30)

    def GetViscosity(self):
        return self._viscosity

    def SetViscosity(self, viscosity):
        """HybridSimulator::SetViscosity (hybrid_simulator.cpp:97-100): > 0 runs ComputeDiffusion every substep
        (pic_simulator.cpp:214-222) with the reference's BackwardEulerDiffusionSolver settings."""
        viscosity = float(viscosity)
        if not viscosity >= 0.0:
            raise ValueError("viscosity must be >= 0")
        if self._scene is not None:
            self._scene.set_viscosity(viscosity)
        self._viscosity = viscosity

    def GetDensity(self):
        return self._density

    def SetDensity(self, density):
        self._density = float(density)  # unused by the projection, as in the reference

    def GetParticlesPerBlock(self):
        return self._particlesPerBlok

    def SetParticlesPerBlock(self, n):
        self._particlesPerBlok = int(n)

    def GetOrigin(self):
        return Vector3D(*self._origin)

    def GetResolution(self):
        return Vector3S(*self._n)

    def GetGridSpacing(self):
        return Vector3D(*self._h)

    def GetNumberOfParticles(self):
        if self._scene is not None:
            return self._scene.num_particles()
        return 0 if self._pending is None else self._pending[0].shape[0]

    def SetPressureSolverSettings(self, cg_rel_tol=None, cg_max_it=None, cg_inner_tol=None, max_refine=None,
                                  pressure_solver=None):
        """Solver settings (the reference swaps LinearSystemSolver objects, pic_simulator.cpp:56-59);
        pressure_solver: fluide_engine_b200.AUTO / MGPCG / CG."""
        upd = {k: v for k, v in dict(cg_rel_tol=cg_rel_tol, cg_max_it=cg_max_it, cg_inner_tol=cg_inner_tol,
                                     max_refine=max_refine, pressure_solver=pressure_solver).items() if v is not None}
        self._rebuild(lambda: self._cg.update(upd))

    # forces / scene contents ----------------------------------------------------------------------
    def AddExternalForce(self, force):
        """PICSimulator::AddExternalForce (pic_simulator.cpp:41-44): DirectionalFields add up to gravity; PointField,
        SwirlField and VolumeField are applied after it on the GPU, in the order added."""
        if isinstance(force, (PointField, SwirlField, VolumeField)):
            self._fieldForces.append(force)
            if self._scene is not None:
                force._add_to(self._scene)
            return
        if not isinstance(force, DirectionalField):
            raise TypeError("AddExternalForce: DirectionalField, PointField, SwirlField or VolumeField expected")
        self._rebuild(lambda: self._forces.append(force))

    def AddCollider(self, collider):
        """PICSimulator::AddCollider (pic_simulator.cpp:66-69): a TriangleMeshCollider, applied on the GPU."""
        if not isinstance(collider, TriangleMeshCollider):
            raise TypeError("AddCollider: a TriangleMeshCollider is expected")
        if self._scene is not None:
            collider._add_to(self._scene)
        self._colliders.append(collider)

    def SetColliders(self, colliders):
        """PICSimulator::SetColliders (pic_simulator.cpp:61-64): replaces the colliders with a ColliderCollection's."""
        cs = list(colliders.GetColliders())
        if not all(isinstance(c, TriangleMeshCollider) for c in cs):
            raise TypeError("SetColliders: TriangleMeshColliders are expected")
        if self._scene is not None:
            self._scene.clear_colliders()
            for c in cs:
                c._add_to(self._scene)
        self._colliders = cs

    def AddEmitter(self, emitter):
        """PICSimulator::AddEmitter (pic_simulator.cpp:46-49); registered with the scene at the next step."""
        if not isinstance(emitter, VolumeEmitter):
            raise TypeError("AddEmitter: a VolumeEmitter is expected")
        self._emitters.append(emitter)

    def InitializeFromTriangleMesh(self, mesh):
        """PICSimulator::InitializeFromTriangleMesh (pic_simulator.cpp:33-39): the mesh SDF becomes the fluid SDF and
        every cell inside it receives GetParticlesPerBlock() particles, appended to those already set.  The fluid SDF
        stays the mesh's until the first substep, also across settings changes that rebuild the scene."""
        self._ensure_scene().init_from_mesh(mesh.vertices, mesh.triangles, self._particlesPerBlok, self._meshSeed)
        self._meshSeed += 1
        self._meshSdfLive = True

    def GetSurface(self, mesh):
        """PICSimulator::GetSurface (pic_simulator.cpp:71-78): appends the marching-cubes surface of the SDF built at
        the start of the last substep to mesh (a TriangleMesh), as the reference's surface tracker does."""
        V, N, T = self._ensure_scene().surface()
        mesh._append(V, N, T)

    def InitializeFromRegions(self, regions, seed=0):
        """Seeds boxes / spheres with the deterministic subcell rule (8 particles per cell)."""
        pos, vel = _abi.seed_regions(regions, self._n, self._origin, self._size, seed)
        self.SetParticles(pos, vel)
        return pos.shape[0]

    def SetParticles(self, pos, vel=None, C=None):
        pos = np.ascontiguousarray(pos, dtype=np.float32)
        vel = np.zeros_like(pos) if vel is None else np.ascontiguousarray(vel, dtype=np.float32)
        self._pending = (pos, vel, C)
        if self._scene is not None:
            self._scene.set_particles(pos, vel, C)
            self._pending = None

    def GetParticles(self):
        if self._scene is not None:
            return self._scene.particles()
        if self._pending is None:
            return np.zeros((0, 3), np.float32), np.zeros((0, 3), np.float32), np.zeros((0, 9), np.float32)
        p, v, c = self._pending
        return p, v, (np.zeros((p.shape[0], 9), np.float32) if c is None else c)

    def GetFluidSdf(self):
        return self._ensure_scene().fluid_sdf()

    def Cfl(self, timeIntervalInSeconds):
        return self._ensure_scene().cfl(timeIntervalInSeconds)

    # PhysicsAnimation -----------------------------------------------------------------------------
    def SetCurrentFrame(self, frame):
        self._currentFrame = frame

    def GetCurrentFrame(self):
        return self._currentFrame

    def GetCurrentTimeInSeconds(self):
        return self._currentTime

    def AdvanceSingleFrame(self):
        """PhysicsAnimation::AdvanceSingleFrame (physics_animation.cpp:17-21, 48-61, 64-92)."""
        scene = self._sync_emitters()
        self._meshSdfLive = False
        self._currentTime = self._currentFrame.GetTimeInSeconds()
        dt = self._currentFrame.GetTimeIntervalInSeconds()
        n = scene.advance_frame(dt)
        self._numberOfTimeSteps = n
        self._currentTime += dt
        self._currentFrame.Advance()
        return n

    def GetNumberOfSubTimeSteps(self):
        """PhysicsAnimation::GetNumberOfSubTimeSteps (physics_animation.cpp:43-46): substeps of the last frame."""
        return self._numberOfTimeSteps

    def AdvanceFixedSubsteps(self, dt, nsub, stats=True):
        """nsub substeps of exactly dt (the benchmark configurations' fixed-dt mode)."""
        scene = self._sync_emitters()
        self._meshSdfLive = False
        self.last_stats = scene.step(dt, nsub, stats=stats) or []
        return self.last_stats

    # internals ------------------------------------------------------------------------------------
    def _gravity(self):
        g = [0.0, 0.0, 0.0]
        for f in self._forces:
            s = f.Sample()
            g = [g[0] + s.x, g[1] + s.y, g[2] + s.z]
        return tuple(g)

    def _ensure_scene(self):
        if self._scene is None:
            self._scene = Scene(self._n, solver=self._solver, origin=self._origin, size=self._size,
                                flip_blend=self._blend, gravity=self._gravity(), max_cfl=self._maxCfl,
                                device=self._device, viscosity=self._viscosity, **self._cg)
            for f in self._fieldForces:
                f._add_to(self._scene)
            for c in self._colliders:
                c._add_to(self._scene)
            if self._pending is not None:
                p, v, c = self._pending
                self._scene.set_particles(p, v, c)
                self._pending = None
        return self._scene

    def _sync_emitters(self):
        """(Re-)registers the emitters when the scene is new or an emitter changed since its registration."""
        scene = self._ensure_scene()
        key = (id(scene), tuple((id(e), e._version) for e in self._emitters))
        if self._registered != key:
            scene.clear_emitters()
            for i, e in enumerate(self._emitters):
                e._add_to(scene, 0x5EED0000 + i)
            self._registered = key
        return scene

    def _rebuild(self, change):
        """Applies a settings change; a live scene is rebuilt with its particles and pressure kept."""
        if self._scene is None:
            change()
            return
        pos, vel, C = self._scene.particles()
        p = self._scene.grid()[3]
        sdf = self._scene.fluid_sdf() if self._meshSdfLive else None
        self._scene.close()
        self._scene = None
        self._registered = None
        change()
        self._pending = (pos, vel, C if self._solver == _abi.APIC else None)
        scene = self._ensure_scene()
        scene.set_pressure(p)
        if sdf is not None:
            scene.set_fluid_sdf(sdf)


class PICSimulator(HybridSimulator):
    _solver = _abi.PIC


class FLIPSimulator(HybridSimulator):
    _solver = _abi.FLIP

    def SetBlendingFactor(self, factor):
        self._rebuild(lambda: setattr(self, "_blend", float(factor)))

    def GetBlendingFactor(self):
        return self._blend


class APICSimulator(HybridSimulator):
    _solver = _abi.APIC


class SimulationStats:
    """SimulationStats (simulation_stats.hpp): per-run statistics of SimulationRunner."""

    def __init__(self):
        self.Clear()

    def Clear(self):
        self.simulatorType = ""
        self.numberOfIterations = 0
        self.gridSize = Vector3S(0, 0, 0)
        self.numberOfParticles = 0
        self.timeIntervalInSeconds = 0.0
        self.simulationTimeInSeconds = 0.0
        self.iterationTimeInSeconds = []
        self.cflPerIteration = []

    @staticmethod
    def _median(v):
        return float(np.median(v)) if len(v) else float("nan")

    def PrintStats(self, out=None):
        import sys

        out = out or sys.stdout
        mean = lambda v: float(np.mean(v)) if len(v) else 0.0  # noqa: E731
        g = self.gridSize
        out.write("================ SIMULATION STATS ================\n")
        out.write("Simulator type: %s\n" % self.simulatorType)
        out.write("Grid resolution: %d x %d x %d\n" % (g.x, g.y, g.z))
        out.write("Number of particles: %d\n" % self.numberOfParticles)
        out.write("Number of Iterations: %d\n" % self.numberOfIterations)
        out.write("Time interval: %g [s]\n" % self.timeIntervalInSeconds)
        out.write("Median CFL: %g\n" % mean(self.cflPerIteration))  # the reference's labels (simulation_stats.cpp:27-28)
        out.write("Mean CFL: %g\n" % self._median(self.cflPerIteration))
        out.write("Median frame: %g [s]\n" % self._median(self.iterationTimeInSeconds))
        out.write("Mean frame: %g [s]\n" % mean(self.iterationTimeInSeconds))
        out.write("Simulation time: %g [s]\n" % self.simulationTimeInSeconds)
        out.write("==================================================\n")


class SimulationRunner:
    """SimulationRunner (simulation_runner.cpp:16-56): AdvanceSingleFrame, GetSurface and OBJ output per
    iteration into <cache>/simulated_frames/<name>_<i>.obj, log in <cache>/log.txt.  Frame i's OBJ is written on a
    host thread while the GPU advances frame i + 1."""

    def __init__(self):
        self._stats = SimulationStats()

    def RunSimulation(self, simulator, timeIntervalInSeconds, numberOfIterations, simulationOutputName, cacheFolderPath):
        import os
        import threading
        import time

        simulator.SetCurrentFrame(Frame(timeIntervalInSeconds))
        os.makedirs(os.path.join(cacheFolderPath, "simulated_frames"), exist_ok=True)
        writer, errors = None, []

        def write(path, mesh):
            try:
                OBJManager().Save(path, mesh)
            except Exception as ex:  # re-raised on the calling thread
                errors.append(ex)

        with open(os.path.join(cacheFolderPath, "log.txt"), "w") as log:
            for i in range(int(numberOfIterations)):
                log.write("Iteration: %d\n" % i)
                t0 = time.perf_counter()
                simulator.AdvanceSingleFrame()
                mesh = TriangleMesh()
                simulator.GetSurface(mesh)
                path = os.path.join(cacheFolderPath, "simulated_frames", "%s_%d.obj" % (simulationOutputName, i))
                if writer is not None:
                    writer.join()
                if errors:
                    raise errors[0]
                writer = threading.Thread(target=write, args=(path, mesh))
                writer.start()
                dt = time.perf_counter() - t0
                self._stats.simulationTimeInSeconds += dt
                self._stats.iterationTimeInSeconds.append(dt)
                self._stats.cflPerIteration.append(simulator.Cfl(timeIntervalInSeconds))
                log.write("\n")
            if writer is not None:
                writer.join()
            if errors:
                raise errors[0]
            self._stats.numberOfIterations = int(numberOfIterations)
            self._stats.timeIntervalInSeconds = timeIntervalInSeconds
            self._stats.simulatorType = type(simulator).__name__
            self._stats.numberOfParticles = simulator.GetNumberOfParticles()
            self._stats.gridSize = simulator.GetResolution()
            self._stats.PrintStats(log)

    def GetStats(self):
        return self._stats

