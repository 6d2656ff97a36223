// fluide_engine.hpp -- the reference's C++ simulator API for the substep path, over the C ABI.
//
// Drop-in for the classes a caller of AleksanderSiwek/Fluide_Engine uses to run the PIC / FLIP / APIC
// substep: PhysicsAnimation (physics_animation.hpp:8-29), HybridSimulator (hybrid_simulator.hpp:10-41),
// PICSimulator (pic_simulator.hpp:27-43), FLIPSimulator (flip_simulator.hpp:9-16), APICSimulator
// (apic_simulator.hpp:9-15), Frame (common/frame.hpp), BoundingBox3D (3d/bounding_box_3d.hpp),
// DirectionalField, PointField, SwirlField, VolumeField (forces/), Vector3 (common/vector3.hpp), TriangleMesh, OBJManager,
// ScalarGrid3D (the node-value subset), VolumeEmitter (emmiter/volume_emmiter.hpp), SimulationStats,
// SimulationRunner, Collider, TriangleMeshCollider and ColliderCollection (3d/), with the same names and argument
// meaning.  State lives on the GPU in one fe_scene (include/fluide_b200.h), created on first use; errors of the
// library throw fluide::Error carrying the fe_status.  Header-only; link with libfluide_b200.so.
#ifndef FLUIDE_ENGINE_HPP
#define FLUIDE_ENGINE_HPP

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstddef>
#include <filesystem>
#include <limits>
#include <numeric>
#include <thread>
#include <typeinfo>
#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "fluide_b200.h"

namespace fluide {
class Error : public std::runtime_error {
  public:
    Error(fe_status s, const std::string& what) : std::runtime_error(what), status(s) {}
    fe_status status;
};
inline void check(fe_status s)
{
    if (s != FE_OK) throw Error(s, std::string("fluide_b200: ") + fe_last_error());
}
}  // namespace fluide

template <typename T>
class Vector3 {
  public:
    Vector3(T v = T()) : x(v), y(v), z(v) {}
    Vector3(T x_, T y_, T z_) : x(x_), y(y_), z(z_) {}
    T x, y, z;
};

class BoundingBox3D {
  public:
    BoundingBox3D(Vector3<double> origin = Vector3<double>(0), Vector3<double> size = Vector3<double>(1))
        : _origin(origin), _size(size) {}
    Vector3<double> GetOrigin() const { return _origin; }
    Vector3<double> GetSize() const { return _size; }
    void SetOrigin(Vector3<double> o) { _origin = o; }
    void SetSize(Vector3<double> s) { _size = s; }

  private:
    Vector3<double> _origin, _size;
};

class Frame {
  public:
    Frame() = default;
    explicit Frame(double timeIntervalInSeconds) : _timeIntervalInSeconds(timeIntervalInSeconds) {}
    void Advance() { ++_index; }
    Frame& operator++() { Advance(); return *this; }
    Frame operator++(int) { Frame r = *this; Advance(); return r; }
    unsigned long GetIndex() const { return _index; }
    double GetTimeIntervalInSeconds() const { return _timeIntervalInSeconds; }
    double GetTimeInSeconds() const { return _index * _timeIntervalInSeconds; }

  private:
    unsigned long _index = 0;
    double _timeIntervalInSeconds = 1 / 60.0f;  // common/frame.hpp:22
};

class ExternalForce {
  public:
    virtual ~ExternalForce() = default;
    virtual Vector3<double> Sample(const Vector3<double>& position) const = 0;
};

class DirectionalField : public ExternalForce {
  public:
    explicit DirectionalField(Vector3<double> strength = Vector3<double>(0.0, -9.81, 0.0)) : _strength(strength) {}
    Vector3<double> Sample(const Vector3<double>&) const override { return _strength; }
    void SetStrength(Vector3<double> s) { _strength = s; }

  private:
    Vector3<double> _strength;
};

namespace fluide {
inline double length3(double x, double y, double z) { return std::sqrt(x * x + y * y + z * z); }  // Vector3::GetLength
// A position-dependent force the GPU substep applies (PointField, SwirlField, VolumeField): its C-ABI record.
class FieldForce : public ExternalForce {
  public:
    virtual fe_force_desc Desc() const = 0;
};
}  // namespace fluide

// PointField (forces/point_field.cpp:3-56): strength / max(|p - origin|, 1) toward the origin.
class PointField : public fluide::FieldForce {
  public:
    PointField(Vector3<double> origin = Vector3<double>(0), double strength = 0, double strengthFallOff = 1)
        : _origin(origin), _strength(strength), _strengthFallOff(strengthFallOff) {}
    Vector3<double> Sample(const Vector3<double>& p) const override
    {
        const double len = fluide::length3(p.x - _origin.x, p.y - _origin.y, p.z - _origin.z);
        const double dist = len >= 1.0 ? len : 1.0;
        const double ex = _origin.x - p.x, ey = _origin.y - p.y, ez = _origin.z - p.z;
        const double el = fluide::length3(ex, ey, ez);
        const double sc = _strength * (1.0 / dist);
        return Vector3<double>(sc * (ex / el), sc * (ey / el), sc * (ez / el));
    }
    void SetPosition(Vector3<double> origin) { _origin = origin; }
    void SetStrength(double strength) { _strength = strength; }
    void SetStrengthFallOff(double f) { _strengthFallOff = f; }
    Vector3<double> GetOrigin() const { return _origin; }
    double GetStrength() const { return _strength; }
    double GetStrengthFallOff() const { return _strengthFallOff; }
    fe_force_desc Desc() const override
    {
        fe_force_desc d{};
        d.kind = FE_FORCE_POINT;
        d.origin[0] = _origin.x; d.origin[1] = _origin.y; d.origin[2] = _origin.z;
        d.strength = _strength;
        d.falloff = _strengthFallOff;
        return d;
    }

  private:
    Vector3<double> _origin;
    double _strength, _strengthFallOff;
};

// SwirlField (forces/swirlf_field.cpp:5-23): strength / max(d, 1)^2 along the displacement of a small rotation about
// the axis (Collisions::RotatePointAroundAxis / DistanceToAxis, 3d/collisions.cpp:219-246).
class SwirlField : public fluide::FieldForce {
  public:
    SwirlField(Vector3<double> origin = Vector3<double>(0), Vector3<double> axisDirection = Vector3<double>(0, 1, 0),
               double strength = 0, double strengthFallOff = 1)
        : _origin(origin), _axisGiven(axisDirection), _strength(strength), _strengthFallOff(strengthFallOff)
    {
        const double l = fluide::length3(axisDirection.x, axisDirection.y, axisDirection.z);
        _axis = Vector3<double>(axisDirection.x / l, axisDirection.y / l, axisDirection.z / l);
    }
    Vector3<double> Sample(const Vector3<double>& p) const override
    {
        const Vector3<double>& o = _origin;
        const Vector3<double>& ax = _axis;
        const double d0 = fluide::length3(o.x - ax.x, o.y - ax.y, o.z - ax.z);
        const double dx = (ax.x - o.x) / d0, dy = (ax.y - o.y) / d0, dz = (ax.z - o.z) / d0;
        const double t = (p.x - o.x) * dx + (p.y - o.y) * dy + (p.z - o.z) * dz;
        double dist = fluide::length3(p.x - (o.x + t * dx), p.y - (o.y + t * dy), p.z - (o.z + t * dz));
        dist = dist >= 1.0 ? dist : 1.0;
        const double angle = 0.0001 * 3.14159265358979323846 / 180, cA = std::cos(angle), sA = std::sin(angle);
        const double al = fluide::length3(ax.x, ax.y, ax.z);
        const double u = ax.x / al, v = ax.y / al, w = ax.z / al, x = p.x, y = p.y, z = p.z, a = o.x, b = o.y, c = o.z;
        const double rx = (a * (v * v + w * w) - u * (b * v + c * w - u * x - v * y - w * z)) * (1 - cA) + x * cA +
                          ((-1.0 * c) * v + b * w - w * y + v * z) * sA;
        const double ry = (b * (u * u + w * w) - v * (a * u + c * w - u * x - v * y - w * z)) * (1 - cA) + y * cA +
                          (c * u - a * w + w * x - u * z) * sA;
        const double rz = (c * (u * u + v * v) - w * (a * u + b * v - u * x - v * y - w * z)) * (1 - cA) + z * cA +
                          ((-1.0 * b) * u + a * v - v * x + u * y) * sA;
        const double fx = x - rx, fy = y - ry, fz = z - rz, fl = fluide::length3(fx, fy, fz);
        const double sc = _strength * (1 / (dist * dist));
        return Vector3<double>(sc * (fx / fl), sc * (fy / fl), sc * (fz / fl));
    }
    void SetOrigin(Vector3<double> origin) { _origin = origin; }
    void SetAxisDirection(Vector3<double>) {}  // the reference's setter assigns its parameter to itself (swirlf_field.cpp:36-39)
    void SetStrength(double strength) { _strength = strength; }
    void SetStrengthFallOff(double f) { _strengthFallOff = f; }
    Vector3<double> GetOrigin() const { return _origin; }
    Vector3<double> GetAxisDirection() const { return _axis; }
    double GetStrength() const { return _strength; }
    double GetStrengthFallOff() const { return _strengthFallOff; }
    fe_force_desc Desc() const override
    {
        fe_force_desc d{};
        d.kind = FE_FORCE_SWIRL;
        d.origin[0] = _origin.x; d.origin[1] = _origin.y; d.origin[2] = _origin.z;
        d.axis[0] = _axisGiven.x; d.axis[1] = _axisGiven.y; d.axis[2] = _axisGiven.z;  // the library normalises it
        d.strength = _strength;
        d.falloff = _strengthFallOff;
        return d;
    }

  private:
    Vector3<double> _origin, _axisGiven, _axis;
    double _strength, _strengthFallOff;
};

// Region description for InitializeFromRegions (layout of the C ABI's fe_seed_regions records).
struct fe_region_desc {
    int32_t kind;     // 0 box, 1 sphere
    double lo[3];     // box lower corner / sphere centre
    double hi[3];     // box upper corner / hi[0] = sphere radius
    double vel[3];    // initial velocity
};

// Triangle3D (3d/triangle_3d.hpp): vertex indices and the normal index, 0-based.
struct Triangle3D {
    size_t point1Idx, point2Idx, point3Idx, normalIdx;
    Triangle3D(size_t p1 = 0, size_t p2 = 1, size_t p3 = 2, size_t normIdx = 0)
        : point1Idx(p1), point2Idx(p2), point3Idx(p3), normalIdx(normIdx) {}
};
typedef Triangle3D Triangle3D_t;

// TriangleMesh (3d/triangle_mesh.hpp): vertices, normals and triangles as the surface tracker appends them.
class TriangleMesh {
  public:
    void Clear() { _vertices.clear(); _normals.clear(); _triangles.clear(); }
    void AddVertex(const Vector3<double>& v) { _vertices.push_back(v); }
    void AddNormal(const Vector3<double>& n) { _normals.push_back(n); }
    void AddTriangle(const Triangle3D_t& t) { _triangles.push_back(t); }
    const std::vector<Vector3<double>>& GetVerticies() const { return _vertices; }
    const std::vector<Vector3<double>>& GetNormals() const { return _normals; }
    const std::vector<Triangle3D_t>& GetTriangles() const { return _triangles; }
    std::vector<Vector3<double>>& GetVerticies() { return _vertices; }
    std::vector<Vector3<double>>& GetNormals() { return _normals; }
    std::vector<Triangle3D_t>& GetTriangles() { return _triangles; }
    std::string GetObjectName() const { return _objectName; }
    void SetObjectName(std::string name) { _objectName = std::move(name); }

  private:
    std::string _objectName;
    std::vector<Vector3<double>> _vertices, _normals;
    std::vector<Triangle3D_t> _triangles;
};

// OBJManager (3d/obj_manager.cpp): Save writes the reference's OBJ text (fe_write_obj); Load reads "o", "v", "vn"
// and three-vertex "f" lines as OBJManager::ParseLine does (:92-161).
class OBJManager {
  public:
    void Save(std::string name, const TriangleMesh& obj)
    {
        const auto& V = obj.GetVerticies();
        const auto& N = obj.GetNormals();
        const auto& T = obj.GetTriangles();
        std::vector<double> v(3 * V.size()), n(3 * N.size());
        std::vector<int64_t> t(4 * T.size());
        for (size_t i = 0; i < V.size(); ++i) { v[3 * i] = V[i].x; v[3 * i + 1] = V[i].y; v[3 * i + 2] = V[i].z; }
        for (size_t i = 0; i < N.size(); ++i) { n[3 * i] = N[i].x; n[3 * i + 1] = N[i].y; n[3 * i + 2] = N[i].z; }
        for (size_t i = 0; i < T.size(); ++i) {
            t[4 * i] = (int64_t)T[i].point1Idx; t[4 * i + 1] = (int64_t)T[i].point2Idx;
            t[4 * i + 2] = (int64_t)T[i].point3Idx; t[4 * i + 3] = (int64_t)T[i].normalIdx;
        }
        if (V.size() != N.size()) throw std::invalid_argument("OBJManager::Save: one normal per vertex expected");
        fluide::check(fe_write_obj(name.c_str(), obj.GetObjectName().c_str(), v.data(), n.data(), V.size(), t.data(),
                                   T.size()));
    }
    void Load(std::string name, TriangleMesh& obj)
    {
        FILE* f = std::fopen(name.c_str(), "rb");
        if (!f) return;  // the reference reports the error on stdout and leaves the mesh unchanged
        std::string line;
        for (int c = std::fgetc(f);; c = std::fgetc(f)) {
            if (c == '\n' || c == EOF) {
                ParseLine(line, obj);
                line.clear();
                if (c == EOF) break;
            } else {
                line.push_back((char)c);
            }
        }
        std::fclose(f);
    }

  private:
    static std::vector<std::string> Split(const std::string& s, char d)
    {
        std::vector<std::string> out;  // std::getline semantics: empty fields kept, no trailing empty field
        size_t b = 0;
        while (b < s.size()) {
            size_t e = s.find(d, b);
            if (e == std::string::npos) e = s.size();
            out.push_back(s.substr(b, e - b));
            b = e + 1;
        }
        return out;
    }
    static void ParseLine(const std::string& line, TriangleMesh& obj)
    {
        const std::vector<std::string> w = Split(line, ' ');
        if (w.empty()) return;
        if (w[0] == "o" && w.size() > 1) obj.SetObjectName(w[1]);
        else if (w[0] == "v" && w.size() > 3) obj.AddVertex(Vector3<double>(std::stod(w[1]), std::stod(w[2]), std::stod(w[3])));
        else if (w[0] == "vn" && w.size() > 3) obj.AddNormal(Vector3<double>(std::stod(w[1]), std::stod(w[2]), std::stod(w[3])));
        else if (w[0] == "f" && w.size() == 4) {
            std::vector<size_t> vs;
            std::vector<std::string> fv;
            for (size_t i = 1; i < w.size(); ++i) {
                fv = Split(w[i], '/');
                if (fv.size() > 1) vs.push_back(std::stoul(fv[0]));
            }
            obj.AddTriangle(Triangle3D_t(vs[0] - 1, vs[1] - 1, vs[2] - 1, std::stoul(fv[fv.size() - 1]) - 1));
        }
    }
};

// ScalarGrid3D (3d/scalar_grid3d.hpp): node values with origin and spacing, index i + nx * (j + ny * k) as
// Array3::GetElement (common/array3.hpp:65-74).  The subset a caller needs to hand an SDF to an emitter.
class ScalarGrid3D {
  public:
    ScalarGrid3D(const Vector3<size_t>& size = Vector3<size_t>(1), const double& initialValue = 0,
                 Vector3<double> origin = Vector3<double>(0), Vector3<double> gridSpacing = Vector3<double>(1))
        : _size(size), _origin(origin), _spacing(gridSpacing), _data(size.x * size.y * size.z, initialValue) {}
    Vector3<size_t> GetSize() const { return _size; }
    Vector3<double> GetOrigin() const { return _origin; }
    Vector3<double> GetGridSpacing() const { return _spacing; }
    Vector3<double> GridIndexToPosition(size_t i, size_t j, size_t k) const
    {
        return Vector3<double>(_origin.x + i * _spacing.x, _origin.y + j * _spacing.y, _origin.z + k * _spacing.z);
    }
    const double& GetElement(size_t i, size_t j, size_t k) const { return _data.at(i + _size.x * (j + _size.y * k)); }
    double& GetElement(size_t i, size_t j, size_t k) { return _data.at(i + _size.x * (j + _size.y * k)); }
    void SetElement(size_t i, size_t j, size_t k, double value) { GetElement(i, j, k) = value; }
    const double& operator()(size_t i, size_t j, size_t k) const { return GetElement(i, j, k); }
    double& operator()(size_t i, size_t j, size_t k) { return GetElement(i, j, k); }
    const std::vector<double>& GetRawData() const { return _data; }

  private:
    Vector3<size_t> _size;
    Vector3<double> _origin, _spacing;
    std::vector<double> _data;
};

namespace fluide {
// A TriangleMesh as the C ABI takes it: 3 doubles per vertex, 4 int64 per triangle (vertex ids, normal id).
inline void flatten_mesh(const TriangleMesh& mesh, std::vector<double>& V, std::vector<int64_t>& T)
{
    V.clear();
    T.clear();
    for (const auto& v : mesh.GetVerticies()) {
        V.push_back(v.x);
        V.push_back(v.y);
        V.push_back(v.z);
    }
    for (const auto& t : mesh.GetTriangles()) {
        T.push_back((int64_t)t.point1Idx);
        T.push_back((int64_t)t.point2Idx);
        T.push_back((int64_t)t.point3Idx);
        T.push_back((int64_t)t.normalIdx);
    }
}
}  // namespace fluide

// VolumeField (forces/volume_field.cpp:5-89): at every node of its grid (`resolution` nodes over `domain`) the
// vector from the node to the closest point of the mesh; Sample interpolates it trilinearly and pushes along its
// negation with strength / max(|vector|, 1)^2.  The vectors are computed on the GPU (fe_volume_field_vectors) on
// first use; the simulators apply the force on the GPU.
class VolumeField : public fluide::FieldForce {
  public:
    VolumeField(const TriangleMesh& mesh, Vector3<size_t> resolution, BoundingBox3D domain, double strength)
        : _resolution(resolution), _strength(strength)
    {
        const Vector3<double> s = domain.GetSize();
        _domainSize = s;
        _origin = domain.GetOrigin();
        _gridSpacing = Vector3<double>(s.x / resolution.x, s.y / resolution.y, s.z / resolution.z);
        fluide::flatten_mesh(mesh, _V, _T);
    }
    Vector3<double> Sample(const Vector3<double>& p) const override
    {
        const std::vector<double>& f = Vectors();
        const size_t n[3] = {_resolution.x, _resolution.y, _resolution.z};
        const double x[3] = {(p.x - _origin.x) / _gridSpacing.x, (p.y - _origin.y) / _gridSpacing.y,
                             (p.z - _origin.z) / _gridSpacing.z};
        size_t i0[3], i1[3];
        double fr[3];
        for (int a = 0; a < 3; ++a) {  // GetBarycentric (common/math_utils.hpp:48-73), iLow 0, iHigh n - 1
            const int hi = (int)n[a] - 1;
            const double fl = std::floor(x[a]);
            int ii = (int)fl;
            if (hi == 0 || ii < 0) { ii = 0; fr[a] = 0.0; }
            else if (ii > hi - 1) { ii = hi - 1; fr[a] = 1.0; }
            else fr[a] = x[a] - fl;
            i0[a] = (size_t)ii;
            i1[a] = std::min((size_t)ii + 1, n[a] - 1);
        }
        auto at = [&](size_t i, size_t j, size_t k, int c) { return f[3 * (i + n[0] * (j + n[1] * k)) + c]; };
        auto lerp = [](double a, double b, double t) { return (1 - t) * a + t * b; };
        double q[3];
        for (int c = 0; c < 3; ++c) {
            const double b0 = lerp(lerp(at(i0[0], i0[1], i0[2], c), at(i1[0], i0[1], i0[2], c), fr[0]),
                                   lerp(at(i0[0], i1[1], i0[2], c), at(i1[0], i1[1], i0[2], c), fr[0]), fr[1]);
            const double b1 = lerp(lerp(at(i0[0], i0[1], i1[2], c), at(i1[0], i0[1], i1[2], c), fr[0]),
                                   lerp(at(i0[0], i1[1], i1[2], c), at(i1[0], i1[1], i1[2], c), fr[0]), fr[1]);
            q[c] = lerp(b0, b1, fr[2]);
        }
        const double len = fluide::length3(q[0], q[1], q[2]);
        const double dist = len >= 1.0 ? len : 1.0;
        const double sc = _strength * (1 / (dist * dist));
        return Vector3<double>(sc * ((q[0] / len) * -1.0), sc * ((q[1] / len) * -1.0), sc * ((q[2] / len) * -1.0));
    }
    void SetStrength(double strength) { _strength = strength; }
    double GetStrength() const { return _strength; }
    // The node vectors (3 per node, x-fastest), computed on the GPU the first time they are needed.
    const std::vector<double>& Vectors() const
    {
        if (_field.empty()) {
            std::vector<double> f(3 * _resolution.x * _resolution.y * _resolution.z);
            const int32_t n[3] = {(int32_t)_resolution.x, (int32_t)_resolution.y, (int32_t)_resolution.z};
            const double o[3] = {_origin.x, _origin.y, _origin.z}, h[3] = {_gridSpacing.x, _gridSpacing.y, _gridSpacing.z};
            fluide::check(fe_volume_field_vectors(_V.data(), _V.size() / 3, _T.data(), _T.size() / 4, n, o, h, f.data(), 0));
            _field = std::move(f);
        }
        return _field;
    }
    fe_force_desc Desc() const override
    {
        fe_force_desc d{};
        d.kind = FE_FORCE_VOLUME;
        d.strength = _strength;
        d.resolution[0] = (int32_t)_resolution.x; d.resolution[1] = (int32_t)_resolution.y;
        d.resolution[2] = (int32_t)_resolution.z;
        d.domain_origin[0] = _origin.x; d.domain_origin[1] = _origin.y; d.domain_origin[2] = _origin.z;
        d.domain_size[0] = _domainSize.x; d.domain_size[1] = _domainSize.y; d.domain_size[2] = _domainSize.z;
        d.field = Vectors().data();
        return d;
    }

  private:
    Vector3<size_t> _resolution;
    Vector3<double> _origin, _gridSpacing, _domainSize;
    double _strength;
    std::vector<double> _V;
    std::vector<int64_t> _T;
    mutable std::vector<double> _field;
};

// Collider (3d/collider.hpp): the base the simulators take in AddCollider.
class Collider {
  public:
    virtual ~Collider() = default;
    virtual bool IsInside(const Vector3<double>& position) = 0;
    virtual double GetClosestDistanceAt(const Vector3<double>& position) = 0;
    virtual Vector3<double> GetVelocityAt(const Vector3<double>& position) = 0;
};

// TriangleMeshCollider (3d/triangle_mesh_collider.cpp:4-100): a static solid given by a mesh with normals and the
// node grid its Mesh2SDF lives on.  The simulators run its boundary condition and collision response on the GPU;
// the distance queries here sample the same SDF (computed on the GPU, fe_mesh_to_sdf, the first time one is asked).
class TriangleMeshCollider : public Collider {
  public:
    TriangleMeshCollider(const Vector3<size_t>& gridSize, const Vector3<double>& gridOrigin,
                         const Vector3<double>& gridSpacing, const TriangleMesh& mesh)
        : _n(gridSize), _origin(gridOrigin), _spacing(gridSpacing)
    {
        fluide::flatten_mesh(mesh, _V, _T);
        for (const auto& nrm : mesh.GetNormals()) {
            _N.push_back(nrm.x);
            _N.push_back(nrm.y);
            _N.push_back(nrm.z);
        }
    }
    bool IsInside(const Vector3<double>& position) override { return GetClosestDistanceAt(position) < 0; }
    // ScalarGrid3D::Sample of the collider's SDF (3d/scalar_grid3d.cpp:33-65)
    double GetClosestDistanceAt(const Vector3<double>& p) override
    {
        const std::vector<double>& f = Sdf();
        const size_t n[3] = {_n.x, _n.y, _n.z};
        const double x[3] = {(p.x - _origin.x) / _spacing.x, (p.y - _origin.y) / _spacing.y, (p.z - _origin.z) / _spacing.z};
        size_t i0[3], i1[3];
        double fr[3];
        for (int a = 0; a < 3; ++a) {
            const int hi = (int)n[a] - 1;
            const double fl = std::floor(x[a]);
            int ii = (int)fl;
            if (hi == 0 || ii < 0) { ii = 0; fr[a] = 0.0; }
            else if (ii > hi - 1) { ii = hi - 1; fr[a] = 1.0; }
            else fr[a] = x[a] - fl;
            i0[a] = (size_t)ii;
            i1[a] = std::min((size_t)ii + 1, n[a] - 1);
        }
        auto at = [&](size_t i, size_t j, size_t k) { return f[i + n[0] * (j + n[1] * k)]; };
        auto lerp = [](double a, double b, double t) { return (1 - t) * a + t * b; };
        const double b0 = lerp(lerp(at(i0[0], i0[1], i0[2]), at(i1[0], i0[1], i0[2]), fr[0]),
                               lerp(at(i0[0], i1[1], i0[2]), at(i1[0], i1[1], i0[2]), fr[0]), fr[1]);
        const double b1 = lerp(lerp(at(i0[0], i0[1], i1[2]), at(i1[0], i0[1], i1[2]), fr[0]),
                               lerp(at(i0[0], i1[1], i1[2]), at(i1[0], i1[1], i1[2]), fr[0]), fr[1]);
        return lerp(b0, b1, fr[2]);
    }
    Vector3<double> GetVelocityAt(const Vector3<double>&) override { return Vector3<double>(0.0); }  // returns 0
    // Registers the collider with a scene (fe_scene_add_mesh_collider).
    void AddTo(fe_scene* scene) const
    {
        const int32_t res[3] = {(int32_t)_n.x, (int32_t)_n.y, (int32_t)_n.z};
        const double o[3] = {_origin.x, _origin.y, _origin.z}, h[3] = {_spacing.x, _spacing.y, _spacing.z};
        fluide::check(fe_scene_add_mesh_collider(scene, _V.data(), _V.size() / 3, _T.data(), _T.size() / 4, _N.data(),
                                                 _N.size() / 3, res, o, h, nullptr));
    }

  private:
    const std::vector<double>& Sdf()
    {
        if (_sdf.empty()) {
            std::vector<double> f(_n.x * _n.y * _n.z);
            const int32_t n[3] = {(int32_t)_n.x, (int32_t)_n.y, (int32_t)_n.z};
            const double o[3] = {_origin.x, _origin.y, _origin.z}, h[3] = {_spacing.x, _spacing.y, _spacing.z};
            fluide::check(fe_mesh_to_sdf(_V.data(), _V.size() / 3, _T.data(), _T.size() / 4, n, o, h, f.data(), 0));
            _sdf = std::move(f);
        }
        return _sdf;
    }
    Vector3<size_t> _n;
    Vector3<double> _origin, _spacing;
    std::vector<double> _V, _N, _sdf;
    std::vector<int64_t> _T;
};

// ColliderCollection (3d/collider_collection.hpp): the colliders of PICSimulator::SetColliders.
class ColliderCollection {
  public:
    ColliderCollection(const Vector3<size_t>& = Vector3<size_t>(1), const Vector3<double>& = Vector3<double>(1),
                       const Vector3<double>& = Vector3<double>(0)) {}
    void AddCollider(std::shared_ptr<Collider> collider) { _colliders.push_back(collider); }
    std::vector<std::shared_ptr<Collider>>& GetColliders() { return _colliders; }
    bool IsInside(const Vector3<double>& position)
    {
        for (auto& c : _colliders)
            if (c->IsInside(position)) return true;
        return false;
    }

  private:
    std::vector<std::shared_ptr<Collider>> _colliders;
};

// Emitter (emmiter/emmiter.hpp): the base the simulators take in AddEmitter.
class Emitter {
  public:
    virtual ~Emitter() = default;
};

// VolumeEmitter (emmiter/volume_emmiter.cpp:8-86): at the start of every substep, each node of its grid
// (`resolution` nodes over `domain`) whose SDF is <= 0 and where the fluid SDF of the previous substep is >= 0
// receives particlesPerBlock particles at node + spacing * U[0,1]^3 with `velocity`.  The SDF comes from the mesh
// (Mesh2SDF, built on the GPU when the emitter is registered with a scene) or from InitializeFromSdf.
// velocityVariance is kept and unused, as in the reference.  The resolution must be within the simulator's grid
// (the emitter indexes the fluid SDF with its own node indices).  Changing the emitter after AddEmitter takes
// effect at the simulator's next step.
class VolumeEmitter : public Emitter {
  public:
    VolumeEmitter(const TriangleMesh& mesh, Vector3<size_t> resolution, BoundingBox3D domain, const size_t& particlesPerBlock,
                  const Vector3<double>& velocity, const Vector3<double>& velocityVariance)
        : _resolution(resolution), _domain(domain), _particlesPerBlock(particlesPerBlock), _velocity(velocity),
          _velocityVariance(velocityVariance)
    {
        InitializeFromTriangleMesh(mesh);
    }
    void InitializeFromTriangleMesh(const TriangleMesh& mesh)
    {
        fluide::flatten_mesh(mesh, _V, _T);
        _sdf.clear();
        ++_version;
    }
    // VolumeEmitter::InitializeFromSdf (:50-56): the emitter's node (i, j, k) takes sdf(i, j, k).
    void InitializeFromSdf(const ScalarGrid3D& sdf)
    {
        const Vector3<size_t> n = sdf.GetSize();
        if (n.x < _resolution.x || n.y < _resolution.y || n.z < _resolution.z)
            throw std::invalid_argument("InitializeFromSdf: the grid must cover the emitter's resolution");
        std::vector<double> v(_resolution.x * _resolution.y * _resolution.z);
        for (size_t k = 0; k < _resolution.z; ++k)
            for (size_t j = 0; j < _resolution.y; ++j)
                for (size_t i = 0; i < _resolution.x; ++i) v[i + _resolution.x * (j + _resolution.y * k)] = sdf(i, j, k);
        _sdf = std::move(v);
        ++_version;
    }
    Vector3<double> GetVelocity() const { return _velocity; }
    Vector3<double> GetVelocityVariance() const { return _velocityVariance; }
    size_t GetParticlesPerBlock() const { return _particlesPerBlock; }
    uint64_t Version() const { return _version; }

    // Registers the emitter with a scene (fe_scene_add_volume_emitter, then fe_scene_set_emitter_sdf for an SDF).
    int32_t AddTo(fe_scene* scene, uint64_t seed) const
    {
        const int32_t res[3] = {(int32_t)_resolution.x, (int32_t)_resolution.y, (int32_t)_resolution.z};
        const Vector3<double> o = _domain.GetOrigin(), sz = _domain.GetSize();
        const double origin[3] = {o.x, o.y, o.z}, size[3] = {sz.x, sz.y, sz.z};
        const double vel[3] = {_velocity.x, _velocity.y, _velocity.z};
        int32_t id = -1;
        fluide::check(fe_scene_add_volume_emitter(scene, _V.data(), _V.size() / 3, _T.data(), _T.size() / 4, res, origin,
                                                  size, (uint32_t)_particlesPerBlock, vel, seed, &id));
        if (!_sdf.empty()) fluide::check(fe_scene_set_emitter_sdf(scene, id, _sdf.data()));
        return id;
    }

  private:
    Vector3<size_t> _resolution;
    BoundingBox3D _domain;
    size_t _particlesPerBlock;
    Vector3<double> _velocity, _velocityVariance;
    std::vector<double> _V, _sdf;
    std::vector<int64_t> _T;
    uint64_t _version = 0;
};

class PhysicsAnimation {
  public:
    virtual ~PhysicsAnimation() = default;
    // physics_animation.cpp:17-21 + OnUpdate :48-61: advance by one frame of the current frame's interval
    void AdvanceSingleFrame()
    {
        Frame f = _currentFrame;
        ++f;
        _currentTime = _currentFrame.GetTimeInSeconds();
        _numberOfTimeSteps = AdvanceTimeStep(f.GetTimeIntervalInSeconds());
        _currentTime += f.GetTimeIntervalInSeconds();
        _currentFrame = f;
    }
    void SetCurrentFrame(const Frame& frame) { _currentFrame = frame; }
    Frame GetCurrentFrame() const { return _currentFrame; }
    double GetCurrentTimeInSeconds() const { return _currentTime; }
    void SetNumberOfSubTimesteps(unsigned n) { _numberOfSubTimesteps = n; }
    unsigned GetNumberOfSubTimeSteps() const { return _numberOfTimeSteps; }

  protected:
    virtual unsigned AdvanceTimeStep(double timeIntervalInSeconds) = 0;
    Frame _currentFrame;
    double _currentTime = 0.0;
    unsigned _numberOfSubTimesteps = 1;
    unsigned _numberOfTimeSteps = 0;
};

class HybridSimulator : public PhysicsAnimation {
  public:
    HybridSimulator(const Vector3<size_t>& gridSize, const BoundingBox3D& domain, fe_solver_kind kind)
        : _n(gridSize), _domain(domain), _kind(kind)
    {
        fluide::check(fe_scene_desc_default(&_desc));
        _desc.n[0] = (int32_t)gridSize.x;
        _desc.n[1] = (int32_t)gridSize.y;
        _desc.n[2] = (int32_t)gridSize.z;
        const Vector3<double> o = domain.GetOrigin(), s = domain.GetSize();
        _desc.origin[0] = o.x; _desc.origin[1] = o.y; _desc.origin[2] = o.z;
        _desc.size[0] = s.x; _desc.size[1] = s.y; _desc.size[2] = s.z;
        _desc.solver = kind;
        _desc.max_cfl = 3.0;  // hybrid_simulator.cpp:21
        _desc.gravity[0] = _desc.gravity[1] = _desc.gravity[2] = 0.0;
    }
    ~HybridSimulator() override
    {
        if (_scene) fe_scene_destroy(_scene);
    }
    HybridSimulator(const HybridSimulator&) = delete;
    HybridSimulator& operator=(const HybridSimulator&) = delete;

    double Cfl(double timeIntervalInSeconds)
    {
        double c = 0.0;
        fluide::check(fe_scene_cfl(Scene(), timeIntervalInSeconds, &c));
        return c;
    }
    double MaxCfl() const { return _desc.max_cfl; }
    double GetViscosity() const { return _desc.viscosity; }
    double GetDensity() const { return _density; }
    size_t GetParticlesPerBlock() const { return _particlesPerBlok; }
    Vector3<double> GetOrigin() const { return _domain.GetOrigin(); }
    Vector3<size_t> GetResolution() const { return _n; }
    Vector3<double> GetGridSpacing() const
    {
        const Vector3<double> s = _domain.GetSize();
        return Vector3<double>(s.x / _n.x, s.y / _n.y, s.z / _n.z);
    }
    size_t GetNumberOfParticles() const
    {
        if (!_scene) return _pos.size() / 3;
        uint64_t n = 0;
        fluide::check(fe_scene_num_particles(_scene, &n));
        return (size_t)n;
    }
    void SetMaxClf(double maxCfl) { Reconfigure([&] { _desc.max_cfl = maxCfl; }); }
    // HybridSimulator::SetViscosity (hybrid_simulator.cpp:97-100): > 0 adds ComputeDiffusion to every substep
    // (pic_simulator.cpp:214-222), the reference's BackwardEulerDiffusionSolver with its Jacobi settings.
    void SetViscosity(double viscosity)
    {
        if (_scene) fluide::check(fe_scene_set_viscosity(_scene, viscosity));
        else if (!(viscosity >= 0.0) || !std::isfinite(viscosity)) throw std::invalid_argument("viscosity must be >= 0");
        _desc.viscosity = viscosity;
    }
    void SetDensity(double density) { _density = density; }  // unused by the projection, as in the reference
    void SetParticlesPerBlock(size_t n) { _particlesPerBlok = n; }

    // Pressure solver settings (the reference swaps LinearSystemSolver objects, pic_simulator.cpp:56-59).
    void SetPressureSolverTolerance(double relTol, int maxIterations)
    {
        Reconfigure([&] { _desc.cg_rel_tol = relTol; _desc.cg_max_it = maxIterations; });
    }
    // Inner solver of the projection: FE_PRESSURE_AUTO (default), FE_PRESSURE_MGPCG or FE_PRESSURE_CG.
    void SetPressureSolverKind(fe_pressure_solver kind) { Reconfigure([&] { _desc.pressure_solver = kind; }); }

    // Particle seeding and access (the reference seeds only through InitializeParticles' std::rand).
    size_t InitializeFromRegions(const std::vector<fe_region_desc>& regions, uint64_t seed = 0);
    void SetParticles(const std::vector<float>& pos, const std::vector<float>& vel, const std::vector<float>& C = {})
    {
        _pos = pos;
        _vel = vel.empty() ? std::vector<float>(pos.size(), 0.f) : vel;
        _C = C;
        if (_scene) Upload();
    }
    void GetParticles(std::vector<float>& pos, std::vector<float>& vel, std::vector<float>* C = nullptr)
    {
        if (!_scene) {
            pos = _pos;
            vel = _vel;
            if (C) *C = _C;
            return;
        }
        const size_t n = GetNumberOfParticles();
        pos.resize(3 * n);
        vel.resize(3 * n);
        if (C) C->resize(9 * n);
        fluide::check(fe_scene_get_particles(_scene, pos.data(), vel.data(), C ? C->data() : nullptr, n));
    }

    // Fixed-dt substeps (the benchmark configurations' mode); stats may be null.
    void AdvanceFixedSubsteps(double dt, int nsub, fe_step_stats* stats = nullptr)
    {
        SyncEmitters();
        _meshSdfLive = false;
        fluide::check(fe_scene_step(Scene(), dt, nsub, stats));
    }

    // PICSimulator::AddExternalForce (pic_simulator.cpp:41-44).  DirectionalFields add up to the scene's gravity;
    // PointField, SwirlField and VolumeField are applied after it on the GPU, in the order added.
    void AddExternalForce(const std::shared_ptr<ExternalForce> newForce)
    {
        if (auto field = std::dynamic_pointer_cast<fluide::FieldForce>(newForce)) {
            const fe_force_desc d = field->Desc();
            if (_scene) fluide::check(fe_scene_add_force(_scene, &d, nullptr));
            _fieldForces.push_back(field);
            _forces.push_back(newForce);
            return;
        }
        if (!std::dynamic_pointer_cast<DirectionalField>(newForce))
            throw std::invalid_argument("AddExternalForce: DirectionalField, PointField, SwirlField or VolumeField expected");
        Reconfigure([&] {
            const Vector3<double> g = newForce->Sample(Vector3<double>(0));
            _desc.gravity[0] += g.x;
            _desc.gravity[1] += g.y;
            _desc.gravity[2] += g.z;
        });
        _forces.push_back(newForce);
    }
    // PICSimulator::AddCollider / SetColliders (pic_simulator.cpp:61-69): TriangleMeshColliders, applied on the GPU
    // (boundary condition, BOUNDRY cells, collision response).  A simulator with colliders cannot have a viscosity.
    void AddCollider(std::shared_ptr<Collider> collider)
    {
        auto m = std::dynamic_pointer_cast<TriangleMeshCollider>(collider);
        if (!m) throw std::invalid_argument("AddCollider: a TriangleMeshCollider is expected");
        if (_scene) m->AddTo(_scene);
        _colliders.push_back(m);
    }
    void SetColliders(std::shared_ptr<ColliderCollection> colliders)
    {
        std::vector<std::shared_ptr<TriangleMeshCollider>> list;
        for (auto& c : colliders->GetColliders()) {
            auto m = std::dynamic_pointer_cast<TriangleMeshCollider>(c);
            if (!m) throw std::invalid_argument("SetColliders: TriangleMeshColliders are expected");
            list.push_back(m);
        }
        if (_scene) fluide::check(fe_scene_clear_colliders(_scene));
        _colliders = list;
        if (_scene)
            for (auto& m : _colliders) m->AddTo(_scene);
    }
    // PICSimulator::AddEmitter (pic_simulator.cpp:46-49); emitters are registered with the scene at the next step.
    void AddEmitter(std::shared_ptr<Emitter> emitter)
    {
        auto v = std::dynamic_pointer_cast<VolumeEmitter>(emitter);
        if (!v) throw std::invalid_argument("AddEmitter: a VolumeEmitter is expected");
        _emitters.push_back(v);
    }
    // PICSimulator::InitializeFromTriangleMesh (pic_simulator.cpp:33-39): the mesh SDF becomes the fluid SDF and
    // every cell inside it receives GetParticlesPerBlock() particles (appended to the particles already set).
    // The fluid SDF stays the mesh's until the first substep, also across settings changes that rebuild the scene.
    void InitializeFromTriangleMesh(const TriangleMesh& mesh)
    {
        std::vector<double> V;
        std::vector<int64_t> T;
        fluide::flatten_mesh(mesh, V, T);
        fluide::check(fe_scene_init_from_mesh(Scene(), V.data(), V.size() / 3, T.data(), T.size() / 4,
                                              (uint32_t)_particlesPerBlok, _meshSeed++));
        _meshSdfLive = true;
    }
    // HybridSimulator::GetFluidSdf (hybrid_simulator.hpp:35): Fluid3::sdf, the SDF built at the start of the last
    // substep (or the mesh SDF of InitializeFromTriangleMesh before any), on the nodes at origin + h / 2.
    ScalarGrid3D GetFluidSdf()
    {
        const Vector3<double> h = GetGridSpacing(), o = GetOrigin();
        ScalarGrid3D g(_n, 0.0, Vector3<double>(o.x + h.x / 2.0, o.y + h.y / 2.0, o.z + h.z / 2.0), h);
        std::vector<double> v(_n.x * _n.y * _n.z);
        fluide::check(fe_scene_get_fluid_sdf(Scene(), v.data()));
        for (size_t k = 0; k < _n.z; ++k)
            for (size_t j = 0; j < _n.y; ++j)
                for (size_t i = 0; i < _n.x; ++i) g(i, j, k) = v[i + _n.x * (j + _n.y * k)];
        return g;
    }
    // PICSimulator::GetSurface (pic_simulator.cpp:71-78): appends the marching-cubes surface of Fluid3::sdf (the
    // SDF built at the start of the last substep) to mesh, exactly as the reference's surface tracker does.
    void GetSurface(TriangleMesh& mesh)
    {
        uint64_t nv = 0, nt = 0;
        fluide::check(fe_scene_build_surface(Scene(), &nv, &nt));
        std::vector<double> v(3 * nv), n(3 * nv);
        std::vector<int64_t> t(4 * nt);
        fluide::check(fe_scene_get_surface(Scene(), v.data(), n.data(), t.data()));
        const size_t base = mesh.GetVerticies().size();  // ids continue after what the mesh holds
        for (uint64_t i = 0; i < nv; ++i) {
            mesh.AddNormal(Vector3<double>(n[3 * i], n[3 * i + 1], n[3 * i + 2]));
            mesh.AddVertex(Vector3<double>(v[3 * i], v[3 * i + 1], v[3 * i + 2]));
        }
        for (uint64_t i = 0; i < nt; ++i)
            mesh.AddTriangle(Triangle3D_t(base + (size_t)t[4 * i], base + (size_t)t[4 * i + 1], base + (size_t)t[4 * i + 2],
                                          base + (size_t)t[4 * i + 3]));
    }

    fe_scene* Scene()
    {
        if (!_scene) {
            fluide::check(fe_scene_create(&_desc, &_scene));
            ++_sceneGeneration;
            for (const auto& f : _fieldForces) {
                const fe_force_desc d = f->Desc();
                fluide::check(fe_scene_add_force(_scene, &d, nullptr));
            }
            for (const auto& c : _colliders) c->AddTo(_scene);
            Upload();
            if (_meshSdfLive && !_sdf.empty()) fluide::check(fe_scene_set_fluid_sdf(_scene, _sdf.data()));
            _sdf.clear();
        }
        return _scene;
    }

  protected:
    unsigned AdvanceTimeStep(double timeIntervalInSeconds) override
    {
        SyncEmitters();
        _meshSdfLive = false;
        int32_t n = 0;
        fluide::check(fe_scene_advance_frame(Scene(), timeIntervalInSeconds, &n));
        return (unsigned)n;
    }
    template <class F>
    void Reconfigure(F change)
    {
        if (_scene) {  // keep the particles (and a mesh-initialised fluid SDF): read back, rebuild with the new settings
            GetParticles(_pos, _vel, _kind == FE_SOLVER_APIC ? &_C : nullptr);
            if (_meshSdfLive) {
                _sdf.resize((size_t)_n.x * _n.y * _n.z);
                fluide::check(fe_scene_get_fluid_sdf(_scene, _sdf.data()));
            }
            fe_scene_destroy(_scene);
            _scene = nullptr;
        }
        change();
    }
    // (Re-)registers the emitters when the scene is new or an emitter changed since its registration.
    void SyncEmitters()
    {
        fe_scene* s = Scene();
        bool stale = _emitterGeneration != _sceneGeneration || _emitterVersions.size() != _emitters.size();
        for (size_t i = 0; !stale && i < _emitters.size(); ++i) stale = _emitterVersions[i] != _emitters[i]->Version();
        if (!stale) return;
        fluide::check(fe_scene_clear_emitters(s));
        _emitterVersions.clear();
        for (size_t i = 0; i < _emitters.size(); ++i) {
            _emitters[i]->AddTo(s, 0x5EED0000ull + i);
            _emitterVersions.push_back(_emitters[i]->Version());
        }
        _emitterGeneration = _sceneGeneration;
    }
    void Upload()
    {
        const size_t n = _pos.size() / 3;
        if (n == 0) return;
        fluide::check(fe_scene_set_particles(_scene, _pos.data(), _vel.data(), _C.empty() ? nullptr : _C.data(), n));
    }

    Vector3<size_t> _n;
    BoundingBox3D _domain;
    fe_solver_kind _kind;
    fe_scene_desc _desc{};
    fe_scene* _scene = nullptr;
    double _density = 1.0;
    size_t _particlesPerBlok = 16;  // hybrid_simulator.cpp:22
    std::vector<float> _pos, _vel, _C;
    std::vector<std::shared_ptr<ExternalForce>> _forces;
    std::vector<std::shared_ptr<fluide::FieldForce>> _fieldForces;
    std::vector<std::shared_ptr<TriangleMeshCollider>> _colliders;
    std::vector<std::shared_ptr<VolumeEmitter>> _emitters;
    std::vector<uint64_t> _emitterVersions;
    uint64_t _sceneGeneration = 0, _emitterGeneration = 0, _meshSeed = 0;
    bool _meshSdfLive = false;  // InitializeFromTriangleMesh ran and no substep since
    std::vector<double> _sdf;   // its SDF while the scene is rebuilt
};

inline size_t HybridSimulator::InitializeFromRegions(const std::vector<fe_region_desc>& regions, uint64_t seed)
{
    const int32_t n[3] = {(int32_t)_n.x, (int32_t)_n.y, (int32_t)_n.z};
    const double o[3] = {_desc.origin[0], _desc.origin[1], _desc.origin[2]};
    const double s[3] = {_desc.size[0], _desc.size[1], _desc.size[2]};
    const uint64_t cnt = fe_seed_regions(regions.data(), (int32_t)regions.size(), n, o, s, seed, nullptr, nullptr, 0);
    std::vector<float> pos(3 * cnt), vel(3 * cnt);
    fe_seed_regions(regions.data(), (int32_t)regions.size(), n, o, s, seed, pos.data(), vel.data(), cnt);
    SetParticles(pos, vel);
    return (size_t)cnt;
}

class PICSimulator : public HybridSimulator {
  public:
    PICSimulator(const Vector3<size_t>& gridSize, const BoundingBox3D& domain)
        : HybridSimulator(gridSize, domain, FE_SOLVER_PIC) {}

  protected:
    PICSimulator(const Vector3<size_t>& gridSize, const BoundingBox3D& domain, fe_solver_kind kind)
        : HybridSimulator(gridSize, domain, kind) {}
};

class FLIPSimulator : public PICSimulator {
  public:
    FLIPSimulator(const Vector3<size_t>& gridSize, const BoundingBox3D& domain)
        : PICSimulator(gridSize, domain, FE_SOLVER_FLIP) {}
    // flip_simulator.cpp:15-23: v = Lerp(flip, pic, factor), default 0.05
    void SetBlendingFactor(double factor) { Reconfigure([&] { _desc.flip_blend = factor; }); }
    double GetBlendingFactor() const { return _desc.flip_blend; }
};

class APICSimulator : public PICSimulator {
  public:
    APICSimulator(const Vector3<size_t>& gridSize, const BoundingBox3D& domain)
        : PICSimulator(gridSize, domain, FE_SOLVER_APIC) {}
};

// SimulationStats (simulation_stats.hpp / .cpp), printed in the reference's format (including its swapped
// "Median CFL" / "Mean CFL" labels, simulation_stats.cpp:27-28).
class SimulationStats {
  public:
    void PrintStats(std::FILE* out = stdout) const
    {
        std::fprintf(out, "================ SIMULATION STATS ================\n");
        std::fprintf(out, "Simulator type: %s\n", simulatorType.c_str());
        std::fprintf(out, "Grid resolution: %zu x %zu x %zu\n", gridSize.x, gridSize.y, gridSize.z);
        std::fprintf(out, "Number of particles: %zu\n", numberOfParticles);
        std::fprintf(out, "Number of Iterations: %zu\n", numberOfIterations);
        std::fprintf(out, "Time interval: %g [s]\n", timeIntervalInSeconds);
        std::fprintf(out, "Median CFL: %g\n", Mean(cflPerIteration));
        std::fprintf(out, "Mean CFL: %g\n", Median(cflPerIteration));
        std::fprintf(out, "Median frame: %g [s]\n", Median(iterationTimeInSeconds));
        std::fprintf(out, "Mean frame: %g [s]\n", Mean(iterationTimeInSeconds));
        std::fprintf(out, "Simulation time: %g [s]\n", simulationTimeInSeconds);
        std::fprintf(out, "==================================================\n");
    }
    void Clear() { *this = SimulationStats(); }
    static double Median(std::vector<double> v)
    {
        if (v.empty()) return std::numeric_limits<double>::signaling_NaN();
        auto i1 = v.begin() + (v.size() - 1) / 2, i2 = v.begin() + v.size() / 2;
        std::nth_element(v.begin(), i1, v.end());
        std::nth_element(i1, i2, v.end());
        return 0.5 * (*i1 + *i2);
    }
    static double Mean(const std::vector<double>& v)
    {
        return v.empty() ? 0.0 : std::accumulate(v.begin(), v.end(), 0.0) / v.size();
    }

    std::string simulatorType;
    size_t numberOfIterations = 0;
    Vector3<size_t> gridSize = Vector3<size_t>(0);
    size_t numberOfParticles = 0;
    double timeIntervalInSeconds = 0;
    double simulationTimeInSeconds = 0;
    std::vector<double> iterationTimeInSeconds;
    std::vector<double> cflPerIteration;
};

// SimulationRunner (simulation_runner.cpp:16-56): for each iteration, AdvanceSingleFrame, GetSurface and
// OBJManager::Save to <cache>/simulated_frames/<name>_<i>.obj, with the log (iterations, stats) in <cache>/log.txt.
// The OBJ of frame i is written by a host thread while the GPU advances frame i + 1 (the mesh is copied to the
// host first); the per-iteration time therefore covers the frame and its surface, and the last write is waited
// for before RunSimulation returns.
class SimulationRunner {
  public:
    void RunSimulation(const std::shared_ptr<HybridSimulator> simulator, double timeIntervalInSeconds,
                       size_t numberOfIterations, std::string simulationOutputName, std::string cacheFolderPath)
    {
        simulator->SetCurrentFrame(Frame(timeIntervalInSeconds));
        std::filesystem::create_directories(cacheFolderPath);
        std::filesystem::create_directories(cacheFolderPath + "/simulated_frames");
        std::FILE* log = std::fopen((cacheFolderPath + "/log.txt").c_str(), "w");
        std::thread writer;
        std::exception_ptr write_error;
        for (size_t i = 0; i < numberOfIterations; ++i) {
            if (log) std::fprintf(log, "Iteration: %zu\n", i);
            const auto start = std::chrono::steady_clock::now();
            simulator->AdvanceSingleFrame();
            auto surface = std::make_shared<TriangleMesh>();
            simulator->GetSurface(*surface);
            const std::string path = cacheFolderPath + "/simulated_frames/" + simulationOutputName + "_" +
                                     std::to_string(i) + ".obj";
            if (writer.joinable()) writer.join();
            if (write_error) std::rethrow_exception(write_error);
            writer = std::thread([surface, path, &write_error] {
                try {
                    OBJManager().Save(path, *surface);
                } catch (...) {
                    write_error = std::current_exception();
                }
            });
            const auto end = std::chrono::steady_clock::now();
            const double duration = std::chrono::duration_cast<std::chrono::nanoseconds>(end - start).count() / 1e9;
            _stats.simulationTimeInSeconds += duration;
            _stats.iterationTimeInSeconds.push_back(duration);
            _stats.cflPerIteration.push_back(simulator->Cfl(timeIntervalInSeconds));
            if (log) std::fprintf(log, "\n");
        }
        if (writer.joinable()) writer.join();
        if (write_error) std::rethrow_exception(write_error);
        _stats.numberOfIterations = numberOfIterations;
        _stats.timeIntervalInSeconds = timeIntervalInSeconds;
        _stats.simulatorType = typeid(*simulator.get()).name();
        _stats.numberOfParticles = simulator->GetNumberOfParticles();
        _stats.gridSize = simulator->GetResolution();
        if (log) {
            _stats.PrintStats(log);
            std::fclose(log);
        }
    }
    SimulationStats GetStats() const { return _stats; }

  private:
    SimulationStats _stats;
};

#endif  // FLUIDE_ENGINE_HPP
