// api_collider.cpp -- the collider scene of the reference's test/pic_simulator_test.cpp:130-165 through the C++
// drop-in API (include/fluide_engine.hpp): meshes loaded with OBJManager::Load, InitializeFromTriangleMesh,
// SetViscosity(0), AddCollider(TriangleMeshCollider(size, origin, spacing, colliderMesh)), SetMaxClf, frames.
// argv[1] = fluid OBJ, argv[2] = collider OBJ (with normals), argv[3] / argv[4] = where to write the particles after
// the initialisation / after the frames (per particle: position then velocity, 6 floats).  Prints
// "particles=<n> substeps=<s> inside=<0|1>" (inside: IsInside of a point in the collider's box).
#include <cstdio>
#include <memory>
#include <vector>

#include "fluide_engine.hpp"

static int dump(const char* path, HybridSimulator& sim)
{
    std::vector<float> pos, vel;
    sim.GetParticles(pos, vel);
    FILE* f = std::fopen(path, "wb");
    if (!f) return 1;
    for (size_t i = 0; i < pos.size() / 3; ++i) {
        std::fwrite(&pos[3 * i], sizeof(float), 3, f);
        std::fwrite(&vel[3 * i], sizeof(float), 3, f);
    }
    std::fclose(f);
    return 0;
}

int main(int argc, char** argv)
{
    if (argc < 5) return 2;
    const Vector3<size_t> size(16, 16, 16);
    const Vector3<double> domainOrigin(0, 0, 0), domainSize(1, 1, 1);
    BoundingBox3D domain(domainOrigin, domainSize);
    TriangleMesh fluidMesh, colliderMesh;
    OBJManager objLoader;
    objLoader.Load(argv[1], fluidMesh);
    objLoader.Load(argv[2], colliderMesh);
    auto collider = std::make_shared<TriangleMeshCollider>(
        size, domainOrigin, Vector3<double>(1.0 / size.x, 1.0 / size.x, 1.0 / size.x), colliderMesh);

    PICSimulator simulator(size, domain);
    simulator.AddExternalForce(std::make_shared<DirectionalField>(Vector3<double>(0, -9.81, 0)));
    simulator.InitializeFromTriangleMesh(fluidMesh);
    simulator.SetViscosity(0);
    simulator.AddCollider(collider);
    simulator.SetMaxClf(2);
    if (dump(argv[3], simulator)) return 3;
    simulator.SetCurrentFrame(Frame(1.0 / 60.0));
    unsigned substeps = 0;
    for (int i = 0; i < 2; ++i) {
        simulator.AdvanceSingleFrame();
        substeps += simulator.GetNumberOfSubTimeSteps();
    }
    if (dump(argv[4], simulator)) return 4;
    std::printf("particles=%zu substeps=%u inside=%d\n", simulator.GetNumberOfParticles(), substeps,
                collider->IsInside(Vector3<double>(0.6, 0.2, 0.5)) ? 1 : 0);
    return 0;
}
