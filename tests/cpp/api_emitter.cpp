// api_emitter.cpp -- the reference's main.cpp scene sequence through the C++ drop-in API (include/fluide_engine.hpp):
// meshes loaded with OBJManager::Load, a FLIP simulator on a 30^3 grid over a 6^3 domain, gravity,
// InitializeFromTriangleMesh(fluid mesh), a VolumeEmitter (12 particles per node, velocity (0, 6, 0)),
// SetViscosity(0.01), SetMaxClf(5), frames of 1/60 s.  A second simulator starts from the emitter alone, a third
// takes its emitter SDF from a ScalarGrid3D (InitializeFromSdf).
// argv[1] = emitter OBJ, argv[2] = fluid OBJ, argv[3] = where to write the fluid SDF after the first substep
// (doubles, x-fastest).  Prints "init=<n> none=<n> first=<n> frames=<n> final=<n> emit_only_first=<n>
// emit_only_frame=<n> sdf_emitter=<n>" for the test to check.
#include <cstdio>
#include <memory>
#include <vector>

#include "fluide_engine.hpp"

int main(int argc, char** argv)
{
    if (argc < 3) return 2;
    const Vector3<size_t> size(30, 30, 30);
    const BoundingBox3D domain(Vector3<double>(0, 0, 0), Vector3<double>(6, 6, 6));
    TriangleMesh fluidMesh, emitterObject;
    OBJManager objLoader;
    objLoader.Load(argv[1], emitterObject);
    objLoader.Load(argv[2], fluidMesh);

    FLIPSimulator sim(size, domain);
    sim.AddExternalForce(std::make_shared<DirectionalField>(Vector3<double>(0, -9.81, 0)));
    sim.InitializeFromTriangleMesh(fluidMesh);
    const size_t init = sim.GetNumberOfParticles();
    sim.AddEmitter(std::make_shared<VolumeEmitter>(emitterObject, size, domain, 12, Vector3<double>(0.0, 6.0, 0.0), 0.0));
    sim.SetViscosity(0.01);
    const ScalarGrid3D meshSdf = sim.GetFluidSdf();
    sim.SetMaxClf(5);  // rebuilds the scene: the particles and the mesh's fluid SDF are carried over
    const ScalarGrid3D kept = sim.GetFluidSdf();
    int sdfKept = kept.GetRawData() == meshSdf.GetRawData() ? 1 : 0;
    sim.AdvanceFixedSubsteps(1.0 / 240.0, 1);  // the first substep emits nothing (collider SDF still 0)
    const size_t none = sim.GetNumberOfParticles();
    const ScalarGrid3D fluidSdf = sim.GetFluidSdf();  // built in that substep; the next one emits where it is >= 0
    sim.AdvanceFixedSubsteps(1.0 / 240.0, 1);
    const size_t first = sim.GetNumberOfParticles();

    sim.SetCurrentFrame(Frame(1.0 / 60.0));
    for (int f = 0; f < 3; ++f) sim.AdvanceSingleFrame();
    const size_t fin = sim.GetNumberOfParticles();

    APICSimulator only(size, domain);
    only.AddExternalForce(std::make_shared<DirectionalField>(Vector3<double>(0, -9.81, 0)));
    only.AddEmitter(std::make_shared<VolumeEmitter>(emitterObject, size, domain, 12, Vector3<double>(0.0, 6.0, 0.0), 0.0));
    only.SetMaxClf(5);
    only.SetCurrentFrame(Frame(1.0 / 60.0));
    only.AdvanceSingleFrame();  // starts without particles: its one substep emits nothing
    const size_t emitOnlyFirst = only.GetNumberOfParticles();
    only.AdvanceSingleFrame();  // now every node inside the emitter emits
    const size_t emitOnlyFrame = only.GetNumberOfParticles();

    // an emitter SDF negative on the nodes 10..12 x 20..21 x 10..13: 3 * 2 * 4 nodes emit 5 particles each
    ScalarGrid3D grid(size, 1.0, Vector3<double>(0.0), Vector3<double>(0.2));
    for (size_t k = 10; k < 14; ++k)
        for (size_t j = 20; j < 22; ++j)
            for (size_t i = 10; i < 13; ++i) grid.SetElement(i, j, k, -0.5);
    auto fromSdf = std::make_shared<VolumeEmitter>(emitterObject, size, domain, 5, Vector3<double>(0.0), 0.0);
    fromSdf->InitializeFromSdf(grid);
    PICSimulator third(size, domain);
    third.AddEmitter(fromSdf);
    third.AdvanceFixedSubsteps(1.0 / 240.0, 2);
    const size_t sdfEmitter = third.GetNumberOfParticles();

    // the fluid SDF the second substep's emission read, written for the test's own count
    if (argc > 3) {
        FILE* f = std::fopen(argv[3], "wb");
        if (!f) return 3;
        for (size_t k = 0; k < size.z; ++k)
            for (size_t j = 0; j < size.y; ++j)
                for (size_t i = 0; i < size.x; ++i) {
                    const double v = fluidSdf(i, j, k);
                    std::fwrite(&v, sizeof(double), 1, f);
                }
        std::fclose(f);
    }
    std::printf("sdf_kept=%d init=%zu none=%zu first=%zu frames=%lu final=%zu emit_only_first=%zu emit_only_frame=%zu sdf_emitter=%zu\n",
                sdfKept, init, none, first, sim.GetCurrentFrame().GetIndex(), fin, emitOnlyFirst, emitOnlyFrame, sdfEmitter);
    return 0;
}
