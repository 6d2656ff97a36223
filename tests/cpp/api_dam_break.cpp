// api_dam_break.cpp -- drives the C++ drop-in API (include/fluide_engine.hpp) the way a caller of the
// reference's simulators would: construct, add gravity, seed, set the frame, AdvanceSingleFrame.
// Then writes the fluid surface the way SimulationRunner does (GetSurface + OBJManager::Save, simulation_runner.cpp:
// 34-36) to the path given as argv[1] (if any).
// Prints "frames=<n> particles=<N> substeps=<s> mean_y=<y> surface_v=<V> surface_t=<T>" for the test to check.
#include <cstdio>
#include <memory>
#include <vector>

#include "fluide_engine.hpp"

int main(int argc, char** argv)
{
    FLIPSimulator sim(Vector3<size_t>(16, 16, 16), BoundingBox3D(Vector3<double>(0.0), Vector3<double>(1.0)));
    sim.AddExternalForce(std::make_shared<DirectionalField>(Vector3<double>(0.0, -9.81, 0.0)));
    sim.SetMaxClf(1.0);
    const size_t n = sim.InitializeFromRegions({fe_region_desc{0, {0.0, 0.0, 0.0}, {0.4, 0.6, 1.0}, {0.0, 0.0, 0.0}}});
    sim.SetCurrentFrame(Frame(1.0 / 60.0));
    unsigned substeps = 0;
    for (int f = 0; f < 3; ++f) {
        sim.AdvanceSingleFrame();
        substeps += sim.GetNumberOfSubTimeSteps();
    }
    std::vector<float> pos, vel;
    sim.GetParticles(pos, vel);
    double my = 0.0;
    for (size_t i = 0; i < pos.size() / 3; ++i) my += pos[3 * i + 1];
    TriangleMesh surface;
    sim.GetSurface(surface);
    if (argc > 1) {
        surface.SetObjectName("fluid");
        OBJManager().Save(argv[1], surface);
    }
    std::printf("frames=%lu particles=%zu substeps=%u mean_y=%.6f surface_v=%zu surface_t=%zu\n",
                sim.GetCurrentFrame().GetIndex(), n, substeps, my / (pos.size() / 3), surface.GetVerticies().size(),
                surface.GetTriangles().size());
    return 0;
}
