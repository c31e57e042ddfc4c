// example_engine.cpp -- the reference's main.cu flow on the C++ mirror classes.
//
//   g++ -std=c++17 example_engine.cpp -I. -L../lib -lvocalsim_b200 -Wl,-rpath,../lib
//   ./a.out [--maps-only]
//
// Prints the frame size, listener cell and (with a GPU) the first listener
// pressures of a uniform 17.5 cm x 3 cm tube with the Gaussian source.
#include <cmath>
#include <cstdio>
#include <cstring>

#include "vocalsim_b200.hpp"

int main(int argc, char** argv) {
    const bool maps_only = argc > 1 && std::strcmp(argv[1], "--maps-only") == 0;
    // FDTD_SOLVER_TYPE 2.5D, tube, circular, open mouth, srate x15, 20 ms, Gaussian, PML on
    vsb::SimulationParams params(1, 1, 1, 1, 1, 0, 15, 0.02f, 1, 1);
    params.raw().uniform_depth_m = 0.02f;
    params.raw().mu3d = 0.005f;
    const float area = (float)(M_PI * 1.5 * 1.5);
    vsb::TubeGeometry tube({17.5f}, {area});
    vsb::FDTDSolver solver(params, &tube);
    solver.setupWaveSolver();
    std::printf("frame %d x %d, listener (%d, %d), %d steps\n", solver.frameH, solver.frameW, solver.listenerY,
                solver.listenerX, solver.num_steps);
    if (maps_only) return 0;
    vsb::FDTDEngineB200 engine(solver, false);
    engine.startSolverEngine();
    double e = 0.0;
    for (float v : engine.record_pressure) e += (double)v * v;
    std::printf("record_pressure: %zu samples, energy %.6e, p[100] %.6e\n", engine.record_pressure.size(), e,
                engine.record_pressure.size() > 100 ? engine.record_pressure[100] : 0.0f);
    return 0;
}
