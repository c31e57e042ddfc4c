// example_engine.cpp -- the reference's main.cu flow on the C++ mirror classes.
//
//   g++ -std=c++17 example_engine.cpp -I. -L../lib -lvocalsim_b200 -Wl,-rpath,../lib
//   ./a.out [--maps-only] [--trace FILE] [--data-dir DIR VOWEL]
//
// Without --data-dir: a uniform 17.5 cm x 3 cm tube with the Gaussian source
// given as an explicit TubeGeometry.  With --data-dir the area function is
// read the reference's way, from DIR/vocaltract_{a,i,u}.txt for VOWEL 1..3
// (cylindrical-tube.txt otherwise).  Prints the frame size, listener cell and
// step count; unless --maps-only, runs the engine on the GPU and prints the
// first listener pressures, and with --trace writes record_pressure to FILE
// as raw float32.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "vocalsim_b200.hpp"

int main(int argc, char** argv) {
    bool maps_only = false;
    const char* trace_file = nullptr;
    const char* data_dir = nullptr;
    int vowel = 1;
    for (int i = 1; i < argc; ++i) {
        if (std::strcmp(argv[i], "--maps-only") == 0) maps_only = true;
        else if (std::strcmp(argv[i], "--trace") == 0 && i + 1 < argc) trace_file = argv[++i];
        else if (std::strcmp(argv[i], "--data-dir") == 0 && i + 2 < argc) {
            data_dir = argv[++i];
            vowel = std::atoi(argv[++i]);
        }
    }
    try {
        if (data_dir) {
            // main.cu's defaults: 2.5D, tube, vocal tract, circular, Dirichlet, x15, 100 ms, Gaussian, no PML
            vsb::SimulationParams params(1, 1, 1, vowel, 1, 1, 15, 0.1f, 1, 0);
            vsb::FDTDSolver solver(params);
            solver.data_dir = std::string(data_dir) + "/";
            solver.setupWaveSolver();
            std::printf("frame %d x %d, listener (%d, %d), %d steps\n", solver.frameH, solver.frameW,
                        solver.listenerY, solver.listenerX, solver.num_steps);
            return 0;
        }
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
        if (trace_file) {
            FILE* f = std::fopen(trace_file, "wb");
            if (!f || std::fwrite(engine.record_pressure.data(), sizeof(float), engine.record_pressure.size(), f) !=
                          engine.record_pressure.size()) {
                std::fprintf(stderr, "cannot write %s\n", trace_file);
                return 1;
            }
            std::fclose(f);
        }
    } catch (const vsb::Error& e) {
        std::fprintf(stderr, "error %d: %s\n", e.status(), e.what());
        return 2;
    }
    return 0;
}
