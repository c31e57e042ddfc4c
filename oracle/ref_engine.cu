/*
 * ref_engine.cu -- runs the reference's own grid setup and CPU engine.
 * TEST INFRASTRUCTURE ONLY: built by oracle/Makefile.ref, straight from the
 * reference tree, into oracle/_ref/ref_engine (git-ignored); used by
 * tests/golden/make_reference_engine.py, the reference-engine tests and the
 * reference arm of bench.py.  Nothing here restates reference logic: it
 * constructs SimulationParams -> FDTDSolver::setupWaveSolver ->
 * FDTDEngineCPU::startSolverEngine (main.cu:114-136) and writes out the
 * public members those classes expose.
 *
 *   ref_engine key=value ...   (run with the working directory two levels
 *                                below a scratch root holding
 *                                data/tube-geometry/<file> and results/, the
 *                                relative paths TubeGeometry.cu:77 and
 *                                FDTDEngineCPU.cpp:438 use)
 *
 * keys: solver (0 2D / 1 2.5D), sim (0 open space / 1 tube), tube (0/1),
 * vowel (1..3), shape (1 circular / 2 elliptical), mouth (0/1), srate_mul,
 * audio_dur (s), source (0 sine / 1 Gaussian / 2 two-mass), pml (0/1),
 * steps (time steps to run, <= the reference's own count for audio_dur),
 * out (directory for the dump), maps (1 = write the maps, default 1).
 *
 * Output in `out`: meta.txt (key value lines) and raw little-endian arrays:
 * cell_type.i32, depth_p/x/y.f32, z_inv.f32 (H x W); the 17 coefficient
 * arrays of calculateSolverCoefficients, each (H-2) x (W-2) .f32;
 * excitation.f32 (the reference's own step count); trace.f32
 * (record_pressure, `steps`); p/vx/vy.f32 (the fields after the run, H x W).
 */
#include "FDTDSolver.h"
#include "FDTDEngineCPU.h"

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <vector>

extern "C" unsigned long long ref_pad_calls;
extern "C" size_t ref_pad_last_request;

namespace {

std::map<std::string, std::string> parse(int argc, char** argv) {
    std::map<std::string, std::string> kv;
    for (int i = 1; i < argc; ++i) {
        const char* eq = std::strchr(argv[i], '=');
        if (!eq) {
            std::fprintf(stderr, "ref_engine: argument '%s' is not key=value\n", argv[i]);
            std::exit(2);
        }
        kv[std::string(argv[i], eq - argv[i])] = std::string(eq + 1);
    }
    return kv;
}

template <class T>
void put(const std::string& dir, const char* name, const T* data, size_t n) {
    const std::string path = dir + "/" + name;
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f || std::fwrite(data, sizeof(T), n, f) != n) {
        std::fprintf(stderr, "ref_engine: cannot write %s\n", path.c_str());
        std::exit(2);
    }
    std::fclose(f);
}

void put_mat(const std::string& dir, const char* name, const std::vector<std::vector<float>>& m) {
    std::vector<float> flat;
    for (const auto& row : m) flat.insert(flat.end(), row.begin(), row.end());
    put(dir, name, flat.data(), flat.size());
}

}  // namespace

int main(int argc, char** argv) {
    auto kv = parse(argc, argv);
    auto geti = [&](const char* k, int d) { return kv.count(k) ? std::atoi(kv[k].c_str()) : d; };
    const int solver = geti("solver", 1), sim = geti("sim", 1), tube = geti("tube", 1), vowel = geti("vowel", 1);
    const int shape = geti("shape", 1), mouth = geti("mouth", 0), srate_mul = geti("srate_mul", 15);
    const int source = geti("source", 1), pml = geti("pml", 1), steps = geti("steps", 100);
    const int with_maps = geti("maps", 1);
    const float audio_dur = kv.count("audio_dur") ? std::strtof(kv["audio_dur"].c_str(), nullptr) : 0.005f;
    if (!kv.count("out")) {
        std::fprintf(stderr, "ref_engine: out=<dir> is required\n");
        return 2;
    }
    const std::string out = kv["out"];
    if (shape == 3) {
        std::fprintf(stderr, "ref_engine: cross_sectional_shape 3 needs Boost.Geometry and is not built\n");
        return 3;
    }

    // Every device allocation must come through the padding cudaMalloc
    // (ref_alloc_pad.cpp) before the reference's setup kernels run.
    {
        const unsigned long long before = ref_pad_calls;
        thrust::device_vector<FDTDSolver::GridCellComponents> probe(3);
        if (ref_pad_calls != before + 1 || ref_pad_last_request != 3 * sizeof(FDTDSolver::GridCellComponents)) {
            std::fprintf(stderr, "ref_engine: device_vector did not allocate through the padded cudaMalloc\n");
            return 4;
        }
    }

    SimulationParams params(solver, sim, tube, vowel, shape, mouth, srate_mul, audio_dur, source, pml);
    FDTDSolver fdtd(params);
    fdtd.setupWaveSolver();
    cudaError_t e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) {
        std::fprintf(stderr, "ref_engine: CUDA error after setup: %s\n", cudaGetErrorString(e));
        return 5;
    }
    const int ref_steps = fdtd.num_steps;
    if (steps < 1 || steps > ref_steps) {
        std::fprintf(stderr, "ref_engine: steps=%d outside 1..%d (the reference's count for audio_dur)\n", steps,
                     ref_steps);
        return 2;
    }
    thrust::host_vector<float> excitation = fdtd.excitation_velocity;

    FDTDEngineCPU engine(fdtd, false);
    fdtd.num_steps = steps;                        // the loop runs _fdtdSolver.num_steps steps
    const auto t0 = std::chrono::steady_clock::now();
    engine.startSolverEngine();
    const auto t1 = std::chrono::steady_clock::now();
    const double loop_s = std::chrono::duration<double>(t1 - t0).count();

    const int H = engine.frameH, W = engine.frameW;
    FILE* m = std::fopen((out + "/meta.txt").c_str(), "w");
    if (!m) {
        std::fprintf(stderr, "ref_engine: cannot write %s/meta.txt\n", out.c_str());
        return 2;
    }
    std::fprintf(m, "frame_h %d\nframe_w %d\nlistener_x %d\nlistener_y %d\nexcitation_x %d\nexcitation_y %d\n", H, W,
                 fdtd.listenerX, fdtd.listenerY, fdtd.excitationX, fdtd.excitationY);
    std::fprintf(m, "ref_steps %d\nsteps %d\nloop_s %.9f\n", ref_steps, steps, loop_s);
    // the loop's start and end on the monotonic clock, comparable across processes
    std::fprintf(m, "loop_t0 %.9f\nloop_t1 %.9f\n", std::chrono::duration<double>(t0.time_since_epoch()).count(),
                 std::chrono::duration<double>(t1.time_since_epoch()).count());
    std::fprintf(m, "dt %.9e\nds %.9e\nkappa %.9e\n", fdtd.dt, fdtd.ds, fdtd.kappa);
    std::fclose(m);

    put(out, "trace.f32", engine.record_pressure.data(), engine.record_pressure.size());
    put(out, "excitation.f32", excitation.data(), excitation.size());
    std::vector<float> p((size_t)H * W), vx((size_t)H * W), vy((size_t)H * W);
    for (int r = 0; r < H; ++r)
        for (int c = 0; c < W; ++c) {
            // after the last step PV_N = PV_Nplus1 holds the final fields
            p[(size_t)r * W + c] = engine.PV_N[r][c].Pr;
            vx[(size_t)r * W + c] = engine.PV_N[r][c].Vx;
            vy[(size_t)r * W + c] = engine.PV_N[r][c].Vy;
        }
    put(out, "p.f32", p.data(), p.size());
    put(out, "vx.f32", vx.data(), vx.size());
    put(out, "vy.f32", vy.data(), vy.size());
    if (with_maps) {
        std::vector<int32_t> ct((size_t)H * W);
        for (int r = 0; r < H; ++r)
            for (int c = 0; c < W; ++c) ct[(size_t)r * W + c] = engine.PV_N[r][c].cell_type;
        put(out, "cell_type.i32", ct.data(), ct.size());
        put_mat(out, "depth_p.f32", engine.depthP);
        put_mat(out, "depth_x.f32", engine.depthX);
        put_mat(out, "depth_y.f32", engine.depthY);
        put_mat(out, "z_inv.f32", engine.z_inv_mat);
        put_mat(out, "N_out.f32", engine.N_out_mat);
        put_mat(out, "N_in.f32", engine.N_in_mat);
        put_mat(out, "minVxBeta.f32", engine.minVxBeta_mat);
        put_mat(out, "minVyBeta.f32", engine.minVyBeta_mat);
        put_mat(out, "maxVxSigmaPrimedt.f32", engine.maxVxSigmaPrimedt_mat);
        put_mat(out, "maxVySigmaPrimedt.f32", engine.maxVySigmaPrimedt_mat);
        put_mat(out, "betaVxSqr_dt_inv_rho_inv_ds.f32", engine.betaVxSqr_dt_inv_rho_inv_ds_mat);
        put_mat(out, "betaVySqr_dt_inv_rho_inv_ds.f32", engine.betaVySqr_dt_inv_rho_inv_ds_mat);
        put_mat(out, "pressureSigmaPrimedt.f32", engine.pressureSigmaPrimedt_mat);
        put_mat(out, "areWeNotExcitationVx.f32", engine.areWeNotExcitationVx_mat);
        put_mat(out, "areWeNotExcitationVy.f32", engine.areWeNotExcitationVy_mat);
        put_mat(out, "excitationWeightVx.f32", engine.excitationWeightVx_mat);
        put_mat(out, "excitationWeightVy.f32", engine.excitationWeightVy_mat);
        put_mat(out, "xor_val1.f32", engine.xor_val1_mat);
        put_mat(out, "xor_val2.f32", engine.xor_val2_mat);
        put_mat(out, "xor_val3.f32", engine.xor_val3_mat);
        put_mat(out, "xor_val4.f32", engine.xor_val4_mat);
    }
    return 0;
}
