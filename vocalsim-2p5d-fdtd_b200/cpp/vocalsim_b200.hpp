// vocalsim_b200.hpp -- C++ host classes with the reference's names and roles,
// over the C ABI of libvocalsim_b200 (include/vocalsim_b200.h).
//
// A program written against the reference (main.cu:203-232):
//
//     SimulationParams simulationParams(FDTD_SOLVER_TYPE, SIMULATION_TYPE, TUBE_GEOMETRY,
//                                       VOWEL_TYPE, CROSS_SECTIONAL_SHAPE, MOUTH_RADIATION,
//                                       SRATE_MUL, AUDIO_DUR, SOURCE_TYPE, PML_FLAG);
//     FDTDSolver fdtdSolver(simulationParams);
//     fdtdSolver.setupWaveSolver();
//     FDTDEngineCPU engine(fdtdSolver, false);
//     engine.startSolverEngine();            // -> engine.record_pressure
//
// keeps its shape with these classes; the area function is passed explicitly
// (TubeGeometry) instead of being read from ../../data/tube-geometry, and the
// engine runs on the current CUDA device.  Errors throw vsb::Error carrying the
// vs_status (the reference prints and continues, SimulationParams.h:17-24).
#pragma once

#include <chrono>
#include <cmath>
#include <cstdint>
#include <fstream>
#include <iostream>
#include <memory>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "../../include/vocalsim_b200.h"

namespace vsb {

class Error : public std::runtime_error {
public:
    Error(int status, const std::string& where)
        : std::runtime_error(where + ": " + vs_last_error()), status_(status) {}
    Error(int status, const char* what) : std::runtime_error(what), status_(status) {}
    int status() const { return status_; }

private:
    int status_;
};

inline void check(int status, const char* where) {
    if (status != VS_OK) throw Error(status, where);
}

// SimulationParams(10 args), SimulationParams.cu:36-57.  tube_geometry and
// vowel_type select a data file in the reference; here the area function is
// given to TubeGeometry, so they are kept only for the caller's bookkeeping.
class SimulationParams {
public:
    SimulationParams(int fdtd_solver_type, int simulation_type, int tube_geometry, int vowel_type,
                     int cross_sectional_shape, int mouth_radiation_cond, int srate_mul, float audio_dur,
                     int source_type, int pml_flag)
        : tube_geometry_(tube_geometry), vowel_type_(vowel_type) {
        check(vs_params_init(&p_), "vs_params_init");
        p_.fdtd_solver_type = fdtd_solver_type;
        p_.simulation_type = simulation_type;
        p_.cross_sectional_shape = cross_sectional_shape;
        p_.mouth_radiation_cond = mouth_radiation_cond;
        p_.srate_mul = srate_mul;
        p_.audio_dur = audio_dur;
        p_.source_type = source_type;
        p_.pml_flag = pml_flag;
    }

    int getFDTDSolverType() const { return p_.fdtd_solver_type; }
    int getSimulationType() const { return p_.simulation_type; }
    int getTubeGeometry() const { return tube_geometry_; }
    int getVowelType() const { return vowel_type_; }
    int getCrossSectionalShape() const { return p_.cross_sectional_shape; }
    int getMouthRadiationCond() const { return p_.mouth_radiation_cond; }
    int getSrateMul() const { return p_.srate_mul; }
    float getAudioDur() const { return p_.audio_dur; }
    int getSourceType() const { return p_.source_type; }
    int getPMLFlag() const { return p_.pml_flag; }

    // Parameters the reference hard-codes, exposed (defaults = reference values).
    vs_params& raw() { return p_; }
    const vs_params& raw() const { return p_; }

private:
    vs_params p_{};
    int tube_geometry_, vowel_type_;
};

// The area function TubeGeometry reads from a data file (TubeGeometry.cu:53-107).
class TubeGeometry {
public:
    TubeGeometry(std::vector<float> segment_length_cm, std::vector<float> cross_sectional_area_cm2)
        : len_(std::move(segment_length_cm)), area_(std::move(cross_sectional_area_cm2)) {
        if (len_.size() != area_.size()) throw std::invalid_argument("one area per segment length");
    }

    // The file the reference's constructor picks (TubeGeometry.cu:57-74):
    // with tube_geometry != 0, vowel 1 / 2 / 3 -> vocaltract_a / _i / _u.txt and
    // any other vowel -> cylindrical-tube.txt (the reference's `else` binds to
    // the inner if).  tube_geometry == 0 selects no file there; it is rejected.
    static std::string data_file(int tube_geometry, int vowel_type) {
        if (!tube_geometry)
            throw Error(VS_ERR_INVALID_ARG, "tube_geometry 0 selects no area-function file (TubeGeometry.cu:60-74)");
        switch (vowel_type) {
            case 1: return "vocaltract_a.txt";
            case 2: return "vocaltract_i.txt";
            case 3: return "vocaltract_u.txt";
            default: return "cylindrical-tube.txt";
        }
    }

    // Whitespace-separated "segment_length_cm area_cm2" pairs, read with
    // operator>> into floats as the reference does (TubeGeometry.cu:83-88).
    static TubeGeometry from_file(const std::string& path) {
        std::ifstream f(path);
        if (!f.is_open()) throw Error(VS_ERR_INVALID_ARG, "cannot open area-function file " + path);
        std::vector<float> len, area;
        float l, a;
        while (f >> l >> a) {
            len.push_back(l);
            area.push_back(a);
        }
        if (len.empty()) throw Error(VS_ERR_GEOMETRY, "no sections in " + path);
        return TubeGeometry(std::move(len), std::move(area));
    }

    const std::vector<float>& segment_length_cm() const { return len_; }
    const std::vector<float>& cross_sectional_area_cm2() const { return area_; }

    vs_geometry view() const {
        vs_geometry g{};
        g.n_sections = (int32_t)len_.size();
        g.section_length_cm = len_.data();
        g.section_area_cm2 = area_.data();
        return g;
    }

private:
    std::vector<float> len_, area_;
};

// FDTDSolver(SimulationParams) + setupWaveSolver() (FDTDSolver.cu:71-83,
// 289-476): builds the maps on the host (bit-identical to the reference's)
// and exposes the fields the engines read.  Without an explicit geometry a
// tube simulation reads the area function the way the reference does, from
// data_dir + TubeGeometry::data_file(tube_geometry, vowel_type); data_dir
// defaults to the reference's relative path ../../data/tube-geometry/.
class FDTDSolver {
public:
    FDTDSolver(const SimulationParams& params, const TubeGeometry* geometry = nullptr)
        : params_(params), geometry_(geometry) {}

    std::string data_dir = "../../data/tube-geometry/";

    void setupWaveSolver() {
        if (!geometry_ && params_.getSimulationType() == 1) {
            owned_ = std::make_shared<TubeGeometry>(TubeGeometry::from_file(
                data_dir + TubeGeometry::data_file(params_.getTubeGeometry(), params_.getVowelType())));
            geometry_ = owned_.get();
        }
        vs_geometry g{};
        const vs_geometry* gp = nullptr;
        if (geometry_) {
            g = geometry_->view();
            gp = &g;
        }
        vs_dims d{};
        check(vs_build_maps(&params_.raw(), gp, &d, nullptr, nullptr, nullptr, nullptr, nullptr), "vs_build_maps");
        const size_t n = (size_t)d.frame_h * d.frame_w;
        cell_type.resize(n);
        depthP.resize(n);
        depthX.resize(n);
        depthY.resize(n);
        z_inv.resize(n);
        check(vs_build_maps(&params_.raw(), gp, &d, cell_type.data(), depthP.data(), depthX.data(), depthY.data(),
                            z_inv.data()),
              "vs_build_maps");
        dims = d;
        frameH = d.frame_h;
        frameW = d.frame_w;
        listenerX = d.listener_x;
        listenerY = d.listener_y;
        excitationX = d.excitation_x;
        excitationY = d.excitation_y;
        num_steps = (int)d.num_steps;
        dt = d.dt;
        ds = d.ds;
    }

    const SimulationParams& params() const { return params_; }
    const TubeGeometry* geometry() const { return geometry_; }

    // public state of the reference class (FDTDSolver.h:39-100)
    int frameH = 0, frameW = 0, listenerX = 0, listenerY = 0, excitationX = 0, excitationY = 0;
    int num_steps = 0;
    float dt = 0.0f, ds = 0.0f;
    std::vector<int32_t> cell_type;      // GridCellComponents::cell_type per frame cell
    std::vector<float> depthP, depthX, depthY, z_inv;
    vs_dims dims{};

private:
    SimulationParams params_;
    const TubeGeometry* geometry_;
    std::shared_ptr<TubeGeometry> owned_;     // the area function read in setupWaveSolver
};

// TubeDepth (TubeDepth.cu:82-265): the depth maps of a set-up solver.  The
// reference computes them with its depth kernels inside setupWaveSolver; here
// vs_build_maps has already produced the same maps, so setTubeDepth() copies
// them out of the solver.
class TubeDepth {
public:
    explicit TubeDepth(FDTDSolver& solver) : solver_(solver) {}

    void setTubeDepth() {
        if (solver_.depthP.empty()) solver_.setupWaveSolver();
        depthP = solver_.depthP;
        depthX = solver_.depthX;
        depthY = solver_.depthY;
    }

    float min_depth = 0.001f;           // TubeDepth.cu:90
    float open_space_depth = 0.50f;     // TubeDepth.cu:91
    std::vector<float> depthP, depthX, depthY;

private:
    FDTDSolver& solver_;
};

// GlottalExcitations (GlottalExcitations.cu:9-52): the per-step source table
// (0 sine, 1 Gaussian, 2 two-mass: zeros, the model runs in the engine).
class GlottalExcitations {
public:
    void setExcitationVelocity(int source_type, int num_steps, double dt) {
        vs_params p{};
        check(vs_params_init(&p), "vs_params_init");
        p.source_type = source_type;
        p.srate_mul = (int)std::lround(1.0 / (dt * 44100.0));
        excitation_.assign((size_t)std::max(num_steps, 0), 0.0f);
        if (num_steps > 0) check(vs_source_table(&p, num_steps, excitation_.data()), "vs_source_table");
    }
    std::vector<float> getExcitationVelocity() const { return excitation_; }

private:
    std::vector<float> excitation_;
};

// Drop-in for FDTDEngineCPU / FDTDEngineEigen (FDTDEngineCPU.cpp:4-304,
// FDTDEngineEigen.cpp:4-189): startSolverEngine() runs num_steps steps on the
// GPU and fills record_pressure.  The arithmetic follows FDTDEngineCPU unless
// the parameters select VS_ENGINE_EIGEN.
class FDTDEngineB200 {
public:
    explicit FDTDEngineB200(FDTDSolver& solver, bool validationFlag = false) : solver_(solver) {
        (void)validationFlag;   // the reference writes CSV dumps; maps are available on FDTDSolver
        vs_geometry g{};
        const vs_geometry* gp = nullptr;
        if (solver.geometry()) {
            g = solver.geometry()->view();
            gp = &g;
        }
        check(vs_create(&solver.params().raw(), gp, &h_), "vs_create");
    }
    FDTDEngineB200(const FDTDEngineB200&) = delete;
    FDTDEngineB200& operator=(const FDTDEngineB200&) = delete;
    ~FDTDEngineB200() { vs_destroy(h_); }

    void startSolverEngine() {
        record_pressure.assign((size_t)solver_.num_steps, 0.0f);
        check(vs_reset(h_), "vs_reset");
        check(vs_run(h_, solver_.num_steps, record_pressure.data(), 0), "vs_run");
    }

    // Advance from the current state (the reference always starts at rest).
    void advance(int64_t steps, std::vector<float>& trace) {
        trace.assign((size_t)steps, 0.0f);
        check(vs_run(h_, steps, trace.data(), 0), "vs_run");
    }

    std::vector<float> record_pressure;   // FDTDEngineCPU.h:69

protected:
    struct Arithmetic {
        int engine;     // VS_ENGINE_CPU or VS_ENGINE_EIGEN
    };
    FDTDEngineB200(FDTDSolver& solver, Arithmetic a) : solver_(solver) {
        vs_params p = solver.params().raw();
        p.engine = a.engine;
        vs_geometry g{};
        const vs_geometry* gp = nullptr;
        if (solver.geometry()) {
            g = solver.geometry()->view();
            gp = &g;
        }
        check(vs_create(&p, gp, &h_), "vs_create");
    }

    // startSolverEngine of the reference engines: run, print the loop time,
    // write record_pressure one value per line to ../../results/
    // (FDTDEngineCPU.cpp:290-303, 435-450).
    void run_and_save(const std::string& results_path) {
        const auto t0 = std::chrono::steady_clock::now();
        startSolverEngine();
        const std::chrono::duration<double> dt = std::chrono::steady_clock::now() - t0;
        std::cout << "Elapsed time [in seconds]: " << dt.count() << " s" << std::endl;
        std::ofstream out(results_path);
        if (!out) throw Error(VS_ERR_INVALID_ARG, "cannot write " + results_path);
        for (float v : record_pressure) out << v << "\n";
    }

private:
    FDTDSolver& solver_;
    vs_solver* h_ = nullptr;
};

// The reference's engine classes by name (FDTDEngineCPU.h, FDTDEngineEigen.h),
// so its driver (main.cu:126-146) builds unchanged against the headers in
// cpp/include: both run on the GPU, in the CPU engine's or the Eigen engine's
// rounding, and save record_pressure where the reference does.
class FDTDEngineCPU : public FDTDEngineB200 {
public:
    explicit FDTDEngineCPU(FDTDSolver& solver, bool validationFlag = false)
        : FDTDEngineB200(solver, Arithmetic{VS_ENGINE_CPU}) {
        (void)validationFlag;
    }
    void startSolverEngine() { run_and_save(results_path); }
    std::string results_path = "../../results/recorded-pressure.txt";
};

class FDTDEngineEigen : public FDTDEngineB200 {
public:
    FDTDEngineEigen(FDTDEngineCPU& cpu, FDTDSolver& solver, bool validationFlag = false)
        : FDTDEngineB200(solver, Arithmetic{VS_ENGINE_EIGEN}) {
        (void)cpu;
        (void)validationFlag;
    }
    void startSolverEngine() { run_and_save(results_path); }
    std::string results_path = "../../results/recorded-pressure.txt";
};

}  // namespace vsb
