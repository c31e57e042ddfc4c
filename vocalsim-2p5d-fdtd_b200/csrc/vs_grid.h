// vs_grid.h -- host-side grid description shared by the map builder, the
// C ABI and the CUDA launchers of libvocalsim_b200.
#pragma once

#include "../../include/vocalsim_b200.h"

#include <cstdint>
#include <string>
#include <vector>

namespace vsb {

// Cell code byte stored per cell on the device: bits 0-3 = reference cell type
// (0..12), bit 4 = "z_inv applies here" (boundary_segment_type != 0).
constexpr uint8_t CODE_TYPE_MASK = 0x0f;
constexpr uint8_t CODE_ZINV_BIT = 0x10;

// Error carried out of the host builders into a vs_status.
struct VsFailure {
    int status;
    std::string what;
};

// Constants of the two-mass vocal fold model (TwoMassModel.cpp:4-87): with
// F = float the values the reference stores in its members, with F = double
// the same expressions evaluated in double (the double-precision model).
template <class F>
struct TmmConstsT {
    F mu, rho, m1, m2, d1, d2, k1, k2, kc, etak1, etak2, h1, h2, etah1, etah2;
    F Ag01, Ag02, lg, r1o, r2o, r1c, r2c, A1, ps, srate;
};
using TmmConsts = TmmConstsT<float>;
using TmmConsts64 = TmmConstsT<double>;

// Per-tube constants of the double two-mass model (tmm_f64), derived once
// from its TmmConsts64 by tmm_derived(): reciprocals of the sample rate and of
// its square, the opening thresholds, the products the step multiplies by,
// and the matrix of the displacement update with its inverse determinant for
// each contact state of the two masses ([0] open, [1] closed).  With them a
// step divides only by the two glottal openings, before and after the update,
// and by the flow denominator.
struct TmmDerived64 {
    double isr, is2, two_lg, g1, g2, c12, cR1, cR2, cL1, cL2, hr, hr137, d1lg, d2lg, iA1, k1e, k2e;
    double a11[2], a22[2], a12, b1c[2], b2c[2], idet[2][2];
};

// Two-mass model state carried from step to step (the members the reference
// reads before writing in runTwoMassModel).
template <class F>
struct TmmStateT {
    F x1_old, x1_curr, x2_old, x2_curr, ug_old, ug_curr;
};
using TmmState = TmmStateT<float>;
using TmmState64 = TmmStateT<double>;

// Everything the device needs for one tube, in host memory.
struct TubeGrid {
    vs_dims dims{};
    int H = 0, W = 0;
    int pitch = 0;                    // row pitch of every device plane, in elements
    bool dirichlet = false;
    bool eigen = false;
    bool tmm = false;
    bool wall_ode = false;            // 2.5D with a nonzero wall coupling
    int srate_mul = 1;
    float K1 = 0, K2 = 0;             // rho c^2 dt / ds, rho c^2 dt (FDTDSolver.cu:311-312)
    float bcoef = 0;                  // dt / (rho ds): betaV*Sqr_dt_inv_rho_inv_ds for beta = 1
    float zinv_val = 0;
    float dt = 0, Mw = 0, Bw = 0, Kw = 0, cpl = 0;
    float beta[16] = {0}, sigma[16] = {0};
    float dir[4] = {0};
    std::vector<int32_t> cell_type;   // H*W, reference values
    std::vector<uint8_t> code;        // H*pitch, padding = dead
    std::vector<float> zinv;          // H*W
    std::vector<float> dP, dX, dY;    // H*W
    std::vector<float> source;        // per-step excitation (empty for the two-mass source)
    TmmConsts tmmc{};
    bool tmm64 = false;               // two-mass model in double (vs_params::tmm_f64)
    TmmConsts64 tmmd{};               // double constants: the double model's, else tmmc widened
    TmmDerived64 tmmx{};              // the double model's derived constants
    vs_params src_params{};           // parameters the source table is rebuilt from
    // tube rasterisation (empty for the open-space domain)
    std::vector<int32_t> upper, lower, colseg;   // per tube column: wall rows, 0-based segment
    std::vector<float> major_m, minor_m;         // per section: width used for walls, minor axis
    // per tube column, after the wall-gap fill: the upper wall occupies rows
    // upper_top .. upper, the lower wall lower .. lower_bot
    std::vector<int32_t> upper_top, lower_bot;
    int pml_layers = 0;                           // graded PML layers painted inside the dead ring
    // the H x W vectors above (cell_type, code, zinv, dP, dX, dY) were not
    // built on the host: the device map builder paints them from the column
    // data (build_tube_columns)
    bool device_maps = false;
};

// Fill p with the reference's defaults.
void default_params(vs_params* p);

// Build a tube (or the open-space domain) exactly as FDTDSolver::setupWaveSolver.
// `steps_for_source` > 0 sizes the source table; 0 uses dims.num_steps.
void build_tube(const vs_params* p, const vs_geometry* g, TubeGrid& out, int64_t steps_for_source);

// Whether the device map builder covers these parameters: a tube simulation
// with circular or elliptical sections (not the open-space domain, not
// single-plane-symmetric sections).
bool device_buildable(const vs_params* p);

// build_tube without any H x W map: the frame, the dims, the constants, the
// source and the per-column wall data (upper, lower, upper_top, lower_bot,
// colseg) that the device map builder paints the maps from
// (out.device_maps = true).  Checks that need the maps (a negative depth
// radicand) are made by the device builder.
void build_tube_columns(const vs_params* p, const vs_geometry* g, TubeGrid& out, int64_t steps_for_source);

// Only the scalar constants and tables of a tube (K1, K2, bcoef, dt, the wall
// parameters, sigma/beta/direction tables, two-mass constants and the flags
// derived from p), without building any map: what a caller that brings its
// own maps needs.  Touches none of the vectors of `out`.
void solver_constants(const vs_params* p, TubeGrid& out);

// The per-step excitation table (GlottalExcitations::setExcitationVelocity).
void build_source(const vs_params* p, float dt, int64_t n, std::vector<float>& out);

// Two-mass model constants (setTwoMassModelParams) for a given subglottal
// pressure, in float (the reference's) or double.
template <class F>
TmmConstsT<F> tmm_consts(float ps, int srate_mul);

// The double model's derived constants (TmmDerived64) of constants k.
TmmDerived64 tmm_derived(const TmmConsts64& k);

}  // namespace vsb
