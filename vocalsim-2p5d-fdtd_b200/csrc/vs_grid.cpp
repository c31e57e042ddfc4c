// vs_grid.cpp -- host map builder of libvocalsim_b200.
//
// Produces, for one tube, the cell-type / boundary / depth maps that the
// reference's FDTDSolver::setupWaveSolver builds with its GPU setup kernels
// (FDTDSolver.cu:289-476), bit for bit, plus the packed per-cell code bytes the
// step kernel reads.  The reference computes its setup on the device in float
// arithmetic; every expression here keeps the reference's operand order and
// precision (this file is compiled with -ffp-contract=off) so the maps agree
// exactly.  The reference quirks that shape the maps are kept on purpose:
//   * section diameters rounded to an odd cell count (TubeGeometry.cu:132-148)
//   * the sequential wall-gap fill stops at column L-2 (TubeGeometry.cu:512)
//   * the excitation column's two wall cells carry no segment id, so no z_inv
//     (TubeGeometry.cu:587-593)
//   * PML rows are painted before PML columns (FDTDSolver.cu:373-464)
//   * depth smoothing pivots on the cell (mid row, tube end) (TubeDepth.cu:642-748)
#include "vs_grid.h"
#include "vs_shapes.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>

namespace vsb {
namespace {

// Units of SimulationUnits.h: float constants from double products.
const float kMeter = 1.0f;
const float kCm = (float)(1e-2 * (double)kMeter);
const float kMm = (float)(1e-3 * (double)kMeter);
const float kSecond = 1.0f;
const float kMs = (float)(1e-3 * (double)kSecond);
const float kHz = 1.0f / kSecond;
const float kKhz = (float)(1e3 * (double)kHz);
const float kKg = 1.0f;
const float kGram = (float)(1e-3 * (double)kKg);
const float kNewton = kKg * kMeter / (kSecond * kSecond);
const float kDyn = (float)(1e-5 * (double)kNewton);
const double kPi = 3.14159265358979323846;

constexpr int kPmlLayers = 6;

struct Physics {
    float c, rho, kappa, dt, ds, max_sigma_dt;
    int srate;
};

Physics physics(int srate_mul) {
    // SimulationParams(int), SimulationParams.cu:7-34
    Physics k;
    k.c = 350.0f * (kMeter / kSecond);
    k.rho = (float)((double)(1.14f * kKg) / std::pow((double)kMeter, 3));
    k.kappa = k.rho * k.c * k.c;
    k.srate = (int)(44100 * kHz) * srate_mul;
    k.dt = 1.0f / (float)k.srate;
    k.ds = k.dt * k.c * sqrtf(2.0f);
    k.max_sigma_dt = 0.5f;
    return k;
}

int64_t float_step_count(float dur, float dt) {
    // SolverParams::setTimeStep (SolverParams.cu:59-66): float accumulation
    int64_t n = 0;
    for (float t = 0.0f; t <= dur - dt; t = t + dt) ++n;
    return n;
}

// Scalar constants and tables of one tube (SimulationParams.cu:7-34,
// SolverParams.cu:5-76, FDTDSolver.cu:311-312): the single source of these
// values for the map builder and for vs_run_noalloc.
void fill_tables(const vs_params& p, const Physics& k, TubeGrid& T) {
    // SolverParams::setBeta / setSigmaPrimeDt / setSourceDirection (SolverParams.cu:5-76)
    static const float beta_fixed[13] = {0, 1, 0, 1, 1, 1, 1, 1, 1, 0, 0, 1, 0};
    for (int i = 0; i < 13; ++i) T.beta[i] = beta_fixed[i];
    const float dt = k.dt;
    const float sig_fixed[13] = {dt, 0, dt, 0, 0, 0, 0, 0, 0, 0, 1000000.0f, 0, dt};
    for (int i = 0; i < 13; ++i) T.sigma[i] = sig_fixed[i];
    for (int l = 0; l < kPmlLayers; ++l)
        T.sigma[VS_CELL_PML0 + l] = ((float)l / (float)(kPmlLayers - 1)) * k.max_sigma_dt;
    T.dir[0] = 0; T.dir[1] = 0; T.dir[2] = 1; T.dir[3] = 0;
    T.K1 = (k.kappa * k.dt) / k.ds;
    T.K2 = k.kappa * k.dt;
    T.bcoef = (1.0f * k.dt) / (k.rho * k.ds);   // (minBeta^2 dt)/(rho ds), minBeta = 1
    T.dt = k.dt;
    T.Mw = 21 * (kKg / (kMeter * kMeter));
    T.Bw = 8000 * (kKg / (kMeter * kMeter * kSecond));
    T.Kw = 845000 * (kKg / (kMeter * kMeter * kSecond * kSecond));
    T.cpl = p.wall_coupling;
    T.srate_mul = p.srate_mul;
    T.dirichlet = p.mouth_radiation_cond != 0;
    T.eigen = p.engine == VS_ENGINE_EIGEN;
    T.tmm = p.source_type == VS_SRC_TMM;
    T.wall_ode = p.fdtd_solver_type == 1 && p.wall_coupling != 0.0f;
    vs_dims& d = T.dims;
    d.dt = k.dt;
    d.ds = k.ds;
    d.num_steps = p.num_steps > 0 ? p.num_steps : float_step_count(p.audio_dur, k.dt);
}

[[noreturn]] void raise(int status, const char* what) { throw VsFailure{status, what}; }

// One tube column: wall rows and the area-function segment it samples.
struct Column {
    int up, down, seg;
};

class Builder {
public:
    // planes = false: columns only (build_tube_columns), no H x W vector
    Builder(const vs_params* p, const vs_geometry* g, TubeGrid& out, bool planes = true)
        : p_(*p), g_(g), T_(out), planes_(planes) {}

    void run() {
        validate();
        k_ = physics(p_.srate_mul);
        pml_ = kPmlLayers * p_.pml_flag;
        T_.pml_layers = pml_;
        T_.device_maps = !planes_;
        tables();
        if (p_.simulation_type == 0) open_space();
        else tube();
        if (planes_) dead_ring_and_pml();
        listener_override();
        pack();
    }

private:
    const vs_params& p_;
    const vs_geometry* g_;
    TubeGrid& T_;
    const bool planes_;
    Physics k_{};
    int pml_ = 0;
    std::vector<int> seg_;      // boundary_segment_type, H*W
    std::vector<std::vector<ShapePt>> shapes_;   // single-plane-symmetric sections (aligned contours)
    float osd_ = 0.5f;          // open_space_depth (FDTDSolver.cu:292, TubeDepth.cu:91)

    int& type(int r, int c) { return T_.cell_type[(size_t)r * T_.W + c]; }
    int& seg(int r, int c) { return seg_[(size_t)r * T_.W + c]; }
    float& dX(int r, int c) { return T_.dX[(size_t)r * T_.W + c]; }
    float& dY(int r, int c) { return T_.dY[(size_t)r * T_.W + c]; }

    void validate() {
        if (p_.srate_mul < 1 || p_.srate_mul > 64) raise(VS_ERR_INVALID_ARG, "srate_mul must be in 1..64");
        if (p_.fdtd_solver_type != 0 && p_.fdtd_solver_type != 1) raise(VS_ERR_INVALID_ARG, "fdtd_solver_type must be 0 or 1");
        if (p_.pml_flag != 0 && p_.pml_flag != 1) raise(VS_ERR_INVALID_ARG, "pml_flag must be 0 or 1");
        if (p_.simulation_type != 0 && p_.simulation_type != 1) raise(VS_ERR_INVALID_ARG, "simulation_type must be 0 or 1");
        if (p_.engine != VS_ENGINE_CPU && p_.engine != VS_ENGINE_EIGEN) raise(VS_ERR_INVALID_ARG, "engine must be VS_ENGINE_CPU or VS_ENGINE_EIGEN");
        if (p_.source_type < 0 || p_.source_type > 3) raise(VS_ERR_INVALID_ARG, "source_type must be 0..3");
        if (p_.tmm_f64 != 0 && p_.tmm_f64 != 1) raise(VS_ERR_INVALID_ARG, "tmm_f64 must be 0 or 1");
        if (p_.fast_math != 0 && p_.fast_math != 1) raise(VS_ERR_INVALID_ARG, "fast_math must be 0 or 1");
        if (p_.fast_math && p_.fdtd_solver_type == 1 && p_.wall_coupling != 0.0f)
            raise(VS_ERR_UNSUPPORTED, "fast_math does not cover the coupled wall oscillator");
        if (p_.num_steps <= 0 && !(p_.audio_dur > 0.0f)) raise(VS_ERR_INVALID_ARG, "need num_steps > 0 or audio_dur > 0");
        if ((p_.source_type == VS_SRC_GAUSS || p_.source_type == VS_SRC_GAUSS_STD) && !(p_.gauss_width_s > 0.0f))
            raise(VS_ERR_INVALID_ARG, "gauss_width_s must be > 0");
        if (p_.simulation_type == 1) {
            if (!g_ || g_->n_sections < 1 || !g_->section_length_cm || !g_->section_area_cm2)
                raise(VS_ERR_GEOMETRY, "tube simulation needs a non-empty area function");
            for (int i = 0; i < g_->n_sections; ++i)
                if (!(g_->section_length_cm[i] > 0.0f) || !(g_->section_area_cm2[i] > 0.0f) ||
                    !std::isfinite(g_->section_length_cm[i]) || !std::isfinite(g_->section_area_cm2[i]))
                    raise(VS_ERR_GEOMETRY, "every section needs a finite length > 0 and area > 0");
            if (p_.cross_sectional_shape < 1 || p_.cross_sectional_shape > 3)
                raise(VS_ERR_UNSUPPORTED,
                      "cross_sectional_shape must be 1 (circular), 2 (elliptical) or 3 (single-plane symmetric)");
            if (p_.cross_sectional_shape == 3 && p_.uniform_depth_m > 0.0f)
                raise(VS_ERR_UNSUPPORTED, "uniform_depth_m applies to circular and elliptical sections");
        }
    }

    void tables() { fill_tables(p_, k_, T_); }

    void alloc_frame(int H, int W) {
        if (H < 3 || W < 3 || (int64_t)H * W > (int64_t)1 << 28) raise(VS_ERR_GEOMETRY, "frame size out of range");
        T_.H = H; T_.W = W;
        size_t n = (size_t)H * W;
        if (planes_) {
            T_.cell_type.assign(n, VS_CELL_AIR);
            seg_.assign(n, 0);
            T_.zinv.assign(n, 0.0f);
            T_.dP.assign(n, 1.0f); T_.dX.assign(n, 1.0f); T_.dY.assign(n, 1.0f);
        }
        T_.dims.frame_h = H; T_.dims.frame_w = W;
        T_.dims.interior_cells = (int64_t)(H - 2) * (W - 2);
    }

    void open_space() {
        // FDTDSolver::openSpaceSimulation (FDTDSolver.cu:479-550)
        alloc_frame(43 + 2 + 2 * pml_, 341 + 2 + 2 * pml_);
        const float d0 = p_.fdtd_solver_type == 1 ? (float)(1.0 * osd_) : 1.0f;
        std::fill(T_.dP.begin(), T_.dP.end(), d0);
        std::fill(T_.dX.begin(), T_.dX.end(), d0);
        std::fill(T_.dY.begin(), T_.dY.end(), d0);
        const int ey = T_.H / 2 - 1, ex = T_.W / 2 - 1;   // ceil() of an integer quotient
        type(ey, ex) = VS_CELL_EXCITATION;
        vs_dims& d = T_.dims;
        d.excitation_x = ex; d.excitation_y = ey;
        d.listener_x = ex + 5; d.listener_y = ey + 5;
        d.tube_mid_y = ey;
    }

    void tube() {
        const int n = g_->n_sections;
        const bool ellipse = p_.cross_sectional_shape == 2;
        const bool sps = p_.cross_sectional_shape == 3;
        // computeTubeWidthCircle / Ellipse / SinglePlaneSymmetry (TubeGeometry.cu:316-431)
        std::vector<float> width(n), minor(n, 0.0f), len_m(n);
        if (sps) shapes_.assign(n, {});
        for (int i = 0; i < n; ++i) {
            const float a = g_->section_area_cm2[i] * kCm * kCm;
            if (sps) {
                std::string err;
                shapes_[i] = sps_shape(a, &width[i], &err);
                if (shapes_[i].empty()) raise(VS_ERR_GEOMETRY, err.c_str());
            } else if (!ellipse) {
                width[i] = (float)(2.0 * std::sqrt((double)a / kPi));
            } else {
                const float lx = sqrtf((float)((double)a / ((double)(3.0f * 1.0f) * kPi)));
                width[i] = lx * 6.0f;
                minor[i] = lx * 2.0f;
            }
            len_m[i] = g_->section_length_cm[i] * kCm;
        }
        const int mic = (int)std::round((3 * kMm) / k_.ds);
        // setComputationalDomain (TubeGeometry.cu:112-179)
        float total = 0.0f;
        for (float v : len_m) total = total + v;
        const int L = (int)std::round(total / k_.ds);
        if (L < 2) raise(VS_ERR_GEOMETRY, "tube shorter than two cells");
        if (p_.fdtd_solver_type == 0) width = scale_2d(width);
        std::vector<int> dcell(n);
        for (int i = 0; i < n; ++i) {
            int c = (int)std::round(width[i] / k_.ds);
            if (c == 0) ++c;
            // an even count rounds down, and always down for shape 3 (TubeGeometry.cu:139-146)
            if (c % 2 == 0) c += (sps || (float)c - (width[i] / k_.ds) > 0) ? -1 : 1;
            dcell[i] = c;
        }
        const int dmax = *std::max_element(dcell.begin(), dcell.end());
        const bool dir = p_.mouth_radiation_cond == 1;
        alloc_frame(dmax + 2 + 2 + 2 * pml_, (dir ? L + 2 : L + 1 + mic) + 2 + 2 * pml_);
        const int W = T_.W;

        // setVocalTractWalls (TubeGeometry.cu:433-484): one column per cell
        const int sx = 2 + pml_;
        const int my = (int)std::ceil(T_.H / 2.0f) - 1;
        const int ex = sx + L - 1;
        std::vector<float> cum(n);
        float acc = 0.0f;
        for (int i = 0; i < n; ++i) { acc = acc + len_m[i]; cum[i] = acc; }
        std::vector<Column> col(L);
        const float half = k_.ds * 0.5f;
        for (int i = 0; i < L; ++i) {
            const float x = (i + 1) * k_.ds;
            int s = 0;
            while (s < n - 1 && x > cum[s] + half) ++s;
            const int r = (dcell[s] - 1) / 2;
            col[i] = {my - r - 1, my + r + 1, s};
            if (col[i].up < 0 || col[i].down >= T_.H) raise(VS_ERR_GEOMETRY, "wall outside the frame");
            if (!planes_) continue;
            type(col[i].up, sx + i) = VS_CELL_WALL;
            type(col[i].down, sx + i) = VS_CELL_WALL;
            seg(col[i].up, sx + i) = s + 1;
            seg(col[i].down, sx + i) = s + 1;
        }
        // the wall-gap fill below paints, in column i, rows up[i-1] .. up[i]
        // (and lower[i] .. lower[i-1]) when the upper wall drops by more than
        // one row from column i-1 (i in 1..L-2), and rows up[i+1] .. up[i]
        // (lower[i] .. lower[i+1]) when it rises by more than one row to
        // column i+1 (i+1 in 1..L-2), always with the column's own segment id
        // (the largest id in a column is its own); so each wall is one run of
        // rows per column, which the device builder paints from these bounds
        T_.upper_top.assign(L, 0);
        T_.lower_bot.assign(L, 0);
        for (int i = 0; i < L; ++i) {
            int top = col[i].up, bot = col[i].down;
            if (i >= 1 && i <= L - 2 && col[i].up - col[i - 1].up > 1) {
                top = std::min(top, col[i - 1].up);
                bot = std::max(bot, col[i - 1].down);
            }
            if (i + 1 >= 1 && i + 1 <= L - 2 && col[i + 1].up - col[i].up < -1) {
                top = std::min(top, col[i + 1].up);
                bot = std::max(bot, col[i + 1].down);
            }
            T_.upper_top[i] = top;
            T_.lower_bot[i] = bot;
        }
        // connectSagittalWallsGap (TubeGeometry.cu:496-569): sequential fill of
        // jumps larger than one row, columns 1..L-2
        auto column_max_seg = [&](int c) {
            if (!planes_) return col[c - sx].seg + 1;     // the column's own id (see above)
            int m = 0;
            for (int r = 0; r < T_.H; ++r) m = std::max(m, seg(r, c));
            return m;
        };
        auto paint = [&](int c, int r0, int r1, int s) {
            for (int r = r0; r <= r1; ++r) { type(r, c) = VS_CELL_WALL; seg(r, c) = s; }
        };
        for (int i = 1; i <= L - 2 && planes_; ++i) {
            const Column& a = col[i - 1];
            const Column& b = col[i];
            const int jump = b.up - a.up;
            if (jump > 1) {
                const int s = column_max_seg(sx + i);
                paint(sx + i, a.up, b.up, s);
                paint(sx + i, b.down, a.down, s);
            } else if (jump < -1) {
                const int s = column_max_seg(sx + i - 1);
                paint(sx + i - 1, b.up, a.up, s);
                paint(sx + i - 1, a.down, b.down, s);
            }
        }
        // setExcitationCells (TubeGeometry.cu:571-594)
        if (planes_) {
            for (int r = col[0].up + 1; r < col[0].down; ++r) type(r, sx - 1) = VS_CELL_EXCITATION;
            type(col[0].up, sx - 1) = VS_CELL_WALL;
            type(col[0].down, sx - 1) = VS_CELL_WALL;
        }
        vs_dims& d = T_.dims;
        // listener / excitation (FDTDSolver.cu:591-611)
        if (dir) {
            if (planes_)
                for (int r = col[L - 1].up; r <= col[L - 1].down; ++r) type(r, ex + 1) = VS_CELL_NOPRESSURE;
            d.listener_x = ex - mic;
        } else {
            d.listener_x = ex + 3 + mic;
        }
        d.listener_y = my;
        d.excitation_x = sx - 1;
        d.excitation_y = my;
        d.tube_length_cells = L;
        d.tube_start_x = sx; d.tube_end_x = ex; d.tube_mid_y = my;

        // semi-reflective walls (FDTDSolver.cu:613-622)
        const float mu3 = p_.mu3d > 0.0f ? p_.mu3d : (p_.fdtd_solver_type == 1 ? 0.025f : 0.005f);
        const float mu2 = (float)((double)mu3 * (((double)(2.0f * 0.5f) * kPi) / (double)1.84f));
        const float alpha = 1.0f / (0.5f + 0.25f * (mu2 + (1 / mu2)));
        const float q = sqrtf(1 - alpha);
        T_.zinv_val = 1 / (k_.rho * k_.c * ((1 + q) / (1 - q)));
        d.z_inv_val = T_.zinv_val;
        for (size_t i = 0; i < seg_.size(); ++i)
            if (seg_[i] != 0) T_.zinv[i] = T_.zinv_val;

        if (p_.fdtd_solver_type == 1 && planes_) depth(col, minor, sx, my, ex, column_max_seg);
        (void)W;
        for (int i = 0; i < L; ++i) {
            T_.upper.push_back(col[i].up);
            T_.lower.push_back(col[i].down);
            T_.colseg.push_back(column_max_seg(sx + i) - 1);
        }
        T_.major_m = width;
        T_.minor_m = minor;
    }

    static std::vector<float> scale_2d(const std::vector<float>& d) {
        // TubeGeometry::tubeAreaScaling (TubeGeometry.cu:241-286)
        const size_t n = d.size();
        const float dm = *std::max_element(d.begin(), d.end());
        size_t im = 0;
        for (size_t i = 0; i < n; ++i) if (d[i] == dm) im = i;
        std::vector<float> out(n, 0.0f), ratio(n, 1.0f);
        out[im] = (float)(((double)dm * 0.5 * kPi) / (double)1.84f);
        for (size_t i = 0; i < n; ++i) {
            if (i == im) continue;
            const float b = i < im ? d[i + 1] : d[i - 1];
            ratio[i] = b != 0.0f ? powf(d[i] / b, 2.0f) : 1.0f;
        }
        for (size_t i = im; i-- > 0;) out[i] = out[i + 1] * ratio[i];
        for (size_t i = im + 1; i < n; ++i) out[i] = out[i - 1] * ratio[i];
        return out;
    }

    template <class ColMax>
    void depth(const std::vector<Column>& col, const std::vector<float>& minor, int sx, int my,
               int ex, ColMax column_max_seg) {
        // TubeDepth::setTubeDepth (TubeDepth.cu:95-169) for circular and
        // elliptical sections, followed by generateDepthP and setMinDepth.
        const float fill = (float)(1.0 * osd_);
        std::fill(T_.dP.begin(), T_.dP.end(), fill);
        std::fill(T_.dX.begin(), T_.dX.end(), fill);
        std::fill(T_.dY.begin(), T_.dY.end(), fill);
        const float ds = k_.ds;
        const bool ellipse = p_.cross_sectional_shape == 2;
        const float ud = p_.uniform_depth_m;
        if (p_.cross_sectional_shape == 3) {
            sps_depth(col, sx, column_max_seg);
            finish_depth(my, ex);
            return;
        }
        for (size_t i = 0; i < col.size(); ++i) {
            const int x = sx + (int)i;
            const int air = col[i].down - col[i].up - 1;
            const int h = (int)std::ceil(air * 0.5f) - 1;
            float r2 = 0, a2 = 0, b2 = 0;
            if (!ellipse) {
                const float r = ((float)air / 2.0f) * ds;
                r2 = r * r;
            } else {
                const int s = column_max_seg(x);
                if (s < 1) raise(VS_ERR_GEOMETRY, "tube column without a segment id");
                const float a = (air * ds) / 2.0f;
                const float b = minor[s - 1] / 2.0f;
                a2 = a * a;
                b2 = b * b;
            }
            // radicand of the half-depth at distance y from the tube axis
            auto radicand = [&](float y) -> float {
                if (!ellipse) {
                    if (p_.depth_fma) return std::fma(-y, y, r2);
                    const float yy = y * y;
                    return r2 - yy;
                }
                const float yy = y * y;
                return b2 * (1.0f - (yy / a2));
            };
            for (int k = h; k >= 0; --k) {
                const int ru = col[i].up + (h - k) + 1;
                const int rl = col[i].down - (h - k) - 1;
                const float rx = radicand((float)k * ds);
                const float rlo = radicand(((float)k - 0.5f) * ds);
                const float rup = k != h ? radicand(((float)k + 0.5f) * ds) : 0.0f;
                if (rx < 0.f || rlo < 0.f || rup < 0.f)
                    raise(VS_ERR_NEGATIVE_SQRT, "negative radicand in the tube depth formula");
                float vx = 2 * sqrtf(rx), vup = 2 * sqrtf(rup), vlo = 2 * sqrtf(rlo);
                if (ud > 0.0f) { vx = ud; vlo = ud; vup = k != h ? ud : 0.0f; }
                dX(ru, x) = vx; dX(rl, x) = vx;
                dY(ru, x) = vup; dY(rl, x) = vlo;
            }
            dX(col[i].up, x) = 0; dX(col[i].down, x) = 0;
            dY(col[i].up, x) = 0; dY(col[i].down, x) = 0;
        }
        finish_depth(my, ex);
    }

    // TubeDepth::generateTubeDepthSinglePlaneSymmetricShape (TubeDepth.cu:493-640):
    // per tube column, with the aligned contour of its section, dX of the
    // k-th air cell above the lower wall = half the contour's z extent along
    // y = minY + (k - 1/2) ds, dY along y = minY + k ds (0 for the top cell);
    // the wall cells 0.
    template <class ColMax>
    void sps_depth(const std::vector<Column>& col, int sx, ColMax column_max_seg) {
        const float ds = k_.ds;
        for (size_t i = 0; i < col.size(); ++i) {
            const int x = sx + (int)i;
            const int up = col[i].up, down = col[i].down;
            const int air = down - up - 1;
            const int s = column_max_seg(x);
            if (s < 1 || s > (int)shapes_.size()) raise(VS_ERR_GEOMETRY, "tube column without a segment id");
            const std::vector<ShapePt>& sh = shapes_[(size_t)s - 1];
            float minZ = std::numeric_limits<float>::infinity(), maxZ = -minZ;
            float minY = minZ;
            for (const ShapePt& p : sh) {
                minZ = std::min(minZ, p.z);
                maxZ = std::max(maxZ, p.z);
                minY = std::min(minY, p.y);
            }
            const float zlo = (float)((double)minZ - 0.001), zhi = (float)((double)maxZ + 0.001);
            for (int k = 1; k <= air; ++k) {
                const int row = down - k;
                const float off_x = (float)((k - 0.5) * (double)ds);
                const float off_y = k * ds;
                float vx = 0.0f, vy = 0.0f;
                if (!sps_half_depth(sh, minY + off_x, zlo, zhi, &vx))
                    raise(VS_ERR_GEOMETRY, "single-plane-symmetric depth: the line misses the section");
                if (k < air && !sps_half_depth(sh, minY + off_y, zlo, zhi, &vy))
                    raise(VS_ERR_GEOMETRY, "single-plane-symmetric depth: the line misses the section");
                if (vx < 0.0f || vy < 0.0f) raise(VS_ERR_GEOMETRY, "negative single-plane-symmetric depth");
                dX(row, x) = vx;
                dY(row, x) = vy;
            }
            dX(down, x) = 0; dX(up, x) = 0;
            dY(down, x) = 0; dY(up, x) = 0;
        }
    }

    // generateDepthP and setMinDepth (TubeDepth.cu:215-253, 642-762)
    void finish_depth(int my, int ex) {
        // generateDepthP (TubeDepth.cu:215-253)
        const int H = T_.H, W = T_.W;
        const size_t n = (size_t)H * W, pivot = (size_t)my * W + ex;
        const float px0 = T_.dX[pivot], py0 = T_.dY[pivot];
        for (size_t i = 0; i < n; ++i) {
            if (T_.dX[i] == osd_) T_.dX[i] = px0;
            if (T_.dY[i] == osd_) T_.dY[i] = py0;
        }
        std::vector<float> sx2(n), sy2(n);
        for (int r = 0; r < H; ++r) {
            for (int c = 0; c < W; ++c) {
                const size_t i = (size_t)r * W + c;
                const float right = c < W - 1 ? T_.dX[i + 1] : T_.dX[pivot];
                const float above = r > 0 ? T_.dY[i - W] : T_.dY[pivot];
                sx2[i] = 0.5f * (T_.dX[i] + right);
                sy2[i] = 0.5f * (T_.dY[i] + above);
            }
        }
        T_.dX.swap(sx2);
        T_.dY.swap(sy2);
        const float px = T_.dX[pivot], py = T_.dY[pivot];
        for (int r = 0; r < H; ++r) {
            for (int c = 0; c < W; ++c) {
                const size_t i = (size_t)r * W + c;
                const float left = c > 0 ? T_.dX[i - 1] : px;
                const float below = r < H - 1 ? T_.dY[i + W] : py;
                T_.dP[i] = 0.25f * (T_.dX[i] + T_.dY[i] + left + below);
            }
        }
        const float lo = 0.001f;   // TubeDepth::min_depth
        for (size_t i = 0; i < n; ++i) {
            if (T_.dP[i] < lo) T_.dP[i] = lo;
            if (T_.dX[i] < lo) T_.dX[i] = lo;
            if (T_.dY[i] < lo) T_.dY[i] = lo;
        }
    }

    void dead_ring_and_pml() {
        const int H = T_.H, W = T_.W;
        for (int c = 0; c < W; ++c) { type(0, c) = VS_CELL_DEAD; type(H - 1, c) = VS_CELL_DEAD; }
        for (int r = 0; r < H; ++r) { type(r, 0) = VS_CELL_DEAD; type(r, W - 1) = VS_CELL_DEAD; }
        if (!p_.pml_flag) return;
        // graded layers, outermost = pml5; rows first, then columns (corners)
        for (int l = 0; l < kPmlLayers; ++l) {
            const int t = VS_CELL_PML5 - l;
            for (int c = 1 + l; c <= W - 2 - l; ++c) { type(1 + l, c) = t; type(H - 2 - l, c) = t; }
        }
        for (int l = 0; l < kPmlLayers; ++l) {
            const int t = VS_CELL_PML5 - l;
            for (int r = 1 + l; r <= H - 2 - l; ++r) { type(r, 1 + l) = t; type(r, W - 2 - l) = t; }
        }
    }

    void listener_override() {
        vs_dims& d = T_.dims;
        if (p_.listener_mode == VS_LISTENER_EXPLICIT) {
            d.listener_x = p_.listener_x;
            d.listener_y = p_.listener_y;
        } else if (p_.listener_mode != VS_LISTENER_REFERENCE) {
            raise(VS_ERR_INVALID_ARG, "listener_mode");
        }
        if (d.listener_x < 1 || d.listener_x > T_.W - 2 || d.listener_y < 1 || d.listener_y > T_.H - 2)
            raise(VS_ERR_INVALID_ARG, "listener must be an interior cell of the frame");
    }

    void pack() {
        // Device planes are padded to a 32-element row pitch; padding cells are
        // dead and never updated.
        T_.pitch = (T_.W + 31) / 32 * 32;
        if (!planes_) return;
        T_.code.assign((size_t)T_.H * T_.pitch, (uint8_t)VS_CELL_DEAD);
        for (int r = 0; r < T_.H; ++r)
            for (int c = 0; c < T_.W; ++c) {
                const size_t i = (size_t)r * T_.W + c;
                uint8_t v = (uint8_t)T_.cell_type[i];
                if (T_.zinv[i] != 0.0f) v |= CODE_ZINV_BIT;
                T_.code[(size_t)r * T_.pitch + c] = v;
            }
    }
};

}  // namespace

void default_params(vs_params* p) {
    std::memset(p, 0, sizeof(*p));
    p->fdtd_solver_type = 1;
    p->simulation_type = 1;
    p->cross_sectional_shape = 1;
    p->mouth_radiation_cond = 0;
    p->srate_mul = 15;
    p->source_type = VS_SRC_GAUSS;
    p->pml_flag = 1;
    p->engine = VS_ENGINE_CPU;
    p->audio_dur = 100 * kMs;
    const float f0 = 10.0f * kKhz;                 // GlottalExcitations.cu:28-31
    p->gauss_peak_s = 0.646f / f0;
    p->gauss_width_s = 0.29f * p->gauss_peak_s;
    p->gauss_amp = 0.025f;
    p->sine_freq_hz = 440 * kHz;                   // GlottalExcitations.cu:20-21
    p->sine_amp = 25;
    p->tmm_ps_pa = 686.46f;                        // TwoMassModel.cpp:52
    p->depth_fma = 1;
    p->listener_mode = VS_LISTENER_REFERENCE;
}

void build_source(const vs_params* p, float dt, int64_t n, std::vector<float>& out) {
    // GlottalExcitations::setExcitationVelocity (GlottalExcitations.cu:9-52);
    // t = idx * dt is formed in double because dt arrives as a double there.
    out.assign((size_t)n, 0.0f);
    const double ddt = (double)dt;
    if (p->source_type == VS_SRC_SINE) {
        for (int64_t i = 0; i < n; ++i) {
            const float t = (float)(i * ddt);
            out[i] = (float)((double)p->sine_amp * std::sin(2 * kPi * (double)p->sine_freq_hz * (double)t));
        }
    } else if (p->source_type == VS_SRC_GAUSS || p->source_type == VS_SRC_GAUSS_STD) {
        const float scale = p->source_type == VS_SRC_GAUSS ? -1.0f : -0.5f;
        for (int64_t i = 0; i < n; ++i) {
            const float t = (float)(i * ddt);
            const float e = (t - p->gauss_peak_s) / p->gauss_width_s;
            out[i] = p->gauss_amp * expf(scale * (e * e));
        }
    }
}

template <class F>
TmmConstsT<F> tmm_consts(float ps, int srate_mul) {
    // TwoMassModel::setTwoMassModelParams (TwoMassModel.cpp:4-87), q = gs = 1.
    // The unit constants and literals are floats; for F = double they are
    // widened before the products, as a double instantiation of the
    // reference's expressions would do.
    TmmConstsT<F> t;
    const F cm = (F)kCm, gram = (F)kGram, dyn = (F)kDyn;
    t.mu = (F)(1.86e-4 * (double)(kDyn * kSecond / (kCm * kCm)));
    t.rho = (F)(1.14 * (double)(kKg / (kMeter * kMeter * kMeter)));
    const F q = 1.0f, gs = 1.0f;
    t.m1 = ((F)0.125f * gram) / q;
    t.m2 = ((F)0.025f * gram) / q;
    t.d1 = ((F)0.25f * cm) / q;
    t.d2 = ((F)0.05f * cm) / q;
    t.k1 = (F)80000.0f * (dyn / cm) * q;
    t.k2 = (F)8000.0f * (dyn / cm) * q;
    t.kc = (F)25000.0f * (dyn / cm) * (q * q);
    t.etak1 = 100 / (cm * cm);
    t.etak2 = 100 / (cm * cm);
    t.h1 = 3 * t.k1;
    t.h2 = 3 * t.k2;
    t.etah1 = (F)500.0f / (cm * cm);
    t.etah2 = (F)500.0f / (cm * cm);
    t.Ag01 = (F)0.05f * (cm * cm);
    t.Ag02 = t.Ag01;
    t.lg = (F)1.40f * cm;
    t.r1o = (2 * (F)0.2f * std::sqrt(t.k1 * t.m1)) / (gs * gs);
    t.r2o = (2 * (F)0.6f * std::sqrt(t.k2 * t.m2)) / (gs * gs);
    t.r1c = (2 * (F)1.1f * std::sqrt(t.k1 * t.m1)) / (gs * gs);
    t.r2c = (2 * (F)1.9f * std::sqrt(t.k2 * t.m2)) / (gs * gs);
    t.A1 = (F)3.0f * (cm * cm);
    t.ps = (F)ps;
    t.srate = 44100 * (F)srate_mul;
    return t;
}

template TmmConstsT<float> tmm_consts<float>(float, int);
template TmmConstsT<double> tmm_consts<double>(float, int);

static TmmConsts64 widen(const TmmConsts& c) {
    return {c.mu, c.rho, c.m1, c.m2, c.d1, c.d2, c.k1, c.k2, c.kc, c.etak1, c.etak2, c.h1, c.h2, c.etah1,
            c.etah2, c.Ag01, c.Ag02, c.lg, c.r1o, c.r2o, c.r1c, c.r2c, c.A1, c.ps, c.srate};
}

TmmDerived64 tmm_derived(const TmmConsts64& k) {
    TmmDerived64 d{};
    d.isr = 1.0 / k.srate;
    d.is2 = d.isr * d.isr;
    d.two_lg = 2.0 * k.lg;
    d.g1 = k.Ag01 / d.two_lg;
    d.g2 = k.Ag02 / d.two_lg;
    d.c12 = 12.0 * k.mu * k.lg * k.lg;
    d.cR1 = d.c12 * k.d1;
    d.cR2 = d.c12 * k.d2;
    d.cL1 = k.rho * k.d1;
    d.cL2 = k.rho * k.d2;
    d.hr = k.rho / 2.0;
    d.hr137 = 1.37 * d.hr;
    d.d1lg = k.d1 * k.lg;
    d.d2lg = k.d2 * k.lg;
    d.iA1 = 1.0 / k.A1;
    d.k1e = k.k1 * k.etak1;
    d.k2e = k.k2 * k.etak2;
    for (int c = 0; c < 2; ++c) {
        const double h1u = c ? k.h1 : 0.0, r1u = c ? k.r1c : k.r1o;
        const double h2u = c ? k.h2 : 0.0, r2u = c ? k.r2c : k.r2o;
        d.a11[c] = (k.k1 + h1u + k.kc) * d.is2 + r1u * d.isr + k.m1;
        d.a22[c] = (k.k2 + h2u + k.kc) * d.is2 + r2u * d.isr + k.m2;
        d.b1c[c] = 2.0 * k.m1 + r1u * d.isr;
        d.b2c[c] = 2.0 * k.m2 + r2u * d.isr;
    }
    d.a12 = -k.kc * d.is2;
    for (int c1 = 0; c1 < 2; ++c1)
        for (int c2 = 0; c2 < 2; ++c2) {
            double det = d.a11[c1] * d.a22[c2] - d.a12 * d.a12;
            if (det == 0.0) det = 1.0;
            d.idet[c1][c2] = 1.0 / det;
        }
    return d;
}

static void fill_tmm(const vs_params* p, TubeGrid& out) {
    out.tmmc = tmm_consts<float>(p->tmm_ps_pa, p->srate_mul);
    out.tmm64 = p->source_type == VS_SRC_TMM && p->tmm_f64 != 0;
    out.tmmd = out.tmm64 ? tmm_consts<double>(p->tmm_ps_pa, p->srate_mul) : widen(out.tmmc);
    out.tmmx = tmm_derived(out.tmmd);
}

void build_tube(const vs_params* p, const vs_geometry* g, TubeGrid& out, int64_t steps_for_source) {
    if (!p) throw VsFailure{VS_ERR_INVALID_ARG, "null vs_params"};
    Builder(p, g, out).run();
    const int64_t n = steps_for_source > 0 ? steps_for_source : out.dims.num_steps;
    if (p->source_type == VS_SRC_TMM) out.source.clear();
    else build_source(p, out.dt, n, out.source);
    fill_tmm(p, out);
}

bool device_buildable(const vs_params* p) {
    return p && p->simulation_type == 1 && (p->cross_sectional_shape == 1 || p->cross_sectional_shape == 2);
}

void build_tube_columns(const vs_params* p, const vs_geometry* g, TubeGrid& out, int64_t steps_for_source) {
    if (!p) throw VsFailure{VS_ERR_INVALID_ARG, "null vs_params"};
    if (!device_buildable(p)) throw VsFailure{VS_ERR_UNSUPPORTED, "the device map builder covers circular and "
                                                                   "elliptical tube sections"};
    Builder(p, g, out, false).run();
    const int64_t n = steps_for_source > 0 ? steps_for_source : out.dims.num_steps;
    if (p->source_type == VS_SRC_TMM) out.source.clear();
    else build_source(p, out.dt, n, out.source);
    fill_tmm(p, out);
}

void solver_constants(const vs_params* p, TubeGrid& out) {
    if (!p) throw VsFailure{VS_ERR_INVALID_ARG, "null vs_params"};
    if (p->srate_mul < 1 || p->srate_mul > 64) throw VsFailure{VS_ERR_INVALID_ARG, "srate_mul must be in 1..64"};
    fill_tables(*p, physics(p->srate_mul), out);
    fill_tmm(p, out);
}

}  // namespace vsb
