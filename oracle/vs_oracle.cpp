/*
 * vs_oracle.cpp -- CPU ORACLE for the 2.5D FDTD time-stepping path.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / reference legs of bench.py may load this library; the
 * product (libvocalsim_b200.so) never links, loads or calls it.
 *
 * It restates, in plain C++ and in the reference's own arithmetic order, the
 * path of Debasishray19/VocalSim-2p5D-FDTD:
 *   setup   SimulationParams.cu:7-34, SolverParams.cu:5-76,
 *           TubeGeometry.cu:53-612 (circular / elliptical only),
 *           TubeDepth.cu:95-490,642-762, FDTDSolver.cu:289-801,806-1070,
 *           GlottalExcitations.cu:9-52
 *   loop    FDTDEngineCPU.cpp:222-433 and FDTDEngineEigen.cpp:121-324
 *   source  TwoMassModel.cpp:4-232
 * The engine is a template over the field type: float reproduces the
 * reference FP32 engine, double gives the double-precision trace of the same
 * discrete system (same maps, same float-rounded primary constants).
 *
 * Pinning.  The reference's setup and engines cannot be compiled here (their
 * headers pull Boost.Geometry and Eigen, neither installed), so the maps and
 * the loop are pinned only through this restatement.  The two-mass model,
 * the excitation tables, the beta / sigma tables, the step count and the
 * physical constants ARE pinned: oracle/Makefile.ref compiles the reference's
 * own TwoMassModel.cpp, GlottalExcitations.cu, SolverParams.cu and
 * SimulationParams.cu into oracle/_ref/, and tests compare them bit for bit.
 *
 * Build: g++ -O2 -ffp-contract=off (no FMA contraction, x86-64 SSE float
 * semantics, matching the reference's MSVC x64 host build).  The one place
 * the reference's GPU setup kernels admit an FMA contraction (the circular
 * depth radicand, TubeDepth.cu:355-370) is reproduced with std::fma when
 * vs_params::depth_fma is set.
 */
#include "../include/vocalsim_b200.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

namespace {

/* ---- SimulationUnits.h:11-25 (float constants built from double products) */
const float U_METER = 1;
const float U_CENTIMETER = (float)(1e-2 * (double)U_METER);
const float U_MILLIMETER = (float)(1e-3 * (double)U_METER);
const float U_SECOND = 1;
const float U_MILLISECOND = (float)(1e-3 * (double)U_SECOND);
const float U_HERTZ = 1 / U_SECOND;
const float U_KILOHERTZ = (float)(1e3 * (double)U_HERTZ);
const float U_KILOGRAM = 1;
const float U_GRAM = (float)(1e-3 * (double)U_KILOGRAM);
const float U_NEWTON = U_KILOGRAM * U_METER / (U_SECOND * U_SECOND);
const float U_DYN = (float)(1e-5 * (double)U_NEWTON);

const double K_PI = 3.14159265358979323846;

struct OracleError {
    int code;
    std::string msg;
};

/* ---- SimulationParams(int srate_mul), SimulationParams.cu:7-34 ---------- */
struct PhysConsts {
    float sound_speed, rho, kappa, dt, ds, max_sigma_dt;
    int base_srate, srate, pml_layers;
    float cpl, Mw, Bw, Kw;
};

PhysConsts phys_consts(int srate_mul) {
    PhysConsts k;
    k.sound_speed = 350.0f * (U_METER / U_SECOND);
    k.rho = (float)((double)(1.14f * U_KILOGRAM) / std::pow((double)U_METER, 3));
    k.base_srate = (int)(44100 * U_HERTZ);
    k.kappa = k.rho * k.sound_speed * k.sound_speed;
    k.srate = k.base_srate * srate_mul;
    k.dt = 1.0f / static_cast<float>(k.srate);
    k.ds = k.dt * k.sound_speed * sqrtf(2.0f);
    k.max_sigma_dt = 0.5f;
    k.pml_layers = 6;
    k.cpl = 0.0f;
    k.Mw = 21 * (U_KILOGRAM / (U_METER * U_METER));
    k.Bw = 8000 * (U_KILOGRAM / (U_METER * U_METER * U_SECOND));
    k.Kw = 845000 * (U_KILOGRAM / (U_METER * U_METER * U_SECOND * U_SECOND));
    return k;
}

/* ---- SolverParams.cu:5-57 ------------------------------------------------ */
void solver_tables(int n_pml, float max_sigma_dt, float dt, float beta[13],
                   float sigma[13], float dir[4]) {
    for (int i = 0; i < 13; i++) { beta[i] = 0; sigma[i] = 0; }
    beta[VS_CELL_WALL] = 0; beta[VS_CELL_AIR] = 1; beta[VS_CELL_EXCITATION] = 0;
    beta[VS_CELL_DYNAMIC] = 0; beta[VS_CELL_DEAD] = 0; beta[VS_CELL_NOPRESSURE] = 1;
    beta[VS_CELL_HEAD] = 0;
    for (int k = 0; k < n_pml; k++) beta[VS_CELL_PML0 + k] = 1;

    sigma[VS_CELL_WALL] = dt; sigma[VS_CELL_AIR] = 0; sigma[VS_CELL_NOPRESSURE] = 0;
    sigma[VS_CELL_EXCITATION] = dt; sigma[VS_CELL_HEAD] = dt; sigma[VS_CELL_DYNAMIC] = 0;
    sigma[VS_CELL_DEAD] = 1000000;
    for (int k = 0; k < n_pml; k++)
        sigma[VS_CELL_PML0 + k] = ((float)k / (float)(n_pml - 1)) * max_sigma_dt;

    /* SolverParams.cu:62-69: left, down, right, up */
    dir[0] = 0; dir[1] = 0; dir[2] = 1; dir[3] = 0;
}

/* SolverParams.cu:59-66: float accumulation of dt (drifts, kept as is) */
long long reference_step_count(float audio_time, float dt) {
    float t = 0;
    long long n = 0;
    while (t <= audio_time - dt) { n++; t = t + dt; }
    return n;
}

/* ---- the built grid ------------------------------------------------------- */
struct Grid {
    PhysConsts k;
    int H = 0, W = 0;
    int listenerX = 0, listenerY = 0, excX = 0, excY = 0;
    int tube_len = 0, tube_start_x = 0, tube_end_x = 0, tube_mid_y = 0;
    long long num_steps = 0;
    float K1 = 0, K2 = 0, zinv_val = 0;
    float beta[13], sigma[13], dir[4];
    std::vector<int> type, bst;
    std::vector<float> zinv, dP, dX, dY;
    double scan_margin = 1e30;   /* min |curr_len - (cum + ds/2)| / cum seen */
};

/* ---- TubeGeometry: widths (TubeGeometry.cu:316-364) ------------------------ */
struct Tube {
    std::vector<float> len_m, diam_m, minor_m;
    std::vector<int> diam_cells;
    int L = 0;
    int mic_cells = 0;
    std::vector<int> upper, lower;
};

/* Section diameters of single-plane-symmetric sections (shape 3) are not
   restated here (their construction needs Boost.Geometry in the reference):
   the tests supply them with orc_set_sps_diameters, and the depth maps with
   orc_run_maps_f32. */
std::vector<float> g_sps_diameters;

void tube_widths(const vs_params* p, const vs_geometry* g, Tube& t) {
    if (p->cross_sectional_shape == 3 && (int)g_sps_diameters.size() != g->n_sections)
        throw OracleError{VS_ERR_UNSUPPORTED, "shape 3 needs the section diameters (orc_set_sps_diameters)"};
    for (int i = 0; i < g->n_sections; i++) {
        float area = g->section_area_cm2[i];
        float a_m2 = area * U_CENTIMETER * U_CENTIMETER;
        if (p->cross_sectional_shape == 3) {
            t.diam_m.push_back(g_sps_diameters[i]);
            t.minor_m.push_back(0.0f);
        } else if (p->cross_sectional_shape == 1) {
            float d = (float)(2.0 * std::sqrt((double)a_m2 / K_PI));
            t.diam_m.push_back(d);
            t.minor_m.push_back(0.0f);
        } else {
            const float semi_major = 3.0f, semi_minor = 1.0f;
            float lenX = sqrtf((float)((double)a_m2 / ((double)(semi_major * semi_minor) * K_PI)));
            float major_len = lenX * (semi_major * 2);
            float minor_len = lenX * (semi_minor * 2);
            t.diam_m.push_back(major_len);
            t.minor_m.push_back(minor_len);
        }
    }
    for (int i = 0; i < g->n_sections; i++)
        t.len_m.push_back(g->section_length_cm[i] * U_CENTIMETER);
}

/* TubeGeometry::tubeAreaScaling, TubeGeometry.cu:241-286 (2D solver only) */
std::vector<float> area_scaling_2d(const std::vector<float>& d3) {
    size_t n = d3.size();
    float dmax = *std::max_element(d3.begin(), d3.end());
    size_t imax = 0;
    for (size_t i = 0; i < n; i++) if (d3[i] == dmax) imax = i;
    std::vector<float> d2(n, 0.0f);
    d2[imax] = (float)(((double)dmax * 0.5 * K_PI) / (double)1.84f);
    std::vector<float> m(n, 1.0f);
    for (size_t i = 0; i < n; i++) {
        if (i < imax) {
            float a = d3[i], b = d3[i + 1];
            m[i] = (b != 0.0f) ? powf(a / b, 2.0f) : 1.0f;
        } else if (i > imax) {
            float a = d3[i], b = d3[i - 1];
            m[i] = (b != 0.0f) ? powf(a / b, 2.0f) : 1.0f;
        }
    }
    for (int i = (int)imax - 1; i >= 0; --i) d2[i] = d2[i + 1] * m[i];
    for (size_t i = imax + 1; i < n; ++i) d2[i] = d2[i - 1] * m[i];
    return d2;
}

/* ---- the whole setup, FDTDSolver::setupWaveSolver (FDTDSolver.cu:289-476) */
void build_grid(const vs_params* p, const vs_geometry* g, Grid& G) {
    if (!p) throw OracleError{VS_ERR_INVALID_ARG, "null params"};
    if (p->srate_mul < 1) throw OracleError{VS_ERR_INVALID_ARG, "srate_mul < 1"};
    if (p->fdtd_solver_type != 0 && p->fdtd_solver_type != 1)
        throw OracleError{VS_ERR_INVALID_ARG, "fdtd_solver_type"};
    if (p->pml_flag != 0 && p->pml_flag != 1) throw OracleError{VS_ERR_INVALID_ARG, "pml_flag"};

    G.k = phys_consts(p->srate_mul);
    PhysConsts& k = G.k;
    k.cpl = p->wall_coupling;
    const float open_space_depth = 0.50f;
    G.K1 = (k.kappa * k.dt) / k.ds;
    G.K2 = k.kappa * k.dt;
    solver_tables(k.pml_layers, k.max_sigma_dt, k.dt, G.beta, G.sigma, G.dir);
    G.num_steps = p->num_steps > 0 ? p->num_steps : reference_step_count(p->audio_dur, k.dt);
    const int pml = k.pml_layers * p->pml_flag;

    if (p->simulation_type == 0) {
        /* openSpaceSimulation, FDTDSolver.cu:479-550 */
        int domainH = 43, domainW = 341;
        G.H = domainH + 2 + 2 * pml;
        G.W = domainW + 2 + 2 * pml;
        size_t N = (size_t)G.H * G.W;
        G.type.assign(N, VS_CELL_AIR);
        G.bst.assign(N, 0);
        G.zinv.assign(N, 0.0f);
        float d0 = p->fdtd_solver_type == 1 ? (float)(1.0 * open_space_depth) : 1.0f;
        G.dP.assign(N, d0); G.dX.assign(N, d0); G.dY.assign(N, d0);
        /* integer division inside ceil(): ceil(frameH / 2) == frameH / 2 */
        int ey = G.H / 2 - 1, ex = G.W / 2 - 1;
        G.listenerY = ey + 5;
        G.listenerX = ex + 5;
        /* the reference assigns these to locals only (FDTDSolver.cu:530-531);
         * the members stay unset.  The oracle records the cell it marks. */
        G.excY = ey; G.excX = ex;
        G.type[(size_t)ey * G.W + ex] = VS_CELL_EXCITATION;
        G.tube_mid_y = ey;
    } else {
        if (!g || g->n_sections < 1 || !g->section_length_cm || !g->section_area_cm2)
            throw OracleError{VS_ERR_GEOMETRY, "empty area function"};
        for (int i = 0; i < g->n_sections; i++) {
            if (!(g->section_area_cm2[i] > 0.0f) || !(g->section_length_cm[i] > 0.0f))
                throw OracleError{VS_ERR_GEOMETRY, "section length / area must be > 0"};
        }
        if (p->cross_sectional_shape < 1 || p->cross_sectional_shape > 3)
            throw OracleError{VS_ERR_UNSUPPORTED, "cross_sectional_shape must be 1, 2 or 3"};
        Tube t;
        tube_widths(p, g, t);
        /* TubeGeometry.cu:105-106 */
        float mic_position = 3 * U_MILLIMETER;
        t.mic_cells = static_cast<int>(std::round(mic_position / k.ds));

        /* setComputationalDomain, TubeGeometry.cu:112-179 */
        float tube_length = 0.0f;
        for (float v : t.len_m) tube_length = tube_length + v;
        t.L = static_cast<int>(std::round(tube_length / k.ds));
        std::vector<float> diam = p->fdtd_solver_type == 1 ? t.diam_m : area_scaling_2d(t.diam_m);
        for (float d : diam) t.diam_cells.push_back(static_cast<int>(std::round(d / k.ds)));
        for (size_t i = 0; i < t.diam_cells.size(); i++) {
            if (t.diam_cells[i] == 0) t.diam_cells[i]++;
            if (t.diam_cells[i] % 2 == 0) {
                float diff = static_cast<float>(t.diam_cells[i]) - (diam[i] / k.ds);
                if (diff > 0 || p->cross_sectional_shape >= 3) t.diam_cells[i]--;
                else t.diam_cells[i]++;
            }
        }
        if (t.L < 2) throw OracleError{VS_ERR_GEOMETRY, "tube shorter than 2 cells"};
        int maxd = *std::max_element(t.diam_cells.begin(), t.diam_cells.end());
        int domainW = p->mouth_radiation_cond == 1 ? t.L + 1 + 1 : t.L + 1 + t.mic_cells;
        int domainH = maxd + 2;
        G.W = domainW + 2 + 2 * pml;
        G.H = domainH + 2 + 2 * pml;
        size_t N = (size_t)G.H * G.W;
        G.type.assign(N, VS_CELL_AIR);
        G.bst.assign(N, 0);
        G.zinv.assign(N, 0.0f);

        /* generateVocalTractWalls, TubeGeometry.cu:182-238 */
        int sx = 0 + 1 + 1 + pml;
        int sy = static_cast<int>(std::ceil(G.H / 2.0f)) - 1;
        int ex = sx + t.L - 1;
        G.tube_len = t.L; G.tube_start_x = sx; G.tube_end_x = ex; G.tube_mid_y = sy;
        /* cumulative section lengths: the reference uses a device
         * thrust::inclusive_scan; restated as a sequential float sum, and the
         * margin of every comparison is recorded so tests can show that no
         * summation order changes a decision. */
        std::vector<float> cum(t.len_m.size());
        std::vector<double> cumd(t.len_m.size());
        {
            float acc = 0; double accd = 0;
            for (size_t i = 0; i < t.len_m.size(); i++) {
                acc = acc + t.len_m[i]; accd += (double)t.len_m[i];
                cum[i] = acc; cumd[i] = accd;
            }
        }
        t.upper.assign(t.L, 0); t.lower.assign(t.L, 0);
        int nseg = (int)t.len_m.size();
        for (int idx = 0; idx < t.L; idx++) {
            int counter = idx + 1;
            float curr_len = counter * k.ds;
            float half = k.ds * 0.5f;
            int seg = 0;
            while (seg < nseg - 1 && curr_len > cum[seg] + half) {
                ++seg;
            }
            for (int s2 = 0; s2 < nseg - 1; s2++) {
                double m = std::fabs((double)curr_len - (cumd[s2] + (double)half)) / cumd[s2];
                if (m < G.scan_margin) G.scan_margin = m;
            }
            int radius = (t.diam_cells[seg] - 1) / 2;
            int x = sx + idx;
            int yu = sy - radius - 1, yd = sy + radius + 1;
            t.upper[idx] = yu; t.lower[idx] = yd;
            if (yu < 0 || yd >= G.H) throw OracleError{VS_ERR_GEOMETRY, "wall outside frame"};
            G.type[(size_t)yu * G.W + x] = VS_CELL_WALL;
            G.type[(size_t)yd * G.W + x] = VS_CELL_WALL;
            G.bst[(size_t)yu * G.W + x] = seg + 1;
            G.bst[(size_t)yd * G.W + x] = seg + 1;
        }
        /* connectSagittalWallsGap, TubeGeometry.cu:496-569 (one thread, in order) */
        auto colmax = [&](int col) {
            int m = 0;
            for (int y = 0; y < G.H; ++y) m = std::max(m, G.bst[(size_t)y * G.W + col]);
            return m;
        };
        {
            int pu = t.upper[0], pux = sx, pl = t.lower[0], plx = sx;
            for (int c = 1; c <= t.L - 2; c++) {
                int cu = t.upper[c], cux = sx + c, cl = t.lower[c], clx = sx + c;
                int diff = cu - pu;
                if (diff > 1) {
                    int sgu = colmax(cux);
                    for (int w = pu; w <= cu; w++) {
                        G.type[(size_t)w * G.W + cux] = VS_CELL_WALL;
                        G.bst[(size_t)w * G.W + cux] = sgu;
                    }
                    for (int w = cl; w <= pl; w++) {
                        G.type[(size_t)w * G.W + clx] = VS_CELL_WALL;
                        G.bst[(size_t)w * G.W + clx] = sgu;
                    }
                } else if (diff < -1) {
                    int sgd = colmax(pux);
                    for (int w = cu; w <= pu; w++) {
                        G.type[(size_t)w * G.W + pux] = VS_CELL_WALL;
                        G.bst[(size_t)w * G.W + pux] = sgd;
                    }
                    for (int w = pl; w <= cl; w++) {
                        G.type[(size_t)w * G.W + plx] = VS_CELL_WALL;
                        G.bst[(size_t)w * G.W + plx] = sgd;
                    }
                }
                pu = cu; pux = cux; pl = cl; plx = clx;
            }
        }
        /* setExcitationCells, TubeGeometry.cu:571-594 (walls get no segment id) */
        {
            int col = sx - 1;
            for (int r = t.upper[0] + 1; r < t.lower[0]; r++)
                G.type[(size_t)r * G.W + col] = VS_CELL_EXCITATION;
            G.type[(size_t)t.upper[0] * G.W + col] = VS_CELL_WALL;
            G.type[(size_t)t.lower[0] * G.W + col] = VS_CELL_WALL;
        }
        /* listener / excitation, FDTDSolver.cu:591-611 */
        if (p->mouth_radiation_cond) {
            int col = ex + 1;  /* setNoPressureCells, TubeGeometry.cu:596-612 */
            for (int r = t.upper[t.L - 1]; r <= t.lower[t.L - 1]; r++)
                G.type[(size_t)r * G.W + col] = VS_CELL_NOPRESSURE;
            G.listenerX = ex - t.mic_cells;
            G.listenerY = sy;
        } else {
            G.listenerX = ex + 3 + t.mic_cells;
            G.listenerY = sy;
        }
        G.excX = sx - 1;
        G.excY = G.listenerY;

        /* z_inv, FDTDSolver.cu:613-622 and setZInverse :1058-1070 */
        float mu_3D = p->mu3d > 0.0f ? p->mu3d : (p->fdtd_solver_type == 1 ? 0.025f : 0.005f);
        float mu_2D = (float)((double)mu_3D * (((double)(2.0f * 0.5F) * K_PI) / (double)1.84f));
        float alpha = 1.0f / (0.5f + 0.25f * (mu_2D + (1 / mu_2D)));
        float sq = sqrtf(1 - alpha);
        G.zinv_val = 1 / (k.rho * k.sound_speed * ((1 + sq) / (1 - sq)));
        for (size_t i = 0; i < N; i++) if (G.bst[i] != 0) G.zinv[i] = G.zinv_val;

        /* depth, FDTDSolver.cu:627-641 */
        G.dP.assign(N, 1.0f); G.dX.assign(N, 1.0f); G.dY.assign(N, 1.0f);
        if (p->fdtd_solver_type == 1 && p->cross_sectional_shape != 3) {
            /* TubeDepth::setTubeDepth, TubeDepth.cu:95-169 */
            const float min_depth = 0.001f;
            float osd = (float)(1.0 * open_space_depth);
            std::fill(G.dP.begin(), G.dP.end(), osd);
            std::fill(G.dX.begin(), G.dX.end(), osd);
            std::fill(G.dY.begin(), G.dY.end(), osd);
            const float ds = k.ds;
            for (int tid = 0; tid < t.L; tid++) {
                int uw = t.upper[tid], lw = t.lower[tid];
                int posX = sx + tid;
                int air = lw - uw - 1;
                int half = (int)std::ceil(air * 0.5f) - 1;
                float ra2 = 0, sma2 = 0, smi2 = 0;
                if (p->cross_sectional_shape == 1) {
                    /* generateTubeDepthCircularShape, TubeDepth.cu:313-391 */
                    float radius = (static_cast<float>(air) / 2.0f) * ds;
                    ra2 = radius * radius;
                } else {
                    /* generateTubeDepthEllipticalShape, TubeDepth.cu:392-490 */
                    int mseg = colmax(posX);
                    if (mseg < 1) throw OracleError{VS_ERR_GEOMETRY, "column without segment id"};
                    float sma = (air * ds) / 2.0f;
                    float smi = t.minor_m[mseg - 1] / 2.0f;
                    sma2 = sma * sma;
                    smi2 = smi * smi;
                }
                for (int cc = half; cc >= 0; cc--) {
                    int pu = uw + (half - cc) + 1;
                    int pl = lw - (half - cc) - 1;
                    float distance = static_cast<float>(cc) * ds;
                    float dlo = (static_cast<float>(cc) - 0.5f) * ds;
                    float dup = (static_cast<float>(cc) + 0.5f) * ds;
                    float rX, rLo, rUp = 0.0f;
                    if (p->cross_sectional_shape == 1) {
                        if (p->depth_fma) {
                            rX = std::fma(-distance, distance, ra2);
                            rLo = std::fma(-dlo, dlo, ra2);
                            if (cc != half) rUp = std::fma(-dup, dup, ra2);
                        } else {
                            float sx2 = distance * distance;
                            rX = ra2 - sx2;
                            float slo = dlo * dlo, sup = dup * dup;
                            rLo = ra2 - slo;
                            if (cc != half) rUp = ra2 - sup;
                        }
                    } else {
                        float sx2 = distance * distance;
                        rX = smi2 * (1.0f - (sx2 / sma2));
                        float slo = dlo * dlo, sup = dup * dup;
                        rLo = smi2 * (1 - (slo / sma2));
                        if (cc != half) rUp = smi2 * (1 - (sup / sma2));
                    }
                    if (rX < 0.f || rLo < 0.f || rUp < 0.f)
                        throw OracleError{VS_ERR_NEGATIVE_SQRT, "negative depth radicand"};
                    float dXv = (float)std::sqrt(rX);
                    float dLo = (float)std::sqrt(rLo);
                    float dUp = (float)std::sqrt(rUp);
                    float vX = 2 * dXv, vUp = 2 * dUp, vLo = 2 * dLo;
                    if (p->uniform_depth_m > 0.0f) {
                        vX = p->uniform_depth_m;
                        vLo = p->uniform_depth_m;
                        vUp = (cc != half) ? p->uniform_depth_m : 0.0f;
                    }
                    G.dX[(size_t)pu * G.W + posX] = vX;
                    G.dX[(size_t)pl * G.W + posX] = vX;
                    G.dY[(size_t)pu * G.W + posX] = vUp;
                    G.dY[(size_t)pl * G.W + posX] = vLo;
                }
                G.dX[(size_t)uw * G.W + posX] = 0;
                G.dX[(size_t)lw * G.W + posX] = 0;
                G.dY[(size_t)uw * G.W + posX] = 0;
                G.dY[(size_t)lw * G.W + posX] = 0;
            }
            /* generateDepthP, TubeDepth.cu:215-253 */
            const int H = G.H, W = G.W;
            size_t mid = (size_t)sy * W + ex;
            {   /* resetOpenSpaceDepth :642-662 */
                float mx = G.dX[mid], my = G.dY[mid];
                for (size_t i = 0; i < N; i++) {
                    if (G.dX[i] == osd) G.dX[i] = mx;
                    if (G.dY[i] == osd) G.dY[i] = my;
                }
            }
            std::vector<float> tx(N), ty(N);
            for (size_t i = 0; i < N; i++) {   /* smoothDepthX :665-687 */
                int col = (int)(i % W);
                float o = G.dX[i];
                float r = (col < W - 1) ? G.dX[i + 1] : G.dX[mid];
                tx[i] = 0.5f * (o + r);
            }
            for (size_t i = 0; i < N; i++) {   /* smoothDepthY :690-712 */
                int row = (int)(i / W);
                float o = G.dY[i];
                float a = (row > 0) ? G.dY[i - W] : G.dY[mid];
                ty[i] = 0.5f * (o + a);
            }
            G.dX.swap(tx); G.dY.swap(ty);
            {   /* updateDepthP :714-748 */
                float px = G.dX[mid], py = G.dY[mid];
                for (size_t i = 0; i < N; i++) {
                    int row = (int)(i / W), col = (int)(i % W);
                    float cX = G.dX[i], cY = G.dY[i];
                    float lX = (col > 0) ? G.dX[(size_t)row * W + (col - 1)] : px;
                    float dY = (row < H - 1) ? G.dY[(size_t)(row + 1) * W + col] : py;
                    G.dP[i] = 0.25f * (cX + cY + lX + dY);
                }
            }
            for (size_t i = 0; i < N; i++) {   /* setMinDepthVals :750-762 */
                if (G.dP[i] < min_depth) G.dP[i] = min_depth;
                if (G.dX[i] < min_depth) G.dX[i] = min_depth;
                if (G.dY[i] < min_depth) G.dY[i] = min_depth;
            }
        }
    }

    /* setupDeadCells, FDTDSolver.cu:816-835 (without its one-past-end write) */
    for (int r = 0; r < G.H; r++)
        for (int c = 0; c < G.W; c++)
            if (r == 0 || r == G.H - 1 || c == 0 || c == G.W - 1)
                G.type[(size_t)r * G.W + c] = VS_CELL_DEAD;
    /* PML rings, FDTDSolver.cu:373-464: rows first, then columns */
    if (p->pml_flag == 1) {
        int t = VS_CELL_PML5, x0 = 1, x1 = G.W - 2;
        for (int k2 = 0; k2 < k.pml_layers; k2++) {
            int ru = 1 + k2, rl = G.H - 1 - 1 - k2;
            for (int c = x0; c <= x1; c++) {
                G.type[(size_t)ru * G.W + c] = t;
                G.type[(size_t)rl * G.W + c] = t;
            }
            x0++; x1--; t--;
        }
        t = VS_CELL_PML5;
        int y0 = 1, y1 = G.H - 2;
        for (int k2 = 0; k2 < k.pml_layers; k2++) {
            int cl = 1 + k2, cr = G.W - 1 - 1 - k2;
            for (int r = y0; r <= y1; r++) {
                G.type[(size_t)r * G.W + cl] = t;
                G.type[(size_t)r * G.W + cr] = t;
            }
            y0++; y1--; t--;
        }
    }
    if (p->listener_mode == VS_LISTENER_EXPLICIT) {
        G.listenerX = p->listener_x;
        G.listenerY = p->listener_y;
    }
    if (G.listenerX < 0 || G.listenerX >= G.W || G.listenerY < 0 || G.listenerY >= G.H)
        throw OracleError{VS_ERR_INVALID_ARG, "listener outside the frame"};
}

/* ---- calculateSolverCoefficients, FDTDSolver.cu:652-801,860-1056 --------- */
struct Coeffs {
    std::vector<float> N_out, N_in, minVxB, minVyB, maxVxS, maxVyS, bX, bY, pS,
        notX, notY, ewX, ewY, x1, x2, x3, x4;
};

int beta_lut(int br, int bt) {
    if (br == VS_CELL_AIR && bt == VS_CELL_AIR) return 0;
    if (br == VS_CELL_AIR && bt == VS_CELL_WALL) return 1;
    if (br == VS_CELL_WALL && bt == VS_CELL_AIR) return 2;
    if (br == VS_CELL_WALL && bt == VS_CELL_WALL) return 3;
    return -1;
}

void build_coeffs(const Grid& G, Coeffs& C) {
    const float airN[4] = {0, 1.0f, 1.0f, 0.707106f};
    const float wallN[4] = {1.0f, 1.0f, 1.0f, 0};
    int ir = G.H - 2, ic = G.W - 2;
    size_t n = (size_t)ir * ic;
    std::vector<float>* all[] = {&C.N_out, &C.N_in, &C.minVxB, &C.minVyB, &C.maxVxS, &C.maxVyS,
                                 &C.bX, &C.bY, &C.pS, &C.notX, &C.notY, &C.ewX, &C.ewY,
                                 &C.x1, &C.x2, &C.x3, &C.x4};
    for (auto* v : all) v->assign(n, 0.0f);
    const float dt = G.k.dt, rho = G.k.rho, ds = G.k.ds;
    for (size_t tid = 0; tid < n; tid++) {
        int col = (int)(tid % ic) + 1, row = (int)(tid / ic) + 1;
        int tc = G.type[(size_t)row * G.W + col];
        int tr = G.type[(size_t)row * G.W + col + 1];
        int tt = G.type[(size_t)(row - 1) * G.W + col];
        float bc = G.beta[tc], br = G.beta[tr], bt = G.beta[tt];
        int lut = beta_lut((int)br, (int)bt);
        if (lut < 0) lut = 0;  /* unreachable: beta is 0 or 1 */
        C.N_out[tid] = airN[lut] * bc;
        C.N_in[tid] = wallN[lut] * (1 - bc);
        float sc = G.sigma[tc], sr = G.sigma[tr], st = G.sigma[tt];
        int ec = tc == VS_CELL_EXCITATION, er = tr == VS_CELL_EXCITATION,
            et = tt == VS_CELL_EXCITATION;
        C.minVxB[tid] = std::min(bc, br);
        C.minVyB[tid] = std::min(bc, bt);
        C.maxVxS[tid] = std::max(sc, sr);
        C.maxVyS[tid] = std::max(sc, st);
        float bxs = C.minVxB[tid] * C.minVxB[tid];
        float bys = C.minVyB[tid] * C.minVyB[tid];
        C.bX[tid] = (bxs * dt) / (rho * ds);
        C.bY[tid] = (bys * dt) / (rho * ds);
        C.pS[tid] = sc;
        C.notX[tid] = (float)((1 - ec) * (1 - er));
        C.notY[tid] = (float)((1 - ec) * (1 - et));
        C.ewX[tid] = (ec * G.dir[2]) + (er * G.dir[0]);
        C.ewY[tid] = (ec * G.dir[3]) + (et * G.dir[1]);
        C.x1[tid] = br * (1 - bc);
        C.x2[tid] = bc * (1 - br);
        C.x3[tid] = bt * (1 - bc);
        C.x4[tid] = bc * (1 - bt);
    }
}

/* ---- GlottalExcitations::setExcitationVelocity, GlottalExcitations.cu:9-52 */
template <typename T>
void source_table(const vs_params* p, long long n, double dt, std::vector<T>& out) {
    out.assign((size_t)n, T(0));
    switch (p->source_type) {
    case VS_SRC_SINE:
        for (long long i = 0; i < n; i++) {
            if (sizeof(T) == 4) {
                float t = (float)(i * dt);
                out[i] = (T)(float)((double)p->sine_amp *
                                    std::sin(2 * K_PI * (double)p->sine_freq_hz * (double)t));
            } else {
                double t = i * dt;
                out[i] = (T)((double)p->sine_amp * std::sin(2 * K_PI * (double)p->sine_freq_hz * t));
            }
        }
        break;
    case VS_SRC_GAUSS:
    case VS_SRC_GAUSS_STD:
        for (long long i = 0; i < n; i++) {
            if (sizeof(T) == 4) {
                float t = (float)(i * dt);
                float e = (t - p->gauss_peak_s) / p->gauss_width_s;
                float sq = e * e;
                float arg = p->source_type == VS_SRC_GAUSS ? -1 * sq : -0.5f * sq;
                out[i] = (T)(p->gauss_amp * expf(arg));
            } else {
                double t = i * dt;
                double e = (t - (double)p->gauss_peak_s) / (double)p->gauss_width_s;
                double arg = p->source_type == VS_SRC_GAUSS ? -e * e : -0.5 * e * e;
                out[i] = (T)((double)p->gauss_amp * std::exp(arg));
            }
        }
        break;
    case VS_SRC_TMM:
        break;
    default:
        throw OracleError{VS_ERR_INVALID_ARG, "source_type"};
    }
}

/* ---- TwoMassModel, TwoMassModel.cpp:4-232 --------------------------------
 * The template keeps the reference's mixed precision for T = float: double
 * literals (1.37, 0.5, 0.37) promote those sub-expressions to double exactly
 * as in the reference; for T = double everything is double. */
template <typename T>
struct TwoMass {
    T mu, rho, q, gs, m1, m2, d1, d2, k1, k2, kc, etak1, etak2, h1, h2, etah1, etah2;
    T Ag0, Ag01, Ag02, lg, z1o, z2o, z1c, z2c, r1o, r2o, r1c, r2c, A1, Ag1, Ag2, ps, p1;
    T fm1, fm2, pm1, pm2, Rv1, Rv2, Lg1, Lg2;
    T ug_old, ug_curr, ug_next, x1_old, x1_curr, x1_next, x2_old, x2_curr, x2_next;
    T a11, a12, a21, a22, b1, b2, s1, s2;

    void init(float ps_pa) {
        mu = (T)(1.86e-4 * (double)(U_DYN * U_SECOND / (U_CENTIMETER * U_CENTIMETER)));
        rho = (T)(1.14 * (double)(U_KILOGRAM / (U_METER * U_METER * U_METER)));
        q = 1.0f; gs = 1.0f;
        m1 = ((T)0.125f * (T)U_GRAM) / q;
        m2 = ((T)0.025f * (T)U_GRAM) / q;
        d1 = ((T)0.25f * (T)U_CENTIMETER) / q;
        d2 = ((T)0.05f * (T)U_CENTIMETER) / q;
        k1 = (T)80000.0f * ((T)U_DYN / (T)U_CENTIMETER) * q;
        k2 = (T)8000.0f * ((T)U_DYN / (T)U_CENTIMETER) * q;
        kc = (T)25000.0f * ((T)U_DYN / (T)U_CENTIMETER) * (q * q);
        etak1 = 100 / ((T)U_CENTIMETER * (T)U_CENTIMETER);
        etak2 = 100 / ((T)U_CENTIMETER * (T)U_CENTIMETER);
        h1 = 3 * k1; h2 = 3 * k2;
        etah1 = (T)500.0f / ((T)U_CENTIMETER * (T)U_CENTIMETER);
        etah2 = (T)500.0f / ((T)U_CENTIMETER * (T)U_CENTIMETER);
        Ag0 = (T)0.05f * ((T)U_CENTIMETER * (T)U_CENTIMETER);
        Ag01 = Ag0; Ag02 = Ag0;
        lg = (T)1.40f * (T)U_CENTIMETER;
        z1o = (T)0.2f; z2o = (T)0.6f; z1c = (T)1.1f; z2c = (T)1.9f;
        r1o = (2 * z1o * std::sqrt(k1 * m1)) / (gs * gs);
        r2o = (2 * z2o * std::sqrt(k2 * m2)) / (gs * gs);
        r1c = (2 * z1c * std::sqrt(k1 * m1)) / (gs * gs);
        r2c = (2 * z2c * std::sqrt(k2 * m2)) / (gs * gs);
        A1 = (T)3.0f * ((T)U_CENTIMETER * (T)U_CENTIMETER);
        Ag1 = 0; Ag2 = 0;
        ps = (T)ps_pa;
        p1 = 0; fm1 = 0; fm2 = 0; pm1 = 0; pm2 = 0; Rv1 = 0; Rv2 = 0; Lg1 = 0; Lg2 = 0;
        ug_old = 0; ug_curr = 0; ug_next = 0;
        x1_old = 0; x1_curr = 0; x1_next = 0; x2_old = 0; x2_curr = 0; x2_next = 0;
        a11 = 0; a12 = 0; a21 = 0; a22 = 0; b1 = 0; b2 = 0; s1 = 0; s2 = 0;
    }

    void step(int srate_mul) {
        T srate = 44100 * static_cast<T>(srate_mul);
        Ag1 = Ag01 + 2 * lg * x1_curr;
        Ag2 = Ag02 + 2 * lg * x2_curr;
        Rv1 = (12 * mu * lg * lg * d1) / (Ag1 * Ag1 * Ag1);
        Lg1 = (rho * d1) / (Ag1);
        Rv2 = (12 * mu * lg * lg * d2) / (Ag2 * Ag2 * Ag2);
        Lg2 = (rho * d2) / (Ag2);
        if (x1_curr > -Ag01 / (2 * lg) && x2_curr > -Ag02 / (2 * lg)) {
            pm1 = (T)(ps - 1.37 * (rho / 2) * (ug_curr / Ag1) * (ug_curr / Ag1) -
                      0.5 * (Rv1 * ug_curr + Lg1 * srate * (ug_curr - ug_old)));
            fm1 = pm1 * d1 * lg;
        } else {
            pm1 = ps;
            fm1 = pm1 * d1 * lg;
        }
        if (x1_curr > -Ag01 / (2 * lg)) {
            if (x2_curr > -Ag02 / (2 * lg)) {
                pm2 = (T)(pm1 - (0.5 * (Rv1 + Rv2) * ug_curr + (Lg1 + Lg2) * (ug_curr - ug_old) * srate) -
                          (rho / 2 * ug_curr * ug_curr) * (1 / (Ag2 * Ag2) - 1 / (Ag1 * Ag1)));
                fm2 = pm2 * d2 * lg;
            } else {
                pm2 = ps;
                fm2 = pm2 * d2 * lg;
            }
        } else {
            pm2 = 0;
            fm2 = pm2 * d2 * lg;
        }
        T h1u, r1u, h2u, r2u;
        if (x1_curr + Ag01 / (2 * lg) < 0) { h1u = h1; r1u = r1c; } else { h1u = 0; r1u = r1o; }
        if (x2_curr + Ag02 / (2 * lg) < 0) { h2u = h2; r2u = r2c; } else { h2u = 0; r2u = r2o; }
        a11 = (k1 + h1u + kc) / (srate * srate) + r1u / srate + m1;
        a12 = -kc / (srate * srate);
        a21 = a12;
        a22 = (k2 + h2u + kc) / (srate * srate) + r2u / srate + m2;
        s1 = k1 * etak1 * x1_curr * x1_curr * x1_curr +
             h1u * (Ag01 / (2 * lg) + etah1 * (Ag01 / (2 * lg) + x1_curr) * (Ag01 / (2 * lg) + x1_curr) *
                                          (Ag01 / (2 * lg) + x1_curr));
        s2 = k2 * etak2 * x2_curr * x2_curr * x2_curr +
             h2u * (Ag02 / (2 * lg) + etah2 * (Ag02 / (2 * lg) + x2_curr) * (Ag02 / (2 * lg) + x2_curr) *
                                          (Ag02 / (2 * lg) + x2_curr));
        b1 = (2 * m1 + r1u / srate) * x1_curr - m1 * x1_old - s1 / (srate * srate) + fm1 / (srate * srate);
        b2 = (2 * m2 + r2u / srate) * x2_curr - m2 * x2_old - s2 / (srate * srate) + fm2 / (srate * srate);
        T det = a11 * a22 - a21 * a12;
        if (det == 0) det = 1;
        x1_next = (a22 * b1 - a12 * b2) / det;
        x2_next = (a11 * b2 - a21 * b1) / det;
        x1_old = x1_curr; x1_curr = x1_next;
        x2_old = x2_curr; x2_curr = x2_next;
        Ag1 = Ag01 + 2 * lg * x1_curr;
        Ag2 = Ag02 + 2 * lg * x2_curr;
        if (Ag1 < 0 || Ag2 < 0) {
            ug_next = 0;
        } else {
            /* TwoMassModel.cpp has no using-directive, so g++/libstdc++ resolve
             * fabs(float) to ::fabs(double): the product (rho/2)*|ug| is
             * formed in double.  This matches the reference compiled here. */
            T Rtot = (T)((rho / 2) * std::fabs((double)ug_curr) *
                             ((0.37 / (Ag1 * Ag1)) + (1 - 2 * (Ag2 / A1) * (1 - Ag2 / A1)) / (Ag2 * Ag2)) +
                         (12 * mu * lg * lg * (d1 / (Ag1 * Ag1 * Ag1) + d2 / (Ag2 * Ag2 * Ag2))));
            T Ltot = rho * (d1 / Ag1 + d2 / Ag2);
            ug_next = ((ps - p1) / srate + Ltot * ug_curr) / (Rtot / srate + Ltot);
        }
        ug_old = ug_curr;
        ug_curr = ug_next;
    }
};

/* ---- the double two-mass model of the tmm_f64 option ------------------------
 * The model of TwoMassModel.cpp:90-232 in double, arranged to divide only by
 * the glottal openings (before and after the displacement update) and by the
 * flow denominator: the per-model constants below (reciprocals of the sample
 * rate, the thresholds, the displacement-update matrix and its inverse
 * determinant per contact state) are formed once.  This is the arrangement
 * the GPU's tmm_f64 model uses, operation for operation, so the FP32 engine
 * with tmm_f64 pins it bit for bit; TwoMass<double> (the literal expressions)
 * stays the FP64 engine's model, the accuracy reference. */
struct TwoMassR {
    TwoMass<double> k;                    /* primaries and state */
    double isr, is2, two_lg, g1, g2, c12, cR1, cR2, cL1, cL2, hr, hr137, d1lg, d2lg, iA1, k1e, k2e;
    double a11[2], a22[2], a12, b1c[2], b2c[2], idet[2][2];
    double srate;

    void init(float ps_pa, int srate_mul) {
        k.init(ps_pa);
        srate = 44100 * static_cast<double>(srate_mul);
        isr = 1.0 / srate;
        is2 = isr * isr;
        two_lg = 2.0 * k.lg;
        g1 = k.Ag01 / two_lg;
        g2 = k.Ag02 / two_lg;
        c12 = 12.0 * k.mu * k.lg * k.lg;
        cR1 = c12 * k.d1;
        cR2 = c12 * k.d2;
        cL1 = k.rho * k.d1;
        cL2 = k.rho * k.d2;
        hr = k.rho / 2.0;
        hr137 = 1.37 * hr;
        d1lg = k.d1 * k.lg;
        d2lg = k.d2 * k.lg;
        iA1 = 1.0 / k.A1;
        k1e = k.k1 * k.etak1;
        k2e = k.k2 * k.etak2;
        for (int c = 0; c < 2; c++) {
            const double h1u = c ? k.h1 : 0.0, r1u = c ? k.r1c : k.r1o;
            const double h2u = c ? k.h2 : 0.0, r2u = c ? k.r2c : k.r2o;
            a11[c] = (k.k1 + h1u + k.kc) * is2 + r1u * isr + k.m1;
            a22[c] = (k.k2 + h2u + k.kc) * is2 + r2u * isr + k.m2;
            b1c[c] = 2.0 * k.m1 + r1u * isr;
            b2c[c] = 2.0 * k.m2 + r2u * isr;
        }
        a12 = -k.kc * is2;
        for (int c1 = 0; c1 < 2; c1++)
            for (int c2 = 0; c2 < 2; c2++) {
                double det = a11[c1] * a22[c2] - a12 * a12;
                if (det == 0.0) det = 1.0;
                idet[c1][c2] = 1.0 / det;
            }
    }

    /* one step with supraglottal pressure p1; returns the new flow */
    double step(double p1) {
        const double x1c = k.x1_curr, x2c = k.x2_curr, ug = k.ug_curr, ugo = k.ug_old;
        const double ia1 = 1.0 / (k.Ag01 + two_lg * x1c);
        const double ia2 = 1.0 / (k.Ag02 + two_lg * x2c);
        const double ia1s = ia1 * ia1, ia2s = ia2 * ia2;
        const double Rv1 = cR1 * (ia1s * ia1), Lg1 = cL1 * ia1;
        const double Rv2 = cR2 * (ia2s * ia2), Lg2 = cL2 * ia2;
        const double dug = ug - ugo;
        const bool open1 = x1c > -g1, open2 = x2c > -g2;
        double pm1 = k.ps;
        if (open1 && open2) {
            const double q = ug * ia1;
            pm1 = k.ps - hr137 * (q * q) - 0.5 * (Rv1 * ug + srate * (Lg1 * dug));
        }
        const double fm1 = d1lg * pm1;
        double pm2 = 0.0;
        if (open1) {
            if (open2)
                pm2 = pm1 - (0.5 * (Rv1 + Rv2) * ug + srate * ((Lg1 + Lg2) * dug)) - hr * (ug * ug) * (ia2s - ia1s);
            else
                pm2 = k.ps;
        }
        const double fm2 = d2lg * pm2;
        const int c1 = x1c + g1 < 0.0, c2 = x2c + g2 < 0.0;
        const double e1 = g1 + x1c, e2 = g2 + x2c;
        const double s1 = k1e * (x1c * x1c * x1c) + (c1 ? k.h1 : 0.0) * (g1 + k.etah1 * (e1 * e1 * e1));
        const double s2 = k2e * (x2c * x2c * x2c) + (c2 ? k.h2 : 0.0) * (g2 + k.etah2 * (e2 * e2 * e2));
        const double b1 = b1c[c1] * x1c - k.m1 * k.x1_old + (fm1 - s1) * is2;
        const double b2 = b2c[c2] * x2c - k.m2 * k.x2_old + (fm2 - s2) * is2;
        const double id = idet[c1][c2];
        const double x1n = (a22[c2] * b1 - a12 * b2) * id;
        const double x2n = (a11[c1] * b2 - a12 * b1) * id;
        const double Ag1 = k.Ag01 + two_lg * x1n;
        const double Ag2 = k.Ag02 + two_lg * x2n;
        double ugn = 0.0;
        if (!(Ag1 < 0 || Ag2 < 0)) {
            const double ja1 = 1.0 / Ag1, ja2 = 1.0 / Ag2;
            const double ja1s = ja1 * ja1, ja2s = ja2 * ja2;
            const double r = Ag2 * iA1;
            const double Rtot = hr * std::fabs(ug) * (0.37 * ja1s + (1.0 - 2.0 * r * (1.0 - r)) * ja2s) +
                                c12 * (k.d1 * (ja1s * ja1) + k.d2 * (ja2s * ja2));
            const double Ltot = cL1 * ja1 + cL2 * ja2;
            ugn = ((k.ps - p1) * isr + Ltot * ug) / (Rtot * isr + Ltot);
        }
        k.x1_old = x1c; k.x1_curr = x1n;
        k.x2_old = x2c; k.x2_curr = x2n;
        k.ug_old = ug; k.ug_curr = ugn;
        return ugn;
    }
};

/* ---- the time loop ---------------------------------------------------------
 * FDTDEngineCPU::startSolverEngine (FDTDEngineCPU.cpp:222-304) with its three
 * passes (:306-433), the full-frame wall ODE and the PV_N = PV_Nplus1 copy.
 * engine == VS_ENGINE_EIGEN switches the one expression that FDTDEngineEigen
 * rounds differently (FDTDEngineEigen.cpp:251). */
template <typename T>
struct Cell { T Pr, Vx, Vy; int cell_type; };

template <typename T>
int run_engine(const vs_params* p, const Grid& G, const Coeffs& C, long long steps,
               T* trace, T* outP, T* outVx, T* outVy,
               const std::vector<double>* ovP = nullptr, const std::vector<double>* ovX = nullptr,
               const std::vector<double>* ovY = nullptr, const std::vector<double>* ovZ = nullptr) {
    const int H = G.H, W = G.W, ir = H - 2, ic = W - 2;
    const size_t N = (size_t)H * W;
    std::vector<Cell<T>> PN(N), PN1(N);
    for (size_t i = 0; i < N; i++) { PN[i] = {T(0), T(0), T(0), G.type[i]}; }
    PN1 = PN;
    std::vector<T> dP(N), dX(N), dY(N), zinv(N);
    for (size_t i = 0; i < N; i++) { dP[i] = G.dP[i]; dX[i] = G.dX[i]; dY[i] = G.dY[i]; zinv[i] = G.zinv[i]; }
    if (ovP) for (size_t i = 0; i < N; i++) dP[i] = (T)(*ovP)[i];
    if (ovX) for (size_t i = 0; i < N; i++) dX[i] = (T)(*ovX)[i];
    if (ovY) for (size_t i = 0; i < N; i++) dY[i] = (T)(*ovY)[i];
    if (ovZ) for (size_t i = 0; i < N; i++) zinv[i] = (T)(*ovZ)[i];
    const size_t n = (size_t)ir * ic;
    auto cv = [&](const std::vector<float>& v) { return std::vector<T>(v.begin(), v.end()); };
    std::vector<T> Nout = cv(C.N_out), Nin = cv(C.N_in), mBx = cv(C.minVxB), mBy = cv(C.minVyB),
                   mSx = cv(C.maxVxS), mSy = cv(C.maxVyS), bX = cv(C.bX), bY = cv(C.bY),
                   pS = cv(C.pS), nX = cv(C.notX), nY = cv(C.notY), ewX = cv(C.ewX),
                   ewY = cv(C.ewY), x1 = cv(C.x1), x2 = cv(C.x2), x3 = cv(C.x3), x4 = cv(C.x4);
    if (sizeof(T) == 8) {
        /* double restatement: derived constants in double from float primaries */
        const double sm = (double)G.k.max_sigma_dt;
        double sig[13];
        for (int i = 0; i < 13; i++) sig[i] = G.sigma[i];
        for (int k2 = 0; k2 < G.k.pml_layers; k2++)
            sig[VS_CELL_PML0 + k2] = ((double)k2 / (double)(G.k.pml_layers - 1)) * sm;
        double bxv = (double)G.k.dt / ((double)G.k.rho * (double)G.k.ds);
        for (size_t tid = 0; tid < n; tid++) {
            int col = (int)(tid % ic) + 1, row = (int)(tid / ic) + 1;
            int tc = G.type[(size_t)row * W + col], tr = G.type[(size_t)row * W + col + 1],
                tt = G.type[(size_t)(row - 1) * W + col];
            pS[tid] = (T)sig[tc];
            mSx[tid] = (T)std::max(sig[tc], sig[tr]);
            mSy[tid] = (T)std::max(sig[tc], sig[tt]);
            bX[tid] = (T)(mBx[tid] * mBx[tid] * bxv);
            bY[tid] = (T)(mBy[tid] * mBy[tid] * bxv);
        }
    }
    std::vector<T> CxVx(n), CyVy(n), CxP(n), CyP(n), VbX(n), VbY(n);
    std::vector<T> w_prev(N, T(0)), w_next(N, T(0)), z_prev(N, T(0)), z_next(N, T(0));
    std::vector<T> src;
    source_table<T>(p, steps, (double)G.k.dt, src);
    TwoMass<T> tmm;
    tmm.init(p->tmm_ps_pa);
    TwoMass<double> tmm64;                /* tmm_f64 with double fields: the literal model in double */
    tmm64.init(p->tmm_ps_pa);
    TwoMassR tmmR;                        /* tmm_f64 with float fields: the GPU's arrangement */
    tmmR.init(p->tmm_ps_pa, p->srate_mul);
    T K1, K2;
    if (sizeof(T) == 4) { K1 = (T)G.K1; K2 = (T)G.K2; }
    else {
        K1 = (T)(((double)G.k.kappa * (double)G.k.dt) / (double)G.k.ds);
        K2 = (T)((double)G.k.kappa * (double)G.k.dt);
    }
    const T dt = (T)G.k.dt, Mw = (T)G.k.Mw, Bw = (T)G.k.Bw, Kw = (T)G.k.Kw, cpl = (T)G.k.cpl;
    const bool eigen = p->engine == VS_ENGINE_EIGEN;
    const bool dirichlet = p->mouth_radiation_cond != 0;
    const bool two5d = p->fdtd_solver_type == 1;
    const size_t lis = (size_t)G.listenerY * W + G.listenerX;
    const size_t exc = (size_t)G.excY * W + G.excX;

    for (long long ts = 0; ts < steps; ts++) {
        T exeV;
        if (p->source_type == VS_SRC_TMM && p->tmm_f64 && sizeof(T) == 4) {
            exeV = (T)tmmR.step((double)PN[exc].Pr);
        } else if (p->source_type == VS_SRC_TMM && p->tmm_f64) {
            tmm64.p1 = (double)PN[exc].Pr;
            tmm64.step(p->srate_mul);
            exeV = (T)tmm64.ug_next;
        } else if (p->source_type == VS_SRC_TMM) {
            tmm.p1 = PN[exc].Pr;
            tmm.step(p->srate_mul);
            exeV = tmm.ug_next;
        } else {
            exeV = src[(size_t)ts];
        }
        std::swap(w_prev, w_next);
        std::swap(z_prev, z_next);
        /* pressure, FDTDEngineCPU.cpp:316-339 */
        for (int r = 0; r < ir; r++) {
            for (int c = 0; c < ic; c++) {
                size_t t = (size_t)r * ic + c;
                size_t cur = (size_t)(r + 1) * W + (c + 1);
                size_t left = (size_t)(r + 1) * W + c;
                size_t down = (size_t)(r + 2) * W + (c + 1);
                CxVx[t] = PN[cur].Vx * dX[cur] - PN[left].Vx * dX[left];
                CyVy[t] = PN[cur].Vy * dY[cur] - PN[down].Vy * dY[down];
                T num = ((PN[cur].Pr * dP[cur]) - (K1 * (CxVx[t] + CyVy[t]))) - (K2 * w_prev[cur]);
                T den = eigen ? (pS[t] * dP[cur] + dP[cur]) : ((1 + pS[t]) * dP[cur]);
                PN1[cur].Pr = num / den;
                if (dirichlet && PN1[cur].cell_type == VS_CELL_NOPRESSURE) PN1[cur].Pr = 0;
            }
        }
        if (trace) trace[ts] = PN1[lis].Pr;
        /* wall ODE over the full frame, FDTDEngineCPU.cpp:345-361 */
        if (two5d) {
            for (size_t i = 0; i < N; i++) {
                z_next[i] = z_prev[i] + w_prev[i] * dt;
                T num = ((Mw * w_prev[i]) + (cpl * dt * PN1[i].Pr)) - (dt * Kw * z_next[i]);
                T den = Mw + (dt * Bw);
                w_next[i] = num / den;
            }
        }
        /* velocity, FDTDEngineCPU.cpp:364-410 */
        for (int r = 0; r < ir; r++) {
            for (int c = 0; c < ic; c++) {
                size_t t = (size_t)r * ic + c;
                size_t cur = (size_t)(r + 1) * W + (c + 1);
                size_t right = (size_t)(r + 1) * W + (c + 2);
                size_t top = (size_t)r * W + (c + 1);
                CxP[t] = PN1[right].Pr - PN1[cur].Pr;
                CyP[t] = PN1[top].Pr - PN1[cur].Pr;
                T vx = (mBx[t] * PN[cur].Vx) - (bX[t] * CxP[t]);
                T vy = (mBy[t] * PN[cur].Vy) - (bY[t] * CyP[t]);
                vx = vx + (exeV * ewX[t] * mSx[t]);
                vy = vy + (exeV * ewY[t] * mSy[t]);
                VbX[t] = (x2[t] * PN1[cur].Pr * Nout[t]) - (x1[t] * PN1[right].Pr * Nin[t]);
                VbY[t] = (x4[t] * PN1[cur].Pr * Nout[t]) - (x3[t] * PN1[top].Pr * Nin[t]);
                VbX[t] = VbX[t] * nX[t] * zinv[cur];
                VbY[t] = VbY[t] * nY[t] * zinv[cur];
                vx += (mSx[t] * VbX[t]);
                vy += (mSy[t] * VbY[t]);
                vx /= (mBx[t] + mSx[t]);
                vy /= (mBy[t] + mSy[t]);
                PN1[cur].Vx = vx;
                PN1[cur].Vy = vy;
            }
        }
        /* update_border_cells, FDTDEngineCPU.cpp:412-433 */
        for (int r = 0; r < H; r++) {
            Cell<T>& a = PN1[(size_t)r * W]; a.Pr = 0; a.Vx = 0; a.Vy = 0;
            Cell<T>& b = PN1[(size_t)r * W + W - 1]; b.Pr = 0; b.Vx = 0; b.Vy = 0;
        }
        for (int c = 0; c < W; c++) {
            Cell<T>& a = PN1[c]; a.Pr = 0; a.Vx = 0; a.Vy = 0;
            Cell<T>& b = PN1[(size_t)(H - 1) * W + c]; b.Pr = 0; b.Vx = 0; b.Vy = 0;
        }
        PN = PN1;
    }
    for (size_t i = 0; i < N; i++) {
        if (outP) outP[i] = PN[i].Pr;
        if (outVx) outVx[i] = PN[i].Vx;
        if (outVy) outVy[i] = PN[i].Vy;
    }
    return VS_OK;
}

int run_engine_maps(const vs_params* p, const Grid& G, const Coeffs& C, long long steps,
                    const std::vector<double>& mP, const std::vector<double>& mX, const std::vector<double>& mY,
                    const std::vector<double>& mZ, double* trace) {
    return run_engine<double>(p, G, C, steps, trace, nullptr, nullptr, nullptr, &mP, &mX, &mY, &mZ);
}

thread_local std::string g_err;

int fail(const OracleError& e) { g_err = e.msg; return e.code; }

void fill_dims(const Grid& G, vs_dims* d) {
    if (!d) return;
    std::memset(d, 0, sizeof(*d));
    d->frame_h = G.H; d->frame_w = G.W;
    d->listener_x = G.listenerX; d->listener_y = G.listenerY;
    d->excitation_x = G.excX; d->excitation_y = G.excY;
    d->tube_length_cells = G.tube_len;
    d->tube_start_x = G.tube_start_x; d->tube_end_x = G.tube_end_x; d->tube_mid_y = G.tube_mid_y;
    d->num_steps = G.num_steps;
    d->interior_cells = (int64_t)(G.H - 2) * (G.W - 2);
    d->dt = G.k.dt; d->ds = G.k.ds; d->z_inv_val = G.zinv_val;
}

}  // namespace

extern "C" {

const char* orc_last_error(void) { return g_err.c_str(); }

/* Diameters (m) of the single-plane-symmetric sections of the next shape-3
   builds (n = 0 clears them). */
int orc_set_sps_diameters(const float* d, int n) {
    g_sps_diameters.assign(d, d + (n > 0 ? n : 0));
    return VS_OK;
}

/* The reference's run configuration: main.cu:160-187 (2.5D, tube, circular,
 * srate_mul 15, Gaussian, 100 ms) with the open mouth and PML on, and the
 * source constants of GlottalExcitations.cu:19-32 / TwoMassModel.cpp:52. */
int orc_params_init(vs_params* p) {
    std::memset(p, 0, sizeof(*p));
    p->fdtd_solver_type = 1;
    p->simulation_type = 1;
    p->cross_sectional_shape = 1;
    p->mouth_radiation_cond = 0;
    p->srate_mul = 15;
    p->source_type = VS_SRC_GAUSS;
    p->pml_flag = 1;
    p->engine = VS_ENGINE_CPU;
    p->audio_dur = 100 * U_MILLISECOND;
    p->num_steps = 0;
    float f0 = 10.0f * U_KILOHERTZ;
    p->gauss_peak_s = 0.646f / f0;
    p->gauss_width_s = 0.29f * p->gauss_peak_s;
    p->gauss_amp = 0.025f;
    p->sine_freq_hz = 440 * U_HERTZ;
    p->sine_amp = 25;
    p->tmm_ps_pa = 686.46f;
    p->mu3d = 0.0f;
    p->wall_coupling = 0.0f;
    p->uniform_depth_m = 0.0f;
    p->depth_fma = 1;
    p->listener_mode = VS_LISTENER_REFERENCE;
    return VS_OK;
}

/* Grid dims + the frame maps (any pointer may be NULL).  bst is the
 * reference's boundary_segment_type map. */
int orc_maps(const vs_params* p, const vs_geometry* g, vs_dims* dims, int32_t* cell_type,
             int32_t* bst, float* dP, float* dX, float* dY, float* zinv, double* scan_margin) {
    try {
        Grid G;
        build_grid(p, g, G);
        fill_dims(G, dims);
        size_t N = (size_t)G.H * G.W;
        for (size_t i = 0; i < N; i++) {
            if (cell_type) cell_type[i] = G.type[i];
            if (bst) bst[i] = G.bst[i];
            if (dP) dP[i] = G.dP[i];
            if (dX) dX[i] = G.dX[i];
            if (dY) dY[i] = G.dY[i];
            if (zinv) zinv[i] = G.zinv[i];
        }
        if (scan_margin) *scan_margin = G.scan_margin;
        return VS_OK;
    } catch (const OracleError& e) { return fail(e); }
}

/* The 17 interior coefficient arrays of calculateSolverCoefficients, packed
 * as out[k * interior + i] in this order: N_out, N_in, minVxBeta, minVyBeta,
 * maxVxSigmaPrimedt, maxVySigmaPrimedt, betaVxSqr_dt_inv_rho_inv_ds,
 * betaVySqr_dt_inv_rho_inv_ds, pressureSigmaPrimedt, areWeNotExcitationVx,
 * areWeNotExcitationVy, excitationWeightVx, excitationWeightVy, xor_val1..4. */
int orc_coeffs(const vs_params* p, const vs_geometry* g, float* out) {
    try {
        Grid G;
        build_grid(p, g, G);
        Coeffs C;
        build_coeffs(G, C);
        const std::vector<float>* all[] = {&C.N_out, &C.N_in, &C.minVxB, &C.minVyB, &C.maxVxS,
                                           &C.maxVyS, &C.bX, &C.bY, &C.pS, &C.notX, &C.notY,
                                           &C.ewX, &C.ewY, &C.x1, &C.x2, &C.x3, &C.x4};
        size_t n = C.N_out.size();
        for (int k2 = 0; k2 < 17; k2++)
            std::memcpy(out + (size_t)k2 * n, all[k2]->data(), n * sizeof(float));
        return VS_OK;
    } catch (const OracleError& e) { return fail(e); }
}

/* Physical constants of SimulationParams(srate_mul) and the derived solver
 * constants: out = {c, rho, kappa, dt, ds, max_sigma_dt, K1, K2, Mw, Bw, Kw}. */
int orc_consts(int srate_mul, float* out) {
    PhysConsts k = phys_consts(srate_mul);
    out[0] = k.sound_speed; out[1] = k.rho; out[2] = k.kappa; out[3] = k.dt; out[4] = k.ds;
    out[5] = k.max_sigma_dt; out[6] = (k.kappa * k.dt) / k.ds; out[7] = k.kappa * k.dt;
    out[8] = k.Mw; out[9] = k.Bw; out[10] = k.Kw;
    return VS_OK;
}

/* beta[13], sigma_prime_dt[13], source_direction[4] of SolverParams. */
int orc_tables(int srate_mul, float* beta, float* sigma, float* dir) {
    PhysConsts k = phys_consts(srate_mul);
    solver_tables(k.pml_layers, k.max_sigma_dt, k.dt, beta, sigma, dir);
    return VS_OK;
}

long long orc_step_count(float audio_time, float dt) { return reference_step_count(audio_time, dt); }

int orc_source_f32(const vs_params* p, long long n, float* out) {
    try {
        PhysConsts k = phys_consts(p->srate_mul);
        std::vector<float> v;
        source_table<float>(p, n, (double)k.dt, v);
        std::memcpy(out, v.data(), (size_t)n * sizeof(float));
        return VS_OK;
    } catch (const OracleError& e) { return fail(e); }
}

/* Two-mass model driven by a given supraglottal pressure sequence. */
int orc_tmm_f32(float ps, int srate_mul, const float* p1, long long n, float* ug) {
    TwoMass<float> m;
    m.init(ps);
    for (long long i = 0; i < n; i++) { m.p1 = p1[i]; m.step(srate_mul); ug[i] = m.ug_next; }
    return VS_OK;
}

int orc_tmm_f64(float ps, int srate_mul, const double* p1, long long n, double* ug) {
    TwoMass<double> m;
    m.init(ps);
    for (long long i = 0; i < n; i++) { m.p1 = p1[i]; m.step(srate_mul); ug[i] = m.ug_next; }
    return VS_OK;
}

/* The tmm_f64 option's arrangement of the double model (TwoMassR). */
int orc_tmm_f64r(float ps, int srate_mul, const double* p1, long long n, double* ug) {
    TwoMassR m;
    m.init(ps, srate_mul);
    for (long long i = 0; i < n; i++) ug[i] = m.step(p1[i]);
    return VS_OK;
}

/* Run `steps` steps of the FP32 engine from rest; trace[steps]; P/Vx/Vy get
 * the final frames (NULL skips). */
int orc_run_f32(const vs_params* p, const vs_geometry* g, long long steps, float* trace,
                float* P, float* Vx, float* Vy) {
    try {
        Grid G;
        build_grid(p, g, G);
        Coeffs C;
        build_coeffs(G, C);
        return run_engine<float>(p, G, C, steps, trace, P, Vx, Vy);
    } catch (const OracleError& e) { return fail(e); }
}

/* The double engine on caller-supplied depth maps (frameH*frameW each) and
 * z_inv value (applied where the reference puts z_inv: boundary segment id
 * != 0); cell types, listener and sources from (p, g).  Finite differences of
 * this function check the adjoint's map and admittance gradients. */
int orc_run_maps_f64(const vs_params* p, const vs_geometry* g, long long steps, const double* dP,
                     const double* dX, const double* dY, double zinv_val, double* trace) {
    try {
        Grid G;
        build_grid(p, g, G);
        Coeffs C;
        build_coeffs(G, C);
        const size_t N = (size_t)G.H * G.W;
        std::vector<double> mP(dP, dP + N), mX(dX, dX + N), mY(dY, dY + N), zin(N, 0.0);
        for (size_t i = 0; i < N; i++) if (G.bst[i] != 0) zin[i] = zinv_val;
        return run_engine_maps(p, G, C, steps, mP, mX, mY, zin, trace);
    } catch (const OracleError& e) { return fail(e); }
}

/* The FP32 engine on caller-supplied depth maps and z_inv value, as
 * orc_run_maps_f64 (the maps are rounded to float as the device copy is). */
int orc_run_maps_f32(const vs_params* p, const vs_geometry* g, long long steps, const float* dP,
                     const float* dX, const float* dY, float zinv_val, float* trace) {
    try {
        Grid G;
        build_grid(p, g, G);
        Coeffs C;
        build_coeffs(G, C);
        const size_t N = (size_t)G.H * G.W;
        std::vector<double> mP(dP, dP + N), mX(dX, dX + N), mY(dY, dY + N), zin(N, 0.0);
        for (size_t i = 0; i < N; i++) if (G.bst[i] != 0) zin[i] = zinv_val;
        return run_engine<float>(p, G, C, steps, trace, nullptr, nullptr, nullptr, &mP, &mX, &mY, &zin);
    } catch (const OracleError& e) { return fail(e); }
}

/* orc_run_maps_f32 that also returns the final P, Vx, Vy frames (any may be NULL). */
int orc_run_maps_f32_fields(const vs_params* p, const vs_geometry* g, long long steps, const float* dP,
                            const float* dX, const float* dY, float zinv_val, float* trace, float* P, float* Vx,
                            float* Vy) {
    try {
        Grid G;
        build_grid(p, g, G);
        Coeffs C;
        build_coeffs(G, C);
        const size_t N = (size_t)G.H * G.W;
        std::vector<double> mP(dP, dP + N), mX(dX, dX + N), mY(dY, dY + N), zin(N, 0.0);
        for (size_t i = 0; i < N; i++) if (G.bst[i] != 0) zin[i] = zinv_val;
        return run_engine<float>(p, G, C, steps, trace, P, Vx, Vy, &mP, &mX, &mY, &zin);
    } catch (const OracleError& e) { return fail(e); }
}

/* The same discrete system in double precision. */
int orc_run_f64(const vs_params* p, const vs_geometry* g, long long steps, double* trace,
                double* P, double* Vx, double* Vy) {
    try {
        Grid G;
        build_grid(p, g, G);
        Coeffs C;
        build_coeffs(G, C);
        return run_engine<double>(p, G, C, steps, trace, P, Vx, Vy);
    } catch (const OracleError& e) { return fail(e); }
}

}  // extern "C"
