// vs_device.h -- device-side descriptors shared by the kernels and the host
// launch code of libvocalsim_b200.
#pragma once

#include <cstdint>
#include <string>

#include <cuda_runtime_api.h>

#include "vs_grid.h"

namespace vsb {

// Flags of a tube descriptor.
enum : int32_t {
    TUBE_DIRICHLET = 1,   // zero P on noPressure cells (FDTDEngineCPU.cpp:336-337)
    TUBE_EIGEN = 2,       // FDTDEngineEigen pressure denominator sigma*dP + dP
    TUBE_TMM = 4,         // two-mass source computed on the device each step
    TUBE_WALL_ODE = 8,    // 2.5D wall oscillator with nonzero pressure coupling
    TUBE_TMM64 = 16,      // with TUBE_TMM: the two-mass model in double
};

// One tube as the step kernel sees it.  All planes share `pitch` and live in
// one device arena; P/Vx/Vy/w/z are ping-ponged by step parity.
struct TubeDev {
    float* P[2];
    float* Vx[2];
    float* Vy[2];
    float* w[2];          // wall velocity (only with TUBE_WALL_ODE)
    float* z[2];          // wall displacement (only with TUBE_WALL_ODE)
    const float* dP;
    const float* dX;
    const float* dY;
    const uint8_t* code;  // type | zinv bit
    const float* src;     // per-step excitation table (nullptr for the two-mass source)
    TmmState* tmm;        // [2], ping-ponged by step parity
    TmmState64* tmm64;    // [2], the double model's state (TUBE_TMM64)
    int64_t src_len;
    int64_t plane;        // elements between consecutive planes: P[k] = P[0] + k*plane,
                          // Vx[k] = P[0] + (2+k)*plane, Vy[k] = P[0] + (4+k)*plane,
                          // dX = dP + plane, dY = dP + 2*plane
    int32_t H, W, pitch, flags;
    int32_t lis_x, lis_y, exc_x, exc_y;
    float K1, K2, bcoef, zinv;
    float dt, Mw, Bw, Kw, cpl;
    float dir0, dir1, dir2, dir3;
    float sigma[13];
    // fast_math: per-cell descriptor bytes (same layout as `code`) into two
    // coefficient tables, desc_a = (alx, aly, g, cex), desc_b = (zox, zix, zoy,
    // ziy): P' = (P - K1 S / dP) g and
    // V' = al (V - bcoef (P'n - P'c)) + zo P'c - zi P'n + ce exeV (x and y).
    // Reference arithmetic (batches without the coupled wall): the same
    // descriptor bytes into tables of the exactly rounded factors of the
    // reference update, desc_a = (sP, den_x, den_y, flag bits EXD_*),
    // desc_b = (mS_x, W_x, mS_y, W_y); see the two-step kernel.
    const uint8_t* desc;
    const float4* desc_a;
    const float4* desc_b;  // = desc_a + kDescEntries (the two tables are contiguous)
    int32_t ndesc;        // descriptors in use (ids 0 .. ndesc-1)
    float* X;             // fast_math: a third P, Vx, Vy set (`plane` apart) for the two-step kernels
    TmmState* tmm_x;      // the two-step kernels' third two-mass state slot (float and double model)
    TmmState64* tmm64_x;
    TmmConsts tmmc;
    TmmConsts64 tmmd;     // the double model's constants, else tmmc widened (adjoint)
    TmmDerived64 tmmx;    // the double model's derived constants
    // state history for the adjoint's recomputation (strip kernel with
    // history capture only): the state after step n goes to slot
    // n + 1 - RunState::run_start, slot = [P, Vx, Vy] planes, `plane` apart
    float* hist;
    double* tmm_hist;     // two-mass state before each step of the segment: 6 values
                          // per slot (x1_old, x1_curr, x2_old, x2_curr, ug_old, ug_curr)
};

// Mutable run bookkeeping kept in device memory so that CUDA graphs captured
// once can be replayed for any run length.
// Entries of each descriptor table (desc_a, desc_b).
constexpr int kDescEntries = 256;

// Flag bits of a reference-arithmetic descriptor (desc_a.w as raw bits): per
// velocity direction (x in bits 0-7, y in bits 8-15) mB = beta_c beta_n, a
// source term (excitation cell or neighbour), the wall term (z_inv bit, no
// excitation, beta_c != beta_n), its pressure (the cell's, else the
// neighbour's) and Nout = 1 (else 1/sqrt 2); the no-pressure cells of a
// Dirichlet mouth.
enum : unsigned {
    EXD_MB = 1u, EXD_SRC = 2u, EXD_WALL = 4u, EXD_WALL_PC = 8u, EXD_NOUT1 = 16u,
    EXD_Y_SHIFT = 8u, EXD_PZERO = 1u << 16,
};

struct RunState {
    int64_t step;         // global step of the next launch with local index 0
    int64_t run_start;    // global step that lands in trace column 0
    float* trace;         // device trace buffer, [ntubes][trace_stride]
    int64_t trace_stride;
    int32_t error;        // sticky device error word (0 = ok): VS_ERR_TIMEOUT, VS_ERR_NONFINITE
    int32_t bsel;         // two-step kernels: 1 = the state of `step` is in TubeDev::X
    uint32_t wait_polls;  // polls of a row-copy wait before it gives up (0 = kWaitPolls);
                          // the drain after a timeout always uses kWaitPolls
};

// Strip geometry of the step kernel: lane i of a warp holds column c0 + i;
// lanes 0 and 31 are halo, so a strip commits the kStripCommit columns
// c0 + 1 .. c0 + 30, and strip k of a tube starts at c0 = 30 k - 1.
constexpr int kStripCommit = 30;
constexpr int kStripLead = 1;
constexpr int kMaxStripRows = 62;

// Quad strips: lane i holds the four columns c0 + 4i .. c0 + 4i + 3 (c0 a
// multiple of 4); lanes 1..30 commit the 120 columns c0 + 4 .. c0 + 123, and
// strip k of a tube starts at c0 = 120 k - 4.
constexpr int kQuadCommit = 120;
constexpr int kQuadLead = 4;

// A strip of one tube processed by one warp: rows [r0, r0+rows), starting
// column c0.  The masks classify its rows once, from the static cell types,
// so the kernel branches uniformly instead of voting per row:
//   p_rows     bit j: row r0-1+j has a computed cell whose type is not air
//              (nonzero sigma or a no-pressure cell)
//   v_beta1    bit j: committed row r0+j needs at least the beta = 1 update
//   v_generic  bit j: committed row r0+j needs the full velocity update
struct Tile {
    int32_t tube, r0, c0, has_exc;
    uint64_t p_rows, v_beta1, v_generic;
};

// Velocity class a committed cell needs, from the codes of the cell and of its
// right and top neighbours.
enum : int { V_PLAIN = 0, V_BETA1 = 1, V_GENERIC = 2 };

__host__ __device__ inline bool beta_one(int t) {
    // air, PML and no-pressure cells have beta = 1 (SolverParams.cu:5-27)
    return t == VS_CELL_AIR || t == VS_CELL_NOPRESSURE || (t >= VS_CELL_PML0 && t <= VS_CELL_PML5);
}

__host__ __device__ inline int velocity_class(int kc, int kr, int kt) {
    const int tc = kc & CODE_TYPE_MASK, tr = kr & CODE_TYPE_MASK, tt = kt & CODE_TYPE_MASK;
    if (kc & CODE_ZINV_BIT) return V_GENERIC;
    if (tc == VS_CELL_AIR && tr == VS_CELL_AIR && tt == VS_CELL_AIR) return V_PLAIN;
    return (beta_one(tc) && beta_one(tr) && beta_one(tt)) ? V_BETA1 : V_GENERIC;
}

// Masks and excitation flag of the strip (r0, rows, c0) of an H x W frame
// that commits columns c0 + lead .. c0 + lead + commit - 1 (and computes P'
// one column further); code(r, c) returns the code byte of a frame cell.
template <class CodeAt>
__host__ __device__ inline void classify_strip(CodeAt code, int H, int W, int r0, int rows, int c0, Tile& t,
                                               int lead = kStripLead, int commit = kStripCommit) {
    t.p_rows = 0;
    t.v_beta1 = 0;
    t.v_generic = 0;
    t.has_exc = 0;
    const int rlast = (r0 + rows - 1 < H - 2) ? r0 + rows - 1 : H - 2;
    const int cfirst = c0 + lead > 1 ? c0 + lead : 1;
    const int plast = c0 + lead + commit < W - 2 ? c0 + lead + commit : W - 2;
    const int vlast = c0 + lead + commit - 1 < W - 2 ? c0 + lead + commit - 1 : W - 2;
    for (int r = r0 - 1; r <= rlast; ++r) {
        if (r >= 1) {
            for (int c = cfirst; c <= plast; ++c)
                if ((code(r, c) & CODE_TYPE_MASK) != VS_CELL_AIR) { t.p_rows |= 1ull << (r - r0 + 1); break; }
        }
        if (r >= r0 && r >= 1) {
            int cls = V_PLAIN;
            for (int c = cfirst; c <= vlast; ++c) {
                const int kc = code(r, c);
                const int k = velocity_class(kc, code(r, c + 1), code(r - 1, c));
                cls = k > cls ? k : cls;
                if ((kc & CODE_TYPE_MASK) == VS_CELL_EXCITATION) t.has_exc = 1;
            }
            if (cls >= V_BETA1) t.v_beta1 |= 1ull << (r - r0);
            if (cls >= V_GENERIC) t.v_generic |= 1ull << (r - r0);
        }
    }
}

// Host-side description of a compiled launch shape.  Strips and quad strips:
// rows per strip, committed columns per strip, warps per CTA.  Bands: rows
// per band (a band spans the full frame width; cols = 0), warps per CTA.
// Quad strips have no wall-oscillator variant.
enum : int { SHAPE_STRIP = 0, SHAPE_BAND = 1, SHAPE_QUAD = 2, SHAPE_QUAD2 = 3, SHAPE_CLUSTER = 4 };

// Two-step quad strips of NC columns per lane start at c0 = 30 NC k - NC,
// commit columns c0 + NC .. c0 + 31 NC - 1 and classify an extended region:
// rows from r0 - 2 (p_rows) / r0 - 1 (velocity masks), columns c0 + NC/2 ..
// c0 + 32 NC - NC/2 - 1.
struct TileShape {
    int rows, cols, warps, kind;
    int lane_cols;        // quad strips: columns per lane
};

int tile_shape_count();
TileShape tile_shape(int i);
// Index of the cluster shape (the last one): a single tube on one
// thread-block cluster, every step of a run in one launch (vs_cluster.cu).
int cluster_shape();

// Launch configuration of the cluster kernel for one tube.
struct ClusterConfig {
    int ctas = 0, threads = 0, rows_max = 0;
    int cols = 0;         // column threads (threads less the two-mass warp of form 2)
    size_t smem = 0;
    int form = 0;         // 0: band in shared memory; 1: register-resident columns (rows_max <= rmax),
                          // cluster barrier per step; 2: the same, neighbour-to-neighbour exchange;
                          // 3: form 2 with the two-mass model in an extra warp
    int rmax = 0;
    int nclusters = 0;    // clusters of this configuration resident on the device at once
};
// Cluster size (16, 8 or 4 CTAs), threads and shared memory for a tube of
// H x W cells (row pitch `pitch`) on the current device, or false when none
// fits; sets the kernel attributes it needs.  `tmm`: the tube has the
// two-mass source (its excitation value reaches every CTA each step, which
// the cluster barrier form does faster than the neighbour exchange).
bool cluster_config(int H, int W, int pitch, bool fast, bool tmm, ClusterConfig* out);
// `steps` time steps of the `ntubes` tubes from `tube` on (device), one
// thread-block cluster per tube (configuration c, sized for the largest of
// them), from RunState::step, in one launch; then RunState::step advances by
// `steps` (a separate launch).  The states must be in their parity sets
// (bsel = 0) and stay there.
cudaError_t launch_cluster_run(const TubeDev* tube, RunState* rs, int64_t steps, bool fast, const ClusterConfig& c,
                               cudaStream_t stream, int ntubes = 1);

// Launch one time step (local index `local` after RunState::step) of every
// strip or band in `tiles` with the compiled shape `shape`; `wall` selects
// the kernel variant with the coupled wall oscillator (needed when any tube
// has it), `fast` the reciprocal-form arithmetic (fast_math; quad strips
// only, never with `wall`); max_pitch sizes a band kernel's shared memory.
cudaError_t launch_step(int shape, bool wall, bool fast, const TubeDev* tubes, const Tile* tiles, int ntiles,
                        RunState* rs, int local, cudaStream_t stream, int max_pitch);
bool shape_has_fast(int shape);
// true when the shape has a reference-arithmetic kernel without the wall oscillator
bool shape_has_plain(int shape);

// Dynamic shared memory a shape needs for frames of row pitch up to
// max_pitch (0 for strips), and the one-time kernel attribute set-up for it.
size_t shape_smem_bytes(int shape, int max_pitch);
cudaError_t prepare_shape(int shape, int max_pitch);

// One step that also stores the new state into the tube's history
// (TubeDev::hist); tubes without a wall oscillator only.  `shape` is
// history_shape() of the batch's interior cell count and arithmetic (strips,
// or quad strips in the reciprocal form for fast_math; the tiles in `tiles`
// must be built for it).
cudaError_t launch_step_history(int shape, const TubeDev* tubes, const Tile* tiles, int ntiles, RunState* rs,
                                int local, cudaStream_t stream);
int history_shape(int64_t cells, bool fast);
// Two steps (launch `local`: steps RunState::step + 2 local and + 1) with both
// new states stored into the history, in the reciprocal form (fast_math):
// the two-step kernel of shape history2_shape() (tiles built for it), with
// the third state set and RunState::bsel as in a forward run.
cudaError_t launch_step_history2(int shape, const TubeDev* tubes, const Tile* tiles, int ntiles, RunState* rs,
                                 int local, cudaStream_t stream);
int history2_shape(int64_t cells);
// The two-step launch shape for a batch of `cells` interior cells (strip
// height by batch size; the default of fast_math batches).
int two_step_shape(int64_t cells);

// Adjoint buffers of one tube (device memory).
struct AdjTube {
    float* lam[2];        // [parity]: lambda P, Vx, Vy planes at +0, +plane, +2*plane
    double* gP;           // per-cell gradient accumulators of dP, dX, dY, z_inv
    double* gX;
    double* gY;
    double* gZ;
    const float* gtrace;  // dL/d trace[step], this tube's row
    double* lam_tmm;      // adjoint of the two-mass state (6 values), then [6 + parity]:
                          // d/d p1 pending for lambda P of that parity at the excitation point
    // the velocities the excitation flow enters: lambda-plane offsets (Vx at
    // plane + o, Vy at 2 plane + o) and dV'/d exeV of each
    const int32_t* exc_off;
    const float* exc_coef;
    int32_t n_exc;
    int32_t tiles;        // 32 x 8 cell tiles of the interior (tile form)
    int32_t strips;       // row-marching strips of the interior (strip forms)
    int32_t ndesc;        // neighbourhood descriptors in use (entries of `tab`)
    // per-cell neighbourhood descriptors (H x pitch bytes) into a table of
    // three float4 per descriptor: (ax, ay, bx, by), (alx, aly, 1 + sigma,
    // Dirichlet no-pressure flag), (zc_out x, zc_in x, zc_out y, zc_in y)
    const uint8_t* desc;
    const float4* tab;
};

// Segment of the reverse sweep, in device memory so that one captured graph
// serves every segment: a launch with reverse-step index `local` reverses
// forward step n = start + len - 1 - local (and, in the two-step form, n - 1
// after it), whose state-before is history slot n - start; launch number
// `phase` of the segment reads the adjoint of the state after its first step
// from lambda parity q0 ^ (phase & 1) and writes the other parity.
struct AdjRun {
    int64_t start;
    int32_t len;
    int32_t q0;
};

// Tile of the reverse step kernel.
constexpr int kAdjTileW = 32, kAdjTileH = 8;

// One reverse step (reverse-step index `local`, launch number `phase` of the
// segment in `run`) for every tube: lambda of the state before the step, the
// map / z_inv gradient terms and, for the two-mass source, its reverse step.
// Three implementations:
//   ADJ_FORM_TILES    32 x 8 tiles with mu in shared memory, one step per
//                     launch: the most parallel form, best for small batches
//   ADJ_FORM_STRIPS2  row-marching warp strips running two reverse steps per
//                     launch (steps n and n - 1; the second one row behind the
//                     first on values held in registers), so lambda and the
//                     gradient accumulators are read and written once per two
//                     steps; table sources only (no two-mass tube)
//   ADJ_FORM_STRIPS   the same strips, one reverse step per launch
// ADJ_FORM_AUTO picks two-step strips for a large batch of table-source tubes
// and tiles otherwise.  `rows` = rows per strip (4, 8 or 16) of the strip
// forms.  max_blocks = the largest block count of a tube in the chosen form,
// plus one when a tube has the two-mass source (its reverse step runs in the
// block after the others).
enum : int { ADJ_FORM_AUTO = 0, ADJ_FORM_TILES = 1, ADJ_FORM_STRIPS2 = 2, ADJ_FORM_STRIPS = 3 };
cudaError_t launch_adjoint_step(const TubeDev* tubes, const AdjTube* adj, int ntubes, int max_blocks,
                                const AdjRun* run, int local, int phase, cudaStream_t stream, int form,
                                int rows);
int adjoint_strips(int H, int W, int form, int rows);   // strips of an H x W frame
int adjoint_strip_blocks(int strips);                   // CTAs those strips take

// Copy each tube's state (parity par) into slot 0 of its history (and the
// two-mass state into slot 0 of tmm_hist).
cudaError_t launch_history_seed(const TubeDev* tubes, int ntubes, int max_plane_cells, int par, cudaStream_t stream);

// ---- device map builder (vs_mapbuild.cu) ------------------------------------
enum : int { MAP_DEPTH_NONE = 0, MAP_DEPTH_CIRCLE = 1, MAP_DEPTH_ELLIPSE = 2 };

// One tube for the device map builder: the frame, the tube's columns (from
// build_tube_columns) and the device planes to paint (row pitch `pitch`).
struct MapBuild {
    int H, W, pitch;
    int sx, L, my, ex;        // first tube column, tube length in cells, axis row, last tube column
    int npc;                  // the no-pressure column (Dirichlet mouth), or -1
    int pml;                  // PML layers (0 or 6)
    int depth;                // MAP_DEPTH_*: 2D solver (unit depths), circular or elliptical sections
    int depth_fma;            // vs_params::depth_fma
    float ds, ud;             // cell size, uniform depth (0: none)
    const int32_t* up;        // per tube column: wall rows, the gap fill's extent, 0-based segment
    const int32_t* down;
    const int32_t* utop;
    const int32_t* dbot;
    const int32_t* seg;
    const float* minor;       // per section: elliptical minor axis (m)
    float* dP;
    float* dX;
    float* dY;
    uint8_t* code;
    float* tmpx;              // two scratch planes (H x pitch)
    float* tmpy;
};

// Paint the maps of `ntubes` tubes (device array `tubes`); max_cells = the
// largest H * pitch.  A negative depth radicand sets *err (device int) to
// VS_ERR_NEGATIVE_SQRT.
cudaError_t launch_build_maps(const MapBuild* tubes, int ntubes, int64_t max_cells, int* err, cudaStream_t stream);

// ---- section depth model (vs_sections.cu) -----------------------------------
// A frame cell the reference's elliptical depth kernel writes: its section,
// the nominal semi-major axis a0 (m) of its column and its distance from the
// tube axis in cells; seg = kSectionZero for the cells it sets to 0 (walls),
// kSectionUnwritten for the cells it leaves (they take the pivot's value).
constexpr int32_t kSectionUnwritten = -1;
constexpr int32_t kSectionZero = -2;

struct SectionCell {
    int32_t seg;
    float dist;
    double a0;
};

struct SectionTube {
    const SectionCell* cx;    // depth_x writes, H x W (unpitched)
    const SectionCell* cy;    // depth_y writes
    const double* w0;         // nominal section widths (m)
    const double* w;          // current section widths and depths (m)
    const double* d;
    double* dw;               // dL/d width, dL/d depth per section (reverse pass)
    double* dd;
    uint8_t* clamp;           // per cell: bit 0 dp, bit 1 xs, bit 2 ys raised to the minimum
    double* gxs;              // reverse-pass scratch planes, H x W
    double* gys;
    double* gx;
    double* gy;
    double* acc;              // 6 pivot accumulators of the reverse pass
    double ds;
    int64_t pivot;            // cell (mid row, tube end), H x W index
    int32_t H, W, nsec, pad;
};

// Depth maps of every tube from its current section parameters, written into
// the tubes' dP / dX / dY planes; max_cells = the largest H x W.
cudaError_t launch_section_maps(const SectionTube* tubes, const TubeDev* devs, int ntubes, int64_t max_cells,
                                cudaStream_t st);
// dL/d width and dL/d depth per section from the per-cell map gradients of
// the last adjoint (AdjTube gP, gX, gY); dw, dd and acc zeroed by the caller.
cudaError_t launch_section_vjp(const SectionTube* tubes, const TubeDev* devs, const AdjTube* adj, int ntubes,
                               int64_t max_cells, cudaStream_t st);

// Formants of ntr device traces of n samples at sampling rate fs (the
// reference's get_formants_bw): out (device) = ntr x [bandwidth, centre,
// level] x nf.  Synchronises `st`; returns a vs_status, err gets the text.
// WAV samples of listener traces (vs_audio.cu).
void audio_filter(int srate_mul, double b[3], double a[3]);
int audio_device(const float* traces, int ntr, int64_t n, int mul, float* out, cudaStream_t st, std::string* err);

int formants_device(const float* traces, int ntr, int64_t n, double fs, int nf, double* out, cudaStream_t st,
                    std::string* err);

// Set the text vs_last_error() returns on this host thread.
void record_error(const char* msg);

// RunState::step += k (the tail node of a captured chunk).
cudaError_t launch_advance(RunState* rs, int k, cudaStream_t stream);
// Two-step kernels: RunState::step += k, RunState::bsel ^= toggle.
cudaError_t launch_advance2(RunState* rs, int k, int toggle, cudaStream_t stream);
// Move each tube's state from TubeDev::X back to the parity set of RunState::step.
cudaError_t launch_copy_back(const TubeDev* tubes, int ntubes, int max_plane_cells, const RunState* rs,
                             cudaStream_t stream);

}  // namespace vsb
