// vs_capi.cpp -- the C ABI of libvocalsim_b200 (include/vocalsim_b200.h).
//
// A vs_batch owns one device arena holding every tube's planes, the tube
// descriptors, the tile work list, the run state and the trace buffer.  A
// vs_solver is a batch of one.  Time steps are issued as CUDA graphs of
// kChunk step launches (captured once per tile shape) plus direct launches
// for the remainder.
#include "vs_device.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <exception>
#include <mutex>
#include <thread>
#include <functional>
#include <cmath>
#include <cstring>
#include <memory>
#include <new>
#include <string>
#include <map>
#include <vector>

namespace vsb {
namespace {

thread_local std::string g_last_error;

int set_error(int status, const std::string& msg) {
    g_last_error = msg;
    return status;
}

struct CudaFail {
    cudaError_t err;
    const char* where;
};

void ck(cudaError_t e, const char* where) {
    if (e != cudaSuccess) throw CudaFail{e, where};
}

}  // namespace

// Error text for entry points defined in other files of the library.
void record_error(const char* msg) { g_last_error = msg; }

namespace {

constexpr int kChunk = 128;   // steps per captured graph
constexpr size_t kAlign = 256;
constexpr size_t kGuard = 1024;  // bytes of slack around the tube planes of an arena

size_t align_up(size_t v) { return (v + kAlign - 1) / kAlign * kAlign; }

// fn(i) for i in [0, n) on up to hardware_concurrency host threads (host
// work only: map building, source tables, staging images); the first
// exception thrown by a call is rethrown here after every thread joined.
void parallel_for(size_t n, const std::function<void(size_t)>& fn) {
    size_t nt = std::min<size_t>(n, std::max(1u, std::thread::hardware_concurrency()));
    nt = std::min<size_t>(nt, 64);
    if (nt <= 1) {
        for (size_t i = 0; i < n; ++i) fn(i);
        return;
    }
    std::atomic<size_t> next{0};
    std::exception_ptr err;
    std::mutex m;
    std::vector<std::thread> pool;
    pool.reserve(nt);
    for (size_t t = 0; t < nt; ++t)
        pool.emplace_back([&] {
            for (size_t i = next.fetch_add(1); i < n; i = next.fetch_add(1)) {
                try {
                    fn(i);
                } catch (...) {
                    std::lock_guard<std::mutex> lock(m);
                    if (!err) err = std::current_exception();
                }
            }
        });
    for (std::thread& t : pool) t.join();
    if (err) std::rethrow_exception(err);
}

}  // namespace
}  // namespace vsb

using namespace vsb;

struct vs_batch {
    std::vector<TubeGrid> grids;
    std::vector<TubeDev> h_tubes;
    std::vector<size_t> src_off;           // arena offset of each tube's source table
    std::vector<int64_t> src_len;
    std::vector<char*> state_base;         // per tube: start of its mutable planes
    std::vector<size_t> state_bytes;
    char* arena = nullptr;
    size_t arena_bytes = 0;
    float* src_arena = nullptr;            // source tables live in their own buffer
    size_t src_bytes = 0;
    TubeDev* d_tubes = nullptr;
    Tile* d_tiles = nullptr;
    int ntiles = 0;
    int tiles_shape = -1;
    RunState* d_rs = nullptr;
    float* d_trace = nullptr;
    int64_t trace_cap = 0;                 // floats
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int shape = -1;                        // chosen tile shape (-1 = not chosen)
    cudaGraphExec_t graph = nullptr;
    int graph_shape = -1;
    int64_t step = 0;                      // host mirror of RunState::step
    int device = 0;
    bool wall = false;                     // some tube has the coupled wall oscillator
    bool fast = false;                     // reciprocal-form arithmetic (vs_params::fast_math)
    bool desc = false;                     // descriptor planes and tables (fast_math, or no wall oscillator)
    int max_pitch = 0;                     // largest row pitch of the batch (band shared memory)
    int cluster_state = 0;                 // cluster shape: 0 = not checked, 1 = fits, -1 = does not
    uint32_t wait_polls = 0;               // RunState::wait_polls of every run (0 = the default limit)
    int adj_form = ADJ_FORM_AUTO;          // reverse-step kernel form (vs_batch_set_adjoint_form)
    int adj_rows = 0;                      // rows per strip of the strip forms (0 = the form's default)
    int adj_graph_rows = 0;
    ClusterConfig cluster{};
    // adjoint: checkpoints of the last checkpointed forward, history, adjoint planes
    int64_t ck_steps = 0;                  // steps of the checkpointed forward (0 = none)
    int ck_every = 0;
    int ck_count = 0;
    char* ckpt = nullptr;                  // [ck_count][sum of state_bytes]
    size_t ckpt_stride = 0;
    char* adj_mem = nullptr;               // history + lambda + gradient planes
    size_t adj_bytes = 0;
    std::vector<size_t> adj_off;           // per tube: offset of its block in adj_mem
    AdjTube* d_adj = nullptr;
    AdjRun* d_adjrun = nullptr;
    float* d_gtrace = nullptr;
    int64_t gtrace_cap = 0;
    char* d_exc = nullptr;                 // excitation velocity lists (offsets, coefficients)
    size_t exc_bytes = 0;
    Tile* d_hist_tiles = nullptr;
    int n_hist_tiles = 0;
    Tile* d_hist2_tiles = nullptr;         // two-step history shape (fast_math batches)
    int n_hist2_tiles = 0;
    Tile* d_odd_tiles = nullptr;           // single-step tiles beside a two-step shape
    char* x_mem = nullptr;                 // third state set of the two-step shapes (TubeDev::X, tmm_x)
    size_t x_bytes = 0;
    int n_odd_tiles = 0;
    int odd_shape = -1;
    // section depth model (vs_batch_set_sections): per-tube descriptors and buffers
    std::vector<SectionTube> h_sec;
    SectionTube* d_sec = nullptr;
    char* sec_mem = nullptr;
    int64_t sec_max_cells = 0;
    bool sec_maps = false;                 // the maps on the device came from set_sections
    cudaGraphExec_t hist_graph = nullptr;  // ck_every history steps
    cudaGraphExec_t adj_graph = nullptr;   // ck_every reverse steps
    int adj_graph_len = 0;
    int adj_graph_form = -1;
    float adj_recompute_ms = 0.0f;         // device time of the last adjoint's recomputation / reverse steps
    float adj_reverse_ms = 0.0f;

    ~vs_batch() { release(); }

    void release() {
        if (graph) cudaGraphExecDestroy(graph);
        graph = nullptr;
        if (arena) cudaFree(arena);
        if (src_arena) cudaFree(src_arena);
        if (d_tubes) cudaFree(d_tubes);
        if (d_tiles) cudaFree(d_tiles);
        if (d_rs) cudaFree(d_rs);
        if (d_trace) cudaFree(d_trace);
        if (ckpt) cudaFree(ckpt);
        if (adj_mem) cudaFree(adj_mem);
        if (d_adj) cudaFree(d_adj);
        if (d_adjrun) cudaFree(d_adjrun);
        if (d_gtrace) cudaFree(d_gtrace);
        if (d_exc) cudaFree(d_exc);
        if (d_hist_tiles) cudaFree(d_hist_tiles);
        if (d_hist2_tiles) cudaFree(d_hist2_tiles);
        if (d_odd_tiles) cudaFree(d_odd_tiles);
        d_odd_tiles = nullptr;
        if (x_mem) cudaFree(x_mem);
        x_mem = nullptr;
        if (d_sec) cudaFree(d_sec);
        if (sec_mem) cudaFree(sec_mem);
        d_sec = nullptr; sec_mem = nullptr;
        if (hist_graph) cudaGraphExecDestroy(hist_graph);
        if (adj_graph) cudaGraphExecDestroy(adj_graph);
        ckpt = nullptr; adj_mem = nullptr; d_adj = nullptr; d_adjrun = nullptr; d_gtrace = nullptr;
        d_exc = nullptr; d_hist_tiles = nullptr; d_hist2_tiles = nullptr; hist_graph = nullptr; adj_graph = nullptr;
        if (own_stream && stream) cudaStreamDestroy(stream);
        arena = nullptr; src_arena = nullptr; d_tubes = nullptr; d_tiles = nullptr;
        d_rs = nullptr; d_trace = nullptr; stream = nullptr;
    }
};

struct vs_solver {
    vs_batch* b = nullptr;
};

namespace vsb {
namespace {

// Default launch shapes when no autotune ran: 16-row strips with 4 warps per
// CTA, and 4-row strips with 2 warps per CTA below kSmallGridCells cells;
// with fast_math the quad strips of the same heights (16 rows x 4 warps,
// 2 rows x 2 warps), and for fast_math batches without the coupled wall
// the two-step strips of 64 columns with the strip height of
// two_step_shape() (2 to 32 rows by batch size).
constexpr int kDefaultShape = 1;
constexpr int kSmallShape = 8;
constexpr int kFastShape = 17;
constexpr int kFastSmallShape = 21;
constexpr int64_t kSmallGridCells = 200000;

int planes_per_tube(const TubeGrid& g) { return g.wall_ode ? 13 : 9; }

void upload_sources(vs_batch* b, int64_t need) {
    // (Re)build every tube's excitation table so that it covers steps [0, need).
    bool ok = true;
    for (size_t i = 0; i < b->grids.size(); ++i)
        if (!b->grids[i].tmm && b->src_len[i] < need) ok = false;
    if (ok && b->src_arena) return;
    parallel_for(b->grids.size(), [&](size_t i) {
        TubeGrid& g = b->grids[i];
        if (g.tmm || (int64_t)g.source.size() >= need) return;
        vs_params p;
        std::memcpy(&p, &g.src_params, sizeof(p));
        build_source(&p, g.dt, need, g.source);
    });
    // identical tables (the same source type and parameters, time step and
    // length) are uploaded once and shared by their tubes
    size_t total = 0;
    std::vector<size_t> off(b->grids.size(), 0);
    std::vector<bool> upload(b->grids.size(), false);
    std::map<std::string, size_t> offset_of;
    for (size_t i = 0; i < b->grids.size(); ++i) {
        const TubeGrid& g = b->grids[i];
        if (g.tmm) continue;
        vs_params p;
        std::memcpy(&p, &g.src_params, sizeof(p));
        const float key_f[7] = {p.sine_amp, p.sine_freq_hz, p.gauss_amp, p.gauss_peak_s, p.gauss_width_s, g.dt,
                                (float)p.source_type};
        const int64_t len = (int64_t)g.source.size();
        std::string key(reinterpret_cast<const char*>(key_f), sizeof(key_f));
        key.append(reinterpret_cast<const char*>(&len), sizeof(len));
        const auto it = offset_of.find(key);
        if (it != offset_of.end()) {
            off[i] = it->second;
            continue;
        }
        off[i] = total;
        offset_of.emplace(key, total);
        upload[i] = true;
        total += align_up(g.source.size() * sizeof(float));
    }
    if (b->src_arena) { cudaFree(b->src_arena); b->src_arena = nullptr; }
    if (total) ck(cudaMalloc(&b->src_arena, total), "cudaMalloc(source tables)");
    for (size_t i = 0; i < b->grids.size(); ++i) {
        TubeGrid& g = b->grids[i];
        TubeDev& t = b->h_tubes[i];
        if (g.tmm) { t.src = nullptr; t.src_len = 0; b->src_len[i] = INT64_MAX; continue; }
        float* dst = (float*)((char*)b->src_arena + off[i]);
        if (upload[i])
            ck(cudaMemcpy(dst, g.source.data(), g.source.size() * sizeof(float), cudaMemcpyHostToDevice),
               "upload source table");
        t.src = dst;
        t.src_len = (int64_t)g.source.size();
        b->src_len[i] = t.src_len;
    }
    ck(cudaMemcpy(b->d_tubes, b->h_tubes.data(), b->h_tubes.size() * sizeof(TubeDev),
                  cudaMemcpyHostToDevice), "upload tube descriptors");
}

// Largest dynamic shared memory a CTA may use on this device.
size_t smem_optin_limit(int device) {
    int v = 0;
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, device) != cudaSuccess) return 0;
    return (size_t)v;
}

// The cluster shape runs each tube of a batch without the coupled wall
// oscillator on its own thread-block cluster, in one launch; the
// configuration is sized for the largest frame of the batch, and every tube
// needs at least one interior row per CTA.
constexpr size_t kMaxClusterTubes = 64;

bool cluster_fits(const vs_batch* b) {
    if (b->cluster_state == 0) {
        vs_batch* m = const_cast<vs_batch*>(b);
        m->cluster_state = -1;
        if (b->grids.size() <= kMaxClusterTubes && !b->wall) {
            int H = 0, W = 0, pitch = 0, min_rows = INT32_MAX;
            bool tmm = false;
            for (const TubeGrid& g : b->grids) {
                H = std::max(H, g.H);
                W = std::max(W, g.W);
                pitch = std::max(pitch, g.pitch);
                min_rows = std::min(min_rows, g.H - 2);
                tmm = tmm || g.tmm;
            }
            if (cluster_config(H, W, pitch, b->fast, tmm, &m->cluster) && m->cluster.ctas <= min_rows)
                m->cluster_state = 1;
        }
    }
    return b->cluster_state == 1;
}

bool shape_fits(const vs_batch* b, int shape) {
    const int kind = tile_shape(shape).kind;
    if (kind == SHAPE_CLUSTER) return cluster_fits(b);
    if (b->wall && (kind == SHAPE_QUAD || kind == SHAPE_QUAD2)) return false;   // no wall-oscillator variant
    // two-step kernels in the reference arithmetic: the 2-column shapes, when
    // every tube's neighbourhoods fit its descriptor tables
    if (kind == SHAPE_QUAD2 && !b->fast) {
        if (!b->desc || !shape_has_plain(shape)) return false;
        for (const TubeDev& t : b->h_tubes)
            if (t.ndesc <= 0) return false;
    }
    if (b->fast && !shape_has_fast(shape)) return false;
    return shape_smem_bytes(shape, b->max_pitch) <= smem_optin_limit(b->device);
}

// single-step default (also the shape of the last step of an odd count
// run with a two-step shape)
int single_step_shape(const vs_batch* b) {
    int64_t cells = 0;
    for (const TubeGrid& g : b->grids) cells += (int64_t)g.H * g.W;
    const bool small = cells < kSmallGridCells;
    if (b->fast) return small ? kFastSmallShape : kFastShape;
    return small ? kSmallShape : kDefaultShape;
}

int default_shape(const vs_batch* b) {
    // a single tube keeps its state on one thread-block cluster for the whole
    // run, and so does every tube of a batch whose clusters (register form)
    // are resident at once (measured, fast_math: 2 and 4 tubes 1.36 us per
    // step against 2.6 on the strips; past one wave of clusters the strips win)
    const int n = (int)b->grids.size();
    if (shape_fits(b, cluster_shape()) && (n == 1 || (b->cluster.form != 0 && n <= b->cluster.nclusters)))
        return cluster_shape();
    int64_t cells = 0;
    for (const TubeGrid& g : b->grids) cells += g.dims.interior_cells;
    const int two = two_step_shape(cells);
    if (tile_shape(two).kind == SHAPE_QUAD2 && shape_fits(b, two)) return two;
    return single_step_shape(b);
}

// Tile list of a launch shape, uploaded to a new device buffer (*n tiles).
Tile* make_tiles(vs_batch* b, int shape, int* n) {
    const TileShape ts = tile_shape(shape);
    if (!shape_fits(b, shape)) throw VsFailure{VS_ERR_UNSUPPORTED, "launch shape unavailable for this batch (shared memory, wall oscillator or fast_math)"};
    ck(prepare_shape(shape, b->max_pitch), "kernel attributes");
    std::vector<std::vector<Tile>> per_tube(b->grids.size());
    parallel_for(b->grids.size(), [&](size_t i) {
        std::vector<Tile>& tiles = per_tube[i];
        const TubeGrid& g = b->grids[i];
        auto code_at = [&g](int r, int c) { return (int)g.code[(size_t)r * g.pitch + c]; };
        for (int r0 = 1; r0 <= g.H - 2; r0 += ts.rows) {
            if (ts.kind == SHAPE_BAND) {
                // a band covers the full width of rows r0 .. r0+rows-1
                Tile t{};
                t.tube = (int32_t)i;
                t.r0 = r0;
                for (int r = r0; r < std::min(r0 + ts.rows, g.H - 1) && !t.has_exc; ++r)
                    for (int c = 0; c < g.W; ++c)
                        if ((code_at(r, c) & CODE_TYPE_MASK) == VS_CELL_EXCITATION) { t.has_exc = 1; break; }
                tiles.push_back(t);
                continue;
            }
            // strips start at c0 = commit*k - lead and commit columns
            // c0+lead .. c0+lead+commit-1; rows r0 .. r0+rows-1
            const bool quad = ts.kind == SHAPE_QUAD || ts.kind == SHAPE_QUAD2;
            const int nc = ts.lane_cols;
            const int lead = ts.kind == SHAPE_QUAD2 ? nc : quad ? kQuadLead : kStripLead;
            const int commit = ts.cols;
            for (int c0 = -lead; c0 + lead <= g.W - 2; c0 += commit) {
                Tile t{};
                t.tube = (int32_t)i;
                t.r0 = r0;
                t.c0 = c0;
                if (ts.kind == SHAPE_QUAD2)
                    classify_strip(code_at, g.H, g.W, r0 - 1, ts.rows + 2, c0, t, nc / 2, 31 * nc);
                else
                    classify_strip(code_at, g.H, g.W, r0, ts.rows, c0, t, lead, commit);
                tiles.push_back(t);
            }
        }
    });
    std::vector<Tile> tiles;
    for (const std::vector<Tile>& v : per_tube) tiles.insert(tiles.end(), v.begin(), v.end());
    if (ts.kind == SHAPE_QUAD2) {
        // tallest strips first: the last strips to start are the short ones
        auto height = [&](const Tile& t) {
            return std::min(t.r0 + ts.rows - 1, b->grids[(size_t)t.tube].H - 2) - t.r0 + 1;
        };
        std::stable_sort(tiles.begin(), tiles.end(),
                         [&](const Tile& x, const Tile& y) { return height(x) > height(y); });
    }
    Tile* d = nullptr;
    ck(cudaMalloc(&d, tiles.size() * sizeof(Tile)), "cudaMalloc(tiles)");
    const cudaError_t e = cudaMemcpy(d, tiles.data(), tiles.size() * sizeof(Tile), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) cudaFree(d);
    ck(e, "upload tiles");
    *n = (int)tiles.size();
    return d;
}

// The third P, Vx, Vy set of the two-step kernels (zero ring cells; kGuard
// bytes around it for the strips' edge reads) and its two-mass slots.
void ensure_third_set(vs_batch* b) {
    if (b->x_mem) return;
    const size_t slots = align_up(sizeof(TmmState)) + align_up(sizeof(TmmState64));
    size_t total = kGuard;
    for (const TubeDev& t : b->h_tubes) total += 3 * (size_t)t.plane * sizeof(float) + slots;
    total += kGuard;
    ck(cudaMalloc(&b->x_mem, total), "cudaMalloc(third state set)");
    ck(cudaMemset(b->x_mem, 0, total), "zero third state set");
    b->x_bytes = total;
    size_t off = kGuard;
    for (TubeDev& t : b->h_tubes) {
        t.X = reinterpret_cast<float*>(b->x_mem + off);
        off += 3 * (size_t)t.plane * sizeof(float);
        t.tmm_x = reinterpret_cast<TmmState*>(b->x_mem + off);
        t.tmm64_x = reinterpret_cast<TmmState64*>(b->x_mem + off + align_up(sizeof(TmmState)));
        off += slots;
    }
    ck(cudaMemcpy(b->d_tubes, b->h_tubes.data(), b->h_tubes.size() * sizeof(TubeDev), cudaMemcpyHostToDevice),
       "upload tube descriptors");
}

void build_tiles(vs_batch* b, int shape) {
    if (tile_shape(shape).kind == SHAPE_CLUSTER) return;     // the cluster kernel needs no tile list
    if (b->tiles_shape == shape && b->d_tiles) return;
    int n = 0;
    Tile* d = make_tiles(b, shape, &n);
    if (b->d_tiles) cudaFree(b->d_tiles);
    b->d_tiles = d;
    b->ntiles = n;
    b->tiles_shape = shape;
    if (b->graph) { cudaGraphExecDestroy(b->graph); b->graph = nullptr; b->graph_shape = -1; }
    if (tile_shape(shape).kind == SHAPE_QUAD2) {
        // a two-step shape advances an odd step count's last step with the
        // single-step shape of the batch
        if (!b->d_odd_tiles) {
            b->odd_shape = single_step_shape(b);
            b->d_odd_tiles = make_tiles(b, b->odd_shape, &b->n_odd_tiles);
        }
        // and alternates the state with a third set of planes
        ensure_third_set(b);
    }
}

void ensure_graph(vs_batch* b) {
    if (b->graph && b->graph_shape == b->shape) return;
    if (b->graph) { cudaGraphExecDestroy(b->graph); b->graph = nullptr; }
    cudaGraph_t g = nullptr;
    ck(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal), "begin capture");
    cudaError_t err = cudaSuccess;
    const bool two = tile_shape(b->shape).kind == SHAPE_QUAD2;
    const int launches = two ? kChunk / 2 : kChunk;     // a two-step launch advances two steps
    for (int i = 0; i < launches && err == cudaSuccess; ++i)
        err = launch_step(b->shape, b->wall, b->fast, b->d_tubes, b->d_tiles, b->ntiles, b->d_rs, i, b->stream, b->max_pitch);
    if (err == cudaSuccess)
        err = two ? launch_advance2(b->d_rs, kChunk, (kChunk / 2) & 1, b->stream) : launch_advance(b->d_rs, kChunk, b->stream);
    cudaError_t e2 = cudaStreamEndCapture(b->stream, &g);
    ck(err, "capture step launches");
    ck(e2, "end capture");
    cudaError_t e3 = cudaGraphInstantiate(&b->graph, g, 0);
    cudaGraphDestroy(g);
    ck(e3, "instantiate graph");
    b->graph_shape = b->shape;
}

// Descriptors of one tube: every interior cell gets the index of its
// (code, right type, top type) neighbourhood; index 0 is plain air, and ring
// cells keep index 0 (they are never computed).  fast_math: the two tables
// hold the velocity and pressure factors of each neighbourhood
// (FDTDSolver.cu:652-801 with every beta 0 or 1), computed in double and
// rounded once:
//   rden = 1 / (mB + mS); al = mB rden; zo = mS zinv n x_out Nout rden;
//   zi = mS zinv n x_in Nin rden; ce = ew mS rden; g = 1 / (1 + sigma_c)
// (g = 0 on the no-pressure cells of a Dirichlet mouth).
// Reference arithmetic (`exact`): the neighbourhood's factors as the per-cell
// update of the strip kernel forms them in float (velocity_generic and the
// pressure denominator), desc_a = (sP, den_x, den_y, EXD_* bits) and desc_b =
// (mS_x, W_x, mS_y, W_y); more than kDescEntries neighbourhoods leave *ndesc
// = 0 there (the two-step shapes are then not offered) instead of failing.
constexpr int kMaxDescriptors = kDescEntries;
constexpr size_t kDescTableBytes = 2 * kMaxDescriptors * 4 * sizeof(float);

// one rounded float product (the host build does not contract, and the
// volatile keeps the product a separate rounding in any case)
float fprod(float a, float b) {
    volatile float p = a * b;
    return p;
}

void exact_descriptor(const TubeGrid& g, int kc, int tr, int tt, float* a, float* bq) {
    const int tc = kc & CODE_TYPE_MASK;
    const bool zbit = (kc & CODE_ZINV_BIT) != 0;
    const bool bc = beta_one(tc), br = beta_one(tr), bt = beta_one(tt);
    const bool ec = tc == VS_CELL_EXCITATION, er = tr == VS_CELL_EXCITATION, et = tt == VS_CELL_EXCITATION;
    const float sc = g.sigma[tc];
    unsigned bits = (g.dirichlet && tc == VS_CELL_NOPRESSURE) ? EXD_PZERO : 0u;
    // one direction: neighbour beta bn / excitation en / sigma sn, the other
    // neighbour's beta bo, the source directions dirc (cell) and dirn (neighbour)
    auto dir = [&](bool bn, bool en, float sn, bool bo, float dirc, float dirn, float* den, float* mS, float* W) {
        const bool mB = bc && bn;
        const bool src = ec || en;
        *mS = std::max(sc, sn);
        *W = fprod(ec ? 1.0f : 0.0f, dirc) + fprod(en ? 1.0f : 0.0f, dirn);
        *den = (mB ? 1.0f : 0.0f) + *mS;
        unsigned f = 0;
        if (mB) f |= EXD_MB;
        if (src) f |= EXD_SRC;
        if (zbit && !src && bc != bn) f |= EXD_WALL;
        if (bc) f |= EXD_WALL_PC;
        if (bo) f |= EXD_NOUT1;
        return f;
    };
    float denx, mSx, Wx, deny, mSy, Wy;
    bits |= dir(br, er, g.sigma[tr], bt, g.dir[2], g.dir[0], &denx, &mSx, &Wx);
    bits |= dir(bt, et, g.sigma[tt], br, g.dir[3], g.dir[1], &deny, &mSy, &Wy) << EXD_Y_SHIFT;
    a[0] = g.eigen ? sc : 1.0f + sc;
    a[1] = denx;
    a[2] = deny;
    std::memcpy(&a[3], &bits, sizeof(float));
    bq[0] = mSx; bq[1] = Wx; bq[2] = mSy; bq[3] = Wy;
}

void build_descriptors(const TubeGrid& g, std::vector<uint8_t>& desc, std::vector<float>& ta,
                       std::vector<float>& tb, int32_t* ndesc = nullptr, bool exact = false) {
    desc.assign((size_t)g.H * g.pitch, 0);
    ta.assign(4 * kMaxDescriptors, 0.0f);
    tb.assign(4 * kMaxDescriptors, 0.0f);
    std::vector<int> key_of_id;
    std::vector<int> id_of_key(32 * 16 * 16, -1);
    auto key = [](int kc, int tr, int tt) { return (kc * 16 + tr) * 16 + tt; };
    id_of_key[key(VS_CELL_AIR, VS_CELL_AIR, VS_CELL_AIR)] = 0;
    key_of_id.push_back(key(VS_CELL_AIR, VS_CELL_AIR, VS_CELL_AIR));
    auto code_at = [&](int r, int c) { return (int)g.code[(size_t)r * g.pitch + c]; };
    for (int r = 1; r <= g.H - 2; ++r)
        for (int c = 1; c <= g.W - 2; ++c) {
            const int k = key(code_at(r, c) & 0x1f, code_at(r, c + 1) & CODE_TYPE_MASK,
                              code_at(r - 1, c) & CODE_TYPE_MASK);
            if (id_of_key[k] < 0) {
                if ((int)key_of_id.size() >= kMaxDescriptors) {
                    if (exact) {
                        desc.assign(desc.size(), 0);
                        if (ndesc) *ndesc = 0;
                        return;
                    }
                    throw VsFailure{VS_ERR_UNSUPPORTED, "fast_math: more than 256 distinct cell neighbourhoods"};
                }
                id_of_key[k] = (int)key_of_id.size();
                key_of_id.push_back(k);
            }
            desc[(size_t)r * g.pitch + c] = (uint8_t)id_of_key[k];
        }
    if (ndesc) *ndesc = (int32_t)key_of_id.size();
    for (size_t id = 0; id < key_of_id.size(); ++id) {
        const int k = key_of_id[id];
        const int kc = k / 256, tr = (k / 16) % 16, tt = k % 16;
        if (exact) {
            exact_descriptor(g, kc, tr, tt, &ta[4 * id], &tb[4 * id]);
            continue;
        }
        const int tc = kc & CODE_TYPE_MASK;
        const bool zbit = (kc & CODE_ZINV_BIT) != 0;
        const double zinv = zbit ? (double)g.zinv_val : 0.0;
        const bool bc = g.beta[tc] != 0.0f, br = g.beta[tr] != 0.0f, bt = g.beta[tt] != 0.0f;
        const bool ec = tc == VS_CELL_EXCITATION, er = tr == VS_CELL_EXCITATION, et = tt == VS_CELL_EXCITATION;
        // one direction: neighbour type tn (beta bn, excitation en), other neighbour's beta bo
        auto dir = [&](int tn, bool bn, bool en, bool bo, double dc, double dn, double* al, double* zo, double* zi,
                       double* ce) {
            const bool mB = bc && bn;
            const double mS = std::max((double)g.sigma[tc], (double)g.sigma[tn]);
            const double rden = 1.0 / ((mB ? 1.0 : 0.0) + mS);
            const double n = (ec || en) ? 0.0 : 1.0;
            const double nout = bo ? 1.0 : (double)0.707106f;
            *al = mB ? rden : 0.0;
            *zo = (bc && !bn) ? mS * zinv * n * nout * rden : 0.0;
            *zi = (bn && !bc) ? mS * zinv * n * rden : 0.0;
            *ce = ((ec ? dc : 0.0) + (en ? dn : 0.0)) * mS * rden;
        };
        double alx, zox, zix, cex, aly, zoy, ziy, cey;
        dir(tr, br, er, bt, g.dir[2], g.dir[0], &alx, &zox, &zix, &cex);
        dir(tt, bt, et, br, g.dir[3], g.dir[1], &aly, &zoy, &ziy, &cey);
        if (cey != 0.0) throw VsFailure{VS_ERR_UNSUPPORTED, "fast_math: source weight on the y velocity"};
        double gp = 1.0 / (1.0 + (double)g.sigma[tc]);
        if (g.dirichlet && tc == VS_CELL_NOPRESSURE) gp = 0.0;
        float* a = &ta[4 * id];
        float* bq = &tb[4 * id];
        a[0] = (float)alx; a[1] = (float)aly; a[2] = (float)gp; a[3] = (float)cex;
        bq[0] = (float)zox; bq[1] = (float)zix; bq[2] = (float)zoy; bq[3] = (float)ziy;
    }
}

// Paint the maps of every device-built tube (TubeGrid::device_maps) into its
// arena planes with the device map builder, then bring the code planes back
// to the host, where the strip lists, the fast_math descriptors and the
// adjoint's tables are derived from them.  The state planes P[0], P[1] serve
// as the builder's scratch (reset_state zeroes them afterwards).
void build_maps_on_device(vs_batch* b) {
    std::vector<size_t> which;
    for (size_t i = 0; i < b->grids.size(); ++i)
        if (b->grids[i].device_maps) which.push_back(i);
    if (which.empty()) return;
    // per tube: up, down, utop, dbot, seg (L ints each), then the minor axes
    std::vector<size_t> ioff(which.size()), foff(which.size());
    size_t ni = 0, nf = 0;
    for (size_t j = 0; j < which.size(); ++j) {
        const TubeGrid& g = b->grids[which[j]];
        ioff[j] = ni;
        ni += 5 * g.upper.size();
        foff[j] = nf;
        nf += std::max<size_t>(g.minor_m.size(), 1);
    }
    std::vector<int32_t> ibuf(ni);
    std::vector<float> fbuf(nf, 0.0f);
    for (size_t j = 0; j < which.size(); ++j) {
        const TubeGrid& g = b->grids[which[j]];
        const size_t L = g.upper.size();
        int32_t* d = ibuf.data() + ioff[j];
        std::copy(g.upper.begin(), g.upper.end(), d);
        std::copy(g.lower.begin(), g.lower.end(), d + L);
        std::copy(g.upper_top.begin(), g.upper_top.end(), d + 2 * L);
        std::copy(g.lower_bot.begin(), g.lower_bot.end(), d + 3 * L);
        std::copy(g.colseg.begin(), g.colseg.end(), d + 4 * L);
        std::copy(g.minor_m.begin(), g.minor_m.end(), fbuf.begin() + (long)foff[j]);
    }
    int32_t* d_i = nullptr;
    float* d_f = nullptr;
    MapBuild* d_m = nullptr;
    int* d_err = nullptr;
    auto release = [&] {
        cudaFree(d_i);
        cudaFree(d_f);
        cudaFree(d_m);
        cudaFree(d_err);
    };
    try {
        ck(cudaMalloc(&d_i, std::max<size_t>(ni, 1) * sizeof(int32_t)), "cudaMalloc(map columns)");
        ck(cudaMalloc(&d_f, nf * sizeof(float)), "cudaMalloc(map sections)");
        ck(cudaMalloc(&d_m, which.size() * sizeof(MapBuild)), "cudaMalloc(map tubes)");
        ck(cudaMalloc(&d_err, sizeof(int)), "cudaMalloc(map status)");
        ck(cudaMemsetAsync(d_err, 0, sizeof(int), b->stream), "zero map status");
        ck(cudaMemcpyAsync(d_i, ibuf.data(), ni * sizeof(int32_t), cudaMemcpyHostToDevice, b->stream),
           "upload map columns");
        ck(cudaMemcpyAsync(d_f, fbuf.data(), nf * sizeof(float), cudaMemcpyHostToDevice, b->stream),
           "upload map sections");
        std::vector<MapBuild> mb(which.size());
        int64_t max_cells = 0;
        for (size_t j = 0; j < which.size(); ++j) {
            const TubeGrid& g = b->grids[which[j]];
            const TubeDev& t = b->h_tubes[which[j]];
            const vs_params& p = g.src_params;
            const int L = (int)g.upper.size();
            MapBuild& m = mb[j];
            m.H = g.H; m.W = g.W; m.pitch = g.pitch;
            m.sx = g.dims.tube_start_x; m.L = L; m.my = g.dims.tube_mid_y; m.ex = g.dims.tube_end_x;
            m.npc = g.dirichlet ? g.dims.tube_end_x + 1 : -1;
            m.pml = g.pml_layers;
            m.depth = p.fdtd_solver_type != 1 ? MAP_DEPTH_NONE
                      : p.cross_sectional_shape == 2 ? MAP_DEPTH_ELLIPSE : MAP_DEPTH_CIRCLE;
            m.depth_fma = p.depth_fma;
            m.ds = g.dims.ds;
            m.ud = p.uniform_depth_m;
            const int32_t* c = d_i + ioff[j];
            m.up = c; m.down = c + L; m.utop = c + 2 * L; m.dbot = c + 3 * L; m.seg = c + 4 * L;
            m.minor = d_f + foff[j];
            m.dP = const_cast<float*>(t.dP);
            m.dX = const_cast<float*>(t.dX);
            m.dY = const_cast<float*>(t.dY);
            m.code = const_cast<uint8_t*>(t.code);
            m.tmpx = t.P[0];
            m.tmpy = t.P[1];
            max_cells = std::max<int64_t>(max_cells, (int64_t)g.H * g.pitch);
        }
        ck(cudaMemcpyAsync(d_m, mb.data(), mb.size() * sizeof(MapBuild), cudaMemcpyHostToDevice, b->stream),
           "upload map tubes");
        ck(launch_build_maps(d_m, (int)which.size(), max_cells, d_err, b->stream), "map builder");
        int err = 0;
        ck(cudaMemcpyAsync(&err, d_err, sizeof(int), cudaMemcpyDeviceToHost, b->stream), "read map status");
        for (size_t j = 0; j < which.size(); ++j) {
            TubeGrid& g = b->grids[which[j]];
            g.code.resize((size_t)g.H * g.pitch);
            ck(cudaMemcpyAsync(g.code.data(), b->h_tubes[which[j]].code, g.code.size(), cudaMemcpyDeviceToHost,
                               b->stream),
               "read codes");
        }
        ck(cudaStreamSynchronize(b->stream), "map builder sync");
        if (err == VS_ERR_NEGATIVE_SQRT)
            throw VsFailure{VS_ERR_NEGATIVE_SQRT, "negative radicand in the tube depth formula"};
    } catch (...) {
        release();
        throw;
    }
    release();
}

// Host copies of a device-built tube's depth maps (frame-shaped), for the
// paths that edit them on the host.
void fetch_device_maps(vs_batch* b, size_t i) {
    TubeGrid& g = b->grids[i];
    if (!g.device_maps || !g.dP.empty()) return;
    const TubeDev& t = b->h_tubes[i];
    const size_t n = (size_t)g.H * g.W;
    g.dP.resize(n);
    g.dX.resize(n);
    g.dY.resize(n);
    for (auto [dst, src] : {std::pair<float*, const float*>{g.dP.data(), t.dP}, {g.dX.data(), t.dX},
                            {g.dY.data(), t.dY}})
        ck(cudaMemcpy2D(dst, g.W * sizeof(float), src, g.pitch * sizeof(float), g.W * sizeof(float), g.H,
                        cudaMemcpyDeviceToHost),
           "read depth maps");
}

// Depth planes, code bytes (and fast_math descriptors) of tube i, padded to
// the row pitch.
void upload_static_tube(vs_batch* b, size_t i) {
    {
        const TubeGrid& g = b->grids[i];
        const TubeDev& t = b->h_tubes[i];
        const size_t pl = (size_t)g.H * g.pitch;
        std::vector<float> buf(pl);
        auto up = [&](const std::vector<float>& src, const float* dst) {
            std::fill(buf.begin(), buf.end(), 0.0f);
            for (int r = 0; r < g.H; ++r)
                std::memcpy(&buf[(size_t)r * g.pitch], &src[(size_t)r * g.W], g.W * sizeof(float));
            ck(cudaMemcpy((void*)dst, buf.data(), pl * sizeof(float), cudaMemcpyHostToDevice), "upload depth");
        };
        up(g.dP, t.dP);
        up(g.dX, t.dX);
        up(g.dY, t.dY);
        ck(cudaMemcpy((void*)t.code, g.code.data(), g.code.size(), cudaMemcpyHostToDevice), "upload codes");
        if (b->desc) {
            std::vector<uint8_t> desc;
            std::vector<float> ta, tb;
            build_descriptors(g, desc, ta, tb, &b->h_tubes[i].ndesc, !b->fast);
            ck(cudaMemcpy((void*)t.desc, desc.data(), desc.size(), cudaMemcpyHostToDevice), "upload descriptors");
            ck(cudaMemcpy((void*)t.desc_a, ta.data(), ta.size() * sizeof(float), cudaMemcpyHostToDevice),
               "upload descriptor table");
            ck(cudaMemcpy((void*)t.desc_b, tb.data(), tb.size() * sizeof(float), cudaMemcpyHostToDevice),
               "upload descriptor table");
        }
    }
}

// Every tube's read-only block (depth planes, codes, fast_math descriptors
// and tables, from TubeDev::dP on, as laid out in the arena), staged on the
// host in parallel and copied with one transfer per tube.
void upload_static(vs_batch* b) {
    const size_t n = b->grids.size();
    std::vector<std::vector<char>> img(n);
    parallel_for(n, [&](size_t i) {
        const TubeGrid& g = b->grids[i];
        const TubeDev& t = b->h_tubes[i];
        const char* base = reinterpret_cast<const char*>(t.dP);
        auto at = [&](const void* p) { return (size_t)(reinterpret_cast<const char*>(p) - base); };
        const size_t end = b->desc ? at(t.desc_b) + kDescTableBytes / 2 : at(t.code) + align_up((size_t)g.H * g.pitch);
        std::vector<char>& m = img[i];
        if (g.device_maps) {
            // the planes and codes are on the device already: the descriptors only
            if (!b->desc) return;
            m.assign(end, 0);
            std::vector<uint8_t> desc;
            std::vector<float> ta, tb;
            build_descriptors(g, desc, ta, tb, &b->h_tubes[i].ndesc, !b->fast);
            std::memcpy(m.data() + at(t.desc), desc.data(), desc.size());
            std::memcpy(m.data() + at(t.desc_a), ta.data(), ta.size() * sizeof(float));
            std::memcpy(m.data() + at(t.desc_b), tb.data(), tb.size() * sizeof(float));
            return;
        }
        m.assign(end, 0);
        auto plane = [&](const std::vector<float>& src, const float* dst) {
            float* d = reinterpret_cast<float*>(m.data() + at(dst));
            for (int r = 0; r < g.H; ++r)
                std::memcpy(d + (size_t)r * g.pitch, &src[(size_t)r * g.W], g.W * sizeof(float));
        };
        plane(g.dP, t.dP);
        plane(g.dX, t.dX);
        plane(g.dY, t.dY);
        std::memcpy(m.data() + at(t.code), g.code.data(), g.code.size());
        if (b->desc) {
            std::vector<uint8_t> desc;
            std::vector<float> ta, tb;
            build_descriptors(g, desc, ta, tb, &b->h_tubes[i].ndesc, !b->fast);
            std::memcpy(m.data() + at(t.desc), desc.data(), desc.size());
            std::memcpy(m.data() + at(t.desc_a), ta.data(), ta.size() * sizeof(float));
            std::memcpy(m.data() + at(t.desc_b), tb.data(), tb.size() * sizeof(float));
        }
    });
    for (size_t i = 0; i < n; ++i) {
        if (img[i].empty()) continue;
        const TubeDev& t = b->h_tubes[i];
        const char* base = reinterpret_cast<const char*>(t.dP);
        // a device-built tube's image starts at its descriptors
        const size_t from = b->grids[i].device_maps ? (size_t)(reinterpret_cast<const char*>(t.desc) - base) : 0;
        ck(cudaMemcpy((void*)(base + from), img[i].data() + from, img[i].size() - from, cudaMemcpyHostToDevice),
           "upload maps");
    }
    // the descriptor counts (TubeDev::ndesc) are known now
    ck(cudaMemcpy(b->d_tubes, b->h_tubes.data(), n * sizeof(TubeDev), cudaMemcpyHostToDevice),
       "upload tube descriptors");
}

void reset_state(vs_batch* b) {
    // fields, wall state and the two-mass state all restart at zero
    for (size_t i = 0; i < b->grids.size(); ++i)
        ck(cudaMemsetAsync(b->state_base[i], 0, b->state_bytes[i], b->stream), "zero state");
    // the two-step kernels' third set: its ring cells must read as zero
    if (b->x_mem) ck(cudaMemsetAsync(b->x_mem, 0, b->x_bytes, b->stream), "zero third state set");
    RunState rs{};
    rs.wait_polls = b->wait_polls;
    ck(cudaMemcpyAsync(b->d_rs, &rs, sizeof(rs), cudaMemcpyHostToDevice, b->stream), "reset run state");
    ck(cudaStreamSynchronize(b->stream), "reset sync");
    b->step = 0;
}

void create_batch(int n, const vs_params* params, const vs_geometry* geoms, vs_batch* b) {
    ck(cudaGetDevice(&b->device), "cudaGetDevice");
    b->grids.resize(n);
    // tubes the device map builder covers get only their per-column data on
    // the host; their maps are painted on the device (build_maps_on_device)
    parallel_for((size_t)n, [&](size_t i) {
        if (device_buildable(&params[i])) build_tube_columns(&params[i], geoms ? &geoms[i] : nullptr, b->grids[i], 0);
        else build_tube(&params[i], geoms ? &geoms[i] : nullptr, b->grids[i], 0);
        std::memcpy(&b->grids[i].src_params, &params[i], sizeof(vs_params));
    });
    // arena layout: per tube, planes of H*pitch floats (+ codes) + two-mass
    // state, with kGuard bytes before the first and after the last tube: the
    // step kernel reads one element before and up to 29 after a plane
    for (const TubeGrid& g : b->grids) {
        b->wall = b->wall || g.wall_ode;
        b->max_pitch = std::max(b->max_pitch, g.pitch);
    }
    b->fast = params[0].fast_math != 0;
    for (int i = 1; i < n; ++i)
        if ((params[i].fast_math != 0) != b->fast)
            throw VsFailure{VS_ERR_INVALID_ARG, "every tube of a batch needs the same fast_math"};
    // descriptor planes for the kernels that read them: fast_math, and the
    // two-step kernel in the reference arithmetic (no coupled wall)
    b->desc = b->fast || !b->wall;
    size_t total = kGuard;
    std::vector<size_t> base(n);
    for (int i = 0; i < n; ++i) {
        const TubeGrid& g = b->grids[i];
        base[i] = total;
        const size_t pl = align_up((size_t)g.H * g.pitch * sizeof(float));
        total += pl * planes_per_tube(g) + align_up((size_t)g.H * g.pitch) + align_up(2 * sizeof(TmmState)) +
                 align_up(2 * sizeof(TmmState64));
        if (b->desc) total += align_up((size_t)g.H * g.pitch) + kDescTableBytes;
    }
    total += kGuard;
    b->arena_bytes = total;
    ck(cudaMalloc(&b->arena, total), "cudaMalloc(arena)");
    b->h_tubes.resize(n);
    b->src_len.assign(n, 0);
    b->state_base.assign(n, nullptr);
    b->state_bytes.assign(n, 0);
    for (int i = 0; i < n; ++i) {
        const TubeGrid& g = b->grids[i];
        TubeDev& t = b->h_tubes[i];
        std::memset(&t, 0, sizeof(t));
        const size_t pl = align_up((size_t)g.H * g.pitch * sizeof(float));
        char* p = b->arena + base[i];
        auto next = [&](size_t bytes) { char* q = p; p += bytes; return q; };
        // mutable state first (one memset resets it), read-only planes after
        b->state_base[i] = p;
        for (int k = 0; k < 2; ++k) t.P[k] = (float*)next(pl);
        for (int k = 0; k < 2; ++k) t.Vx[k] = (float*)next(pl);
        for (int k = 0; k < 2; ++k) t.Vy[k] = (float*)next(pl);
        if (g.wall_ode) {
            for (int k = 0; k < 2; ++k) t.w[k] = (float*)next(pl);
            for (int k = 0; k < 2; ++k) t.z[k] = (float*)next(pl);
        }
        t.tmm = (TmmState*)next(align_up(2 * sizeof(TmmState)));
        t.tmm64 = (TmmState64*)next(align_up(2 * sizeof(TmmState64)));
        b->state_bytes[i] = (size_t)(p - b->state_base[i]);
        t.dP = (const float*)next(pl);
        t.dX = (const float*)next(pl);
        t.dY = (const float*)next(pl);
        t.code = (const uint8_t*)next(align_up((size_t)g.H * g.pitch));
        if (b->desc) {
            t.desc = (const uint8_t*)next(align_up((size_t)g.H * g.pitch));
            t.desc_a = (const float4*)next(kDescTableBytes / 2);
            t.desc_b = (const float4*)next(kDescTableBytes / 2);    // desc_a + kDescEntries
        }
        t.H = g.H; t.W = g.W; t.pitch = g.pitch;
        t.plane = (int64_t)(pl / sizeof(float));
        t.flags = (g.dirichlet ? TUBE_DIRICHLET : 0) | (g.eigen ? TUBE_EIGEN : 0) |
                  (g.tmm ? TUBE_TMM : 0) | (g.wall_ode ? TUBE_WALL_ODE : 0) | (g.tmm64 ? TUBE_TMM64 : 0);
        t.lis_x = g.dims.listener_x; t.lis_y = g.dims.listener_y;
        t.exc_x = g.dims.excitation_x; t.exc_y = g.dims.excitation_y;
        t.K1 = g.K1; t.K2 = g.K2; t.bcoef = g.bcoef; t.zinv = g.zinv_val;
        t.dt = g.dt; t.Mw = g.Mw; t.Bw = g.Bw; t.Kw = g.Kw; t.cpl = g.cpl;
        t.dir0 = g.dir[0]; t.dir1 = g.dir[1]; t.dir2 = g.dir[2]; t.dir3 = g.dir[3];
        for (int k = 0; k < 13; ++k) t.sigma[k] = g.sigma[k];
        t.tmmc = g.tmmc;
        t.tmmd = g.tmmd;
        t.tmmx = g.tmmx;
    }
    ck(cudaMalloc(&b->d_tubes, n * sizeof(TubeDev)), "cudaMalloc(tubes)");
    ck(cudaMalloc(&b->d_rs, sizeof(RunState)), "cudaMalloc(run state)");
    ck(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking), "cudaStreamCreate");
    b->own_stream = true;
    int64_t need = 0;
    for (const TubeGrid& g : b->grids) need = std::max<int64_t>(need, g.dims.num_steps);
    upload_sources(b, need);
    build_maps_on_device(b);
    upload_static(b);
    reset_state(b);
    // small grids (a single tube) need short strips to spread over the SMs
    b->shape = default_shape(b);
}

// Issue `count` steps from the device step counter (graph chunks of kChunk
// plus direct launches), RunState already set with bsel = 0.  With a
// two-step shape the launches alternate between the parity set and the third
// set; an odd number of them is followed by a copy back, and an odd step
// count ends with one launch of the batch's single-step shape, so the state
// of the final step is in its parity set (bsel = 0) when the call returns.
void issue_steps(vs_batch* b, int64_t count) {
    if (tile_shape(b->shape).kind == SHAPE_CLUSTER) {
        ck(launch_cluster_run(b->d_tubes, b->d_rs, count, b->fast, b->cluster, b->stream, (int)b->grids.size()),
           "cluster launch");
        return;
    }
    const bool two = tile_shape(b->shape).kind == SHAPE_QUAD2;
    int64_t done = 0;
    if (count >= kChunk) {
        ensure_graph(b);
        for (; done + kChunk <= count; done += kChunk) ck(cudaGraphLaunch(b->graph, b->stream), "graph launch");
    }
    const int rem = (int)(count - done);
    if (!two) {
        for (int i = 0; i < rem; ++i)
            ck(launch_step(b->shape, b->wall, b->fast, b->d_tubes, b->d_tiles, b->ntiles, b->d_rs, i, b->stream,
                           b->max_pitch),
               "step launch");
        if (rem) ck(launch_advance(b->d_rs, rem, b->stream), "advance");
        return;
    }
    const int pairs = rem / 2;
    for (int i = 0; i < pairs; ++i)
        ck(launch_step(b->shape, b->wall, b->fast, b->d_tubes, b->d_tiles, b->ntiles, b->d_rs, i, b->stream,
                       b->max_pitch),
           "two-step launch");
    if (pairs) ck(launch_advance2(b->d_rs, 2 * pairs, pairs & 1, b->stream), "advance");
    if (pairs & 1) {
        int64_t max_plane = 0;
        for (const TubeDev& t : b->h_tubes) max_plane = std::max<int64_t>(max_plane, t.plane);
        ck(launch_copy_back(b->d_tubes, (int)b->grids.size(), (int)max_plane, b->d_rs, b->stream), "copy back");
        ck(launch_advance2(b->d_rs, 0, 1, b->stream), "advance");
    }
    if (rem & 1) {
        ck(launch_step(b->odd_shape, b->wall, b->fast, b->d_tubes, b->d_odd_tiles, b->n_odd_tiles, b->d_rs, 0,
                       b->stream, b->max_pitch),
           "step launch");
        ck(launch_advance(b->d_rs, 1, b->stream), "advance");
    }
}

void run_batch(vs_batch* b, int64_t steps, float* traces, int on_device) {
    const int n = (int)b->grids.size();
    if (b->shape < 0) b->shape = default_shape(b);
    build_tiles(b, b->shape);
    upload_sources(b, b->step + steps);
    const int64_t need = (int64_t)n * steps;
    if (need > b->trace_cap) {
        if (b->d_trace) cudaFree(b->d_trace);
        b->d_trace = nullptr;
        ck(cudaMalloc(&b->d_trace, need * sizeof(float)), "cudaMalloc(trace)");
        b->trace_cap = need;
    }
    RunState rs{};
    rs.wait_polls = b->wait_polls;
    rs.step = b->step;
    rs.run_start = b->step;
    rs.trace = b->d_trace;
    rs.trace_stride = steps;
    ck(cudaMemcpyAsync(b->d_rs, &rs, sizeof(rs), cudaMemcpyHostToDevice, b->stream), "set run state");
    issue_steps(b, steps);
    b->step += steps;
    if (traces) {
        ck(cudaMemcpyAsync(traces, b->d_trace, need * sizeof(float),
                           on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, b->stream),
           "copy traces");
    }
    ck(cudaStreamSynchronize(b->stream), "run sync");
    int32_t dev_error = 0;
    ck(cudaMemcpy(&dev_error, &b->d_rs->error, sizeof(dev_error), cudaMemcpyDeviceToHost), "read run status");
    if (dev_error == VS_ERR_NONFINITE) throw VsFailure{dev_error, "non-finite listener pressure"};
    if (dev_error != 0) throw VsFailure{dev_error, "a bounded device wait gave up; the state is not valid"};
    if (traces && !on_device) {
        for (int64_t i = 0; i < need; ++i)
            if (!std::isfinite(traces[i])) throw VsFailure{VS_ERR_NONFINITE, "non-finite listener pressure"};
    }
}

// ---- adjoint -------------------------------------------------------------

void check_adjoint_support(const vs_batch* b) {
    for (const TubeGrid& g : b->grids) {
        if (g.wall_ode) throw VsFailure{VS_ERR_UNSUPPORTED, "adjoint of the coupled wall oscillator is not implemented"};
    }
}

void copy_state(vs_batch* b, int k, bool save) {
    size_t off = 0;
    for (size_t i = 0; i < b->grids.size(); ++i) {
        char* slot = b->ckpt + (size_t)k * b->ckpt_stride + off;
        ck(cudaMemcpyAsync(save ? slot : b->state_base[i], save ? b->state_base[i] : slot, b->state_bytes[i],
                           cudaMemcpyDeviceToDevice, b->stream),
           save ? "save checkpoint" : "restore checkpoint");
        off += b->state_bytes[i];
    }
}

void forward_checkpointed(vs_batch* b, int64_t steps, int every, float* traces, bool traces_on_device = false) {
    check_adjoint_support(b);
    const int n = (int)b->grids.size();
    if (b->shape < 0) b->shape = default_shape(b);
    build_tiles(b, b->shape);
    reset_state(b);
    upload_sources(b, steps);
    const int64_t need = (int64_t)n * steps;
    if (need > b->trace_cap) {
        if (b->d_trace) cudaFree(b->d_trace);
        b->d_trace = nullptr;
        ck(cudaMalloc(&b->d_trace, need * sizeof(float)), "cudaMalloc(trace)");
        b->trace_cap = need;
    }
    const int count = (int)((steps + every - 1) / every);
    size_t stride = 0;
    for (size_t bytes : b->state_bytes) stride += bytes;
    if (b->ckpt) { cudaFree(b->ckpt); b->ckpt = nullptr; }
    ck(cudaMalloc(&b->ckpt, stride * count), "cudaMalloc(checkpoints)");
    b->ckpt_stride = stride;
    RunState rs{};
    rs.wait_polls = b->wait_polls;
    rs.trace = b->d_trace;
    rs.trace_stride = steps;
    ck(cudaMemcpyAsync(b->d_rs, &rs, sizeof(rs), cudaMemcpyHostToDevice, b->stream), "set run state");
    for (int k = 0; k < count; ++k) {
        copy_state(b, k, true);
        issue_steps(b, std::min<int64_t>(every, steps - (int64_t)k * every));
    }
    b->step = steps;
    b->ck_steps = steps;
    b->ck_every = every;
    b->ck_count = count;
    if (traces)
        ck(cudaMemcpyAsync(traces, b->d_trace, need * sizeof(float),
                           traces_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, b->stream),
           "copy traces");
    ck(cudaStreamSynchronize(b->stream), "forward sync");
}

// Velocities the excitation flow enters, per tube with the two-mass source:
// lambda-plane offset and dV'/d exeV = ew mS / (mB + mS) (the source term of
// FDTDEngineCPU.cpp:364-410 divided by the velocity denominator).
void excitation_list(const TubeGrid& g, int64_t plane, std::vector<int32_t>& off, std::vector<float>& coef) {
    off.clear();
    coef.clear();
    if (!g.tmm) return;
    const int ex = g.dims.excitation_x;
    auto type = [&](int r, int c) { return g.code[(size_t)r * g.pitch + c] & CODE_TYPE_MASK; };
    for (int r = 1; r <= g.H - 2; ++r)
        for (int c = std::max(ex - 1, 1); c <= std::min(ex, g.W - 2); ++c) {
            const int tc = type(r, c), tr = type(r, c + 1), tt = type(r - 1, c);
            const float ec = tc == VS_CELL_EXCITATION, er = tr == VS_CELL_EXCITATION, et = tt == VS_CELL_EXCITATION;
            const float ewx = ec * g.dir[2] + er * g.dir[0], ewy = ec * g.dir[3] + et * g.dir[1];
            const int64_t o = (int64_t)r * g.pitch + c;
            if (ewx != 0.0f) {
                const float mb = std::min(g.beta[tc], g.beta[tr]), ms = std::max(g.sigma[tc], g.sigma[tr]);
                off.push_back((int32_t)(plane + o));
                coef.push_back(ewx * ms / (mb + ms));
            }
            if (ewy != 0.0f) {
                const float mb = std::min(g.beta[tc], g.beta[tt]), ms = std::max(g.sigma[tc], g.sigma[tt]);
                off.push_back((int32_t)(2 * plane + o));
                coef.push_back(ewy * ms / (mb + ms));
            }
        }
}

// Adjoint coefficients of one velocity component (the transposed forward
// update, FDTDEngineCPU.cpp:364-410 with calculateSolverCoefficients,
// FDTDSolver.cu:652-801): V' = al V + a P'_c - b P'_nbr + source, and
// dV'/dzinv = zc_out P'_c - zc_in P'_nbr.  dirx: Vx of a cell with code kc,
// right neighbour kr, top neighbour kt; else Vy (neighbour = the top cell).
struct AdjCoef {
    float al, a, b, zc_out, zc_in;
};

AdjCoef adjoint_direction(const TubeGrid& g, bool dirx, int kc, int kr, int kt) {
    static const float air_n[4] = {0.0f, 1.0f, 1.0f, 0.707106f};    // DeviceSymbols.cu:20-21
    static const float wall_n[4] = {1.0f, 1.0f, 1.0f, 0.0f};
    const int tc = kc & CODE_TYPE_MASK, tr = kr & CODE_TYPE_MASK, tt = kt & CODE_TYPE_MASK;
    const float bc = g.beta[tc], br = g.beta[tr], bt = g.beta[tt];
    const int lut = (br == 0.0f ? 2 : 0) + (bt == 0.0f ? 1 : 0);
    const float nout = air_n[lut] * bc, nin = wall_n[lut] * (1.0f - bc);
    const int tn = dirx ? tr : tt;
    const float bn = dirx ? br : bt;
    const float mB = std::min(bc, bn), mS = std::max(g.sigma[tc], g.sigma[tn]);
    const float bxy = mB != 0.0f ? g.bcoef : 0.0f;
    const int ec = tc == VS_CELL_EXCITATION, en = tn == VS_CELL_EXCITATION;
    const float nn = (float)((1 - ec) * (1 - en));
    const float xout = bc * (1.0f - bn), xin = bn * (1.0f - bc);
    const bool zc = (kc & CODE_ZINV_BIT) != 0;
    const float z = zc ? g.zinv_val : 0.0f;
    const float gi = 1.0f / (mB + mS);
    AdjCoef v;
    v.al = mB * gi;
    v.a = gi * (bxy + mS * z * nn * xout * nout);
    v.b = gi * (bxy + mS * z * nn * xin * nin);
    v.zc_out = zc ? gi * mS * nn * xout * nout : 0.0f;
    v.zc_in = zc ? gi * mS * nn * xin * nin : 0.0f;
    return v;
}

// Neighbourhood descriptors of a tube's interior cells, (code, right type,
// top type), and the adjoint coefficient table (three float4 each, see
// AdjTube); at most kMaxDescriptors distinct neighbourhoods.
void adjoint_coefficients(const TubeGrid& g, std::vector<uint8_t>& desc, std::vector<float>& tab) {
    desc.assign((size_t)g.H * g.pitch, 0);
    tab.assign(12 * kMaxDescriptors, 0.0f);
    std::vector<int> key_of_id, id_of_key(32 * 16 * 16, -1);
    auto code_at = [&](int r, int c) { return (int)g.code[(size_t)r * g.pitch + c]; };
    for (int r = 1; r <= g.H - 2; ++r)
        for (int c = 1; c <= g.W - 2; ++c) {
            const int k = ((code_at(r, c) & 0x1f) * 16 + (code_at(r, c + 1) & CODE_TYPE_MASK)) * 16 +
                          (code_at(r - 1, c) & CODE_TYPE_MASK);
            if (id_of_key[k] < 0) {
                if ((int)key_of_id.size() >= kMaxDescriptors)
                    throw VsFailure{VS_ERR_UNSUPPORTED, "adjoint: more than 256 distinct cell neighbourhoods"};
                id_of_key[k] = (int)key_of_id.size();
                key_of_id.push_back(k);
            }
            desc[(size_t)r * g.pitch + c] = (uint8_t)id_of_key[k];
        }
    for (size_t id = 0; id < key_of_id.size(); ++id) {
        const int k = key_of_id[id];
        const int kc = k / 256, tr = (k / 16) % 16, tt = k % 16;
        const AdjCoef x = adjoint_direction(g, true, kc, tr, tt);
        const AdjCoef y = adjoint_direction(g, false, kc, tr, tt);
        const int tc = kc & CODE_TYPE_MASK;
        float* e = &tab[12 * id];
        e[0] = x.a; e[1] = y.a; e[2] = x.b; e[3] = y.b;
        e[4] = x.al; e[5] = y.al; e[6] = 1.0f + g.sigma[tc];
        e[7] = (g.dirichlet && tc == VS_CELL_NOPRESSURE) ? 1.0f : 0.0f;
        e[8] = x.zc_out; e[9] = x.zc_in; e[10] = y.zc_out; e[11] = y.zc_in;
    }
    tab.resize(12 * std::max<size_t>(key_of_id.size(), 1));     // the descriptors in use
}

void capture(vs_batch* b, cudaGraphExec_t* out, const char* what, const std::function<cudaError_t(int)>& launch,
             int count) {
    if (*out) { cudaGraphExecDestroy(*out); *out = nullptr; }
    cudaGraph_t g = nullptr;
    ck(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal), "begin capture");
    cudaError_t err = cudaSuccess;
    for (int i = 0; i < count && err == cudaSuccess; ++i) err = launch(i);
    cudaError_t e2 = cudaStreamEndCapture(b->stream, &g);
    ck(err, what);
    ck(e2, "end capture");
    cudaError_t e3 = cudaGraphInstantiate(out, g, 0);
    cudaGraphDestroy(g);
    ck(e3, "instantiate graph");
}

void run_adjoint(vs_batch* b, const float* gtrace, float* gdP, float* gdX, float* gdY, float* gz,
                 bool gtrace_on_device = false) {
    if (b->ck_steps <= 0) throw VsFailure{VS_ERR_INVALID_ARG, "run vs_batch_forward_ckpt before vs_batch_adjoint"};
    check_adjoint_support(b);
    const int n = (int)b->grids.size();
    const int64_t steps = b->ck_steps;
    const int K = b->ck_every;
    // the form of this call's reverse steps.  Automatic: two-step strips of 8
    // rows when the batch has table sources only and gives every SM at least
    // four strips, else tiles (the strips' row march is latency-bound with
    // few warps).  The two-step strips need table sources (the two-mass
    // reverse step runs beside each single step), so a two-mass batch runs
    // them one step per launch.
    bool any_tmm = false;
    int64_t strips8 = 0;
    for (const TubeGrid& g : b->grids) {
        any_tmm = any_tmm || g.tmm;
        strips8 += adjoint_strips(g.H, g.W, ADJ_FORM_STRIPS2, 8);
    }
    int sms = 148;
    ck(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device), "device attribute");
    int form = b->adj_form;
    if (form == ADJ_FORM_AUTO) form = (!any_tmm && strips8 >= 4 * (int64_t)sms) ? ADJ_FORM_STRIPS2 : ADJ_FORM_TILES;
    if (form == ADJ_FORM_STRIPS2 && any_tmm) form = ADJ_FORM_STRIPS;
    const int rows = b->adj_rows ? b->adj_rows : (form == ADJ_FORM_STRIPS2 ? 8 : 4);
    // a single tube that steps on the cluster kernel (register form) recomputes
    // each segment with one cluster launch that stores every step's state;
    // otherwise, with fast_math, a full segment (K even) is recomputed two
    // steps per launch by the two-step kernel, which needs the third state set
    const bool hist_cluster = n == 1 && tile_shape(b->shape).kind == SHAPE_CLUSTER && b->cluster.form != 0;
    const bool hist_two = !hist_cluster && b->fast && K % 2 == 0;
    if (hist_two) ensure_third_set(b);
    // device memory per tube, all zeroed per call: history (K+1 slots x 3
    // planes), lambda (2 x 3 planes), gradients (4 double planes) and, with
    // the two-mass source, its state history (K+1) and adjoint (6)
    std::vector<size_t> off(n), zero_off(n);
    size_t total = 0;
    int max_tiles = 0, max_plane = 0;
    for (int i = 0; i < n; ++i) {
        const size_t pe = (size_t)b->h_tubes[i].plane;
        const TubeGrid& g = b->grids[i];
        off[i] = total;
        total += align_up(pe * sizeof(float) * 3 * (size_t)(K + 1));
        zero_off[i] = total;
        total += align_up(pe * sizeof(float) * 6) + align_up(pe * sizeof(double) * 4);
        if (g.tmm) total += align_up((size_t)(K + 1) * 6 * sizeof(double)) + align_up(8 * sizeof(double));
        const int tiles = ((g.W - 2 + kAdjTileW - 1) / kAdjTileW) * ((g.H - 2 + kAdjTileH - 1) / kAdjTileH);
        const int blocks = form == ADJ_FORM_TILES ? tiles : adjoint_strip_blocks(adjoint_strips(g.H, g.W, form, rows));
        max_tiles = std::max(max_tiles, blocks);
        max_plane = std::max(max_plane, g.H * g.pitch);
    }
    if (total != b->adj_bytes) {
        if (b->adj_mem) { cudaFree(b->adj_mem); b->adj_mem = nullptr; b->adj_bytes = 0; }
        ck(cudaMalloc(&b->adj_mem, total), "cudaMalloc(adjoint)");
        b->adj_bytes = total;
    }
    // everything starts at zero: lambda, the accumulators and the history,
    // whose ring and row padding the history-capturing steps never write
    // (the forward keeps those cells at zero; the reverse steps read them as
    // neighbours of edge cells)
    ck(cudaMemsetAsync(b->adj_mem, 0, total, b->stream), "zero adjoint");
    if ((int64_t)n * steps > b->gtrace_cap) {
        if (b->d_gtrace) { cudaFree(b->d_gtrace); b->d_gtrace = nullptr; }
        ck(cudaMalloc(&b->d_gtrace, (size_t)n * steps * sizeof(float)), "cudaMalloc(trace gradient)");
        b->gtrace_cap = (int64_t)n * steps;
    }
    ck(cudaMemcpyAsync(b->d_gtrace, gtrace, (size_t)n * steps * sizeof(float),
                       gtrace_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, b->stream),
       "upload trace gradient");
    // excitation lists, neighbourhood descriptors and coefficient tables
    std::vector<std::vector<int32_t>> eoff(n);
    std::vector<std::vector<float>> ecoef(n);
    std::vector<std::vector<uint8_t>> adesc(n);
    std::vector<std::vector<float>> atab(n);
    size_t exc_total = 0;
    for (int i = 0; i < n; ++i) {
        excitation_list(b->grids[i], b->h_tubes[i].plane, eoff[i], ecoef[i]);
        adjoint_coefficients(b->grids[i], adesc[i], atab[i]);
        exc_total += align_up(eoff[i].size() * sizeof(int32_t)) + align_up(ecoef[i].size() * sizeof(float)) +
                     align_up(adesc[i].size()) + align_up(atab[i].size() * sizeof(float));
    }
    if (exc_total > b->exc_bytes) {
        if (b->d_exc) { cudaFree(b->d_exc); b->d_exc = nullptr; b->exc_bytes = 0; }
        ck(cudaMalloc(&b->d_exc, exc_total), "cudaMalloc(excitation lists)");
        b->exc_bytes = exc_total;
    }
    std::vector<AdjTube> adj(n);
    size_t eo = 0;
    for (int i = 0; i < n; ++i) {
        const TubeGrid& g = b->grids[i];
        const size_t pe = (size_t)b->h_tubes[i].plane;
        b->h_tubes[i].hist = reinterpret_cast<float*>(b->adj_mem + off[i]);
        float* lam = reinterpret_cast<float*>(b->adj_mem + zero_off[i]);
        adj[i].lam[0] = lam;
        adj[i].lam[1] = lam + 3 * pe;
        char* gbase = b->adj_mem + zero_off[i] + align_up(pe * sizeof(float) * 6);
        double* gp = reinterpret_cast<double*>(gbase);
        adj[i].gP = gp;
        adj[i].gX = gp + pe;
        adj[i].gY = gp + 2 * pe;
        adj[i].gZ = gp + 3 * pe;
        adj[i].gtrace = b->d_gtrace + (size_t)i * steps;
        adj[i].lam_tmm = nullptr;
        b->h_tubes[i].tmm_hist = nullptr;
        if (g.tmm) {
            char* tbase = gbase + align_up(pe * sizeof(double) * 4);
            b->h_tubes[i].tmm_hist = reinterpret_cast<double*>(tbase);
            adj[i].lam_tmm = reinterpret_cast<double*>(tbase + align_up((size_t)(K + 1) * 6 * sizeof(double)));
        }
        const size_t nb = eoff[i].size();
        int32_t* d_off = reinterpret_cast<int32_t*>(b->d_exc + eo);
        eo += align_up(nb * sizeof(int32_t));
        float* d_coef = reinterpret_cast<float*>(b->d_exc + eo);
        eo += align_up(nb * sizeof(float));
        if (nb) {
            ck(cudaMemcpyAsync(d_off, eoff[i].data(), nb * sizeof(int32_t), cudaMemcpyHostToDevice, b->stream),
               "upload excitation offsets");
            ck(cudaMemcpyAsync(d_coef, ecoef[i].data(), nb * sizeof(float), cudaMemcpyHostToDevice, b->stream),
               "upload excitation coefficients");
        }
        uint8_t* d_desc = reinterpret_cast<uint8_t*>(b->d_exc + eo);
        eo += align_up(adesc[i].size());
        float* d_tab = reinterpret_cast<float*>(b->d_exc + eo);
        eo += align_up(atab[i].size() * sizeof(float));
        ck(cudaMemcpyAsync(d_desc, adesc[i].data(), adesc[i].size(), cudaMemcpyHostToDevice, b->stream),
           "upload adjoint descriptors");
        ck(cudaMemcpyAsync(d_tab, atab[i].data(), atab[i].size() * sizeof(float), cudaMemcpyHostToDevice,
                           b->stream),
           "upload adjoint coefficient table");
        adj[i].desc = d_desc;
        adj[i].tab = reinterpret_cast<const float4*>(d_tab);
        adj[i].ndesc = (int32_t)(atab[i].size() / 12);
        adj[i].exc_off = d_off;
        adj[i].exc_coef = d_coef;
        adj[i].n_exc = (int32_t)nb;
        adj[i].tiles = ((g.W - 2 + kAdjTileW - 1) / kAdjTileW) * ((g.H - 2 + kAdjTileH - 1) / kAdjTileH);
        adj[i].strips = adjoint_strips(g.H, g.W, form, rows);
        const int blocks = form == ADJ_FORM_TILES ? adj[i].tiles : adjoint_strip_blocks(adj[i].strips);
        if (g.tmm) max_tiles = std::max(max_tiles, blocks + 1);
    }
    if (!b->d_adj) ck(cudaMalloc(&b->d_adj, n * sizeof(AdjTube)), "cudaMalloc(adjoint descriptors)");
    if (!b->d_adjrun) ck(cudaMalloc(&b->d_adjrun, sizeof(AdjRun)), "cudaMalloc(adjoint run state)");
    ck(cudaMemcpyAsync(b->d_adj, adj.data(), n * sizeof(AdjTube), cudaMemcpyHostToDevice, b->stream),
       "upload adjoint descriptors");
    ck(cudaMemcpyAsync(b->d_tubes, b->h_tubes.data(), n * sizeof(TubeDev), cudaMemcpyHostToDevice, b->stream),
       "upload tube descriptors");
    // strip list of the history-capturing step kernel (static per batch)
    int64_t cells = 0;
    for (const TubeGrid& g : b->grids) cells += (int64_t)(g.H - 2) * (g.W - 2);
    const int hshape = history_shape(cells, b->fast);
    if (!b->d_hist_tiles) b->d_hist_tiles = make_tiles(b, hshape, &b->n_hist_tiles);
    auto hist_step = [&](int j) {
        return launch_step_history(hshape, b->d_tubes, b->d_hist_tiles, b->n_hist_tiles, b->d_rs, j, b->stream);
    };
    const int h2shape = hist_two ? history2_shape(cells) : -1;
    if (hist_two && !b->d_hist2_tiles) b->d_hist2_tiles = make_tiles(b, h2shape, &b->n_hist2_tiles);
    auto hist2_step = [&](int j) {
        return launch_step_history2(h2shape, b->d_tubes, b->d_hist2_tiles, b->n_hist2_tiles, b->d_rs, j, b->stream);
    };
    // reverse launches of a segment of len steps: one per step, or in the
    // two-step form len / 2 two-step launches and, for odd len, one single
    // step last; launch j reads lambda parity q0 ^ (j & 1)
    const bool two = form == ADJ_FORM_STRIPS2;
    auto launches = [&](int len) { return two ? len / 2 + (len & 1) : len; };
    auto adj_launch = [&](int j, int len) {
        if (two && 2 * j + 1 < len)
            return launch_adjoint_step(b->d_tubes, b->d_adj, n, max_tiles, b->d_adjrun, 2 * j, j, b->stream,
                                       ADJ_FORM_STRIPS2, rows);
        const int local = two ? 2 * j : j;
        return launch_adjoint_step(b->d_tubes, b->d_adj, n, max_tiles, b->d_adjrun, local, j, b->stream,
                                   two ? ADJ_FORM_STRIPS : form, rows);
    };
    if (b->adj_graph_len != K || b->adj_graph_form != form || b->adj_graph_rows != rows || !b->hist_graph ||
        !b->adj_graph) {
        if (hist_two) capture(b, &b->hist_graph, "capture history steps", hist2_step, K / 2);
        else capture(b, &b->hist_graph, "capture history steps", hist_step, K);
        capture(b, &b->adj_graph, "capture reverse steps", [&](int j) { return adj_launch(j, K); }, launches(K));
        b->adj_graph_len = K;
        b->adj_graph_form = form;
        b->adj_graph_rows = rows;
    }
    int q = 0;                    // lambda parity holding the adjoint of the later state
    // events around each segment's recomputation and reverse steps, for the
    // time split vs_batch_adjoint_times reports
    std::vector<cudaEvent_t> ev(3 * (size_t)b->ck_count, nullptr);
    for (cudaEvent_t& e : ev) ck(cudaEventCreate(&e), "event");
    for (int k = b->ck_count - 1; k >= 0; --k) {
        const int64_t start = (int64_t)k * K;
        const int len = (int)std::min<int64_t>(K, steps - start);
        copy_state(b, k, false);
        RunState rs{};
        rs.wait_polls = b->wait_polls;
        rs.step = start;
        rs.run_start = start;
        rs.trace = b->d_trace;
        rs.trace_stride = len;
        ck(cudaMemcpyAsync(b->d_rs, &rs, sizeof(rs), cudaMemcpyHostToDevice, b->stream), "set run state");
        const AdjRun ar{start, len, q};
        ck(cudaMemcpyAsync(b->d_adjrun, &ar, sizeof(ar), cudaMemcpyHostToDevice, b->stream), "set adjoint run");
        ck(cudaEventRecord(ev[3 * k], b->stream), "event");
        ck(launch_history_seed(b->d_tubes, n, max_plane, (int)(start & 1), b->stream), "history seed");
        if (hist_cluster) {
            ck(launch_cluster_run(b->d_tubes, b->d_rs, len, b->fast, b->cluster, b->stream), "history (cluster)");
            ck(cudaEventRecord(ev[3 * k + 1], b->stream), "event");
            if (len == K) ck(cudaGraphLaunch(b->adj_graph, b->stream), "reverse graph");
            else
                for (int j = 0; j < launches(len); ++j) ck(adj_launch(j, len), "adjoint step");
        } else if (len == K) {
            ck(cudaGraphLaunch(b->hist_graph, b->stream), "history graph");
            ck(cudaEventRecord(ev[3 * k + 1], b->stream), "event");
            ck(cudaGraphLaunch(b->adj_graph, b->stream), "reverse graph");
        } else {
            for (int j = 0; j < len; ++j) ck(hist_step(j), "history step");
            ck(cudaEventRecord(ev[3 * k + 1], b->stream), "event");
            for (int j = 0; j < launches(len); ++j) ck(adj_launch(j, len), "adjoint step");
        }
        ck(cudaEventRecord(ev[3 * k + 2], b->stream), "event");
        q ^= launches(len) & 1;
    }
    ck(cudaStreamSynchronize(b->stream), "adjoint sync");
    b->adj_recompute_ms = 0.0f;
    b->adj_reverse_ms = 0.0f;
    for (int k = 0; k < b->ck_count; ++k) {
        float a = 0.0f, r = 0.0f;
        ck(cudaEventElapsedTime(&a, ev[3 * k], ev[3 * k + 1]), "elapsed");
        ck(cudaEventElapsedTime(&r, ev[3 * k + 1], ev[3 * k + 2]), "elapsed");
        b->adj_recompute_ms += a;
        b->adj_reverse_ms += r;
    }
    for (cudaEvent_t e : ev) cudaEventDestroy(e);
    // gradients to the caller, frame by frame (unpadded)
    size_t cell_off = 0;
    for (int i = 0; i < n; ++i) {
        const TubeGrid& g = b->grids[i];
        const size_t pe = (size_t)b->h_tubes[i].plane;
        std::vector<double> host(4 * pe);
        ck(cudaMemcpy(host.data(), adj[i].gP, 4 * pe * sizeof(double), cudaMemcpyDeviceToHost), "read gradients");
        double z = 0.0;
        for (int r = 0; r < g.H; ++r)
            for (int c = 0; c < g.W; ++c) {
                const size_t src = (size_t)r * g.pitch + c, dst = cell_off + (size_t)r * g.W + c;
                if (gdP) gdP[dst] = (float)host[src];
                if (gdX) gdX[dst] = (float)host[pe + src];
                if (gdY) gdY[dst] = (float)host[2 * pe + src];
                z += host[3 * pe + src];
            }
        if (gz) gz[i] = (float)z;
        cell_off += (size_t)g.H * g.W;
    }
    for (int i = 0; i < n; ++i) {
        b->h_tubes[i].hist = nullptr;
        b->h_tubes[i].tmm_hist = nullptr;
    }
    ck(cudaMemcpy(b->d_tubes, b->h_tubes.data(), n * sizeof(TubeDev), cudaMemcpyHostToDevice), "restore descriptors");
    b->step = steps;
}

// The depth kernel's writes of one tube, as autograd.SectionDepthModel lists
// them (TubeDepth.cu:392-490): for each tube column from the first, the air
// cells from the axis outwards on both sides, then the two wall rows (zero);
// a later write to a cell replaces an earlier one.
void section_cells(const TubeGrid& g, std::vector<SectionCell>& cx, std::vector<SectionCell>& cy) {
    const int H = g.H, W = g.W;
    cx.assign((size_t)H * W, SectionCell{kSectionUnwritten, 0.0f, 0.0});
    cy = cx;
    const double ds = (double)g.dims.ds;
    const int sx = g.dims.tube_start_x;
    for (size_t i = 0; i < g.upper.size(); ++i) {
        const int x = sx + (int)i, u = g.upper[i], lo = g.lower[i], sg = g.colseg[i];
        const int air = lo - u - 1;
        const int half = (int)std::ceil(air * 0.5) - 1;
        const double a0 = (air * ds) / 2.0;
        for (int cc = half; cc >= 0; --cc) {
            const int pu = u + (half - cc) + 1, pl = lo - (half - cc) - 1;
            cx[(size_t)pu * W + x] = SectionCell{sg, (float)cc, a0};
            cx[(size_t)pl * W + x] = SectionCell{sg, (float)cc, a0};
            cy[(size_t)pu * W + x] = cc != half ? SectionCell{sg, (float)cc + 0.5f, a0}
                                                : SectionCell{kSectionZero, 0.0f, a0};
            cy[(size_t)pl * W + x] = SectionCell{sg, (float)cc - 0.5f, a0};
        }
        for (int r : {u, lo}) {
            cx[(size_t)r * W + x] = SectionCell{kSectionZero, 0.0f, a0};
            cy[(size_t)r * W + x] = SectionCell{kSectionZero, 0.0f, a0};
        }
    }
}

void section_setup(vs_batch* b) {
    if (b->d_sec) return;
    const int n = (int)b->grids.size();
    std::vector<std::vector<SectionCell>> cx(n), cy(n);
    std::vector<size_t> off(n);
    size_t total = 0;
    for (int i = 0; i < n; ++i) {
        const TubeGrid& g = b->grids[i];
        const vs_params& p = g.src_params;
        if (p.fdtd_solver_type != 1 || p.cross_sectional_shape != 2 || g.upper.empty())
            throw VsFailure{VS_ERR_UNSUPPORTED, "section maps cover 2.5D tubes with 3:1 elliptical sections"};
        section_cells(g, cx[i], cy[i]);
        const int64_t pv = (int64_t)g.dims.tube_mid_y * g.W + g.dims.tube_end_x;
        if (cx[i][pv].seg < 0 || cy[i][pv].seg < 0)
            throw VsFailure{VS_ERR_UNSUPPORTED, "section maps: the pivot cell is not an air cell"};
        const size_t cells = (size_t)g.H * g.W, ns = g.major_m.size();
        off[i] = total;
        total += align_up(2 * cells * sizeof(SectionCell)) + align_up(cells) + align_up(4 * cells * sizeof(double)) +
                 align_up(5 * ns * sizeof(double)) + align_up(6 * sizeof(double));
        b->sec_max_cells = std::max<int64_t>(b->sec_max_cells, (int64_t)cells);
    }
    ck(cudaMalloc(&b->sec_mem, total), "cudaMalloc(section model)");
    b->h_sec.assign(n, SectionTube{});
    for (int i = 0; i < n; ++i) {
        const TubeGrid& g = b->grids[i];
        const size_t cells = (size_t)g.H * g.W, ns = g.major_m.size();
        char* p = b->sec_mem + off[i];
        auto next = [&](size_t bytes) { char* q = p; p += align_up(bytes); return q; };
        SectionTube& t = b->h_sec[i];
        SectionCell* dcx = reinterpret_cast<SectionCell*>(next(2 * cells * sizeof(SectionCell)));
        t.cx = dcx;
        t.cy = dcx + cells;
        t.clamp = reinterpret_cast<uint8_t*>(next(cells));
        double* sc = reinterpret_cast<double*>(next(4 * cells * sizeof(double)));
        t.gxs = sc; t.gys = sc + cells; t.gx = sc + 2 * cells; t.gy = sc + 3 * cells;
        double* pr = reinterpret_cast<double*>(next(5 * ns * sizeof(double)));
        t.w0 = pr; t.w = pr + ns; t.d = pr + 2 * ns; t.dw = pr + 3 * ns; t.dd = pr + 4 * ns;
        t.acc = reinterpret_cast<double*>(next(6 * sizeof(double)));
        t.ds = (double)g.dims.ds;
        t.pivot = (int64_t)g.dims.tube_mid_y * g.W + g.dims.tube_end_x;
        t.H = g.H; t.W = g.W; t.nsec = (int32_t)ns;
        ck(cudaMemcpy(dcx, cx[i].data(), cells * sizeof(SectionCell), cudaMemcpyHostToDevice), "upload section cells");
        ck(cudaMemcpy(dcx + cells, cy[i].data(), cells * sizeof(SectionCell), cudaMemcpyHostToDevice),
           "upload section cells");
        std::vector<double> w0(g.major_m.begin(), g.major_m.end());
        ck(cudaMemcpy(const_cast<double*>(t.w0), w0.data(), ns * sizeof(double), cudaMemcpyHostToDevice),
           "upload nominal widths");
    }
    ck(cudaMalloc(&b->d_sec, n * sizeof(SectionTube)), "cudaMalloc(section descriptors)");
    ck(cudaMemcpy(b->d_sec, b->h_sec.data(), n * sizeof(SectionTube), cudaMemcpyHostToDevice),
       "upload section descriptors");
}

void set_sections(vs_batch* b, const double* width, const double* depth, const double* zinv) {
    section_setup(b);
    const int n = (int)b->grids.size();
    size_t k = 0;
    for (int i = 0; i < n; ++i) {
        const SectionTube& t = b->h_sec[i];
        for (int j = 0; j < t.nsec; ++j)
            if (!(width[k + j] > 0.0) || !(depth[k + j] > 0.0) || !std::isfinite(width[k + j]) ||
                !std::isfinite(depth[k + j]))
                throw VsFailure{VS_ERR_INVALID_ARG, "section widths and depths must be finite and > 0"};
        if (zinv && (!(zinv[i] >= 0.0) || !std::isfinite(zinv[i])))
            throw VsFailure{VS_ERR_INVALID_ARG, "z_inv must be finite and >= 0"};
        ck(cudaMemcpyAsync(const_cast<double*>(t.w), width + k, t.nsec * sizeof(double), cudaMemcpyHostToDevice,
                           b->stream), "upload widths");
        ck(cudaMemcpyAsync(const_cast<double*>(t.d), depth + k, t.nsec * sizeof(double), cudaMemcpyHostToDevice,
                           b->stream), "upload depths");
        k += t.nsec;
        if (zinv) {
            b->grids[i].zinv_val = (float)zinv[i];
            b->h_tubes[i].zinv = (float)zinv[i];
        }
    }
    ck(cudaMemcpyAsync(b->d_tubes, b->h_tubes.data(), n * sizeof(TubeDev), cudaMemcpyHostToDevice, b->stream),
       "upload tube descriptors");
    if (b->fast && zinv) {
        // the fast_math coefficient tables hold z_inv
        for (int i = 0; i < n; ++i) {
            std::vector<uint8_t> desc;
            std::vector<float> ta, tb;
            build_descriptors(b->grids[i], desc, ta, tb);
            const TubeDev& t = b->h_tubes[i];
            ck(cudaMemcpyAsync((void*)t.desc_a, ta.data(), ta.size() * sizeof(float), cudaMemcpyHostToDevice,
                               b->stream), "upload descriptor table");
            ck(cudaMemcpyAsync((void*)t.desc_b, tb.data(), tb.size() * sizeof(float), cudaMemcpyHostToDevice,
                               b->stream), "upload descriptor table");
        }
    }
    ck(launch_section_maps(b->d_sec, b->d_tubes, n, b->sec_max_cells, b->stream), "section maps");
    ck(cudaStreamSynchronize(b->stream), "section maps sync");
    b->sec_maps = true;
    b->ck_steps = 0;    // checkpoints no longer match the maps
}

void section_gradients(vs_batch* b, double* dwidth, double* ddepth) {
    if (!b->d_sec || !b->sec_maps || !b->d_adj || b->ck_steps <= 0)
        throw VsFailure{VS_ERR_INVALID_ARG,
                        "vs_batch_section_gradients needs vs_batch_set_sections, vs_batch_forward_ckpt and "
                        "vs_batch_adjoint first"};
    const int n = (int)b->grids.size();
    for (int i = 0; i < n; ++i) {
        const SectionTube& t = b->h_sec[i];
        ck(cudaMemsetAsync(t.dw, 0, 2 * t.nsec * sizeof(double), b->stream), "zero section gradients");
        ck(cudaMemsetAsync(t.acc, 0, 6 * sizeof(double), b->stream), "zero accumulators");
    }
    ck(launch_section_vjp(b->d_sec, b->d_tubes, b->d_adj, n, b->sec_max_cells, b->stream), "section vjp");
    ck(cudaStreamSynchronize(b->stream), "section vjp sync");
    size_t k = 0;
    for (int i = 0; i < n; ++i) {
        const SectionTube& t = b->h_sec[i];
        if (dwidth) ck(cudaMemcpy(dwidth + k, t.dw, t.nsec * sizeof(double), cudaMemcpyDeviceToHost), "read dwidth");
        if (ddepth) ck(cudaMemcpy(ddepth + k, t.dd, t.nsec * sizeof(double), cudaMemcpyDeviceToHost), "read ddepth");
        k += t.nsec;
    }
}

void set_maps(vs_batch* b, int i, const float* dP, const float* dX, const float* dY, float zinv) {
    fetch_device_maps(b, (size_t)i);
    TubeGrid& g = b->grids[i];
    const size_t n = (size_t)g.H * g.W;
    if (dP) std::memcpy(g.dP.data(), dP, n * sizeof(float));
    if (dX) std::memcpy(g.dX.data(), dX, n * sizeof(float));
    if (dY) std::memcpy(g.dY.data(), dY, n * sizeof(float));
    for (size_t k = 0; k < n; ++k)
        if (!(g.dP[k] > 0.0f) || !(g.dX[k] > 0.0f) || !(g.dY[k] > 0.0f) || !std::isfinite(g.dP[k]) ||
            !std::isfinite(g.dX[k]) || !std::isfinite(g.dY[k]))
            throw VsFailure{VS_ERR_INVALID_ARG, "depth maps must be finite and > 0"};
    if (!(zinv >= 0.0f) || !std::isfinite(zinv)) throw VsFailure{VS_ERR_INVALID_ARG, "z_inv must be finite and >= 0"};
    g.zinv_val = zinv;
    b->h_tubes[i].zinv = zinv;
    upload_static_tube(b, (size_t)i);
    b->sec_maps = false;
    ck(cudaMemcpy(b->d_tubes, b->h_tubes.data(), b->h_tubes.size() * sizeof(TubeDev), cudaMemcpyHostToDevice),
       "upload tube descriptors");
    b->ck_steps = 0;    // checkpoints no longer match the maps
}

template <class F>
int guarded(F&& f) {
    try {
        f();
        return VS_OK;
    } catch (const VsFailure& e) {
        return set_error(e.status, e.what);
    } catch (const CudaFail& e) {
        return set_error(VS_ERR_CUDA, std::string(e.where) + ": " + cudaGetErrorString(e.err));
    } catch (const std::bad_alloc&) {
        return set_error(VS_ERR_ALLOC, "host allocation failed");
    }
}

}  // namespace
}  // namespace vsb

extern "C" {

int vs_version(void) { return VS_ABI_VERSION; }

const char* vs_last_error(void) { return vsb::g_last_error.c_str(); }

int vs_params_init(vs_params* p) {
    if (!p) return set_error(VS_ERR_INVALID_ARG, "null vs_params");
    default_params(p);
    return VS_OK;
}

int vs_build_maps(const vs_params* p, const vs_geometry* g, vs_dims* dims, int32_t* cell_type,
                  float* depth_p, float* depth_x, float* depth_y, float* z_inv) {
    return guarded([&] {
        TubeGrid t;
        build_tube(p, g, t, 1);
        if (dims) *dims = t.dims;
        const size_t n = (size_t)t.H * t.W;
        if (cell_type) std::memcpy(cell_type, t.cell_type.data(), n * sizeof(int32_t));
        if (depth_p) std::memcpy(depth_p, t.dP.data(), n * sizeof(float));
        if (depth_x) std::memcpy(depth_x, t.dX.data(), n * sizeof(float));
        if (depth_y) std::memcpy(depth_y, t.dY.data(), n * sizeof(float));
        if (z_inv) std::memcpy(z_inv, t.zinv.data(), n * sizeof(float));
    });
}

int vs_tube_layout(const vs_params* p, const vs_geometry* g, vs_dims* dims, int32_t* upper_wall,
                   int32_t* lower_wall, int32_t* column_segment, float* major_axis_m, float* minor_axis_m) {
    return guarded([&] {
        TubeGrid t;
        build_tube(p, g, t, 1);
        if (dims) *dims = t.dims;
        if (upper_wall) std::copy(t.upper.begin(), t.upper.end(), upper_wall);
        if (lower_wall) std::copy(t.lower.begin(), t.lower.end(), lower_wall);
        if (column_segment) std::copy(t.colseg.begin(), t.colseg.end(), column_segment);
        if (major_axis_m) std::copy(t.major_m.begin(), t.major_m.end(), major_axis_m);
        if (minor_axis_m) std::copy(t.minor_m.begin(), t.minor_m.end(), minor_axis_m);
    });
}

int vs_source_table(const vs_params* p, int64_t num_steps, float* out) {
    if (!p || !out || num_steps < 0) return set_error(VS_ERR_INVALID_ARG, "vs_source_table arguments");
    return guarded([&] {
        const float dt = 1.0f / (float)(44100 * p->srate_mul);
        std::vector<float> v;
        build_source(p, dt, num_steps, v);
        std::memcpy(out, v.data(), (size_t)num_steps * sizeof(float));
    });
}

int vs_batch_create(int32_t n, const vs_params* params, const vs_geometry* geoms, vs_batch** out) {
    if (!out || !params || n < 1) return set_error(VS_ERR_INVALID_ARG, "vs_batch_create arguments");
    *out = nullptr;
    std::unique_ptr<vs_batch> b(new (std::nothrow) vs_batch());
    if (!b) return set_error(VS_ERR_ALLOC, "host allocation failed");
    int st = guarded([&] { create_batch(n, params, geoms, b.get()); });
    if (st == VS_OK) *out = b.release();
    return st;
}

int vs_batch_get_dims(const vs_batch* b, int32_t i, vs_dims* dims) {
    if (!b || !dims || i < 0 || i >= (int)b->grids.size()) return set_error(VS_ERR_INVALID_ARG, "vs_batch_get_dims");
    *dims = b->grids[i].dims;
    return VS_OK;
}

int vs_batch_run(vs_batch* b, int64_t steps, float* traces, int traces_on_device) {
    if (!b || steps < 0) return set_error(VS_ERR_INVALID_ARG, "vs_batch_run arguments");
    if (steps == 0) return VS_OK;
    return guarded([&] { run_batch(b, steps, traces, traces_on_device); });
}

int vs_batch_reset(vs_batch* b) {
    if (!b) return set_error(VS_ERR_INVALID_ARG, "null batch");
    return guarded([&] { reset_state(b); });
}

int vs_batch_set_tile(vs_batch* b, int32_t tile_index) {
    if (!b || tile_index < -1 || tile_index >= tile_shape_count())
        return set_error(VS_ERR_INVALID_ARG, "tile index out of range");
    const int s = tile_index < 0 ? default_shape(b) : tile_index;
    if (!shape_fits(b, s)) return set_error(VS_ERR_UNSUPPORTED, "launch shape unavailable for this batch (shared memory, wall oscillator or fast_math)");
    b->shape = s;
    return VS_OK;
}

int vs_batch_adjoint_times(const vs_batch* b, float* recompute_ms, float* reverse_ms) {
    if (!b) return set_error(VS_ERR_INVALID_ARG, "null batch");
    if (recompute_ms) *recompute_ms = b->adj_recompute_ms;
    if (reverse_ms) *reverse_ms = b->adj_reverse_ms;
    return VS_OK;
}

int vs_batch_set_adjoint_form(vs_batch* b, int32_t form) {
    if (!b || form < ADJ_FORM_AUTO || form > ADJ_FORM_STRIPS)
        return set_error(VS_ERR_INVALID_ARG, "vs_batch_set_adjoint_form: form must be 0 (automatic), 1 (tiles), "
                                             "2 (two-step strips) or 3 (one-step strips)");
    b->adj_form = form;
    return VS_OK;
}

int vs_batch_set_adjoint_rows(vs_batch* b, int32_t rows) {
    if (!b || (rows != 0 && rows != 4 && rows != 8 && rows != 16))
        return set_error(VS_ERR_INVALID_ARG, "vs_batch_set_adjoint_rows: rows must be 0 (default), 4, 8 or 16");
    b->adj_rows = rows;
    return VS_OK;
}

int vs_batch_set_wait_limit(vs_batch* b, uint32_t polls) {
    if (!b) return set_error(VS_ERR_INVALID_ARG, "null batch");
    b->wait_polls = polls;
    return VS_OK;
}

int vs_batch_autotune(vs_batch* b, int64_t steps, int32_t* best_index, float* best_ms) {
    if (!b || steps < 1) return set_error(VS_ERR_INVALID_ARG, "vs_batch_autotune arguments");
    return guarded([&] {
        cudaEvent_t e0, e1;
        ck(cudaEventCreate(&e0), "event");
        ck(cudaEventCreate(&e1), "event");
        float best = 1e30f;
        int best_i = default_shape(b);
        for (int s = 0; s < tile_shape_count(); ++s) {
            if (!shape_fits(b, s)) continue;
            b->shape = s;
            run_batch(b, std::min<int64_t>(steps, kChunk), nullptr, 1);   // warm: tiles + graph
            ck(cudaEventRecord(e0, b->stream), "record");
            run_batch(b, steps, nullptr, 1);
            ck(cudaEventRecord(e1, b->stream), "record");
            ck(cudaEventSynchronize(e1), "sync");
            float ms = 0;
            ck(cudaEventElapsedTime(&ms, e0, e1), "elapsed");
            if (ms < best) { best = ms; best_i = s; }
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        b->shape = best_i;
        build_tiles(b, best_i);
        reset_state(b);
        if (best_index) *best_index = best_i;
        if (best_ms) *best_ms = best;
    });
}

int vs_formants(const float* traces, int32_t n_traces, int64_t n, double fs, int32_t num_formants, double* out,
                void* cuda_stream) {
    if (!traces || !out || n_traces < 1 || n < 3 || num_formants < 1 || !(fs > 0.0) || n > INT32_MAX)
        return set_error(VS_ERR_INVALID_ARG, "vs_formants arguments");
    std::string err;
    const int st = formants_device(traces, n_traces, n, fs, num_formants, out,
                                   static_cast<cudaStream_t>(cuda_stream), &err);
    if (st != VS_OK) return set_error(st, err.c_str());
    return VS_OK;
}

int vs_audio(const float* traces, int32_t n_traces, int64_t n, int32_t srate_mul, float* out, void* cuda_stream) {
    if (!traces || !out || n_traces < 1 || n < 1 || srate_mul < 1 || srate_mul > 64)
        return set_error(VS_ERR_INVALID_ARG, "vs_audio arguments");
    std::string err;
    const int st = audio_device(traces, n_traces, n, srate_mul, out, static_cast<cudaStream_t>(cuda_stream), &err);
    if (st != VS_OK) return set_error(st, err.c_str());
    return VS_OK;
}

int vs_audio_filter(int32_t srate_mul, double* b3, double* a3) {
    if (!b3 || !a3 || srate_mul < 2 || srate_mul > 64) return set_error(VS_ERR_INVALID_ARG, "vs_audio_filter arguments");
    audio_filter(srate_mul, b3, a3);
    return VS_OK;
}

int vs_tile_shape_count(void) { return tile_shape_count(); }

int vs_tile_shape(int32_t i, int32_t* rows, int32_t* cols) {
    if (i < 0 || i >= tile_shape_count()) return set_error(VS_ERR_INVALID_ARG, "tile index out of range");
    const TileShape s = tile_shape(i);
    if (rows) *rows = s.rows;
    if (cols) *cols = s.cols * s.warps;
    return VS_OK;
}

int vs_tile_shape_steps(int32_t i, int32_t* steps_per_launch) {
    if (i < 0 || i >= tile_shape_count() || !steps_per_launch)
        return set_error(VS_ERR_INVALID_ARG, "vs_tile_shape_steps arguments");
    const int kind = tile_shape(i).kind;
    *steps_per_launch = kind == SHAPE_QUAD2 ? 2 : kind == SHAPE_CLUSTER ? 0 : 1;
    return VS_OK;
}

void vs_batch_destroy(vs_batch* b) { delete b; }

int vs_batch_set_maps(vs_batch* b, int32_t tube, const float* depth_p, const float* depth_x, const float* depth_y,
                      float z_inv) {
    if (!b || tube < 0 || tube >= (int)b->grids.size()) return set_error(VS_ERR_INVALID_ARG, "vs_batch_set_maps");
    return guarded([&] { set_maps(b, tube, depth_p, depth_x, depth_y, z_inv); });
}

int vs_batch_get_maps(const vs_batch* b, int32_t tube, int32_t* cell_type, float* depth_p, float* depth_x,
                      float* depth_y, float* z_inv) {
    if (!b || tube < 0 || tube >= (int)b->grids.size()) return set_error(VS_ERR_INVALID_ARG, "vs_batch_get_maps");
    return guarded([&] {
        const TubeGrid& g = b->grids[tube];
        const TubeDev& t = b->h_tubes[tube];
        ck(cudaStreamSynchronize(b->stream), "sync");
        const size_t row = g.W * sizeof(float), dpitch = g.pitch * sizeof(float);
        if (depth_p) ck(cudaMemcpy2D(depth_p, row, t.dP, dpitch, row, g.H, cudaMemcpyDeviceToHost), "read depth_p");
        if (depth_x) ck(cudaMemcpy2D(depth_x, row, t.dX, dpitch, row, g.H, cudaMemcpyDeviceToHost), "read depth_x");
        if (depth_y) ck(cudaMemcpy2D(depth_y, row, t.dY, dpitch, row, g.H, cudaMemcpyDeviceToHost), "read depth_y");
        if (cell_type || z_inv) {
            std::vector<uint8_t> code((size_t)g.H * g.W);
            ck(cudaMemcpy2D(code.data(), g.W, t.code, g.pitch, g.W, g.H, cudaMemcpyDeviceToHost), "read codes");
            for (size_t k = 0; k < code.size(); ++k) {
                if (cell_type) cell_type[k] = code[k] & CODE_TYPE_MASK;
                if (z_inv) z_inv[k] = (code[k] & CODE_ZINV_BIT) ? t.zinv : 0.0f;
            }
        }
    });
}

int vs_batch_set_sections(vs_batch* b, const double* width_m, const double* depth_m, const double* z_inv) {
    if (!b || !width_m || !depth_m) return set_error(VS_ERR_INVALID_ARG, "vs_batch_set_sections arguments");
    return guarded([&] { set_sections(b, width_m, depth_m, z_inv); });
}

int vs_batch_section_gradients(vs_batch* b, double* grad_width, double* grad_depth) {
    if (!b) return set_error(VS_ERR_INVALID_ARG, "null batch");
    return guarded([&] { section_gradients(b, grad_width, grad_depth); });
}

int vs_batch_forward_ckpt(vs_batch* b, int64_t steps, int32_t ckpt_every, float* traces) {
    if (!b || steps < 1 || ckpt_every < 1) return set_error(VS_ERR_INVALID_ARG, "vs_batch_forward_ckpt arguments");
    return guarded([&] { forward_checkpointed(b, steps, ckpt_every, traces); });
}

int vs_batch_adjoint(vs_batch* b, const float* dL_dtrace, float* grad_depth_p, float* grad_depth_x,
                     float* grad_depth_y, float* grad_z_inv) {
    if (!b || !dL_dtrace) return set_error(VS_ERR_INVALID_ARG, "vs_batch_adjoint arguments");
    return guarded([&] { run_adjoint(b, dL_dtrace, grad_depth_p, grad_depth_x, grad_depth_y, grad_z_inv); });
}

int vs_batch_forward_ckpt_device(vs_batch* b, int64_t steps, int32_t ckpt_every, float* traces) {
    if (!b || steps < 1 || ckpt_every < 1 || !traces)
        return set_error(VS_ERR_INVALID_ARG, "vs_batch_forward_ckpt_device arguments");
    return guarded([&] { forward_checkpointed(b, steps, ckpt_every, traces, true); });
}

int vs_batch_adjoint_device(vs_batch* b, const float* dL_dtrace, float* grad_depth_p, float* grad_depth_x,
                            float* grad_depth_y, float* grad_z_inv) {
    if (!b || !dL_dtrace) return set_error(VS_ERR_INVALID_ARG, "vs_batch_adjoint_device arguments");
    return guarded([&] { run_adjoint(b, dL_dtrace, grad_depth_p, grad_depth_x, grad_depth_y, grad_z_inv, true); });
}

int vs_create(const vs_params* p, const vs_geometry* g, vs_solver** out) {
    if (!out || !p) return set_error(VS_ERR_INVALID_ARG, "vs_create arguments");
    *out = nullptr;
    vs_batch* b = nullptr;
    int st = vs_batch_create(1, p, g, &b);
    if (st != VS_OK) return st;
    vs_solver* s = new (std::nothrow) vs_solver();
    if (!s) { delete b; return set_error(VS_ERR_ALLOC, "host allocation failed"); }
    s->b = b;
    *out = s;
    return VS_OK;
}

int vs_get_dims(const vs_solver* s, vs_dims* dims) {
    if (!s) return set_error(VS_ERR_INVALID_ARG, "null solver");
    return vs_batch_get_dims(s->b, 0, dims);
}

int vs_run(vs_solver* s, int64_t steps, float* trace, int trace_on_device) {
    if (!s) return set_error(VS_ERR_INVALID_ARG, "null solver");
    return vs_batch_run(s->b, steps, trace, trace_on_device);
}

int vs_reset(vs_solver* s) {
    if (!s) return set_error(VS_ERR_INVALID_ARG, "null solver");
    return vs_batch_reset(s->b);
}

int vs_get_fields(const vs_solver* s, float* p, float* vx, float* vy) {
    if (!s) return set_error(VS_ERR_INVALID_ARG, "null solver");
    return vs_batch_get_fields(s->b, 0, p, vx, vy);
}

int vs_batch_get_fields(const vs_batch* b, int32_t tube, float* p, float* vx, float* vy) {
    if (!b || tube < 0 || tube >= (int)b->grids.size()) return set_error(VS_ERR_INVALID_ARG, "vs_batch_get_fields");
    return guarded([&] {
        const TubeGrid& g = b->grids[(size_t)tube];
        const TubeDev& t = b->h_tubes[(size_t)tube];
        const int par = (int)(b->step & 1);
        const float* src[3] = {t.P[par], t.Vx[par], t.Vy[par]};
        float* dst[3] = {p, vx, vy};
        for (int k = 0; k < 3; ++k) {
            if (!dst[k]) continue;
            ck(cudaMemcpy2DAsync(dst[k], g.W * sizeof(float), src[k], g.pitch * sizeof(float),
                                 g.W * sizeof(float), g.H, cudaMemcpyDeviceToHost, b->stream),
               "copy fields");
        }
        ck(cudaStreamSynchronize(b->stream), "fields sync");
    });
}

int vs_batch_set_stream(vs_batch* b, void* cuda_stream) {
    if (!b) return set_error(VS_ERR_INVALID_ARG, "null batch");
    return guarded([&] {
        ck(cudaStreamSynchronize(b->stream), "sync old stream");
        if (b->own_stream && b->stream) cudaStreamDestroy(b->stream);
        if (cuda_stream) {
            b->stream = (cudaStream_t)cuda_stream;
            b->own_stream = false;
        } else {
            ck(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking), "cudaStreamCreate");
            b->own_stream = true;
        }
    });
}

int vs_set_stream(vs_solver* s, void* cuda_stream) {
    if (!s) return set_error(VS_ERR_INVALID_ARG, "null solver");
    return vs_batch_set_stream(s->b, cuda_stream);
}

void vs_destroy(vs_solver* s) {
    if (!s) return;
    delete s->b;
    delete s;
}

}  // extern "C"
