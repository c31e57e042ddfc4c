// vs_noalloc.cu -- vs_run_noalloc: one tube, no device allocation.
//
// Some callers cannot call cudaMalloc at the moment they want to step a tube:
// a real-time audio host running the solver on its processing thread, where
// an allocation may block for an unbounded time, or an application whose
// device memory is already reserved by another allocator (a framework's
// caching allocator), where a direct cudaMalloc can fail.  They own their
// buffers already.  This entry point takes those buffers (the maps from
// vs_build_maps, the table from vs_source_table, a trace buffer, all in
// device memory the caller owns) and keeps everything else it needs -- the
// ping-pong field planes, padded copies of the maps, the tube descriptor,
// the strip list and the run bookkeeping -- in one file-scope __device__
// array of fixed size.  It calls no cudaMalloc, cudaFree or other allocating
// routine, and runs the same strip kernel as vs_run.
//
// The array is shared by every call in the process: each call re-initialises
// the parts that must start at zero, but two calls whose work overlaps on the
// GPU (different streams, or different host threads on the same device)
// race on it.  Every GPU that loads the library holds the array until exit.
#include "vs_device.h"

#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>

namespace vsb {
namespace {

// Fixed scratch size per device: 16 MiB.  A frame of H x W cells needs
// about 37 * H * roundup(W, 32) bytes (49 with a coupled wall), e.g. a
// 57 x 253 tube needs 0.55 MiB; frames up to ~400k padded cells fit.
constexpr size_t kScratchBytes = size_t(16) << 20;

__device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
constexpr int kShape = 1;          // 16-row strips, 4 warps per CTA

std::mutex g_mu;
unsigned char* g_scratch_addr[kMaxDevices] = {};

size_t up256(size_t v) { return (v + 255) / 256 * 256; }

// Device address of the scratch array on the current device; looked up once
// per device with that device current.
cudaError_t scratch_address(unsigned char** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_scratch_addr[dev] = static_cast<unsigned char*>(p);
    }
    *out = g_scratch_addr[dev];
    return cudaSuccess;
}

// Copy the caller's H x W maps into the padded planes of the scratch layout.
__global__ void pack_maps(const int32_t* __restrict__ cell_type, const float* __restrict__ dp,
                          const float* __restrict__ dx, const float* __restrict__ dy,
                          const float* __restrict__ zinv, float* __restrict__ odp, float* __restrict__ odx,
                          float* __restrict__ ody, uint8_t* __restrict__ ocode, int H, int W, int pitch,
                          int32_t* __restrict__ bad) {
    const int64_t n = (int64_t)H * pitch;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int r = (int)(i / pitch), c = (int)(i - (int64_t)r * pitch);
        if (c < W) {
            const int64_t s = (int64_t)r * W + c;
            odp[i] = dp[s];
            odx[i] = dx[s];
            ody[i] = dy[s];
            const int32_t ty = cell_type[s];
            uint8_t k;
            if (ty < 0 || ty >= 13) {          // not a reference cell type: kept out of the tables
                k = (uint8_t)VS_CELL_DEAD;
                *bad = 1;
            } else {
                k = (uint8_t)ty;
                if (zinv[s] != 0.0f) k |= CODE_ZINV_BIT;
            }
            ocode[i] = k;
        } else {
            odp[i] = 0.0f;
            odx[i] = 0.0f;
            ody[i] = 0.0f;
            ocode[i] = (uint8_t)VS_CELL_DEAD;
        }
    }
}

// Strip work items of one tube, in the order vs_batch builds them, classified
// from the packed code bytes.
__global__ void make_strips(Tile* __restrict__ tiles, const uint8_t* __restrict__ code, int H, int W, int pitch,
                            int rows, int nstrips, int nitems) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nitems) return;
    Tile t{};
    t.tube = 0;
    t.r0 = 1 + (i / nstrips) * rows;
    t.c0 = -kStripLead + (i % nstrips) * kStripCommit;
    auto code_at = [=](int r, int c) { return (int)code[(int64_t)r * pitch + c]; };
    classify_strip(code_at, H, W, t.r0, rows, t.c0, t);
    tiles[i] = t;
}

// Descriptors of the run, passed by value (kernel parameters are copied at
// launch, so no host buffer has to stay alive and nothing is staged through
// pageable memory).
__global__ void init_run(TubeDev t, RunState rs, TubeDev* __restrict__ dt, RunState* __restrict__ drs,
                         int32_t* __restrict__ bad) {
    *dt = t;
    *drs = rs;
    *bad = 0;
}

// A map with a cell type outside 0..12 has no defined update: its trace is
// returned as NaN so the caller cannot mistake it for a result.
__global__ void poison_trace(const int32_t* __restrict__ bad, float* __restrict__ trace, int64_t n) {
    if (!*bad) return;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        trace[i] = __int_as_float(0x7fc00000);
}

int fail(int status, const char* msg) {
    record_error(msg);
    return status;
}

}  // namespace
}  // namespace vsb

using namespace vsb;

extern "C" int vs_run_noalloc(const vs_params* p, const vs_dims* dims, const int32_t* cell_type,
                              const float* depth_p, const float* depth_x, const float* depth_y,
                              const float* z_inv, const float* source, int64_t steps, float* trace,
                              void* cuda_stream) {
    if (!p || !dims || !cell_type || !depth_p || !depth_x || !depth_y || !z_inv || !trace)
        return fail(VS_ERR_INVALID_ARG, "vs_run_noalloc: null argument");
    if (steps < 1 || steps > INT32_MAX) return fail(VS_ERR_INVALID_ARG, "vs_run_noalloc: steps must be in 1..2^31-1");
    if (p->source_type != VS_SRC_TMM && !source)
        return fail(VS_ERR_INVALID_ARG, "vs_run_noalloc: this source type needs the excitation table");
    if (p->srate_mul < 1 || p->srate_mul > 64 || (p->engine != VS_ENGINE_CPU && p->engine != VS_ENGINE_EIGEN))
        return fail(VS_ERR_INVALID_ARG, "vs_run_noalloc: invalid vs_params");
    if (p->fast_math) return fail(VS_ERR_UNSUPPORTED, "vs_run_noalloc runs the reference arithmetic only (fast_math = 0)");
    const int H = dims->frame_h, W = dims->frame_w;
    if (H < 3 || W < 3) return fail(VS_ERR_INVALID_ARG, "vs_run_noalloc: frame smaller than 3 x 3");
    // the same ranges the map builder guarantees: interior cells only
    if (dims->listener_x < 1 || dims->listener_x > W - 2 || dims->listener_y < 1 || dims->listener_y > H - 2)
        return fail(VS_ERR_INVALID_ARG, "vs_run_noalloc: listener cell outside the frame's interior");
    if (dims->excitation_x < 1 || dims->excitation_x > W - 2 || dims->excitation_y < 1 || dims->excitation_y > H - 2)
        return fail(VS_ERR_INVALID_ARG, "vs_run_noalloc: excitation cell outside the frame's interior");
    const int pitch = (W + 31) / 32 * 32;
    const bool wall = p->fdtd_solver_type == 1 && p->wall_coupling != 0.0f;
    const size_t plane_bytes = up256((size_t)H * pitch * sizeof(float));
    const int nstate = wall ? 10 : 6;
    const int rows = tile_shape(kShape).rows;
    const int nstrips = (W - 2) / kStripCommit + 1;
    const int nitems = ((H - 3) / rows + 1) * nstrips;
    size_t off = 256;                                        // guard ahead of the first plane
    const size_t off_state = off;             off += plane_bytes * nstate;
    const size_t off_depth = off;             off += plane_bytes * 3;
    const size_t off_code = off;              off += up256((size_t)H * pitch);
    const size_t off_tmm = off;               off += up256(2 * sizeof(TmmState)) + up256(2 * sizeof(TmmState64));
    const size_t off_tube = off;              off += up256(sizeof(TubeDev));
    const size_t off_rs = off;                off += up256(sizeof(RunState));
    const size_t off_bad = off;               off += 256;
    const size_t off_tiles = off;             off += up256((size_t)nitems * sizeof(Tile));
    if (off > kScratchBytes)
        return fail(VS_ERR_INVALID_ARG, "vs_run_noalloc: frame too large for the 16 MiB static scratch");

    // K1, K2, bcoef, dt, wall parameters, sigma table and two-mass constants
    // from the map builder's own source of them
    TubeGrid k;
    try {
        solver_constants(p, k);
    } catch (const VsFailure& f) {
        return fail(f.status, f.what.c_str());
    }

    unsigned char* base = nullptr;
    cudaError_t e = scratch_address(&base);
    if (e != cudaSuccess) return fail(VS_ERR_CUDA, cudaGetErrorString(e));
    cudaStream_t st = static_cast<cudaStream_t>(cuda_stream);

    TubeDev t;
    std::memset(&t, 0, sizeof(t));
    const size_t pe = plane_bytes / sizeof(float);
    float* s0 = reinterpret_cast<float*>(base + off_state);
    for (int j = 0; j < 2; ++j) {
        t.P[j] = s0 + j * pe;
        t.Vx[j] = s0 + (2 + j) * pe;
        t.Vy[j] = s0 + (4 + j) * pe;
        if (wall) { t.w[j] = s0 + (6 + j) * pe; t.z[j] = s0 + (8 + j) * pe; }
    }
    float* d0 = reinterpret_cast<float*>(base + off_depth);
    t.dP = d0;
    t.dX = d0 + pe;
    t.dY = d0 + 2 * pe;
    t.code = base + off_code;
    t.src = p->source_type == VS_SRC_TMM ? nullptr : source;
    t.src_len = p->source_type == VS_SRC_TMM ? 0 : steps;
    t.tmm = reinterpret_cast<TmmState*>(base + off_tmm);
    t.tmm64 = reinterpret_cast<TmmState64*>(base + off_tmm + up256(2 * sizeof(TmmState)));
    t.plane = (int64_t)pe;
    t.H = H; t.W = W; t.pitch = pitch;
    t.flags = (k.dirichlet ? TUBE_DIRICHLET : 0) | (k.eigen ? TUBE_EIGEN : 0) | (k.tmm ? TUBE_TMM : 0) |
              (k.wall_ode ? TUBE_WALL_ODE : 0) | (k.tmm64 ? TUBE_TMM64 : 0);
    t.lis_x = dims->listener_x; t.lis_y = dims->listener_y;
    t.exc_x = dims->excitation_x; t.exc_y = dims->excitation_y;
    t.K1 = k.K1; t.K2 = k.K2; t.bcoef = k.bcoef;
    t.zinv = dims->z_inv_val;
    t.dt = k.dt; t.Mw = k.Mw; t.Bw = k.Bw; t.Kw = k.Kw; t.cpl = k.cpl;
    t.dir0 = k.dir[0]; t.dir1 = k.dir[1]; t.dir2 = k.dir[2]; t.dir3 = k.dir[3];
    for (int j = 0; j < 13; ++j) t.sigma[j] = k.sigma[j];
    t.tmmc = k.tmmc;
    t.tmmd = k.tmmd;
    t.tmmx = k.tmmx;

    RunState rs;
    std::memset(&rs, 0, sizeof(rs));
    rs.trace = trace;
    rs.trace_stride = steps;

    TubeDev* d_tube = reinterpret_cast<TubeDev*>(base + off_tube);
    RunState* d_rs = reinterpret_cast<RunState*>(base + off_rs);
    int32_t* d_bad = reinterpret_cast<int32_t*>(base + off_bad);
    Tile* d_tiles = reinterpret_cast<Tile*>(base + off_tiles);
    // fields, wall state and the two-mass state restart at zero on every call
    e = cudaMemsetAsync(base + off_state, 0, plane_bytes * nstate, st);
    if (e == cudaSuccess)
        e = cudaMemsetAsync(base + off_tmm, 0, up256(2 * sizeof(TmmState)) + up256(2 * sizeof(TmmState64)), st);
    if (e != cudaSuccess) return fail(VS_ERR_CUDA, cudaGetErrorString(e));
    init_run<<<1, 1, 0, st>>>(t, rs, d_tube, d_rs, d_bad);
    pack_maps<<<592, 256, 0, st>>>(cell_type, depth_p, depth_x, depth_y, z_inv, d0, d0 + pe,
                                   d0 + 2 * pe, base + off_code, H, W, pitch, d_bad);
    make_strips<<<(nitems + 127) / 128, 128, 0, st>>>(d_tiles, base + off_code, H, W, pitch, rows, nstrips, nitems);
    e = cudaGetLastError();
    for (int64_t i = 0; i < steps && e == cudaSuccess; ++i)
        e = launch_step(kShape, wall, false, d_tube, d_tiles, nitems, d_rs, (int)i, st, pitch);
    if (e == cudaSuccess) {
        poison_trace<<<64, 256, 0, st>>>(d_bad, trace, steps);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) return fail(VS_ERR_CUDA, cudaGetErrorString(e));
    return VS_OK;
}
