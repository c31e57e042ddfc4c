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
                          float* __restrict__ ody, uint8_t* __restrict__ ocode, int H, int W, int pitch) {
    const int64_t n = (int64_t)H * pitch;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int r = (int)(i / pitch), c = (int)(i - (int64_t)r * pitch);
        if (c < W) {
            const int64_t s = (int64_t)r * W + c;
            odp[i] = dp[s];
            odx[i] = dx[s];
            ody[i] = dy[s];
            uint8_t k = (uint8_t)(cell_type[s] & CODE_TYPE_MASK);
            if (zinv[s] != 0.0f) k |= CODE_ZINV_BIT;
            ocode[i] = k;
        } else {
            odp[i] = 0.0f;
            odx[i] = 0.0f;
            ody[i] = 0.0f;
            ocode[i] = (uint8_t)VS_CELL_DEAD;
        }
    }
}

// Strip work items of one tube, in the order vs_batch builds them.
__global__ void make_strips(Tile* __restrict__ tiles, const int32_t* __restrict__ cell_type,
                            const float* __restrict__ zinv, int H, int W, int rows, int nstrips, int nitems) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nitems) return;
    Tile t{};
    t.tube = 0;
    t.r0 = 1 + (i / nstrips) * rows;
    t.c0 = -kStripLead + (i % nstrips) * kStripCommit;
    auto code_at = [=](int r, int c) {
        const int64_t s = (int64_t)r * W + c;
        return (cell_type[s] & CODE_TYPE_MASK) | (zinv[s] != 0.0f ? CODE_ZINV_BIT : 0);
    };
    classify_strip(code_at, H, W, t.r0, rows, t.c0, t);
    tiles[i] = t;
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
    const size_t off_tiles = off;             off += up256((size_t)nitems * sizeof(Tile));
    if (off > kScratchBytes)
        return fail(VS_ERR_INVALID_ARG, "vs_run_noalloc: frame too large for the 16 MiB static scratch");

    unsigned char* base = nullptr;
    cudaError_t e = scratch_address(&base);
    if (e != cudaSuccess) return fail(VS_ERR_CUDA, cudaGetErrorString(e));
    cudaStream_t st = static_cast<cudaStream_t>(cuda_stream);

    // constants of SimulationParams(srate_mul) / SolverParams / FDTDSolver.cu:311-312
    const float c = 350.0f, rho = (float)((double)1.14f / std::pow(1.0, 3));
    const float kappa = rho * c * c;
    const float dt = 1.0f / (float)(44100 * p->srate_mul);
    const float ds = dt * c * sqrtf(2.0f);

    TubeDev t;
    std::memset(&t, 0, sizeof(t));
    const size_t pe = plane_bytes / sizeof(float);
    float* s0 = reinterpret_cast<float*>(base + off_state);
    for (int k = 0; k < 2; ++k) {
        t.P[k] = s0 + k * pe;
        t.Vx[k] = s0 + (2 + k) * pe;
        t.Vy[k] = s0 + (4 + k) * pe;
        if (wall) { t.w[k] = s0 + (6 + k) * pe; t.z[k] = s0 + (8 + k) * pe; }
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
    t.flags = (p->mouth_radiation_cond ? TUBE_DIRICHLET : 0) | (p->engine == VS_ENGINE_EIGEN ? TUBE_EIGEN : 0) |
              (p->source_type == VS_SRC_TMM ? TUBE_TMM : 0) | (wall ? TUBE_WALL_ODE : 0) |
              (p->source_type == VS_SRC_TMM && p->tmm_f64 ? TUBE_TMM64 : 0);
    t.lis_x = dims->listener_x; t.lis_y = dims->listener_y;
    t.exc_x = dims->excitation_x; t.exc_y = dims->excitation_y;
    t.K1 = (kappa * dt) / ds;
    t.K2 = kappa * dt;
    t.bcoef = (1.0f * dt) / (rho * ds);
    t.zinv = dims->z_inv_val;
    t.dt = dt;
    t.Mw = 21.0f; t.Bw = 8000.0f; t.Kw = 845000.0f;
    t.cpl = p->wall_coupling;
    t.dir0 = 0.0f; t.dir1 = 0.0f; t.dir2 = 1.0f; t.dir3 = 0.0f;
    const float sig[13] = {dt, 0, dt, 0, 0, 0, 0, 0, 0, 0, 1000000.0f, 0, dt};
    for (int k = 0; k < 13; ++k) t.sigma[k] = sig[k];
    for (int l = 0; l < 6; ++l) t.sigma[VS_CELL_PML0 + l] = ((float)l / (float)5) * 0.5f;
    t.tmmc = tmm_consts<float>(p->tmm_ps_pa, p->srate_mul);
    t.tmmd = tmm_consts<double>(p->tmm_ps_pa, p->srate_mul);

    RunState rs;
    std::memset(&rs, 0, sizeof(rs));
    rs.trace = trace;
    rs.trace_stride = steps;

    TubeDev* d_tube = reinterpret_cast<TubeDev*>(base + off_tube);
    RunState* d_rs = reinterpret_cast<RunState*>(base + off_rs);
    Tile* d_tiles = reinterpret_cast<Tile*>(base + off_tiles);
    // fields, wall state and the two-mass state restart at zero on every call
    e = cudaMemsetAsync(base + off_state, 0, plane_bytes * nstate, st);
    if (e == cudaSuccess)
        e = cudaMemsetAsync(base + off_tmm, 0, up256(2 * sizeof(TmmState)) + up256(2 * sizeof(TmmState64)), st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_tube, &t, sizeof(t), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_rs, &rs, sizeof(rs), cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return fail(VS_ERR_CUDA, cudaGetErrorString(e));
    pack_maps<<<592, 256, 0, st>>>(cell_type, depth_p, depth_x, depth_y, z_inv, d0, d0 + pe,
                                   d0 + 2 * pe, base + off_code, H, W, pitch);
    make_strips<<<(nitems + 127) / 128, 128, 0, st>>>(d_tiles, cell_type, z_inv, H, W, rows, nstrips, nitems);
    e = cudaGetLastError();
    for (int64_t i = 0; i < steps && e == cudaSuccess; ++i)
        e = launch_step(kShape, wall, false, d_tube, d_tiles, nitems, d_rs, (int)i, st, pitch);
    if (e != cudaSuccess) return fail(VS_ERR_CUDA, cudaGetErrorString(e));
    return VS_OK;
}
