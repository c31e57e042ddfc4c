// vs_device.h -- device-side descriptors shared by the kernels and the host
// launch code of libvocalsim_b200.
#pragma once

#include <cstdint>

#include <cuda_runtime_api.h>

#include "vs_grid.h"

namespace vsb {

// Flags of a tube descriptor.
enum : int32_t {
    TUBE_DIRICHLET = 1,   // zero P on noPressure cells (FDTDEngineCPU.cpp:336-337)
    TUBE_EIGEN = 2,       // FDTDEngineEigen pressure denominator sigma*dP + dP
    TUBE_TMM = 4,         // two-mass source computed on the device each step
    TUBE_WALL_ODE = 8,    // 2.5D wall oscillator with nonzero pressure coupling
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
    TmmConsts tmmc;
};

// Mutable run bookkeeping kept in device memory so that CUDA graphs captured
// once can be replayed for any run length.
struct RunState {
    int64_t step;         // global step of the next launch with local index 0
    int64_t run_start;    // global step that lands in trace column 0
    float* trace;         // device trace buffer, [ntubes][trace_stride]
    int64_t trace_stride;
    int32_t error;        // sticky device error word (0 = ok)
    int32_t pad;
};

// A strip of one tube processed by one warp: rows [r0, r0+rows), lanes on
// columns c0 .. c0+31, committing columns c0+1 .. c0+cols.
struct Tile {
    int32_t tube, r0, c0, has_exc;
};

// Host-side description of a compiled launch shape: strip rows, committed
// columns per strip, warps per CTA.
struct TileShape {
    int rows, cols, warps;
};

int tile_shape_count();
TileShape tile_shape(int i);

// Launch one time step (local index `local` after RunState::step) of every
// tile in `tiles` with the compiled tile shape `shape`.
cudaError_t launch_step(int shape, const TubeDev* tubes, const Tile* tiles, int ntiles,
                        RunState* rs, int local, cudaStream_t stream);

// Set the text vs_last_error() returns on this host thread.
void record_error(const char* msg);

// RunState::step += k (the tail node of a captured chunk).
cudaError_t launch_advance(RunState* rs, int k, cudaStream_t stream);

}  // namespace vsb
