// vs_mapbuild.cu -- batched device map builder.
//
// Paints, for every tube of a batch at once, the maps the reference's setup
// kernels build (FDTDSolver::setupWaveSolver, FDTDSolver.cu:289-476): the cell
// types with the wall-gap fill (TubeGeometry.cu:433-569), the excitation and
// no-pressure columns (:571-612, FDTDSolver.cu:591-611), the dead ring and the
// graded PML (FDTDSolver.cu:373-464), the z_inv bit of every wall cell that
// carries a segment id (FDTDSolver.cu:613-622), and for the 2.5D solver the
// depth maps of circular and elliptical sections (TubeDepth.cu:95-169) with
// generateDepthP and setMinDepth (:215-253, 642-762).  The host computes only
// what is per column (wall rows, the rows the gap fill adds, segment ids:
// build_tube_columns); every cell is painted here, straight into the batch's
// device planes, with the host builder's float expressions in its operand
// order (this file is compiled with --fmad=false), so the maps equal the
// host builder's bit for bit.
//
// Three launches over all tubes' cells: paint (types, codes, pre-smoothing
// dX / dY with the open-space value replaced by the pivot's), smooth (the
// half-sums of dX with its right and dY with its upper neighbour) and
// depth P (the quarter-sum, then the minimum depth on all three planes).
#include <cuda_runtime.h>

#include "vs_device.h"

namespace vsb {
namespace {

constexpr float kOpenSpaceDepth = 0.5f;   // FDTDSolver.cu:292, TubeDepth.cu:91
constexpr float kMinDepth = 0.001f;       // TubeDepth::min_depth

struct DepthVal {
    float dx, dy;
};

// Radicand of the half-depth at distance y from the axis of tube column k.
__device__ __forceinline__ float radicand(const MapBuild& m, int k, float y) {
    const int air = m.down[k] - m.up[k] - 1;
    if (m.depth == MAP_DEPTH_CIRCLE) {
        const float r = ((float)air / 2.0f) * m.ds;
        const float r2 = r * r;
        if (m.depth_fma) return fmaf(-y, y, r2);
        const float yy = y * y;
        return r2 - yy;
    }
    const float a = (air * m.ds) / 2.0f;
    const float b = m.minor[m.seg[k]] / 2.0f;
    const float a2 = a * a, b2 = b * b;
    const float yy = y * y;
    return b2 * (1.0f - (yy / a2));
}

// dX, dY of row r of tube column k before generateDepthP, as
// TubeDepth::setTubeDepth leaves them.  Ring kk of the air rows (kk = h at the
// walls, 0 at the axis) has dX from the half-depth at distance kk ds, dY from
// kk + 1/2 for its upper row (0 for kk = h) and from kk - 1/2 for its lower
// row; the reference writes the rings from the walls in, the upper row before
// the lower, so a row that is both (the axis row) keeps the lower value.  The
// column's two wall rows get 0, every other cell the open-space value.
__device__ DepthVal column_depth(const MapBuild& m, int k, int r, int* err) {
    const int up = m.up[k], down = m.down[k];
    if (r == up || r == down) return {0.0f, 0.0f};
    if (r < up || r > down) return {kOpenSpaceDepth, kOpenSpaceDepth};
    const int air = down - up - 1;
    const int h = (int)ceilf(air * 0.5f) - 1;
    const int du = r - up - 1, dl = down - 1 - r;           // rows from the upper / lower wall
    int kk;
    bool lower;
    const bool as_up = du <= h, as_lo = dl <= h;
    if (as_up && as_lo) {
        const int ku = h - du, kl = h - dl;
        lower = kl <= ku;          // the later write: smaller ring, and the lower row on a tie
        kk = lower ? kl : ku;
    } else if (as_up) {
        kk = h - du;
        lower = false;
    } else if (as_lo) {
        kk = h - dl;
        lower = true;
    } else {
        return {kOpenSpaceDepth, kOpenSpaceDepth};
    }
    const float ds = m.ds;
    const float rx = radicand(m, k, (float)kk * ds);
    const float rlo = radicand(m, k, ((float)kk - 0.5f) * ds);
    const float rup = kk != h ? radicand(m, k, ((float)kk + 0.5f) * ds) : 0.0f;
    if (rx < 0.f || rlo < 0.f || rup < 0.f) atomicExch(err, VS_ERR_NEGATIVE_SQRT);
    float vx = 2 * sqrtf(rx), vup = 2 * sqrtf(rup), vlo = 2 * sqrtf(rlo);
    if (m.ud > 0.0f) {
        vx = m.ud;
        vlo = m.ud;
        vup = kk != h ? m.ud : 0.0f;
    }
    return {vx, lower ? vlo : vup};
}

// Pre-smoothing dX, dY of frame cell (r, c), with the open-space value
// replaced by the pivot cell's (generateDepthP's first step).
__device__ DepthVal raw_depth(const MapBuild& m, int r, int c, int* err) {
    auto at = [&](int rr, int cc) -> DepthVal {
        const int k = cc - m.sx;
        if (k < 0 || k >= m.L) return {kOpenSpaceDepth, kOpenSpaceDepth};
        return column_depth(m, k, rr, err);
    };
    DepthVal v = at(r, c);
    if (v.dx == kOpenSpaceDepth || v.dy == kOpenSpaceDepth) {
        const DepthVal pv = at(m.my, m.ex);
        if (v.dx == kOpenSpaceDepth) v.dx = pv.dx;
        if (v.dy == kOpenSpaceDepth) v.dy = pv.dy;
    }
    return v;
}

// Cell type and segment-id flag of frame cell (r, c).
__device__ uint8_t cell_code(const MapBuild& m, int r, int c) {
    const int H = m.H, W = m.W;
    int type = VS_CELL_AIR;
    bool segment = false;
    const int k = c - m.sx;
    if (k >= 0 && k < m.L) {
        if ((r >= m.utop[k] && r <= m.up[k]) || (r >= m.down[k] && r <= m.dbot[k])) {
            type = VS_CELL_WALL;
            segment = true;
        }
    } else if (k == -1) {
        // the excitation column: its wall cells carry no segment id
        if (r == m.up[0] || r == m.down[0]) type = VS_CELL_WALL;
        else if (r > m.up[0] && r < m.down[0]) type = VS_CELL_EXCITATION;
    } else if (c == m.npc) {
        if (r >= m.up[m.L - 1] && r <= m.down[m.L - 1]) type = VS_CELL_NOPRESSURE;
    }
    if (r == 0 || r == H - 1 || c == 0 || c == W - 1) {
        type = VS_CELL_DEAD;
    } else if (m.pml) {
        // graded layers, outermost = pml5: rows first, then columns (corners)
        for (int l = 0; l < m.pml; ++l)
            if ((r == 1 + l || r == H - 2 - l) && c >= 1 + l && c <= W - 2 - l) type = VS_CELL_PML5 - l;
        for (int l = 0; l < m.pml; ++l)
            if ((c == 1 + l || c == W - 2 - l) && r >= 1 + l && r <= H - 2 - l) type = VS_CELL_PML5 - l;
    }
    return (uint8_t)(type | (segment ? CODE_ZINV_BIT : 0));
}

__global__ void paint_kernel(const MapBuild* __restrict__ tubes, int* __restrict__ err) {
    const MapBuild m = tubes[blockIdx.y];
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= (int64_t)m.H * m.pitch) return;
    const int r = (int)(i / m.pitch), c = (int)(i % m.pitch);
    if (c >= m.W) {                      // row padding: dead, zero depth
        m.code[i] = (uint8_t)VS_CELL_DEAD;
        m.dP[i] = 0.0f;
        m.dX[i] = 0.0f;
        m.dY[i] = 0.0f;
        return;
    }
    m.code[i] = cell_code(m, r, c);
    if (m.depth == MAP_DEPTH_NONE) {     // 2D solver: unit depths
        m.dP[i] = 1.0f;
        m.dX[i] = 1.0f;
        m.dY[i] = 1.0f;
        return;
    }
    const DepthVal v = raw_depth(m, r, c, err);
    m.dX[i] = v.dx;
    m.dY[i] = v.dy;
}

// half-sums: dX with its right neighbour, dY with its upper one (the pivot's
// value beyond the frame), into the scratch planes
__global__ void smooth_kernel(const MapBuild* __restrict__ tubes) {
    const MapBuild m = tubes[blockIdx.y];
    if (m.depth == MAP_DEPTH_NONE) return;
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= (int64_t)m.H * m.pitch) return;
    const int r = (int)(i / m.pitch), c = (int)(i % m.pitch);
    if (c >= m.W) return;
    const int64_t pivot = (int64_t)m.my * m.pitch + m.ex;
    const float right = c < m.W - 1 ? m.dX[i + 1] : m.dX[pivot];
    const float above = r > 0 ? m.dY[i - m.pitch] : m.dY[pivot];
    m.tmpx[i] = 0.5f * (m.dX[i] + right);
    m.tmpy[i] = 0.5f * (m.dY[i] + above);
}

// the quarter-sum of dP, then the minimum depth on dP, dX and dY
__global__ void depthp_kernel(const MapBuild* __restrict__ tubes) {
    const MapBuild m = tubes[blockIdx.y];
    if (m.depth == MAP_DEPTH_NONE) return;
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= (int64_t)m.H * m.pitch) return;
    const int r = (int)(i / m.pitch), c = (int)(i % m.pitch);
    if (c >= m.W) return;
    const int64_t pivot = (int64_t)m.my * m.pitch + m.ex;
    const float x = m.tmpx[i], y = m.tmpy[i];
    const float left = c > 0 ? m.tmpx[i - 1] : m.tmpx[pivot];
    const float below = r < m.H - 1 ? m.tmpy[i + m.pitch] : m.tmpy[pivot];
    float p = 0.25f * (x + y + left + below);
    float dx = x, dy = y;
    if (p < kMinDepth) p = kMinDepth;
    if (dx < kMinDepth) dx = kMinDepth;
    if (dy < kMinDepth) dy = kMinDepth;
    m.dP[i] = p;
    m.dX[i] = dx;
    m.dY[i] = dy;
}

}  // namespace

cudaError_t launch_build_maps(const MapBuild* tubes, int ntubes, int64_t max_cells, int* err, cudaStream_t stream) {
    if (ntubes <= 0) return cudaSuccess;
    const dim3 grid((unsigned)((max_cells + 255) / 256), (unsigned)ntubes);
    paint_kernel<<<grid, 256, 0, stream>>>(tubes, err);
    smooth_kernel<<<grid, 256, 0, stream>>>(tubes);
    depthp_kernel<<<grid, 256, 0, stream>>>(tubes);
    return cudaGetLastError();
}

}  // namespace vsb
