// vs_sections.cu -- depth maps of a batch of tubes as a function of their
// section widths and depths, and the vector-Jacobian product of that
// function, on the device.
//
// The map is the reference's elliptical depth kernel and post-processing
// (TubeDepth.cu:392-490, 642-762) on each tube's nominal rasterisation: the
// wall rows stay where the nominal widths put them, and every cell the depth
// kernel writes keeps its (section, semi-major axis a0, distance from the
// axis in cells) record, with a = a0 x width / nominal width, b = depth / 2:
//   raw      = 2 b sqrt(max(0, 1 - (dist ds)^2 / a^2))   (0 for the zero writes)
//   x, y     = raw, or raw at the pivot cell (mid row, tube end) where the
//              kernel wrote nothing (resetOpenSpaceDepth)
//   xs       = (x + x_right) / 2,  ys = (y + y_above) / 2   (edges: pivot values)
//   dp       = (xs + ys + xs_left + ys_below) / 4           (edges: pivot values)
// and depth_p, depth_x, depth_y = dp, xs, ys raised to 0.001 (TubeDepth.cu:90).
// Everything is evaluated in double and rounded to float once.  The reverse
// pass walks the same chain backwards; a clamped value passes no gradient.
#include <cuda_runtime.h>

#include "vs_device.h"

namespace vsb {
namespace {

constexpr double kMinDepth = (double)0.001f;

__device__ __forceinline__ double raw_value(const SectionCell& s, const SectionTube& t, const double* w,
                                            const double* d) {
    if (s.seg < 0) return 0.0;                               // zero write (or unwritten: not called)
    const double a = s.a0 * (w[s.seg] / t.w0[s.seg]);
    const double b = d[s.seg] / 2.0;
    const double y = (double)s.dist * t.ds;
    const double arg = 1.0 - (y * y) / (a * a);
    return arg > 0.0 ? 2.0 * b * sqrt(arg) : 0.0;
}

struct Frame {
    const SectionTube* t;
    const double* w;
    const double* d;
    __device__ double x(int64_t c) const {       // raw x with the unwritten cells at the pivot's value
        const SectionCell& s = t->cx[c];
        return raw_value(s.seg == kSectionUnwritten ? t->cx[t->pivot] : s, *t, w, d);
    }
    __device__ double y(int64_t c) const {
        const SectionCell& s = t->cy[c];
        return raw_value(s.seg == kSectionUnwritten ? t->cy[t->pivot] : s, *t, w, d);
    }
};

__global__ void section_maps_kernel(const SectionTube* __restrict__ tubes, const TubeDev* __restrict__ devs) {
    const SectionTube& T = tubes[blockIdx.y];
    const int H = T.H, W = T.W;
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= (int64_t)H * W) return;
    const int r = (int)(i / W), c = (int)(i % W);
    const Frame f{&T, T.w, T.d};
    const int64_t pv = T.pivot;
    const double xc = f.x(i), yc = f.y(i);
    const double xs = 0.5 * (xc + (c < W - 1 ? f.x(i + 1) : f.x(pv)));
    const double ys = 0.5 * (yc + (r > 0 ? f.y(i - W) : f.y(pv)));
    const double xl = c > 0 ? 0.5 * (f.x(i - 1) + xc) : 0.5 * (f.x(pv) + f.x(pv + 1));
    const double yb = r < H - 1 ? 0.5 * (f.y(i + W) + yc) : 0.5 * (f.y(pv) + f.y(pv - W));
    const double dp = 0.25 * (xs + ys + xl + yb);
    const TubeDev& D = devs[blockIdx.y];
    const int64_t o = (int64_t)r * D.pitch + c;
    const uint8_t m = (dp < kMinDepth ? 1 : 0) | (xs < kMinDepth ? 2 : 0) | (ys < kMinDepth ? 4 : 0);
    T.clamp[i] = m;
    float* dP = const_cast<float*>(D.dP);
    dP[o] = (float)(m & 1 ? kMinDepth : dp);
    dP[D.plane + o] = (float)(m & 2 ? kMinDepth : xs);
    dP[2 * D.plane + o] = (float)(m & 4 ? kMinDepth : ys);
}

// g_dp = dL/d dp (0 where clamped), read from the adjoint's depth_p gradient
__device__ __forceinline__ double g_dp(const SectionTube& T, const TubeDev& D, const double* gP, int r, int c) {
    const int64_t i = (int64_t)r * T.W + c;
    return (T.clamp[i] & 1) ? 0.0 : gP[(int64_t)r * D.pitch + c];
}

// pass 1: dL/d xs and dL/d ys (without the pivot's extra terms, which go to acc[0], acc[1])
__global__ void section_vjp1_kernel(const SectionTube* __restrict__ tubes, const TubeDev* __restrict__ devs,
                                    const AdjTube* __restrict__ adj) {
    const SectionTube& T = tubes[blockIdx.y];
    const TubeDev& D = devs[blockIdx.y];
    const AdjTube& A = adj[blockIdx.y];
    const int H = T.H, W = T.W;
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= (int64_t)H * W) return;
    const int r = (int)(i / W), c = (int)(i % W);
    const int64_t o = (int64_t)r * D.pitch + c;
    const double gd = g_dp(T, D, A.gP, r, c);
    double gxs = ((T.clamp[i] & 2) ? 0.0 : A.gX[o]) + 0.25 * gd;
    if (c + 1 < W) gxs += 0.25 * g_dp(T, D, A.gP, r, c + 1);
    double gys = ((T.clamp[i] & 4) ? 0.0 : A.gY[o]) + 0.25 * gd;
    if (r >= 1) gys += 0.25 * g_dp(T, D, A.gP, r - 1, c);
    T.gxs[i] = gxs;
    T.gys[i] = gys;
    if (c == 0 && gd != 0.0) atomicAdd(&T.acc[0], 0.25 * gd);       // xs_left = xs(pivot)
    if (r == H - 1 && gd != 0.0) atomicAdd(&T.acc[1], 0.25 * gd);   // ys_below = ys(pivot)
}

// pass 2: dL/d x and dL/d y of the filled raw maps
__global__ void section_vjp2_kernel(const SectionTube* __restrict__ tubes) {
    const SectionTube& T = tubes[blockIdx.y];
    const int H = T.H, W = T.W;
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= (int64_t)H * W) return;
    const int r = (int)(i / W), c = (int)(i % W);
    const int64_t pv = T.pivot;
    auto gxs = [&](int64_t k) { return T.gxs[k] + (k == pv ? T.acc[0] : 0.0); };
    auto gys = [&](int64_t k) { return T.gys[k] + (k == pv ? T.acc[1] : 0.0); };
    const double a = gxs(i), b = gys(i);
    double gx = 0.5 * a + (c >= 1 ? 0.5 * gxs(i - 1) : 0.0);
    double gy = 0.5 * b + (r + 1 <= H - 1 ? 0.5 * gys(i + W) : 0.0);
    if (c == W - 1 && a != 0.0) atomicAdd(&T.acc[2], 0.5 * a);      // x_right = x(pivot)
    if (r == 0 && b != 0.0) atomicAdd(&T.acc[3], 0.5 * b);          // y_above = y(pivot)
    if (T.cx[i].seg == kSectionUnwritten) {
        if (gx != 0.0) atomicAdd(&T.acc[4], gx);                    // x = x(pivot)
        gx = 0.0;
    }
    if (T.cy[i].seg == kSectionUnwritten) {
        if (gy != 0.0) atomicAdd(&T.acc[5], gy);
        gy = 0.0;
    }
    T.gx[i] = gx;
    T.gy[i] = gy;
}

// pass 3: dL/d width and dL/d depth of each section
__device__ __forceinline__ void raw_vjp(const SectionCell& s, const SectionTube& T, double g, double* dw,
                                        double* dd) {
    if (s.seg < 0 || g == 0.0) return;
    const double a = s.a0 * (T.w[s.seg] / T.w0[s.seg]);
    const double y = (double)s.dist * T.ds;
    const double arg = 1.0 - (y * y) / (a * a);
    if (!(arg > 0.0)) return;
    const double sq = sqrt(arg);
    const double b = T.d[s.seg] / 2.0;
    // v = 2 b sqrt(1 - y^2 / a^2): dv/db = 2 sqrt(arg), dv/da = 2 b y^2 / (a^3 sqrt(arg)), a = a0 w / w0
    atomicAdd(&dd[s.seg], g * sq);                                  // db/dd = 1/2
    atomicAdd(&dw[s.seg], g * (2.0 * b * y * y / (a * a * a * sq)) * (s.a0 / T.w0[s.seg]));
}

__global__ void section_vjp3_kernel(const SectionTube* __restrict__ tubes) {
    const SectionTube& T = tubes[blockIdx.y];
    const int64_t n = (int64_t)T.H * T.W;
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int64_t pv = T.pivot;
    const double gx = T.gx[i] + (i == pv ? T.acc[2] + T.acc[4] : 0.0);
    const double gy = T.gy[i] + (i == pv ? T.acc[3] + T.acc[5] : 0.0);
    raw_vjp(T.cx[i], T, gx, T.dw, T.dd);
    raw_vjp(T.cy[i], T, gy, T.dw, T.dd);
}

}  // namespace

cudaError_t launch_section_maps(const SectionTube* tubes, const TubeDev* devs, int ntubes, int64_t max_cells,
                                cudaStream_t st) {
    const dim3 grid((unsigned)((max_cells + 255) / 256), ntubes);
    section_maps_kernel<<<grid, 256, 0, st>>>(tubes, devs);
    return cudaGetLastError();
}

cudaError_t launch_section_vjp(const SectionTube* tubes, const TubeDev* devs, const AdjTube* adj, int ntubes,
                               int64_t max_cells, cudaStream_t st) {
    const dim3 grid((unsigned)((max_cells + 255) / 256), ntubes);
    section_vjp1_kernel<<<grid, 256, 0, st>>>(tubes, devs, adj);
    section_vjp2_kernel<<<grid, 256, 0, st>>>(tubes);
    section_vjp3_kernel<<<grid, 256, 0, st>>>(tubes);
    return cudaGetLastError();
}

}  // namespace vsb
