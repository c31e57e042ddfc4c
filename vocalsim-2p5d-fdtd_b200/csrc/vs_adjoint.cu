// vs_adjoint.cu -- reverse-time discrete adjoint of one FDTD step.
//
// For a table source the forward step (FDTDEngineCPU.cpp:316-410) is linear in
// the state.  Per interior cell c, with right / left / top / down neighbours:
//
//   P'_c  = (P_c dP_c - K1 S_c) / D_c,   D_c = (1 + s_c) dP_c,
//           S_c = U_c - U_left + W_c - W_down,  U = Vx dX,  W = Vy dY
//   Vx'_c = alx_c Vx_c + ax_c P'_c - bx_c P'_right + src,
//   Vy'_c = aly_c Vy_c + ay_c P'_c - by_c P'_top + src,
//
// with  g = 1/(mB + mS),  al = mB g,  a = g (bXY + mS zinv n x_out Nout),
// b = g (bXY + mS zinv n x_in Nin)  from the same cell codes the forward uses.
// The listener records P'_lis.  Transposing, with lamX' the adjoint of the
// state after the step:
//
//   mu_c   = lamP'_c + ax_c lamVx'_c - bx_left lamVx'_left
//                    + ay_c lamVy'_c - by_down lamVy'_down + dL/dtrace[n] [c = lis]
//            (mu = 0 on no-pressure cells of a Dirichlet mouth, where P' := 0)
//   lamU_c = K1 (mu_right / D_right - mu_c / D_c),   lamW_c = K1 (mu_top / D_top - mu_c / D_c)
//   lamVx_c = alx_c lamVx'_c + dX_c lamU_c,  lamVy_c = aly_c lamVy'_c + dY_c lamW_c,
//   lamP_c  = mu_c dP_c / D_c
//
// and the map gradients accumulate (in double, per cell)
//
//   dL/d dP_c += mu_c K1 S_c / ((1 + s_c) dP_c^2),   dL/d dX_c += Vx_c lamU_c,
//   dL/d dY_c += Vy_c lamW_c,
//   dL/d zinv  += g_x mS_x n_x (x2 Nout P'_c - x1 Nin P'_right) lamVx'_c + (same in y)
//
// The adjoint is evaluated in float with float coefficients (it is not meant
// to be bit-identical to anything); accumulators are double.
#include <cuda_runtime.h>

#include "vs_device.h"

namespace vsb {
namespace {

__constant__ float a_beta[16] = {0, 1, 0, 1, 1, 1, 1, 1, 1, 0, 0, 1, 0, 0, 0, 0};
__constant__ float a_airN[4] = {0.0f, 1.0f, 1.0f, 0.707106f};
__constant__ float a_wallN[4] = {1.0f, 1.0f, 1.0f, 0.0f};

// Coefficients of one velocity component of a cell (see the file comment).
struct VCoef {
    float al, a, b;      // V' = al V + a P'_c - b P'_nbr + source
    float zc_out, zc_in; // dV'/dzinv = zc_out P'_c - zc_in P'_nbr
};

// dirx = true: Vx of cell with code kc, right neighbour kn, top neighbour kt
// dirx = false: Vy of cell with code kc, top neighbour kn (= kt), right kr
__device__ inline VCoef vcoef(bool dirx, int kc, int kr, int kt, float zval, float bco,
                              const float* __restrict__ sig) {
    const int tc = kc & CODE_TYPE_MASK, tr = kr & CODE_TYPE_MASK, tt = kt & CODE_TYPE_MASK;
    const float bc = a_beta[tc], br = a_beta[tr], bt = a_beta[tt];
    const int lut = (br == 0.0f ? 2 : 0) + (bt == 0.0f ? 1 : 0);
    const float Nout = a_airN[lut] * bc, Nin = a_wallN[lut] * (1.0f - bc);
    const int tn = dirx ? tr : tt;
    const float bn = dirx ? br : bt;
    const float mB = fminf(bc, bn), mS = fmaxf(sig[tc], sig[tn]);
    const float bxy = mB != 0.0f ? bco : 0.0f;
    const int ec = tc == VS_CELL_EXCITATION, en = tn == VS_CELL_EXCITATION;
    const float nn = (float)((1 - ec) * (1 - en));
    const float xout = bc * (1.0f - bn), xin = bn * (1.0f - bc);
    const float z = (kc & CODE_ZINV_BIT) ? zval : 0.0f;
    const float g = 1.0f / (mB + mS);
    VCoef v;
    v.al = mB * g;
    v.a = g * (bxy + mS * z * nn * xout * Nout);
    v.b = g * (bxy + mS * z * nn * xin * Nin);
    const bool zc = (kc & CODE_ZINV_BIT) != 0;
    v.zc_out = zc ? g * mS * nn * xout * Nout : 0.0f;
    v.zc_in = zc ? g * mS * nn * xin * Nin : 0.0f;
    return v;
}

__global__ void adjoint_mu_kernel(const TubeDev* __restrict__ tubes, const AdjTube* __restrict__ adj, int64_t n,
                                  int par) {
    const TubeDev& T = tubes[blockIdx.y];
    const AdjTube& A = adj[blockIdx.y];
    const int W = T.W, H = T.H, pitch = T.pitch;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (H - 2) * (W - 2)) return;
    const int r = 1 + i / (W - 2), c = 1 + i % (W - 2);
    const int64_t pl = T.plane;
    const int64_t o = (int64_t)r * pitch + c;
    const uint8_t* __restrict__ code = T.code;
    const float* __restrict__ lam = A.lam[par];
    const float* __restrict__ sig = T.sigma;
    const int kc = code[o];
    if ((T.flags & TUBE_DIRICHLET) && (kc & CODE_TYPE_MASK) == VS_CELL_NOPRESSURE) {
        A.mu[o] = 0.0f;
        return;
    }
    const int kr = code[o + 1], kt = code[o - pitch];
    const VCoef cx = vcoef(true, kc, kr, kt, T.zinv, T.bcoef, sig);
    const VCoef cy = vcoef(false, kc, kr, kt, T.zinv, T.bcoef, sig);
    float mu = lam[o] + cx.a * lam[pl + o] + cy.a * lam[2 * pl + o];
    if (c - 1 >= 1) {   // the left cell's Vx' depends on this P' as its right neighbour
        const VCoef cl = vcoef(true, code[o - 1], kc, code[o - 1 - pitch], T.zinv, T.bcoef, sig);
        mu -= cl.b * lam[pl + o - 1];
    }
    if (r + 1 <= H - 2) {   // the cell below's Vy' depends on this P' as its top neighbour
        const VCoef cd = vcoef(false, code[o + pitch], code[o + pitch + 1], kc, T.zinv, T.bcoef, sig);
        mu -= cd.b * lam[2 * pl + o + pitch];
    }
    if (r == T.lis_y && c == T.lis_x) mu += A.gtrace[n];
    A.mu[o] = mu;
}

__global__ void adjoint_lambda_kernel(const TubeDev* __restrict__ tubes, const AdjTube* __restrict__ adj,
                                      int64_t slot, int par) {
    const TubeDev& T = tubes[blockIdx.y];
    const AdjTube& A = adj[blockIdx.y];
    const int W = T.W, H = T.H, pitch = T.pitch;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (H - 2) * (W - 2)) return;
    const int r = 1 + i / (W - 2), c = 1 + i % (W - 2);
    const int64_t pl = T.plane;
    const int64_t o = (int64_t)r * pitch + c;
    const uint8_t* __restrict__ code = T.code;
    const float* __restrict__ sig = T.sigma;
    const float* __restrict__ lam = A.lam[par];
    float* __restrict__ lout = A.lam[par ^ 1];
    const float* __restrict__ mu = A.mu;
    const float* __restrict__ dP = T.dP;
    const float* __restrict__ dX = T.dP + pl;
    const float* __restrict__ dY = T.dP + 2 * pl;
    const float K1 = T.K1;
    auto D = [&](int64_t q) { return (1.0f + sig[code[q] & CODE_TYPE_MASK]) * dP[q]; };
    const int kc = code[o], kr = code[o + 1], kt = code[o - pitch];
    const float muc = mu[o], Dc = D(o);
    // ring cells keep mu = 0, so the neighbours' terms vanish there
    const float lamU = K1 * (mu[o + 1] / D(o + 1) - muc / Dc);
    const float lamW = K1 * (mu[o - pitch] / D(o - pitch) - muc / Dc);
    const VCoef cx = vcoef(true, kc, kr, kt, T.zinv, T.bcoef, sig);
    const VCoef cy = vcoef(false, kc, kr, kt, T.zinv, T.bcoef, sig);
    const float lvx1 = lam[pl + o], lvy1 = lam[2 * pl + o];
    lout[o] = muc * dP[o] / Dc;
    lout[pl + o] = cx.al * lvx1 + dX[o] * lamU;
    lout[2 * pl + o] = cy.al * lvy1 + dY[o] * lamW;
    // state before the step (slot) and P' after it (slot + 1)
    const float* __restrict__ s0 = T.hist + slot * 3 * pl;
    const float* __restrict__ s1 = s0 + 3 * pl;
    const float vx = s0[pl + o], vy = s0[2 * pl + o];
    const float S = (vx * dX[o] - s0[pl + o - 1] * dX[o - 1]) + (vy * dY[o] - s0[2 * pl + o + pitch] * dY[o + pitch]);
    const float sc = sig[kc & CODE_TYPE_MASK];
    if (!((T.flags & TUBE_DIRICHLET) && (kc & CODE_TYPE_MASK) == VS_CELL_NOPRESSURE))
        A.gP[o] += (double)muc * (double)K1 * (double)S / ((1.0 + (double)sc) * (double)dP[o] * (double)dP[o]);
    A.gX[o] += (double)vx * (double)lamU;
    A.gY[o] += (double)vy * (double)lamW;
    if (kc & CODE_ZINV_BIT) {
        const float pc = s1[o], pr = s1[o + 1], pt = s1[o - pitch];
        A.gZ[o] += (double)(cx.zc_out * pc - cx.zc_in * pr) * (double)lvx1 +
                   (double)(cy.zc_out * pc - cy.zc_in * pt) * (double)lvy1;
    }
}

// Slot 0 of every tube's history = the state before the first step of a
// segment (P, Vx, Vy of parity par).
__global__ void history_seed_kernel(const TubeDev* __restrict__ tubes, int par) {
    const TubeDev& T = tubes[blockIdx.y];
    const int64_t pl = T.plane;
    const int64_t n = (int64_t)T.H * T.pitch;
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* P = T.P[0] + par * pl;
    T.hist[i] = P[i];
    T.hist[pl + i] = P[2 * pl + i];
    T.hist[2 * pl + i] = P[4 * pl + i];
}

}  // namespace

cudaError_t launch_history_seed(const TubeDev* tubes, int ntubes, int max_plane_cells, int par, cudaStream_t stream) {
    const dim3 grid((max_plane_cells + 255) / 256, ntubes);
    history_seed_kernel<<<grid, 256, 0, stream>>>(tubes, par);
    return cudaGetLastError();
}

cudaError_t launch_adjoint_step(const TubeDev* tubes, const AdjTube* adj, int ntubes, int max_cells, int64_t n,
                                int64_t slot, int par, cudaStream_t stream) {
    const dim3 grid((max_cells + 255) / 256, ntubes);
    adjoint_mu_kernel<<<grid, 256, 0, stream>>>(tubes, adj, n, par);
    adjoint_lambda_kernel<<<grid, 256, 0, stream>>>(tubes, adj, slot, par);
    return cudaGetLastError();
}

}  // namespace vsb
