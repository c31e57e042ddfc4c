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
// to be bit-identical to anything); accumulators are double.  The static
// coefficients (al, a, b, zc of each direction, 1 + sigma) of every cell come
// from a per-tube table indexed by the cell's neighbourhood descriptor
// (adjoint_coefficients, vs_capi.cpp).
#include <cuda_runtime.h>

#include "vs_device.h"

namespace vsb {
namespace {

// Fields of a tube the reverse step reads, held in registers (the kernel's
// stores go through other pointers, so nothing here changes during a launch).
struct AdjView {
    const float* lam;         // adjoint of the state after the step (read only)
    const uint8_t* desc;
    const float4* tab;
    const float* dP;
    const float* gtrace;
    int64_t pl;
    int pitch, H, lis_y, lis_x, exc_y, exc_x;
    bool tmm;
    float pending;            // d/d p1 of the step after this one, at the excitation point
};

// mu of interior cell (r, c), the adjoint of P' (see the file comment), and
// q = mu / D.  The coefficients come from the cell's neighbourhood
// descriptor: A = (ax, ay, bx, by), B = (alx, aly, 1 + sigma, Dirichlet
// no-pressure flag); the left cell's bx and the lower cell's by from theirs.
__device__ __forceinline__ float mu_at(const AdjView& v, int r, int c, int64_t n, float* q) {
    const int64_t o = (int64_t)r * v.pitch + c;
    const int d = __ldg(v.desc + o);
    const int dl = c - 1 >= 1 ? __ldg(v.desc + o - 1) : -1;
    const int dd = r + 1 <= v.H - 2 ? __ldg(v.desc + o + v.pitch) : -1;
    const float l0 = __ldg(v.lam + o), lx = __ldg(v.lam + v.pl + o), ly = __ldg(v.lam + 2 * v.pl + o);
    const float lxl = dl >= 0 ? __ldg(v.lam + v.pl + o - 1) : 0.0f;
    const float lyd = dd >= 0 ? __ldg(v.lam + 2 * v.pl + o + v.pitch) : 0.0f;
    const float dpc = __ldg(v.dP + o);
    const float4 ea = __ldg(v.tab + 3 * d), eb = __ldg(v.tab + 3 * d + 1);
    if (eb.w != 0.0f) { *q = 0.0f; return 0.0f; }    // P' := 0 on a Dirichlet mouth
    float mu = l0 + ea.x * lx + ea.y * ly;
    if (dl >= 0) mu -= __ldg(v.tab + 3 * dl).z * lxl;
    if (dd >= 0) mu -= __ldg(v.tab + 3 * dd).w * lyd;
    if (r == v.lis_y && c == v.lis_x) mu += __ldg(v.gtrace + n);
    // the two-mass flow of the step after this one read P' here
    if (v.tmm && r == v.exc_y && c == v.exc_x) mu += v.pending;
    *q = mu / (eb.z * dpc);
    return mu;
}

// ---- two-mass source ------------------------------------------------------
// With the two-mass source, exeV_n = ug_n = TMM(state_n, p1 = P_n[exc]) feeds
// the velocity of the excitation cells.  Its reverse step needs the Jacobian
// of one model step (TwoMassModel.cpp:90-232) with respect to the six state
// values and p1.  Lane j of a warp evaluates the step's expressions in
// double on a dual number carrying the derivative along input j (forward
// mode; branches follow the primal values), so lanes 0..6 hold the seven
// columns of the Jacobian.
struct Dual {
    double v, d;
};

__device__ inline Dual dc(double v) { return {v, 0.0}; }
__device__ inline Dual operator+(Dual a, Dual b) { return {a.v + b.v, a.d + b.d}; }
__device__ inline Dual operator-(Dual a, Dual b) { return {a.v - b.v, a.d - b.d}; }
__device__ inline Dual operator*(Dual a, Dual b) { return {a.v * b.v, a.d * b.v + a.v * b.d}; }
__device__ inline Dual operator*(double a, Dual b) { return {a * b.v, a * b.d}; }
__device__ inline Dual operator+(double a, Dual b) { return {a + b.v, b.d}; }
__device__ inline Dual operator-(double a, Dual b) { return {a - b.v, -b.d}; }
__device__ inline Dual dabs(Dual a) { return a.v < 0.0 ? Dual{-a.v, -a.d} : a; }

__device__ inline Dual dinv(Dual b) {
    const double r = 1.0 / b.v;
    return {r, -b.d * r * r};
}

// One model step on st = {x1_old, x1_curr, x2_old, x2_curr, ug_old, ug_curr}.
// The divisions by state-dependent quantities go through one reciprocal
// each (Ag1, Ag2 before and after the update, the flow denominator), so the
// chain holds three dependent double divisions; the values agree with the
// forward model to rounding, which is all its derivative needs.
__device__ void tmm_math(const TmmConsts64& k, Dual st[6], Dual p1) {
    const double srate = k.srate, isr = 1.0 / srate, is2 = isr * isr;
    const double lg = k.lg, two_lg = 2.0 * lg, rho = k.rho, ps = k.ps;
    const double thr1 = -k.Ag01 / two_lg, thr2 = -k.Ag02 / two_lg;
    const double g1 = k.Ag01 / two_lg, g2 = k.Ag02 / two_lg;
    const double iA1 = 1.0 / k.A1;
    const Dual x1o = st[0], x1 = st[1], x2o = st[2], x2 = st[3], ugo = st[4], ug = st[5];
    const Dual ia1 = dinv(k.Ag01 + two_lg * x1), ia2 = dinv(k.Ag02 + two_lg * x2);
    const Dual ia1s = ia1 * ia1, ia2s = ia2 * ia2;
    const double c12 = 12.0 * k.mu * lg * lg;
    const Dual Rv1 = (c12 * k.d1) * (ia1s * ia1), Lg1 = (rho * k.d1) * ia1;
    const Dual Rv2 = (c12 * k.d2) * (ia2s * ia2), Lg2 = (rho * k.d2) * ia2;
    Dual pm1 = dc(ps), pm2;
    if (x1.v > thr1 && x2.v > thr2) {
        const Dual q = ug * ia1;
        pm1 = ps - 1.37 * (rho / 2.0) * q * q - 0.5 * (Rv1 * ug + srate * (Lg1 * (ug - ugo)));
    }
    const Dual fm1 = (k.d1 * lg) * pm1;
    if (x1.v > thr1) {
        if (x2.v > thr2)
            pm2 = pm1 - (0.5 * (Rv1 + Rv2) * ug + srate * ((Lg1 + Lg2) * (ug - ugo))) -
                  (rho / 2.0) * ug * ug * (ia2s - ia1s);
        else
            pm2 = dc(ps);
    } else {
        pm2 = dc(0.0);
    }
    const Dual fm2 = (k.d2 * lg) * pm2;
    const bool c1 = x1.v + g1 < 0.0, c2 = x2.v + g2 < 0.0;
    const double h1u = c1 ? k.h1 : 0.0, r1u = c1 ? k.r1c : k.r1o;
    const double h2u = c2 ? k.h2 : 0.0, r2u = c2 ? k.r2c : k.r2o;
    const double a11 = (k.k1 + h1u + k.kc) * is2 + r1u * isr + k.m1;
    const double a12 = -k.kc * is2;
    const double a22 = (k.k2 + h2u + k.kc) * is2 + r2u * isr + k.m2;
    const Dual e1 = g1 + x1, e2 = g2 + x2;
    const Dual sp1 = (k.k1 * k.etak1) * x1 * x1 * x1 + h1u * (g1 + k.etah1 * e1 * e1 * e1);
    const Dual sp2 = (k.k2 * k.etak2) * x2 * x2 * x2 + h2u * (g2 + k.etah2 * e2 * e2 * e2);
    const Dual b1 = (2.0 * k.m1 + r1u * isr) * x1 - k.m1 * x1o + is2 * (fm1 - sp1);
    const Dual b2 = (2.0 * k.m2 + r2u * isr) * x2 - k.m2 * x2o + is2 * (fm2 - sp2);
    double det = a11 * a22 - a12 * a12;
    if (det == 0.0) det = 1.0;
    const double idet = 1.0 / det;
    const Dual x1n = idet * (a22 * b1 - a12 * b2);
    const Dual x2n = idet * (a11 * b2 - a12 * b1);
    const Dual A1n = k.Ag01 + two_lg * x1n, A2n = k.Ag02 + two_lg * x2n;
    Dual ugn = dc(0.0);
    if (!(A1n.v < 0.0 || A2n.v < 0.0)) {
        const Dual ib1 = dinv(A1n), ib2 = dinv(A2n);
        const Dual ib1s = ib1 * ib1, ib2s = ib2 * ib2;
        const Dual r = iA1 * A2n;
        const Dual Rtot = (rho / 2.0) * dabs(ug) * (0.37 * ib1s + (1.0 - 2.0 * r * (1.0 - r)) * ib2s) +
                          c12 * (k.d1 * (ib1s * ib1) + k.d2 * (ib2s * ib2));
        const Dual Ltot = rho * (k.d1 * ib1 + k.d2 * ib2);
        ugn = (isr * (ps - p1) + Ltot * ug) * dinv(isr * Rtot + Ltot);
    }
    st[0] = x1; st[1] = x1n; st[2] = x2; st[3] = x2n; st[4] = ug; st[5] = ugn;
}

// Reverse of the two-mass step n, by one warp: lam holds the adjoint of the
// state after step n.  d/d p1 belongs to the adjoint of the state before the
// step at the excitation point; it is left in lam_tmm[6 + (par ^ 1)] for the
// next reverse step's mu there, so this warp runs beside the cell blocks.
__device__ void tmm_reverse(const TubeDev& T, const AdjTube& A, const float* __restrict__ lam, int par,
                            int64_t slot) {
    const int lane = threadIdx.x & 31;
    // dL/d exeV = sum over the velocities it enters of lambda' * dV'/d exeV
    double lexe = 0.0;
    for (int i = lane; i < A.n_exc; i += 32) lexe += (double)A.exc_coef[i] * (double)lam[A.exc_off[i]];
    for (int m = 16; m > 0; m >>= 1) lexe += __shfl_xor_sync(0xffffffffu, lexe, m);
    const int64_t pl = T.plane;
    const int64_t oexc = (int64_t)T.exc_y * T.pitch + T.exc_x;
    const double* sv = T.tmm_hist + 6 * slot;
    double lo[6];
    for (int i = 0; i < 6; ++i) lo[i] = A.lam_tmm[i];
    lo[5] += lexe;                          // ug_curr after the step is exeV_n
    __syncwarp();
    if (lane < 7) {
        Dual st[6];
        for (int i = 0; i < 6; ++i) st[i] = Dual{sv[i], i == lane ? 1.0 : 0.0};
        const Dual p1{(double)T.hist[slot * 3 * pl + oexc], lane == 6 ? 1.0 : 0.0};
        tmm_math(T.tmmd, st, p1);
        double lin = 0.0;
        for (int i = 0; i < 6; ++i) lin += lo[i] * st[i].d;
        if (lane < 6) A.lam_tmm[lane] = lin;
        else A.lam_tmm[6 + (par ^ 1)] = lin;
    }
}

// One reverse step: block (tile, tube) computes mu over its 32 x 8 cells
// plus the row above and the column to the right into shared memory, then
// lambda of the state before the step and the gradient terms of its cells;
// the block holding the excitation point also runs the two-mass reverse step.
__global__ void __launch_bounds__(kAdjTileW * kAdjTileH, 3)
adjoint_step_kernel(const TubeDev* __restrict__ tubes, const AdjTube* __restrict__ adj,
                    const AdjRun* __restrict__ run, int local) {
    const TubeDev& T = tubes[blockIdx.y];
    const AdjTube& A = adj[blockIdx.y];
    const AdjRun ar = *run;
    const int64_t n = ar.start + ar.len - 1 - local;
    const int64_t slot = n - ar.start;
    const int par = ar.q0 ^ (local & 1);
    if ((int)blockIdx.x >= A.tiles) {
        // the block after the last tile reverses the two-mass step
        if ((int)blockIdx.x == A.tiles && (T.flags & TUBE_TMM) && threadIdx.x < 32)
            tmm_reverse(T, A, A.lam[par], par, slot);
        return;
    }
    const int W = T.W, H = T.H, pitch = T.pitch;
    const int tiles_x = (W - 2 + kAdjTileW - 1) / kAdjTileW;
    const int c0 = 1 + (int)(blockIdx.x % tiles_x) * kAdjTileW, r0 = 1 + (int)(blockIdx.x / tiles_x) * kAdjTileH;
    const int tx = threadIdx.x % kAdjTileW, ty = threadIdx.x / kAdjTileW;
    AdjView v;
    v.lam = A.lam[par];
    v.desc = A.desc;
    v.tab = A.tab;
    v.dP = T.dP;
    v.gtrace = A.gtrace;
    v.pl = T.plane;
    v.pitch = pitch; v.H = H;
    v.lis_y = T.lis_y; v.lis_x = T.lis_x; v.exc_y = T.exc_y; v.exc_x = T.exc_x;
    v.tmm = (T.flags & TUBE_TMM) != 0;
    v.pending = v.tmm ? (float)A.lam_tmm[6 + par] : 0.0f;
    float* __restrict__ lout = A.lam[par ^ 1];
    double* __restrict__ gP = A.gP;
    double* __restrict__ gX = A.gX;
    double* __restrict__ gY = A.gY;
    const int64_t pl = v.pl;
    const float K1 = T.K1;
    const float* __restrict__ s0 = T.hist + slot * 3 * pl;   // state before the step
    const float* __restrict__ s1 = s0 + 3 * pl;              // P' after it
    const int r = r0 + ty, c = c0 + tx;
    const bool in = r <= H - 2 && c <= W - 2;
    const int64_t o = (int64_t)r * pitch + c;

    // loads of this cell's update that do not depend on mu, issued before it
    float lvx1 = 0.0f, lvy1 = 0.0f, dpc = 1.0f, dxc = 0.0f, dyc = 0.0f, dxl = 0.0f, dyd = 0.0f;
    float vx = 0.0f, vy = 0.0f, vxl = 0.0f, vyd = 0.0f;
    double gx0 = 0.0, gy0 = 0.0, gp0 = 0.0;
    float4 eb = make_float4(0.0f, 0.0f, 1.0f, 0.0f);
    int d = 0;
    if (in) {
        d = __ldg(v.desc + o);
        eb = __ldg(v.tab + 3 * d + 1);
        lvx1 = __ldg(v.lam + pl + o);
        lvy1 = __ldg(v.lam + 2 * pl + o);
        dpc = __ldg(T.dP + o);
        dxc = __ldg(T.dP + pl + o);
        dyc = __ldg(T.dP + 2 * pl + o);
        dxl = __ldg(T.dP + pl + o - 1);
        dyd = __ldg(T.dP + 2 * pl + o + pitch);
        vx = __ldg(s0 + pl + o);
        vy = __ldg(s0 + 2 * pl + o);
        vxl = __ldg(s0 + pl + o - 1);
        vyd = __ldg(s0 + 2 * pl + o + pitch);
        gx0 = gX[o];
        gy0 = gY[o];
        gp0 = gP[o];
    }

    // mu and q = mu / D of the tile, the row above (row 0) and the column to the right (column 32)
    __shared__ float smu[kAdjTileH + 1][kAdjTileW + 1];
    __shared__ float sq[kAdjTileH + 1][kAdjTileW + 1];
    {
        float q = 0.0f;
        smu[ty + 1][tx] = in ? mu_at(v, r, c, n, &q) : 0.0f;
        sq[ty + 1][tx] = q;
    }
    if (threadIdx.x < kAdjTileW) {
        const int rr = r0 - 1, cc = c0 + (int)threadIdx.x;
        float q = 0.0f;
        smu[0][threadIdx.x] = (rr >= 1 && cc <= W - 2) ? mu_at(v, rr, cc, n, &q) : 0.0f;
        sq[0][threadIdx.x] = q;
    } else if (threadIdx.x < kAdjTileW + kAdjTileH) {
        const int k = threadIdx.x - kAdjTileW, rr = r0 + k, cc = c0 + kAdjTileW;
        float q = 0.0f;
        smu[k + 1][kAdjTileW] = (rr <= H - 2 && cc <= W - 2) ? mu_at(v, rr, cc, n, &q) : 0.0f;
        sq[k + 1][kAdjTileW] = q;
    }
    __syncthreads();
    if (in) {
        const float muc = smu[ty + 1][tx];
        // ring cells and no-pressure cells of a Dirichlet mouth have mu = q = 0
        const float qc = sq[ty + 1][tx], qr = sq[ty + 1][tx + 1], qt = sq[ty][tx];
        const float lamU = K1 * (qr - qc);
        const float lamW = K1 * (qt - qc);
        lout[o] = qc * dpc;
        lout[pl + o] = eb.x * lvx1 + dxc * lamU;
        lout[2 * pl + o] = eb.y * lvy1 + dyc * lamW;
        const float S = (vx * dxc - vxl * dxl) + (vy * dyc - vyd * dyd);
        if (muc != 0.0f) gP[o] = gp0 + (double)qc * (double)K1 * (double)S / (double)dpc;
        gX[o] = gx0 + (double)vx * (double)lamU;
        gY[o] = gy0 + (double)vy * (double)lamW;
        if (T.code[o] & CODE_ZINV_BIT) {
            const float4 ez = __ldg(v.tab + 3 * d + 2);
            const float pc = s1[o], pr = s1[o + 1], pt = s1[o - pitch];
            A.gZ[o] += (double)(ez.x * pc - ez.y * pr) * (double)lvx1 + (double)(ez.z * pc - ez.w * pt) * (double)lvy1;
        }
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
    if (i == 0 && (T.flags & TUBE_TMM)) {
        double* h = T.tmm_hist;
        if (T.flags & TUBE_TMM64) {
            const TmmState64 s = T.tmm64[par];
            h[0] = s.x1_old; h[1] = s.x1_curr; h[2] = s.x2_old; h[3] = s.x2_curr; h[4] = s.ug_old; h[5] = s.ug_curr;
        } else {
            const TmmState s = T.tmm[par];
            h[0] = s.x1_old; h[1] = s.x1_curr; h[2] = s.x2_old; h[3] = s.x2_curr; h[4] = s.ug_old; h[5] = s.ug_curr;
        }
    }
}

}  // namespace

cudaError_t launch_history_seed(const TubeDev* tubes, int ntubes, int max_plane_cells, int par, cudaStream_t stream) {
    const dim3 grid((max_plane_cells + 255) / 256, ntubes);
    history_seed_kernel<<<grid, 256, 0, stream>>>(tubes, par);
    return cudaGetLastError();
}

cudaError_t launch_adjoint_step(const TubeDev* tubes, const AdjTube* adj, int ntubes, int max_tiles,
                                const AdjRun* run, int local, cudaStream_t stream) {
    const dim3 grid(max_tiles, ntubes);
    adjoint_step_kernel<<<grid, kAdjTileW * kAdjTileH, 0, stream>>>(tubes, adj, run, local);
    return cudaGetLastError();
}

}  // namespace vsb
