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

// ---------------------------------------------------------------------------
// The same reverse step in strip form: one warp per strip of TR rows x
// 30 NC columns, NC consecutive columns per lane (one aligned NC-float load
// per plane row), lanes 1..30 commit; strip k of a tube starts at column
// c0 = 30 NC k - NC.  The warp marches down its rows: mu and q of row r come
// from the row's own lambda' and that of the row below (kept one row ahead
// in registers), the left neighbour's bx lambdaVx' and Vx dX by one shuffle;
// the commit of row r takes q of the right neighbour by one shuffle and q of
// the row above from the previous iteration (the row above the strip is
// computed, not committed).  No shared memory and no block barrier.  The
// per-cell gradient terms are formed in float and added to the double
// accumulators; q = mu / D uses the fast division (the adjoint is not meant
// to be bit-identical to anything).
template <int NC>
struct Row {
    float v[NC];
};

template <int NC>
__device__ __forceinline__ void ldrow(float (&d)[NC], const float* p, bool ok) {
    if (!ok) {
#pragma unroll
        for (int q = 0; q < NC; ++q) d[q] = 0.0f;
        return;
    }
    if constexpr (NC == 4) {
        const float4 t = __ldg(reinterpret_cast<const float4*>(p));
        d[0] = t.x; d[1] = t.y; d[2] = t.z; d[3] = t.w;
    } else if constexpr (NC == 2) {
        const float2 t = __ldg(reinterpret_cast<const float2*>(p));
        d[0] = t.x; d[1] = t.y;
    } else {
#pragma unroll
        for (int q = 0; q < NC; ++q) d[q] = __ldg(p + q);
    }
}

template <int NC>
__device__ __forceinline__ uint32_t ldbytes(const uint8_t* p, bool ok) {
    if (!ok) return 0u;
    if constexpr (NC == 4) return __ldg(reinterpret_cast<const uint32_t*>(p));
    else if constexpr (NC == 2) return (uint32_t)__ldg(reinterpret_cast<const uint16_t*>(p));
    else return (uint32_t)__ldg(p);
}

__device__ __forceinline__ int byte_at(uint32_t k, int q) { return (int)((k >> (8 * q)) & 0xffu); }

template <int NC, int TR, int WARPS>
__global__ void __launch_bounds__(WARPS * 32)
adjoint_strip_kernel(const TubeDev* __restrict__ tubes, const AdjTube* __restrict__ adj,
                     const AdjRun* __restrict__ run, int local) {
    const TubeDev& T = tubes[blockIdx.y];
    const AdjTube& A = adj[blockIdx.y];
    const AdjRun ar = *run;
    const int64_t n = ar.start + ar.len - 1 - local;
    const int64_t slot = n - ar.start;
    const int par = ar.q0 ^ (local & 1);
    const int nblk = (A.strips + WARPS - 1) / WARPS;
    if ((int)blockIdx.x >= nblk) {
        // the block after the last strip block reverses the two-mass step
        if ((int)blockIdx.x == nblk && (T.flags & TUBE_TMM) && threadIdx.x < 32)
            tmm_reverse(T, A, A.lam[par], par, slot);
        return;
    }
    const int s = (int)blockIdx.x * WARPS + (int)(threadIdx.x >> 5);
    if (s >= A.strips) return;
    constexpr unsigned kAll = 0xffffffffu;
    constexpr int kCommit = 30 * NC;
    const int lane = threadIdx.x & 31;
    const int W = T.W, H = T.H, pitch = T.pitch;
    const int nsx = (W - 2) / kCommit + 1;
    const int c0 = kCommit * (s % nsx) - NC;
    const int r0 = 1 + (s / nsx) * TR;
    const int rlast = min(r0 + TR - 1, H - 2);
    const int x0 = c0 + NC * lane;
    const bool ok = x0 >= 0 && x0 < pitch;          // the lane's NC columns lie in the pitched row
    unsigned inter = 0, commit = 0;
#pragma unroll
    for (int q = 0; q < NC; ++q) {
        const int x = x0 + q;
        const bool in = x >= 1 && x <= W - 2;
        inter |= (unsigned)in << q;
        commit |= (unsigned)(in && lane >= 1 && lane <= 30) << q;
    }
    const int64_t pl = T.plane;
    const float* __restrict__ lam = A.lam[par];
    float* __restrict__ lout = A.lam[par ^ 1];
    const float* __restrict__ s0 = T.hist + slot * 3 * pl;   // state before the step (P, Vx, Vy)
    const float* __restrict__ s1 = s0 + 3 * pl;              // P' after it
    const float* __restrict__ mP = T.dP;
    const uint8_t* __restrict__ dsc = A.desc;
    const uint8_t* __restrict__ code = T.code;
    const float4* __restrict__ tab = A.tab;
    const float K1 = T.K1;
    const int lis_y = T.lis_y, lis_q = T.lis_x - x0;
    const bool tmm = (T.flags & TUBE_TMM) != 0;
    const int exc_y = T.exc_y, exc_q = T.exc_x - x0;
    const float glis = (lis_y >= r0 - 1 && lis_y <= rlast && lis_q >= 0 && lis_q < NC) ? __ldg(A.gtrace + n) : 0.0f;
    const float pend = (tmm && exc_y >= r0 - 1 && exc_y <= rlast && exc_q >= 0 && exc_q < NC)
                           ? (float)A.lam_tmm[6 + par] : 0.0f;

    // row r = r0 - 1 and the row below it
    int r = r0 - 1;
    int64_t o = (int64_t)r * pitch + x0;
    float lP[NC], lX[NC], lY[NC], dp[NC], dx[NC], dy[NC], vx[NC], vy[NC];
    float lYn[NC], dyn[NC], vyn[NC], qa[NC];
    uint32_t d_c, d_n;
    ldrow<NC>(lP, lam + o, ok);
    ldrow<NC>(lX, lam + pl + o, ok);
    ldrow<NC>(lY, lam + 2 * pl + o, ok);
    ldrow<NC>(dp, mP + o, ok);
    ldrow<NC>(dx, mP + pl + o, ok);
    ldrow<NC>(dy, mP + 2 * pl + o, ok);
    ldrow<NC>(vx, s0 + pl + o, ok);
    ldrow<NC>(vy, s0 + 2 * pl + o, ok);
    d_c = ldbytes<NC>(dsc + o, ok);
    ldrow<NC>(lYn, lam + 2 * pl + o + pitch, ok);
    ldrow<NC>(dyn, mP + 2 * pl + o + pitch, ok);
    ldrow<NC>(vyn, s0 + 2 * pl + o + pitch, ok);
    d_n = ldbytes<NC>(dsc + o + pitch, ok);
#pragma unroll
    for (int q = 0; q < NC; ++q) qa[q] = 0.0f;

    for (int j = 0; r <= rlast; ++j, ++r, o += pitch) {
        // ---- loads for the next row: its own values and the row below it
        const int64_t o1 = o + pitch;
        const bool more = r + 1 <= rlast;
        float lP1[NC], lX1[NC], dp1[NC], dx1[NC], vx1[NC], lY2[NC], dy2[NC], vy2[NC];
        uint32_t d_2 = 0;
        ldrow<NC>(lP1, lam + o1, ok && more);
        ldrow<NC>(lX1, lam + pl + o1, ok && more);
        ldrow<NC>(dp1, mP + o1, ok && more);
        ldrow<NC>(dx1, mP + pl + o1, ok && more);
        ldrow<NC>(vx1, s0 + pl + o1, ok && more);
        ldrow<NC>(lY2, lam + 2 * pl + o1 + pitch, ok && more);
        ldrow<NC>(dy2, mP + 2 * pl + o1 + pitch, ok && more);
        ldrow<NC>(vy2, s0 + 2 * pl + o1 + pitch, ok && more);
        d_2 = ldbytes<NC>(dsc + o1 + pitch, ok && more);

        // ---- mu and q of row r
        const unsigned rowm = r >= 1 ? inter : 0u;
        float4 eb[NC];
        float mu[NC], qc[NC], bxl[NC], ux[NC];
#pragma unroll
        for (int q = 0; q < NC; ++q) {
            const float4 ea = __ldg(tab + 3 * byte_at(d_c, q));
            eb[q] = __ldg(tab + 3 * byte_at(d_c, q) + 1);
            const float byd = __ldg(tab + 3 * byte_at(d_n, q)).w;
            bxl[q] = ea.z * lX[q];                 // this cell's bx lambdaVx', for its right neighbour
            ux[q] = vx[q] * dx[q];                 // this cell's Vx dX, for its right neighbour
            mu[q] = lP[q] + ea.x * lX[q] + ea.y * lY[q] - byd * lYn[q];
        }
        const float bx_in = __shfl_up_sync(kAll, bxl[NC - 1], 1);
        const float ux_in = __shfl_up_sync(kAll, ux[NC - 1], 1);
#pragma unroll
        for (int q = 0; q < NC; ++q) {
            mu[q] -= q > 0 ? bxl[q - 1] : bx_in;
            if (r == lis_y && q == lis_q) mu[q] += glis;
            if (tmm && r == exc_y && q == exc_q) mu[q] += pend;
            if (!((rowm >> q) & 1u) || eb[q].w != 0.0f) mu[q] = 0.0f;   // ring / Dirichlet no-pressure
            qc[q] = mu[q] == 0.0f ? 0.0f : __fdividef(mu[q], eb[q].z * dp[q]);
        }
        // ---- commit row r (FDTDEngineCPU.cpp:316-410 transposed)
        if (j >= 1) {
            const float q_in = __shfl_down_sync(kAll, qc[0], 1);
            const uint32_t kc = ldbytes<NC>(code + o, ok);
            float oP[NC], oX[NC], oY[NC];
            float tP[NC], tX[NC], tY[NC];
#pragma unroll
            for (int q = 0; q < NC; ++q) {
                const float qr = q < NC - 1 ? qc[q + 1] : q_in;
                const float lamU = K1 * (qr - qc[q]);
                const float lamW = K1 * (qa[q] - qc[q]);
                oP[q] = qc[q] * dp[q];
                oX[q] = eb[q].x * lX[q] + dx[q] * lamU;
                oY[q] = eb[q].y * lY[q] + dy[q] * lamW;
                const float uxl = q > 0 ? ux[q - 1] : ux_in;
                const float S = (ux[q] - uxl) + (vy[q] * dy[q] - vyn[q] * dyn[q]);
                tP[q] = mu[q] != 0.0f ? qc[q] * K1 * S / dp[q] : 0.0f;
                tX[q] = vx[q] * lamU;
                tY[q] = vy[q] * lamW;
            }
            if (commit) {
                const int64_t ob = o;
#pragma unroll
                for (int q = 0; q < NC; ++q) {
                    if (!((commit >> q) & 1u)) continue;
                    lout[ob + q] = oP[q];
                    lout[pl + ob + q] = oX[q];
                    lout[2 * pl + ob + q] = oY[q];
                    if (tP[q] != 0.0f) A.gP[ob + q] += (double)tP[q];
                    A.gX[ob + q] += (double)tX[q];
                    A.gY[ob + q] += (double)tY[q];
                    if (byte_at(kc, q) & CODE_ZINV_BIT) {
                        const float4 ez = __ldg(tab + 3 * byte_at(d_c, q) + 2);
                        const float pc = s1[ob + q], pr = s1[ob + q + 1], pt = s1[ob + q - pitch];
                        A.gZ[ob + q] += (double)(ez.x * pc - ez.y * pr) * (double)lX[q] +
                                        (double)(ez.z * pc - ez.w * pt) * (double)lY[q];
                    }
                }
            }
        }
        // ---- shift the row pipeline
#pragma unroll
        for (int q = 0; q < NC; ++q) {
            qa[q] = qc[q];
            lP[q] = lP1[q]; lX[q] = lX1[q]; lY[q] = lYn[q];
            dp[q] = dp1[q]; dx[q] = dx1[q]; dy[q] = dyn[q];
            vx[q] = vx1[q]; vy[q] = vyn[q];
            lYn[q] = lY2[q]; dyn[q] = dy2[q]; vyn[q] = vy2[q];
        }
        d_c = d_n;
        d_n = d_2;
    }
}

constexpr int kAdjNC = 2, kAdjTR = 16, kAdjWarps = 4;

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

cudaError_t launch_adjoint_step(const TubeDev* tubes, const AdjTube* adj, int ntubes, int max_blocks,
                                const AdjRun* run, int local, cudaStream_t stream, int form) {
    const dim3 grid(max_blocks, ntubes);
    if (form == ADJ_FORM_TILES)
        adjoint_step_kernel<<<grid, kAdjTileW * kAdjTileH, 0, stream>>>(tubes, adj, run, local);
    else
        adjoint_strip_kernel<kAdjNC, kAdjTR, kAdjWarps><<<grid, kAdjWarps * 32, 0, stream>>>(tubes, adj, run, local);
    return cudaGetLastError();
}

int adjoint_strips(int H, int W) { return ((W - 2) / (30 * kAdjNC) + 1) * ((H - 2 + kAdjTR - 1) / kAdjTR); }

int adjoint_strip_blocks(int strips) { return (strips + kAdjWarps - 1) / kAdjWarps; }

}  // namespace vsb
