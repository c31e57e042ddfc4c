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
                    const AdjRun* __restrict__ run, int local, int phase) {
    const TubeDev& T = tubes[blockIdx.y];
    const AdjTube& A = adj[blockIdx.y];
    const AdjRun ar = *run;
    const int64_t n = ar.start + ar.len - 1 - local;
    const int64_t slot = n - ar.start;
    const int par = ar.q0 ^ (phase & 1);
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
                     const AdjRun* __restrict__ run, int local, int phase) {
    const TubeDev& T = tubes[blockIdx.y];
    const AdjTube& A = adj[blockIdx.y];
    const AdjRun ar = *run;
    const int64_t n = ar.start + ar.len - 1 - local;
    const int64_t slot = n - ar.start;
    const int par = ar.q0 ^ (phase & 1);
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
        float mu[NC], qc[NC], bxl[NC], ux[NC], rD[NC];
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
            rD[q] = __fdividef(1.0f, eb[q].z * dp[q]);               // 1 / D
            qc[q] = mu[q] == 0.0f ? 0.0f : mu[q] * rD[q];
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
                tP[q] = mu[q] != 0.0f ? qc[q] * K1 * S * (rD[q] * eb[q].z) : 0.0f;   // / dP
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

// ---------------------------------------------------------------------------
// Two reverse steps per launch in strip form (table sources only).  The warp
// geometry is that of the one-step strips (NC columns per lane, lanes 1..30
// commit, strips of TR rows); the warp marches rows r = r0-2 .. rlast+1 and,
// at row r, runs
//   stage 0 (step n):      mu, q of row r from lambda' (the launch's input),
//                          then lambda^n of row r (kept in registers);
//   stage 1 (step n - 1):  mu, q of row r-1 from lambda^n of rows r-1 and r,
//                          then lambda^(n-1) of row r-1, which is stored.
// The valid region shrinks by one column on each side and one row per stage,
// which the extra rows (two above the strip, one below) and the halo lanes
// (0 and 31) absorb; those are recomputed by the neighbouring strips, so
// lambda^n is never written or read back.  The gradient terms of both steps
// at a cell go to its double accumulators in one read-modify-write (stage
// 0's terms of row r wait one iteration in registers for stage 1's).
// Per cell and step the arithmetic is that of the one-step strip kernel.
//
// Row supply: each lane streams its own NC-column pieces of the ten float
// plane rows an iteration reads (lambda' P, X, Y; dP, dX, dY; Vx, Vy before
// step n; Vx, Vy before step n-1) and of the three double gradient rows it
// updates into a per-warp ring of kAdjDepth + 1 shared-memory stages with
// cp.async, kAdjDepth rows ahead of their use; out-of-frame pieces are
// zero-filled by the copy.  A lane reads back only what it copied, after
// cp.async.wait_group, so no barrier is involved.  A stage is refilled one
// iteration after its values were last read.  Each gradient cell is updated
// once per launch, so its prefetched old value is current.
constexpr int kAdjDepth = 2;          // rows in flight per warp
constexpr int kAdjPieces = 10;        // float plane-row pieces per stage
constexpr int kAdjGPieces = 3;        // double gradient-row pieces per stage

// One piece of BYTES (4, 8 or 16) into shared memory; src and dst aligned to BYTES.
template <int BYTES>
__device__ __forceinline__ void cp_async_piece(void* dst, const void* src, bool ok, const void* dummy) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    const void* s = ok ? src : dummy;         // a valid address; nothing is read when ok is false
    const int n = ok ? BYTES : 0;             // 0 source bytes: the piece is zero-filled
    if constexpr (BYTES == 16)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(s), "r"(n) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;\n" ::"r"(d), "l"(s), "n"(BYTES), "r"(n)
                     : "memory");
}

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }

template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

template <int NC>
__device__ __forceinline__ void ldsrow(float (&d)[NC], const float* p) {
    if constexpr (NC == 2) {
        const float2 t = *reinterpret_cast<const float2*>(p);
        d[0] = t.x; d[1] = t.y;
    } else {
#pragma unroll
        for (int q = 0; q < NC; ++q) d[q] = p[q];
    }
}

template <int NC, int TR, int WARPS>
__global__ void __launch_bounds__(WARPS * 32, 3)
adjoint2_kernel(const TubeDev* __restrict__ tubes, const AdjTube* __restrict__ adj,
                const AdjRun* __restrict__ run, int local, int phase) {
    extern __shared__ float4 adj2_smem[];
    const TubeDev& T = tubes[blockIdx.y];
    const AdjTube& A = adj[blockIdx.y];
    const AdjRun ar = *run;
    const int64_t n = ar.start + ar.len - 1 - local;    // stage 0 reverses step n, stage 1 step n - 1
    const int64_t slot = n - ar.start;                  // >= 1
    const int par = ar.q0 ^ (phase & 1);
    // the tube's coefficient table (A.ndesc descriptors x 3 float4) in shared
    // memory after the row rings, loaded once per block
    constexpr int kSlots = kAdjDepth + 1;
    constexpr int kStage = (kAdjPieces + 2 * kAdjGPieces) * 32 * NC;   // floats per stage
    float4* stab = adj2_smem + WARPS * kSlots * kStage / 4;
    if ((int)blockIdx.x * WARPS >= A.strips) return;                   // the whole block: no strip
    for (int j = threadIdx.x; j < 3 * A.ndesc; j += WARPS * 32) stab[j] = __ldg(A.tab + j);
    __syncthreads();
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
    const bool ok = x0 >= 0 && x0 < pitch;
    unsigned inter = 0, commit = 0;
#pragma unroll
    for (int q = 0; q < NC; ++q) {
        const int x = x0 + q;
        const bool in = x >= 1 && x <= W - 2;
        inter |= (unsigned)in << q;
        commit |= (unsigned)(in && lane >= 1 && lane <= 30) << q;
    }
    const int pl = (int)T.plane;                             // plane offsets fit in 32 bits
    const float* __restrict__ lam = A.lam[par];
    float* __restrict__ lout = A.lam[par ^ 1];
    const float* __restrict__ hn = T.hist + slot * 3 * T.plane;   // state before step n (P, Vx, Vy)
    const float* __restrict__ hm = hn - 3 * pl;              // state before step n - 1
    const float* __restrict__ pn = hn + 3 * pl;              // P after step n (P after n - 1 = hn)
    const float* __restrict__ mP = T.dP;
    const uint8_t* __restrict__ dsc = A.desc;
    const uint8_t* __restrict__ code = T.code;
    const float4* tab = stab;
    const float K1 = T.K1;
    const int lis_y = T.lis_y, lis_q = T.lis_x - x0;
    const bool lis_col = lis_q >= 0 && lis_q < NC;
    const float g0 = (lis_col && lis_y >= r0 - 2 && lis_y <= rlast + 1) ? __ldg(A.gtrace + n) : 0.0f;
    const float g1 = (lis_col && lis_y >= r0 - 1 && lis_y <= rlast) ? __ldg(A.gtrace + n - 1) : 0.0f;
    auto rv = [&](int rr) { return ok && rr >= 0 && rr <= H - 1; };
    // stage t holds the pieces of row j = r0 - 2 + t: lambda' P(j), X(j), Y(j+1), dP(j), dX(j),
    // dY(j+1), Vx_n(j), Vy_n(j+1), Vx_(n-1)(j-1), Vy_(n-1)(j) as floats, then gP, gX, gY of
    // row j-1 (the row stage 1 commits at iteration j) as doubles; this lane's float piece k
    // sits at stage + (k * 32 + lane) * NC, its double piece k at gstage + (k * 32 + lane) * NC
    float* ring = reinterpret_cast<float*>(adj2_smem) + (threadIdx.x >> 5) * (kSlots * kStage);
    const int t_last = rlast - r0 + 3;                       // stage of row rlast + 1
    auto issue = [&](int t) {
        if (t > t_last) {                                    // past the strip: keep the group count
            cp_async_commit();
            return;
        }
        float* d = ring + (t % kSlots) * kStage + lane * NC;
        double* g = reinterpret_cast<double*>(ring + (t % kSlots) * kStage + kAdjPieces * 32 * NC) + lane * NC;
        const int j = r0 - 2 + t;
        const int o = j * pitch + x0;
        const bool a = rv(j), b = rv(j + 1), c = rv(j - 1);
        const bool gc = commit && j - 1 >= r0 && j - 1 <= rlast;
        constexpr int B = 4 * NC;
        cp_async_piece<B>(d + 0 * 32 * NC, lam + o, a, lam);
        cp_async_piece<B>(d + 1 * 32 * NC, lam + pl + o, a, lam);
        cp_async_piece<B>(d + 2 * 32 * NC, lam + 2 * pl + o + pitch, b, lam);
        cp_async_piece<B>(d + 3 * 32 * NC, mP + o, a, lam);
        cp_async_piece<B>(d + 4 * 32 * NC, mP + pl + o, a, lam);
        cp_async_piece<B>(d + 5 * 32 * NC, mP + 2 * pl + o + pitch, b, lam);
        cp_async_piece<B>(d + 6 * 32 * NC, hn + pl + o, a, lam);
        cp_async_piece<B>(d + 7 * 32 * NC, hn + 2 * pl + o + pitch, b, lam);
        cp_async_piece<B>(d + 8 * 32 * NC, hm + pl + o - pitch, c, lam);
        cp_async_piece<B>(d + 9 * 32 * NC, hm + 2 * pl + o, a, lam);
        cp_async_piece<2 * B>(g + 0 * 32 * NC, A.gP + (o - pitch), gc, A.gP);
        cp_async_piece<2 * B>(g + 1 * 32 * NC, A.gX + (o - pitch), gc, A.gP);
        cp_async_piece<2 * B>(g + 2 * 32 * NC, A.gY + (o - pitch), gc, A.gP);
        cp_async_commit();
    };

    // rows held at iteration r (u = r-1, c = r, d = r+1)
    float lPc[NC], lXc[NC], lYc[NC], lYd[NC];            // lambda' rows r (P, X, Y), r+1 (Y)
    float dpu[NC], dpc[NC], dxu[NC], dxc[NC];            // dP, dX rows r-1, r
    float dyu[NC], dyc[NC], dyd[NC];                     // dY rows r-1, r, r+1
    float vxc[NC], vyc[NC], vyd[NC];                     // step n state: Vx row r, Vy rows r, r+1
    float wxu[NC], wyu[NC], wyc[NC];                     // step n-1 state: Vx row r-1, Vy rows r-1, r
    uint32_t du = 0, dc = 0, dd = 0;                     // descriptors rows r-1, r, r+1
    uint32_t ku = 0, kc = 0;                             // cell codes rows r-1, r
    float LPp[NC], LXp[NC], LYp[NC];                     // lambda^n of row r-1
    float qa0[NC], qa1[NC];                              // q of step n at row r-1, of step n-1 at row r-2
    float h0P[NC], h0X[NC], h0Y[NC];                     // step n's gradient terms of row r-1
    double h0Z[NC];                                      // and its z_inv term there
    {
        const int r = r0 - 2;
        const int o = r * pitch + x0;
        const bool a = rv(r), b = rv(r + 1);
        ldrow<NC>(lPc, lam + o, a);
        ldrow<NC>(lXc, lam + pl + o, a);
        ldrow<NC>(lYc, lam + 2 * pl + o, a);
        ldrow<NC>(lYd, lam + 2 * pl + o + pitch, b);
        ldrow<NC>(dpc, mP + o, a);
        ldrow<NC>(dxc, mP + pl + o, a);
        ldrow<NC>(dyc, mP + 2 * pl + o, a);
        ldrow<NC>(dyd, mP + 2 * pl + o + pitch, b);
        ldrow<NC>(vxc, hn + pl + o, a);
        ldrow<NC>(vyc, hn + 2 * pl + o, a);
        ldrow<NC>(vyd, hn + 2 * pl + o + pitch, b);
        ldrow<NC>(wyc, hm + 2 * pl + o, a);
        dc = ldbytes<NC>(dsc + o, a);
        dd = ldbytes<NC>(dsc + o + pitch, b);
        kc = ldbytes<NC>(code + o, a);
#pragma unroll
        for (int q = 0; q < NC; ++q) {
            dpu[q] = 1.0f; dxu[q] = 0.0f; dyu[q] = 0.0f; wxu[q] = 0.0f; wyu[q] = 0.0f;
            LPp[q] = 0.0f; LXp[q] = 0.0f; LYp[q] = 0.0f;
            qa0[q] = 0.0f; qa1[q] = 0.0f; h0P[q] = 0.0f; h0X[q] = 0.0f; h0Y[q] = 0.0f; h0Z[q] = 0.0;
        }
    }
#pragma unroll
    for (int t = 1; t < kAdjDepth; ++t) issue(t);

    for (int r = r0 - 2; r <= rlast + 1; ++r) {
        const int tr = r - (r0 - 2);
        issue(tr + kAdjDepth);            // into the stage moved to registers two iterations ago
        const int o = r * pitch + x0;
        const bool nx = r + 1 <= rlast + 1;
        const uint32_t d2 = ldbytes<NC>(dsc + o + 2 * pitch, nx && rv(r + 2));
        const uint32_t k1 = ldbytes<NC>(code + o + pitch, nx && rv(r + 1));

        // ---- stage 0: mu and q of row r (step n)
        const unsigned m0 = (r >= 1 && r <= H - 2) ? inter : 0u;
        float4 eb0[NC];
        float mu0[NC], q0[NC], bxl[NC], ux[NC], rD0[NC];
#pragma unroll
        for (int q = 0; q < NC; ++q) {
            const float4 ea = tab[3 * byte_at(dc, q)];
            eb0[q] = tab[3 * byte_at(dc, q) + 1];
            const float byd = tab[3 * byte_at(dd, q)].w;
            bxl[q] = ea.z * lXc[q];
            ux[q] = vxc[q] * dxc[q];
            mu0[q] = lPc[q] + ea.x * lXc[q] + ea.y * lYc[q] - byd * lYd[q];
        }
        {
            const float bx_in = __shfl_up_sync(kAll, bxl[NC - 1], 1);
#pragma unroll
            for (int q = 0; q < NC; ++q) {
                mu0[q] -= q > 0 ? bxl[q - 1] : bx_in;
                if (r == lis_y && q == lis_q) mu0[q] += g0;
                if (!((m0 >> q) & 1u) || eb0[q].w != 0.0f) mu0[q] = 0.0f;   // ring / Dirichlet no-pressure
                rD0[q] = __fdividef(1.0f, eb0[q].z * dpc[q]);                  // 1 / D
                q0[q] = mu0[q] == 0.0f ? 0.0f : mu0[q] * rD0[q];
            }
        }
        // ---- stage 0: lambda^n of row r (registers) and step n's gradient terms there
        float LPn[NC], LXn[NC], LYn[NC], t0P[NC], t0X[NC], t0Y[NC];
        double t0Z[NC];
        const bool own0 = r >= r0 && r <= rlast;
        {
            const float q_in = __shfl_down_sync(kAll, q0[0], 1);
            const float ux_in = __shfl_up_sync(kAll, ux[NC - 1], 1);
#pragma unroll
            for (int q = 0; q < NC; ++q) {
                const float qr = q < NC - 1 ? q0[q + 1] : q_in;
                const float lamU = K1 * (qr - q0[q]);
                const float lamW = K1 * (qa0[q] - q0[q]);
                const bool in = (m0 >> q) & 1u;
                LPn[q] = in ? q0[q] * dpc[q] : 0.0f;
                LXn[q] = in ? eb0[q].x * lXc[q] + dxc[q] * lamU : 0.0f;
                LYn[q] = in ? eb0[q].y * lYc[q] + dyc[q] * lamW : 0.0f;
                const float uxl = q > 0 ? ux[q - 1] : ux_in;
                const float S = (ux[q] - uxl) + (vyc[q] * dyc[q] - vyd[q] * dyd[q]);
                t0P[q] = mu0[q] != 0.0f ? q0[q] * K1 * S * (rD0[q] * eb0[q].z) : 0.0f;   // / dP
                t0X[q] = vxc[q] * lamU;
                t0Y[q] = vyc[q] * lamW;
                t0Z[q] = 0.0;
                if (own0 && ((commit >> q) & 1u) && (byte_at(kc, q) & CODE_ZINV_BIT)) {
                    const float4 ez = tab[3 * byte_at(dc, q) + 2];
                    const float pc = pn[o + q], pr = pn[o + q + 1], pt = pn[o + q - pitch];
                    t0Z[q] = (double)(ez.x * pc - ez.y * pr) * (double)lXc[q] +
                             (double)(ez.z * pc - ez.w * pt) * (double)lYc[q];
                }
            }
        }
        // ---- stage 1: mu and q of row r-1 (step n-1) from lambda^n of rows r-1 and r
        if (r >= r0) {
            const int r1 = r - 1;
            const int o1 = o - pitch;
            const unsigned m1 = (r1 >= 1 && r1 <= H - 2) ? inter : 0u;
            float4 eb1[NC];
            float mu1[NC], q1[NC], bxl1[NC], wx[NC], rD1[NC];
#pragma unroll
            for (int q = 0; q < NC; ++q) {
                const float4 ea = tab[3 * byte_at(du, q)];
                eb1[q] = tab[3 * byte_at(du, q) + 1];
                const float byd = tab[3 * byte_at(dc, q)].w;
                bxl1[q] = ea.z * LXp[q];
                wx[q] = wxu[q] * dxu[q];
                mu1[q] = LPp[q] + ea.x * LXp[q] + ea.y * LYp[q] - byd * LYn[q];
            }
            const float bx_in = __shfl_up_sync(kAll, bxl1[NC - 1], 1);
#pragma unroll
            for (int q = 0; q < NC; ++q) {
                mu1[q] -= q > 0 ? bxl1[q - 1] : bx_in;
                if (r1 == lis_y && q == lis_q) mu1[q] += g1;
                if (!((m1 >> q) & 1u) || eb1[q].w != 0.0f) mu1[q] = 0.0f;
                rD1[q] = __fdividef(1.0f, eb1[q].z * dpu[q]);
                q1[q] = mu1[q] == 0.0f ? 0.0f : mu1[q] * rD1[q];
            }
            // ---- stage 1: lambda^(n-1) of row r-1 (stored) and the gradient terms of both steps there
            if (r >= r0 + 1) {
                const float q_in = __shfl_down_sync(kAll, q1[0], 1);
                const float wx_in = __shfl_up_sync(kAll, wx[NC - 1], 1);
                float oP[NC], oX[NC], oY[NC], tP[NC], tX[NC], tY[NC];
#pragma unroll
                for (int q = 0; q < NC; ++q) {
                    const float qr = q < NC - 1 ? q1[q + 1] : q_in;
                    const float lamU = K1 * (qr - q1[q]);
                    const float lamW = K1 * (qa1[q] - q1[q]);
                    oP[q] = q1[q] * dpu[q];
                    oX[q] = eb1[q].x * LXp[q] + dxu[q] * lamU;
                    oY[q] = eb1[q].y * LYp[q] + dyu[q] * lamW;
                    const float wxl = q > 0 ? wx[q - 1] : wx_in;
                    const float S = (wx[q] - wxl) + (wyu[q] * dyu[q] - wyc[q] * dyc[q]);
                    tP[q] = mu1[q] != 0.0f ? q1[q] * K1 * S * (rD1[q] * eb1[q].z) : 0.0f;
                    tX[q] = wxu[q] * lamU;
                    tY[q] = wyu[q] * lamW;
                }
                if (commit) {
                    // the old gradient values of row r-1 arrived with stage tr
                    const double* gs = reinterpret_cast<const double*>(ring + (tr % kSlots) * kStage +
                                                                       kAdjPieces * 32 * NC) + lane * NC;
#pragma unroll
                    for (int q = 0; q < NC; ++q) {
                        if (!((commit >> q) & 1u)) continue;
                        lout[o1 + q] = oP[q];
                        lout[pl + o1 + q] = oX[q];
                        lout[2 * pl + o1 + q] = oY[q];
                        if (tP[q] != 0.0f || h0P[q] != 0.0f)
                            A.gP[o1 + q] = gs[q] + ((double)h0P[q] + (double)tP[q]);
                        A.gX[o1 + q] = gs[32 * NC + q] + ((double)h0X[q] + (double)tX[q]);
                        A.gY[o1 + q] = gs[64 * NC + q] + ((double)h0Y[q] + (double)tY[q]);
                        if (byte_at(ku, q) & CODE_ZINV_BIT) {
                            // P after step n-1 is the P plane of the state before step n;
                            // both steps' z_inv terms go in with one read-modify-write
                            const float4 ez = tab[3 * byte_at(du, q) + 2];
                            const float pc = hn[o1 + q], pr = hn[o1 + q + 1], pt = hn[o1 + q - pitch];
                            A.gZ[o1 + q] += h0Z[q] + ((double)(ez.x * pc - ez.y * pr) * (double)LXp[q] +
                                                      (double)(ez.z * pc - ez.w * pt) * (double)LYp[q]);
                        }
                    }
                }
            }
#pragma unroll
            for (int q = 0; q < NC; ++q) qa1[q] = q1[q];
        }
        if (!nx) break;

        // ---- shift the row pipeline; row r+1's pieces come from its ring stage
#pragma unroll
        for (int q = 0; q < NC; ++q) {
            LPp[q] = LPn[q]; LXp[q] = LXn[q]; LYp[q] = LYn[q];
            qa0[q] = q0[q];
            h0P[q] = t0P[q]; h0X[q] = t0X[q]; h0Y[q] = t0Y[q]; h0Z[q] = t0Z[q];
            lYc[q] = lYd[q];
            dpu[q] = dpc[q]; dxu[q] = dxc[q];
            dyu[q] = dyc[q]; dyc[q] = dyd[q];
            vyc[q] = vyd[q];
            wyu[q] = wyc[q];
        }
        du = dc; dc = dd; dd = d2;
        ku = kc; kc = k1;
        cp_async_wait<kAdjDepth - 1>();
        const float* st = ring + ((tr + 1) % kSlots) * kStage + lane * NC;
        ldsrow<NC>(lPc, st + 0 * 32 * NC);
        ldsrow<NC>(lXc, st + 1 * 32 * NC);
        ldsrow<NC>(lYd, st + 2 * 32 * NC);
        ldsrow<NC>(dpc, st + 3 * 32 * NC);
        ldsrow<NC>(dxc, st + 4 * 32 * NC);
        ldsrow<NC>(dyd, st + 5 * 32 * NC);
        ldsrow<NC>(vxc, st + 6 * 32 * NC);
        ldsrow<NC>(vyd, st + 7 * 32 * NC);
        ldsrow<NC>(wxu, st + 8 * 32 * NC);
        ldsrow<NC>(wyc, st + 9 * 32 * NC);
    }
    cp_async_wait<0>();                   // no copy outlives the warp
}

// Dynamic shared memory of adjoint2_kernel per block.
constexpr size_t adj2_smem_bytes(int nc, int warps) {
    return (size_t)warps * (kAdjDepth + 1) * (kAdjPieces + 2 * kAdjGPieces) * 32 * nc * sizeof(float);
}

// ... plus the coefficient table of up to kMaxAdjDescriptors descriptors.
constexpr int kMaxAdjDescriptors = 256;
constexpr size_t adj2_smem_max(int nc, int warps) {
    return adj2_smem_bytes(nc, warps) + (size_t)kMaxAdjDescriptors * 3 * sizeof(float4);
}

constexpr int kAdjNC = 2, kAdjWarps = 4;

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

// The two-step kernel's shared memory (row rings + the coefficient table)
// exceeds the default 48 KB: the attribute is set on every launch (it is per
// device, and cheap; graph replays do not repeat it).
template <int TR>
cudaError_t launch_adj2(dim3 grid, const TubeDev* tubes, const AdjTube* adj, const AdjRun* run, int local,
                        int phase, cudaStream_t stream) {
    constexpr size_t smem = adj2_smem_max(kAdjNC, kAdjWarps);
    static_assert(smem <= 200 * 1024, "two-step shared memory exceeds a third of the SM's");
    const cudaError_t e = cudaFuncSetAttribute(adjoint2_kernel<kAdjNC, TR, kAdjWarps>,
                                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    adjoint2_kernel<kAdjNC, TR, kAdjWarps><<<grid, kAdjWarps * 32, smem, stream>>>(tubes, adj, run, local, phase);
    return cudaGetLastError();
}

cudaError_t launch_adjoint_step(const TubeDev* tubes, const AdjTube* adj, int ntubes, int max_blocks,
                                const AdjRun* run, int local, int phase, cudaStream_t stream, int form,
                                int rows) {
    const dim3 grid(max_blocks, ntubes);
    constexpr int kThreads = kAdjWarps * 32;
    if (form == ADJ_FORM_TILES) {
        adjoint_step_kernel<<<grid, kAdjTileW * kAdjTileH, 0, stream>>>(tubes, adj, run, local, phase);
    } else if (form == ADJ_FORM_STRIPS2) {
        if (rows == 4)
            return launch_adj2<4>(grid, tubes, adj, run, local, phase, stream);
        if (rows == 8)
            return launch_adj2<8>(grid, tubes, adj, run, local, phase, stream);
        return launch_adj2<16>(grid, tubes, adj, run, local, phase, stream);
    } else {
        if (rows == 4)
            adjoint_strip_kernel<kAdjNC, 4, kAdjWarps><<<grid, kThreads, 0, stream>>>(tubes, adj, run, local, phase);
        else if (rows == 8)
            adjoint_strip_kernel<kAdjNC, 8, kAdjWarps><<<grid, kThreads, 0, stream>>>(tubes, adj, run, local, phase);
        else
            adjoint_strip_kernel<kAdjNC, 16, kAdjWarps><<<grid, kThreads, 0, stream>>>(tubes, adj, run, local, phase);
    }
    return cudaGetLastError();
}

int adjoint_strips(int H, int W, int form, int rows) {
    (void)form;   // both strip forms use the same geometry
    return ((W - 2) / (30 * kAdjNC) + 1) * ((H - 2 + rows - 1) / rows);
}

int adjoint_strip_blocks(int strips) { return (strips + kAdjWarps - 1) / kAdjWarps; }

}  // namespace vsb
