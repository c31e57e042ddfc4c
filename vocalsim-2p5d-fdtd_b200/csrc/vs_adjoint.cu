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

// ---- two-mass source ------------------------------------------------------
// With the two-mass source, exeV_n = ug_n = TMM(state_n, p1 = P_n[exc]) feeds
// the velocity of the excitation cells.  Its reverse step needs the Jacobian
// of one model step (TwoMassModel.cpp:90-232) with respect to the six state
// values and p1; it is evaluated by forward-mode dual numbers over the same
// expressions in double (branches on the primal values).
constexpr int kTmmIn = 7;

struct Dual {
    double v;
    double d[kTmmIn];
};

__device__ inline Dual dconst(double v) {
    Dual r;
    r.v = v;
    for (int i = 0; i < kTmmIn; ++i) r.d[i] = 0.0;
    return r;
}
__device__ inline Dual operator+(const Dual& a, const Dual& b) {
    Dual r;
    r.v = a.v + b.v;
    for (int i = 0; i < kTmmIn; ++i) r.d[i] = a.d[i] + b.d[i];
    return r;
}
__device__ inline Dual operator-(const Dual& a, const Dual& b) {
    Dual r;
    r.v = a.v - b.v;
    for (int i = 0; i < kTmmIn; ++i) r.d[i] = a.d[i] - b.d[i];
    return r;
}
__device__ inline Dual operator*(const Dual& a, const Dual& b) {
    Dual r;
    r.v = a.v * b.v;
    for (int i = 0; i < kTmmIn; ++i) r.d[i] = a.d[i] * b.v + a.v * b.d[i];
    return r;
}
__device__ inline Dual operator/(const Dual& a, const Dual& b) {
    Dual r;
    r.v = a.v / b.v;
    for (int i = 0; i < kTmmIn; ++i) r.d[i] = (a.d[i] - r.v * b.d[i]) / b.v;
    return r;
}
__device__ inline Dual operator*(double a, const Dual& b) { return dconst(a) * b; }
__device__ inline Dual operator+(double a, const Dual& b) { return dconst(a) + b; }
__device__ inline Dual operator-(double a, const Dual& b) { return dconst(a) - b; }
__device__ inline Dual operator/(double a, const Dual& b) { return dconst(a) / b; }
__device__ inline Dual operator/(const Dual& a, double b) { return a / dconst(b); }
__device__ inline Dual dabs(const Dual& a) { return a.v < 0.0 ? dconst(0.0) - a : a; }

// One model step on st = {x1_old, x1_curr, x2_old, x2_curr, ug_old, ug_curr}.
__device__ void tmm_math(const TmmConsts64& k, Dual st[6], const Dual& p1) {
    const double srate = k.srate, s2 = srate * srate;
    const double lg = k.lg, two_lg = 2.0 * lg, rho = k.rho, ps = k.ps;
    const Dual x1o = st[0], x1 = st[1], x2o = st[2], x2 = st[3], ugo = st[4], ug = st[5];
    const Dual Ag1 = k.Ag01 + two_lg * x1, Ag2 = k.Ag02 + two_lg * x2;
    const double c12 = 12.0 * k.mu * lg * lg;
    const Dual Rv1 = (c12 * k.d1) / (Ag1 * Ag1 * Ag1), Lg1 = (rho * k.d1) / Ag1;
    const Dual Rv2 = (c12 * k.d2) / (Ag2 * Ag2 * Ag2), Lg2 = (rho * k.d2) / Ag2;
    const double thr1 = -k.Ag01 / two_lg, thr2 = -k.Ag02 / two_lg;
    Dual pm1 = dconst(ps), pm2;
    if (x1.v > thr1 && x2.v > thr2) {
        const Dual q = ug / Ag1;
        pm1 = ps - 1.37 * (rho / 2.0) * q * q - 0.5 * (Rv1 * ug + srate * (Lg1 * (ug - ugo)));
    }
    const Dual fm1 = (k.d1 * lg) * pm1;
    if (x1.v > thr1) {
        if (x2.v > thr2)
            pm2 = pm1 - (0.5 * (Rv1 + Rv2) * ug + srate * ((Lg1 + Lg2) * (ug - ugo))) -
                  (rho / 2.0) * ug * ug * (1.0 / (Ag2 * Ag2) - 1.0 / (Ag1 * Ag1));
        else
            pm2 = dconst(ps);
    } else {
        pm2 = dconst(0.0);
    }
    const Dual fm2 = (k.d2 * lg) * pm2;
    const double g1 = k.Ag01 / two_lg, g2 = k.Ag02 / two_lg;
    const bool c1 = x1.v + g1 < 0.0, c2 = x2.v + g2 < 0.0;
    const double h1u = c1 ? k.h1 : 0.0, r1u = c1 ? k.r1c : k.r1o;
    const double h2u = c2 ? k.h2 : 0.0, r2u = c2 ? k.r2c : k.r2o;
    const double a11 = (k.k1 + h1u + k.kc) / s2 + r1u / srate + k.m1;
    const double a12 = -k.kc / s2;
    const double a22 = (k.k2 + h2u + k.kc) / s2 + r2u / srate + k.m2;
    const Dual e1 = g1 + x1, e2 = g2 + x2;
    const Dual sp1 = (k.k1 * k.etak1) * x1 * x1 * x1 + h1u * (g1 + k.etah1 * e1 * e1 * e1);
    const Dual sp2 = (k.k2 * k.etak2) * x2 * x2 * x2 + h2u * (g2 + k.etah2 * e2 * e2 * e2);
    const Dual b1 = (2.0 * k.m1 + r1u / srate) * x1 - k.m1 * x1o - sp1 / s2 + fm1 / s2;
    const Dual b2 = (2.0 * k.m2 + r2u / srate) * x2 - k.m2 * x2o - sp2 / s2 + fm2 / s2;
    double det = a11 * a22 - a12 * a12;
    if (det == 0.0) det = 1.0;
    const Dual x1n = (a22 * b1 - a12 * b2) / dconst(det);
    const Dual x2n = (a11 * b2 - a12 * b1) / dconst(det);
    const Dual A1n = k.Ag01 + two_lg * x1n, A2n = k.Ag02 + two_lg * x2n;
    Dual ugn = dconst(0.0);
    if (!(A1n.v < 0.0 || A2n.v < 0.0)) {
        const Dual r = A2n / dconst(k.A1);
        const Dual Rtot = (rho / 2.0) * dabs(ug) * (0.37 / (A1n * A1n) + (1.0 - 2.0 * r * (1.0 - r)) / (A2n * A2n)) +
                          c12 * (k.d1 / (A1n * A1n * A1n) + k.d2 / (A2n * A2n * A2n));
        const Dual Ltot = rho * (k.d1 / A1n + k.d2 / A2n);
        ugn = ((ps - p1) / dconst(srate) + Ltot * ug) / (Rtot / dconst(srate) + Ltot);
    }
    st[0] = x1; st[1] = x1n; st[2] = x2; st[3] = x2n; st[4] = ug; st[5] = ugn;
}

// Reverse of the two-mass step n: one thread per tube.  lam[par] holds the
// adjoint of the state after step n, lam[par ^ 1] the (already computed)
// adjoint of the state before it, which receives d/d p1 at the excitation cell.
__global__ void tmm_adjoint_kernel(const TubeDev* __restrict__ tubes, const AdjTube* __restrict__ adj, int ntubes,
                                   int64_t slot, int par) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ntubes) return;
    const TubeDev& T = tubes[t];
    const AdjTube& A = adj[t];
    if (!(T.flags & TUBE_TMM)) return;
    const int64_t pl = T.plane;
    const int pitch = T.pitch;
    const float* __restrict__ lam = A.lam[par];
    // dL/d exeV: a velocity whose cell (or right / top neighbour) is an
    // excitation cell carries exeV * ew * mS / (mB + mS); every excitation
    // cell lies in column exc_x, so columns exc_x - 1 and exc_x cover them
    const float* sig = T.sigma;
    double lexe = 0.0;
    for (int r = 1; r <= T.H - 2; ++r) {
        for (int c = max(T.exc_x - 1, 1); c <= min(T.exc_x, T.W - 2); ++c) {
            const int64_t o = (int64_t)r * pitch + c;
            const int tc = T.code[o] & CODE_TYPE_MASK, tr = T.code[o + 1] & CODE_TYPE_MASK;
            const int tt = T.code[o - pitch] & CODE_TYPE_MASK;
            const double ec = tc == VS_CELL_EXCITATION, er = tr == VS_CELL_EXCITATION, et = tt == VS_CELL_EXCITATION;
            const double ewx = ec * T.dir2 + er * T.dir0, ewy = ec * T.dir3 + et * T.dir1;
            if (ewx != 0.0) {
                const double mb = fmin(a_beta[tc], a_beta[tr]), ms = fmax(sig[tc], sig[tr]);
                lexe += ewx * ms / (mb + ms) * lam[pl + o];
            }
            if (ewy != 0.0) {
                const double mb = fmin(a_beta[tc], a_beta[tt]), ms = fmax(sig[tc], sig[tt]);
                lexe += ewy * ms / (mb + ms) * lam[2 * pl + o];
            }
        }
    }
    const double* sv = T.tmm_hist + 6 * slot;
    const float p1v = T.hist[slot * 3 * pl + (int64_t)T.exc_y * pitch + T.exc_x];
    Dual st[6];
    for (int i = 0; i < 6; ++i) {
        st[i] = dconst(sv[i]);
        st[i].d[i] = 1.0;
    }
    Dual p1 = dconst(p1v);
    p1.d[6] = 1.0;
    tmm_math(T.tmmd, st, p1);
    double lout[6];
    for (int i = 0; i < 6; ++i) lout[i] = A.lam_tmm[i];
    lout[5] += lexe;                       // ug_curr after the step is exeV_n
    double lin[kTmmIn];
    for (int j = 0; j < kTmmIn; ++j) {
        lin[j] = 0.0;
        for (int i = 0; i < 6; ++i) lin[j] += lout[i] * st[i].d[j];
    }
    for (int i = 0; i < 6; ++i) A.lam_tmm[i] = lin[i];
    A.lam[par ^ 1][(int64_t)T.exc_y * pitch + T.exc_x] += (float)lin[6];
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

cudaError_t launch_adjoint_step(const TubeDev* tubes, const AdjTube* adj, int ntubes, int max_cells, int64_t n,
                                int64_t slot, int par, bool tmm, cudaStream_t stream) {
    const dim3 grid((max_cells + 255) / 256, ntubes);
    adjoint_mu_kernel<<<grid, 256, 0, stream>>>(tubes, adj, n, par);
    adjoint_lambda_kernel<<<grid, 256, 0, stream>>>(tubes, adj, slot, par);
    if (tmm) tmm_adjoint_kernel<<<(ntubes + 31) / 32, 32, 0, stream>>>(tubes, adj, ntubes, slot, par);
    return cudaGetLastError();
}

}  // namespace vsb
