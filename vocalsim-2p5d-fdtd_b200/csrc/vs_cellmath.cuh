// vs_cellmath.cuh -- per-cell arithmetic shared by the step kernels of
// libvocalsim_b200 (vs_step.cu, vs_cluster.cu): round-to-nearest float and
// double operations in the reference's operand order, the two-mass model
// steps, and the velocity update with the coefficients of
// calculateSolverCoefficients derived from the cell codes.
#pragma once

#include <cuda_runtime.h>

#include "vs_device.h"

namespace vsb {
namespace {

__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fdiv(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dadd_rn(a, -b); }
__device__ __forceinline__ double dd(float a) { return (double)a; }
__device__ __forceinline__ float tof(double a) { return __double2float_rn(a); }

constexpr unsigned kFull = 0xffffffffu;

// One step of the Ishizaka-Flanagan two-mass model, TwoMassModel.cpp:90-232,
// in the reference's mixed float/double precision and operand order.  The
// reference's host build (g++) forms (rho/2)*fabs(ug) in double.
// The model step split at its one use of the supraglottal pressure p1: the
// first part depends on the state alone (the new displacements and the flow
// equation's coefficients), so a caller can evaluate it before p1 is known;
// tmm_finish applies p1 and commits the state.  prepare + finish performs
// exactly the operations of one step, in the same order.
struct TmmPrep {
    float x1, x1n, x2, x2n, ug;     // state before / after the displacement update, flow before
    float Lug, den, srate, ps;      // ugn = ((ps - p1) / srate + Lug) / den
    bool closed;                    // glottis closed: ugn = 0
};

__device__ __forceinline__ TmmPrep tmm_prepare(const TmmConsts& k, const TmmState& s) {
    const float srate = k.srate;
    const float two_lg = fmul(2.0f, k.lg);
    float Ag1 = fadd(k.Ag01, fmul(two_lg, s.x1_curr));
    float Ag2 = fadd(k.Ag02, fmul(two_lg, s.x2_curr));
    const float mu12lglg = fmul(fmul(fmul(12.0f, k.mu), k.lg), k.lg);
    const float Rv1 = fdiv(fmul(mu12lglg, k.d1), fmul(fmul(Ag1, Ag1), Ag1));
    const float Lg1 = fdiv(fmul(k.rho, k.d1), Ag1);
    const float Rv2 = fdiv(fmul(mu12lglg, k.d2), fmul(fmul(Ag2, Ag2), Ag2));
    const float Lg2 = fdiv(fmul(k.rho, k.d2), Ag2);
    const float thr1 = fdiv(-k.Ag01, two_lg);
    const float thr2 = fdiv(-k.Ag02, two_lg);
    const float ug = s.ug_curr, ugo = s.ug_old;
    const float dug = fsub(ug, ugo);
    const float half_rho = fdiv(k.rho, 2.0f);
    float pm1, pm2;
    if (s.x1_curr > thr1 && s.x2_curr > thr2) {
        const float q = fdiv(ug, Ag1);
        const double a = dmul(dmul(dmul(1.37, dd(half_rho)), dd(q)), dd(q));
        const double b = dmul(0.5, dd(fadd(fmul(Rv1, ug), fmul(fmul(Lg1, srate), dug))));
        pm1 = tof(dsub(dsub(dd(k.ps), a), b));
    } else {
        pm1 = k.ps;
    }
    const float fm1 = fmul(fmul(pm1, k.d1), k.lg);
    if (s.x1_curr > thr1) {
        if (s.x2_curr > thr2) {
            const double u = dadd(dmul(dmul(0.5, dd(fadd(Rv1, Rv2))), dd(ug)),
                                  dd(fmul(fmul(fadd(Lg1, Lg2), dug), srate)));
            const float v = fmul(fmul(fmul(half_rho, ug), ug),
                                 fsub(fdiv(1.0f, fmul(Ag2, Ag2)), fdiv(1.0f, fmul(Ag1, Ag1))));
            pm2 = tof(dsub(dsub(dd(pm1), u), dd(v)));
        } else {
            pm2 = k.ps;
        }
    } else {
        pm2 = 0.0f;
    }
    const float fm2 = fmul(fmul(pm2, k.d2), k.lg);
    const float g1 = fdiv(k.Ag01, two_lg), g2 = fdiv(k.Ag02, two_lg);
    float h1u, r1u, h2u, r2u;
    if (fadd(s.x1_curr, g1) < 0.0f) { h1u = k.h1; r1u = k.r1c; } else { h1u = 0.0f; r1u = k.r1o; }
    if (fadd(s.x2_curr, g2) < 0.0f) { h2u = k.h2; r2u = k.r2c; } else { h2u = 0.0f; r2u = k.r2o; }
    const float s2 = fmul(srate, srate);
    const float a11 = fadd(fadd(fdiv(fadd(fadd(k.k1, h1u), k.kc), s2), fdiv(r1u, srate)), k.m1);
    const float a12 = fdiv(-k.kc, s2);
    const float a21 = a12;
    const float a22 = fadd(fadd(fdiv(fadd(fadd(k.k2, h2u), k.kc), s2), fdiv(r2u, srate)), k.m2);
    const float x1 = s.x1_curr, x2 = s.x2_curr;
    const float e1 = fadd(g1, x1), e2 = fadd(g2, x2);
    const float sp1 = fadd(fmul(fmul(fmul(fmul(k.k1, k.etak1), x1), x1), x1),
                           fmul(h1u, fadd(g1, fmul(fmul(fmul(k.etah1, e1), e1), e1))));
    const float sp2 = fadd(fmul(fmul(fmul(fmul(k.k2, k.etak2), x2), x2), x2),
                           fmul(h2u, fadd(g2, fmul(fmul(fmul(k.etah2, e2), e2), e2))));
    const float b1 = fadd(fsub(fsub(fmul(fadd(fmul(2.0f, k.m1), fdiv(r1u, srate)), x1), fmul(k.m1, s.x1_old)),
                               fdiv(sp1, s2)), fdiv(fm1, s2));
    const float b2 = fadd(fsub(fsub(fmul(fadd(fmul(2.0f, k.m2), fdiv(r2u, srate)), x2), fmul(k.m2, s.x2_old)),
                               fdiv(sp2, s2)), fdiv(fm2, s2));
    float det = fsub(fmul(a11, a22), fmul(a21, a12));
    if (det == 0.0f) det = 1.0f;
    const float x1n = fdiv(fsub(fmul(a22, b1), fmul(a12, b2)), det);
    const float x2n = fdiv(fsub(fmul(a11, b2), fmul(a21, b1)), det);
    TmmPrep o;
    o.x1 = x1; o.x1n = x1n; o.x2 = x2; o.x2n = x2n; o.ug = ug;
    o.srate = srate; o.ps = k.ps;
    Ag1 = fadd(k.Ag01, fmul(two_lg, x1n));
    Ag2 = fadd(k.Ag02, fmul(two_lg, x2n));
    o.closed = Ag1 < 0.0f || Ag2 < 0.0f;
    o.Lug = 0.0f;
    o.den = 1.0f;
    if (!o.closed) {
        const float r = fdiv(Ag2, k.A1);
        const float f = fdiv(fsub(1.0f, fmul(fmul(2.0f, r), fsub(1.0f, r))), fmul(Ag2, Ag2));
        const double t1 = dmul(dmul(dd(half_rho), fabs(dd(ug))),
                               dadd(__ddiv_rn(0.37, dd(fmul(Ag1, Ag1))), dd(f)));
        const float t2 = fmul(mu12lglg, fadd(fdiv(k.d1, fmul(fmul(Ag1, Ag1), Ag1)),
                                             fdiv(k.d2, fmul(fmul(Ag2, Ag2), Ag2))));
        const float Rtot = tof(dadd(t1, dd(t2)));
        const float Ltot = fmul(k.rho, fadd(fdiv(k.d1, Ag1), fdiv(k.d2, Ag2)));
        o.Lug = fmul(Ltot, ug);
        o.den = fadd(fdiv(Rtot, srate), Ltot);
    }
    return o;
}

__device__ __forceinline__ float tmm_finish(const TmmPrep& o, TmmState& s, float p1) {
    const float ugn = o.closed ? 0.0f : fdiv(fadd(fdiv(fsub(o.ps, p1), o.srate), o.Lug), o.den);
    s.x1_old = o.x1; s.x1_curr = o.x1n;
    s.x2_old = o.x2; s.x2_curr = o.x2n;
    s.ug_old = o.ug;
    s.ug_curr = ugn;
    return ugn;
}

__device__ __noinline__ float tmm_step(const TmmConsts& k, TmmState& s, float p1) {
    const TmmPrep o = tmm_prepare(k, s);
    return tmm_finish(o, s, p1);
}

// The same model step with every quantity in double (tmm_f64): the
// expressions of TwoMassModel.cpp:90-232 with the per-tube constants taken
// from TmmDerived64 (reciprocals of the sample rate, the thresholds, the
// displacement-update matrix and its inverse determinant per contact state),
// so that a step divides only by the glottal openings before and after the
// displacement update and by the flow denominator.  The order of operations
// is the model's own (it is this build's option, not the reference's float
// arithmetic): the FP32 oracle's tmm_f64 path performs the same operations,
// and the FP64 oracle keeps the literal expressions as the accuracy reference.
// The caller's pressure is widened and the flow rounded to float for the
// field update.
struct TmmPrep64 {
    double x1, x1n, x2, x2n, ug;
    double Lug, den, isr, ps;       // ugn = ((ps - p1) isr + Lug) / den
    bool closed;
};

__device__ __forceinline__ TmmPrep64 tmm_prepare64(const TmmConsts64& k, const TmmDerived64& d,
                                                   const TmmState64& s) {
    const double x1c = s.x1_curr, x2c = s.x2_curr, ug = s.ug_curr, ugo = s.ug_old;
    const double ia1 = 1.0 / (k.Ag01 + d.two_lg * x1c);
    const double ia2 = 1.0 / (k.Ag02 + d.two_lg * x2c);
    const double ia1s = ia1 * ia1, ia2s = ia2 * ia2;
    const double Rv1 = d.cR1 * (ia1s * ia1), Lg1 = d.cL1 * ia1;
    const double Rv2 = d.cR2 * (ia2s * ia2), Lg2 = d.cL2 * ia2;
    const double dug = ug - ugo;
    const bool open1 = x1c > -d.g1, open2 = x2c > -d.g2;
    double pm1 = k.ps;
    if (open1 && open2) {
        const double q = ug * ia1;
        pm1 = k.ps - d.hr137 * (q * q) - 0.5 * (Rv1 * ug + k.srate * (Lg1 * dug));
    }
    const double fm1 = d.d1lg * pm1;
    double pm2 = 0.0;
    if (open1)
        pm2 = open2 ? pm1 - (0.5 * (Rv1 + Rv2) * ug + k.srate * ((Lg1 + Lg2) * dug)) - d.hr * (ug * ug) * (ia2s - ia1s)
                    : k.ps;
    const double fm2 = d.d2lg * pm2;
    const int c1 = x1c + d.g1 < 0.0, c2 = x2c + d.g2 < 0.0;
    const double e1 = d.g1 + x1c, e2 = d.g2 + x2c;
    const double s1 = d.k1e * (x1c * x1c * x1c) + (c1 ? k.h1 : 0.0) * (d.g1 + k.etah1 * (e1 * e1 * e1));
    const double s2 = d.k2e * (x2c * x2c * x2c) + (c2 ? k.h2 : 0.0) * (d.g2 + k.etah2 * (e2 * e2 * e2));
    const double b1 = d.b1c[c1] * x1c - k.m1 * s.x1_old + (fm1 - s1) * d.is2;
    const double b2 = d.b2c[c2] * x2c - k.m2 * s.x2_old + (fm2 - s2) * d.is2;
    const double idet = d.idet[c1][c2];
    const double x1n = (d.a22[c2] * b1 - d.a12 * b2) * idet;
    const double x2n = (d.a11[c1] * b2 - d.a12 * b1) * idet;
    TmmPrep64 o;
    o.x1 = x1c; o.x1n = x1n; o.x2 = x2c; o.x2n = x2n; o.ug = ug;
    o.isr = d.isr; o.ps = k.ps;
    const double Ag1 = k.Ag01 + d.two_lg * x1n;
    const double Ag2 = k.Ag02 + d.two_lg * x2n;
    o.closed = Ag1 < 0 || Ag2 < 0;
    o.Lug = 0;
    o.den = 1;
    if (!o.closed) {
        const double ja1 = 1.0 / Ag1, ja2 = 1.0 / Ag2;
        const double ja1s = ja1 * ja1, ja2s = ja2 * ja2;
        const double r = Ag2 * d.iA1;
        const double Rtot = d.hr * fabs(ug) * (0.37 * ja1s + (1.0 - 2.0 * r * (1.0 - r)) * ja2s) +
                            d.c12 * (k.d1 * (ja1s * ja1) + k.d2 * (ja2s * ja2));
        const double Ltot = d.cL1 * ja1 + d.cL2 * ja2;
        o.Lug = Ltot * ug;
        o.den = Rtot * d.isr + Ltot;
    }
    return o;
}

__device__ __forceinline__ float tmm_finish64(const TmmPrep64& o, TmmState64& s, float p1f) {
    const double p1 = (double)p1f;
    const double ugn = o.closed ? 0.0 : ((o.ps - p1) * o.isr + o.Lug) / o.den;
    s.x1_old = o.x1; s.x1_curr = o.x1n;
    s.x2_old = o.x2; s.x2_curr = o.x2n;
    s.ug_old = o.ug;
    s.ug_curr = ugn;
    return (float)ugn;
}

__device__ __noinline__ float tmm_step64(const TmmConsts64& k, const TmmDerived64& d, TmmState64& s, float p1f) {
    const TmmPrep64 o = tmm_prepare64(k, d, s);
    return tmm_finish64(o, s, p1f);
}

// One two-mass step of tube T from the state of parity par and the pressure
// p1 at the excitation point; with `store` the new state is written to parity
// par ^ 1 (and, when hist is given, as 6 doubles to hist).
__device__ __noinline__ float glottal_step(const TubeDev* T, int par, float p1, bool store, double* hist) {
    if (T->flags & TUBE_TMM64) {
        TmmState64 s = T->tmm64[par];
        const float e = tmm_step64(T->tmmd, T->tmmx, s, p1);
        if (store) {
            T->tmm64[par ^ 1] = s;
            if (hist) {
                hist[0] = s.x1_old; hist[1] = s.x1_curr; hist[2] = s.x2_old;
                hist[3] = s.x2_curr; hist[4] = s.ug_old; hist[5] = s.ug_curr;
            }
        }
        return e;
    }
    TmmState s = T->tmm[par];
    const float e = tmm_step(T->tmmc, s, p1);
    if (store) {
        T->tmm[par ^ 1] = s;
        if (hist) {
            hist[0] = s.x1_old; hist[1] = s.x1_curr; hist[2] = s.x2_old;
            hist[3] = s.x2_curr; hist[4] = s.ug_old; hist[5] = s.ug_curr;
        }
    }
    return e;
}

// The six state values of a two-mass state as the adjoint's history keeps them.
template <class S>
__device__ __forceinline__ void tmm_to_hist(const S& s, double* h) {
    h[0] = s.x1_old; h[1] = s.x1_curr; h[2] = s.x2_old;
    h[3] = s.x2_curr; h[4] = s.ug_old; h[5] = s.ug_curr;
}

// Two-mass steps n and n+1 for the two-step kernels: the state of step n is
// in the parity slot (from_x = false) or the third slot, that of step n+2
// goes to the other one (stored by the owning strip only, which also writes
// the states after steps n and n+1 to hist[0..5] and hist[6..11] when given).
__device__ __noinline__ float2 glottal_two_steps(const TubeDev* T, int par, bool from_x, float p1, float p2,
                                                 bool store, double* hist = nullptr) {
    float2 e;
    if (T->flags & TUBE_TMM64) {
        TmmState64 s = from_x ? *T->tmm64_x : T->tmm64[par];
        e.x = tmm_step64(T->tmmd, T->tmmx, s, p1);
        if (store && hist) tmm_to_hist(s, hist);
        e.y = tmm_step64(T->tmmd, T->tmmx, s, p2);
        if (store && hist) tmm_to_hist(s, hist + 6);
        if (store) *(from_x ? &T->tmm64[par] : T->tmm64_x) = s;
    } else {
        TmmState s = from_x ? *T->tmm_x : T->tmm[par];
        e.x = tmm_step(T->tmmc, s, p1);
        if (store && hist) tmm_to_hist(s, hist);
        e.y = tmm_step(T->tmmc, s, p2);
        if (store && hist) tmm_to_hist(s, hist + 6);
        if (store) *(from_x ? &T->tmm[par] : T->tmm_x) = s;
    }
    return e;
}

// a / b for b > 0 with the signed zero returned directly when a is zero:
// the same value as the division, without sending the zero fields of a cold
// start through the slow path of the IEEE divide.
__device__ __forceinline__ float fdiv_z(float a, float b) { return a == 0.0f ? a : fdiv(a, b); }

// Velocity update of one cell, FDTDEngineCPU.cpp:364-410, with the 17
// coefficient arrays of calculateSolverCoefficients (FDTDSolver.cu:652-801)
// derived from the cell codes of the cell, its right and its top neighbour.
//
// Every beta is 0 or 1, so minBeta, x1..x4, the no-excitation factors and
// the excitation weights multiply by exact 0 / 1 and the normal components
// are 1 or 0.707106 chosen by the neighbours' betas (betaLookUpTable,
// FDTDSolver.cu:1047-1056, with the tables of DeviceSymbols.cu:20-21).  The reference expression
//   V' = ((mB V - bX dP) + exeV ew mS + mS zinv n (x2 Pc Nout - x1 Pn Nin)) / (mB + mS)
// is evaluated here with those exact factors resolved by selects: the
// remaining products, sums and the division are the reference's, in its
// order, so the values are equal (a dropped term only ever adds an exact 0).
struct VelocityOut { float vx, vy; };

// beta per cell type (SolverParams::setBeta, SolverParams.cu:5-27): 1 for
// air, PML 0..5 and no-pressure cells, 0 otherwise
constexpr uint32_t kBetaMask = 0x9FAu;

__device__ __forceinline__ bool beta_bit(int t) { return (kBetaMask >> t) & 1u; }

__device__ __forceinline__ float velocity_dir(bool bc, bool bn, bool bo, bool ec, bool en, float dirc, float dirn,
                                              float v0, float pc, float pn, float exeV, float mS, float zinv,
                                              float bco) {
    const bool mB = bc && bn;
    float v = mB ? fsub(v0, fmul(bco, fsub(pn, pc))) : 0.0f;
    if (ec || en) v = fadd(v, fmul(fmul(exeV, fadd(fmul((float)ec, dirc), fmul((float)en, dirn))), mS));
    if (zinv != 0.0f && !(ec || en) && bc != bn) {
        // x2 = bc (1 - bn): Pc * Nout, Nout = 1/sqrt(2) when the other neighbour is
        // a wall (beta 0), else 1; x1 = bn (1 - bc): -Pn * Nin with Nin = 1
        const float vb = bc ? fmul(pc, bo ? 1.0f : 0.707106f) : -pn;
        v = fadd(v, fmul(mS, fmul(vb, zinv)));
    }
    return fdiv_z(v, fadd(mB ? 1.0f : 0.0f, mS));
}

__device__ __forceinline__ VelocityOut velocity_generic(
        int kc, int kr, int kt, float pc, float pr, float pt, float vx0, float vy0, float exeV,
        const float* __restrict__ sig, float zval, float bco, float dir0, float dir1, float dir2, float dir3) {
    const int tc = kc & CODE_TYPE_MASK, tr = kr & CODE_TYPE_MASK, tt = kt & CODE_TYPE_MASK;
    const bool bc = beta_bit(tc), br = beta_bit(tr), bt = beta_bit(tt);
    const bool ec = tc == VS_CELL_EXCITATION, er = tr == VS_CELL_EXCITATION, et = tt == VS_CELL_EXCITATION;
    const float sc = sig[tc];
    const float zinv = (kc & CODE_ZINV_BIT) ? zval : 0.0f;
    return {velocity_dir(bc, br, bt, ec, er, dir2, dir0, vx0, pc, pr, exeV, fmaxf(sc, sig[tr]), zinv, bco),
            velocity_dir(bc, bt, br, ec, et, dir3, dir1, vy0, pc, pt, exeV, fmaxf(sc, sig[tt]), zinv, bco)};
}

// velocity_dir with its neighbourhood resolved ahead: `bits` = the EXD_*
// flags of one direction, den = mB + mS rounded, mS and the source weight
// W = ec dirc + en dirn rounded as velocity_dir forms them.  The same
// products, sums and division in the same order; the division by den = 1 is
// the identity and is skipped.
__device__ __forceinline__ float velocity_tab(unsigned bits, float den, float mS, float W, float v0, float pc,
                                              float pn, float exeV, float zval, float bco) {
    float v = (bits & EXD_MB) ? fsub(v0, fmul(bco, fsub(pn, pc))) : 0.0f;
    if (bits & EXD_SRC) v = fadd(v, fmul(fmul(exeV, W), mS));
    if ((bits & EXD_WALL) && zval != 0.0f) {
        const float vb = (bits & EXD_WALL_PC) ? fmul(pc, (bits & EXD_NOUT1) ? 1.0f : 0.707106f) : -pn;
        v = fadd(v, fmul(mS, fmul(vb, zval)));
    }
    return den != 1.0f ? fdiv_z(v, den) : v;
}

// Pressure denominator of a cell, (1 + sigma) dP (FDTDEngineCPU.cpp:330) with
// sP = 1 + sigma rounded, or sigma dP + dP (FDTDEngineEigen.cpp:251) with
// sP = sigma.
__device__ __forceinline__ float pressure_den(float sP, float dp, bool eigen) {
    return eigen ? fadd(fmul(sP, dp), dp) : fmul(sP, dp);
}

// Listener sample of a step; a non-finite value (an unstable tube) also
// raises the run's sticky error word, so runs that keep their traces on the
// device report VS_ERR_NONFINITE too.
__device__ __forceinline__ void store_trace(RunState* rs, float* dst, float v) {
    *dst = v;
    if (!isfinite(v)) atomicExch(&rs->error, VS_ERR_NONFINITE);
}

// Approximate reciprocal (PTX rcp.approx.f32, at most 1 ulp from 1/x).
__device__ __forceinline__ float rcp_approx(float x) {
    float r;
    asm("rcp.approx.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

}  // namespace
}  // namespace vsb
