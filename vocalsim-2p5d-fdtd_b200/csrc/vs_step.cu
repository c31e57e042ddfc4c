// vs_step.cu -- fused FDTD time step for sm_100a.
//
// One launch advances every strip of every tube by one time step of the
// reference loop (FDTDEngineCPU.cpp:257-288):
//   exeV (table or on-device two-mass model) -> pressure pass with the 2.5D
//   depth fluxes, PML sigma and Dirichlet column -> listener readout -> wall
//   oscillator (when coupled) -> velocity pass with PML, boundary admittance
//   and source injection.
// The outer ring is never written, so it keeps the zeros that
// update_border_cells (:412-433) re-imposes each step, and the ping-pong by
// step parity replaces the PV_N = PV_Nplus1 copy (:287).
//
// Work decomposition: one warp owns a strip of 32 columns x TR rows and
// marches down the rows.  Lane i holds column x0 + i; strips overlap by two
// columns (stride 30), so lane 0 only supplies the left depth flux and
// lane 31 only the right P' neighbour, and lanes 1..30 commit.  Vertical
// neighbours (P' above, Vy*dY below) stay in registers, horizontal ones move
// by shuffles: no shared memory and no block barrier.  The next row's loads
// are issued before the current row is computed.
//
// Arithmetic: round-to-nearest intrinsics in the reference's operand order,
// no FMA contraction, so results equal the reference FP32 engine on the same
// maps.  A warp whose 32 cells are all plain air takes a shortened path that
// drops only operations the reference performs with exact 0 / 1 operands
// (x*1, x+0, x/1): the values are identical.
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

// SolverParams::setBeta (SolverParams.cu:5-27) for 6 PML layers; the normal
// component tables of DeviceSymbols.cu:20-21.
__constant__ float c_beta[16] = {0, 1, 0, 1, 1, 1, 1, 1, 1, 0, 0, 1, 0, 0, 0, 0};
__constant__ float c_airN[4] = {0.0f, 1.0f, 1.0f, 0.707106f};
__constant__ float c_wallN[4] = {1.0f, 1.0f, 1.0f, 0.0f};

constexpr unsigned kFull = 0xffffffffu;
constexpr int kStride = 30;      // committed columns per strip

// betaLookUpTable (FDTDSolver.cu:1047-1056) for beta in {0, 1}:
// (air, air) -> 0, (air, wall) -> 1, (wall, air) -> 2, (wall, wall) -> 3.
__device__ __forceinline__ int beta_lut(float br, float bt) {
    return (br == 0.0f ? 2 : 0) + (bt == 0.0f ? 1 : 0);
}

// One step of the Ishizaka-Flanagan two-mass model, TwoMassModel.cpp:90-232,
// in the reference's mixed float/double precision and operand order.  The
// reference's host build (g++) forms (rho/2)*fabs(ug) in double.
__device__ __noinline__ float tmm_step(const TmmConsts& k, TmmState& s, float p1) {
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
    s.x1_old = x1; s.x1_curr = x1n;
    s.x2_old = x2; s.x2_curr = x2n;
    Ag1 = fadd(k.Ag01, fmul(two_lg, x1n));
    Ag2 = fadd(k.Ag02, fmul(two_lg, x2n));
    float ugn;
    if (Ag1 < 0.0f || Ag2 < 0.0f) {
        ugn = 0.0f;
    } else {
        const float r = fdiv(Ag2, k.A1);
        const float f = fdiv(fsub(1.0f, fmul(fmul(2.0f, r), fsub(1.0f, r))), fmul(Ag2, Ag2));
        const double t1 = dmul(dmul(dd(half_rho), fabs(dd(ug))),
                               dadd(__ddiv_rn(0.37, dd(fmul(Ag1, Ag1))), dd(f)));
        const float t2 = fmul(mu12lglg, fadd(fdiv(k.d1, fmul(fmul(Ag1, Ag1), Ag1)),
                                             fdiv(k.d2, fmul(fmul(Ag2, Ag2), Ag2))));
        const float Rtot = tof(dadd(t1, dd(t2)));
        const float Ltot = fmul(k.rho, fadd(fdiv(k.d1, Ag1), fdiv(k.d2, Ag2)));
        ugn = fdiv(fadd(fdiv(fsub(k.ps, p1), srate), fmul(Ltot, ug)), fadd(fdiv(Rtot, srate), Ltot));
    }
    s.ug_old = ug;
    s.ug_curr = ugn;
    return ugn;
}

// Velocity update of one cell, FDTDEngineCPU.cpp:364-410, with the 17
// coefficient arrays of calculateSolverCoefficients (FDTDSolver.cu:652-801)
// derived from the cell codes of the cell, its right and its top neighbour.
struct VelocityOut { float vx, vy; };

__device__ __forceinline__ VelocityOut velocity_generic(
        int kc, int kr, int kt, float pc, float pr, float pt, float vx0, float vy0, float exeV,
        const float* sig, float zval, float bco, float dir0, float dir1, float dir2, float dir3) {
    const int tc = kc & CODE_TYPE_MASK, tr = kr & CODE_TYPE_MASK, tt = kt & CODE_TYPE_MASK;
    const float bc = c_beta[tc], br = c_beta[tr], bt = c_beta[tt];
    const int lut = beta_lut(br, bt);
    const float Nout = fmul(c_airN[lut], bc);
    const float Nin = fmul(c_wallN[lut], fsub(1.0f, bc));
    const float sc = sig[tc], sr = sig[tr], st = sig[tt];
    const int ec = tc == VS_CELL_EXCITATION, er = tr == VS_CELL_EXCITATION, et = tt == VS_CELL_EXCITATION;
    const float mBx = fminf(bc, br), mBy = fminf(bc, bt);
    const float mSx = fmaxf(sc, sr), mSy = fmaxf(sc, st);
    // (minBeta^2 * dt) / (rho * ds) with minBeta in {0, 1}
    const float bX = mBx != 0.0f ? bco : 0.0f;
    const float bY = mBy != 0.0f ? bco : 0.0f;
    const float nX = (float)((1 - ec) * (1 - er));
    const float nY = (float)((1 - ec) * (1 - et));
    const float ewX = fadd(fmul((float)ec, dir2), fmul((float)er, dir0));
    const float ewY = fadd(fmul((float)ec, dir3), fmul((float)et, dir1));
    const float x1 = fmul(br, fsub(1.0f, bc)), x2 = fmul(bc, fsub(1.0f, br));
    const float x3 = fmul(bt, fsub(1.0f, bc)), x4 = fmul(bc, fsub(1.0f, bt));
    const float zinv = (kc & CODE_ZINV_BIT) ? zval : 0.0f;
    const float CxP = fsub(pr, pc), CyP = fsub(pt, pc);
    float vx = fsub(fmul(mBx, vx0), fmul(bX, CxP));
    float vy = fsub(fmul(mBy, vy0), fmul(bY, CyP));
    vx = fadd(vx, fmul(fmul(exeV, ewX), mSx));
    vy = fadd(vy, fmul(fmul(exeV, ewY), mSy));
    float vbx = fsub(fmul(fmul(x2, pc), Nout), fmul(fmul(x1, pr), Nin));
    float vby = fsub(fmul(fmul(x4, pc), Nout), fmul(fmul(x3, pt), Nin));
    vbx = fmul(fmul(vbx, nX), zinv);
    vby = fmul(fmul(vby, nY), zinv);
    vx = fadd(vx, fmul(mSx, vbx));
    vy = fadd(vy, fmul(mSy, vby));
    return {fdiv(vx, fadd(mBx, mSx)), fdiv(vy, fadd(mBy, mSy))};
}

template <int TR>
__global__ void __launch_bounds__(256, 4)
strip_kernel(const TubeDev* __restrict__ tubes, const Tile* __restrict__ items, int nitems,
             RunState* __restrict__ rs, int local) {
    const int lane = threadIdx.x & 31;
    const int wi = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (wi >= nitems) return;
    const Tile it = items[wi];
    const TubeDev* __restrict__ T = tubes + it.tube;
    const int64_t n = rs->step + local;
    const int par = (int)(n & 1);
    const int H = T->H, W = T->W, pitch = T->pitch, flags = T->flags;
    const int r0 = it.r0, x = it.c0 + lane;
    const bool col_ok = x >= 0 && x < W;
    const bool col_in = x >= 1 && x <= W - 2;
    const bool commit_lane = lane >= 1 && lane <= kStride;
    // planes are laid out P0 P1 Vx0 Vx1 Vy0 Vy1 and dP dX dY, `plane` apart
    const int64_t pl = T->plane;
    const float* __restrict__ Pin = T->P[0] + par * pl;
    float* __restrict__ Pout = T->P[0] + (par ^ 1) * pl;
    const float* __restrict__ Vxin = Pin + 2 * pl;
    const float* __restrict__ Vyin = Pin + 4 * pl;
    float* __restrict__ Vxout = Pout + 2 * pl;
    float* __restrict__ Vyout = Pout + 4 * pl;
    const float* __restrict__ dPp = T->dP;
    const float* __restrict__ dXp = dPp + pl;
    const float* __restrict__ dYp = dPp + 2 * pl;
    const uint8_t* __restrict__ code = T->code;
    const float K1 = T->K1, K2 = T->K2, bco = T->bcoef, zval = T->zinv;
    const bool eigen = flags & TUBE_EIGEN, dirichlet = flags & TUBE_DIRICHLET;
    const bool wall = flags & TUBE_WALL_ODE;
    const float* __restrict__ sig = T->sigma;

    // excitation velocity of this step (only strips holding excitation cells need it)
    float exeV = 0.0f;
    if (it.has_exc) {
        if (flags & TUBE_TMM) {
            if (lane == 0) {
                // every strip holding excitation cells advances the same state from
                // the same input; the strip that commits the excitation cell stores it
                TmmState s = T->tmm[par];
                exeV = tmm_step(T->tmmc, s, Pin[(size_t)T->exc_y * pitch + T->exc_x]);
                const int ex = T->exc_x - it.c0;
                if (T->exc_y >= r0 && T->exc_y < r0 + TR && ex >= 1 && ex <= kStride) T->tmm[par ^ 1] = s;
            }
            exeV = __shfl_sync(kFull, exeV, 0);
        } else {
            exeV = n < T->src_len ? T->src[n] : 0.0f;
        }
    }
    const int rlast = min(r0 + TR - 1, H - 2);

    // prologue: the row above the strip (r0 - 1) supplies P' and codes for the
    // top neighbours of row r0; its own P' is recomputed, not committed.
    int r = r0 - 1;
    size_t o = (size_t)r * pitch + x;
    float vy_c = 0.0f, uy_c = 0.0f;
    if (col_ok) { vy_c = Vyin[o]; uy_c = fmul(vy_c, dYp[o]); }
    float vx_c = 0.0f, ux_c = 0.0f, p_c = 0.0f, dp_c = 1.0f;
    int k_c = VS_CELL_DEAD;
    if (col_ok) {
        vx_c = Vxin[o]; ux_c = fmul(vx_c, dXp[o]); p_c = Pin[o]; dp_c = dPp[o]; k_c = code[o];
    }
    float p_above = 0.0f;
    int k_above = VS_CELL_DEAD;

    for (; r <= rlast; ++r) {
        // ---- issue next-row loads first (row r+1 fields, row r+2 Vy/dY)
        const size_t on = o + pitch;
        float vy_n = 0.0f, uy_n = 0.0f;
        float vx_n = 0.0f, ux_n = 0.0f, p_n = 0.0f, dp_n = 1.0f;
        int k_n = VS_CELL_DEAD;
        if (col_ok) {                       // r + 1 <= H - 1 always holds here
            vy_n = Vyin[on]; uy_n = fmul(vy_n, dYp[on]);
            vx_n = Vxin[on]; ux_n = fmul(vx_n, dXp[on]); p_n = Pin[on]; dp_n = dPp[on]; k_n = code[on];
        }
        // ---- pressure of row r (FDTDEngineCPU.cpp:316-339)
        const float ux_l = __shfl_up_sync(kFull, ux_c, 1);
        const bool in = col_in && r >= 1;
        const int tc = k_c & CODE_TYPE_MASK;
        const bool plain_p = (tc == VS_CELL_AIR) || !(in && lane >= 1);
        float pn = 0.0f;
        float w = 0.0f;
        if (__all_sync(kFull, plain_p) && !wall) {
            if (in && lane >= 1) {
                // sigma = 0: (1 + 0) * dP == 0 * dP + dP == dP exactly
                const float cx = fsub(ux_c, ux_l), cy = fsub(uy_c, uy_n);
                pn = fdiv(fsub(fmul(p_c, dp_c), fmul(K1, fadd(cx, cy))), dp_c);
            }
        } else if (in && lane >= 1) {
            const float cx = fsub(ux_c, ux_l), cy = fsub(uy_c, uy_n);
            float num = fsub(fmul(p_c, dp_c), fmul(K1, fadd(cx, cy)));
            if (wall) {
                w = T->w[par][o];
                num = fsub(num, fmul(K2, w));
            }
            const float s = sig[tc];
            const float den = eigen ? fadd(fmul(s, dp_c), dp_c) : fmul(fadd(1.0f, s), dp_c);
            pn = fdiv(num, den);
            if (dirichlet && tc == VS_CELL_NOPRESSURE) pn = 0.0f;
        }
        // ---- commit row r and its velocity (FDTDEngineCPU.cpp:364-410)
        const float p_right = __shfl_down_sync(kFull, pn, 1);
        const int k_right = __shfl_down_sync(kFull, k_c, 1);
        if (r >= r0) {
            const bool mine = in && commit_lane;
            if (mine) {
                Pout[o] = pn;
                if (r == T->lis_y && x == T->lis_x)
                    rs->trace[(int64_t)it.tube * rs->trace_stride + (n - rs->run_start)] = pn;
                if (wall) {
                    // wall oscillator, FDTDEngineCPU.cpp:345-361
                    const float dt = T->dt;
                    const float zn = fadd(T->z[par][o], fmul(w, dt));
                    const float wn = fdiv(fsub(fadd(fmul(T->Mw, w), fmul(fmul(T->cpl, dt), pn)),
                                              fmul(fmul(dt, T->Kw), zn)),
                                         fadd(T->Mw, fmul(dt, T->Bw)));
                    T->z[par ^ 1][o] = zn;
                    T->w[par ^ 1][o] = wn;
                }
            }
            const int tr = k_right & CODE_TYPE_MASK, tt = k_above & CODE_TYPE_MASK;
            const bool plain_v = !mine || (tc == VS_CELL_AIR && tr == VS_CELL_AIR && tt == VS_CELL_AIR &&
                                           !(k_c & CODE_ZINV_BIT));
            if (__all_sync(kFull, plain_v)) {
                if (mine) {
                    // beta = 1, sigma = 0, no source, no boundary term:
                    // V' = V - (dt/(rho ds)) * dP' exactly as the full expression
                    Vxout[o] = fsub(vx_c, fmul(bco, fsub(p_right, pn)));
                    Vyout[o] = fsub(vy_c, fmul(bco, fsub(p_above, pn)));
                }
            } else if (mine) {
                const VelocityOut v = velocity_generic(k_c, k_right, k_above, pn, p_right, p_above, vx_c, vy_c,
                                                       exeV, sig, zval, bco, T->dir0, T->dir1, T->dir2, T->dir3);
                Vxout[o] = v.vx;
                Vyout[o] = v.vy;
            }
        }
        // ---- shift the row pipeline
        p_above = pn; k_above = k_c;
        vy_c = vy_n; uy_c = uy_n;
        vx_c = vx_n; ux_c = ux_n; p_c = p_n; dp_c = dp_n; k_c = k_n;
        o = on;
    }
}

__global__ void advance_kernel(RunState* rs, int k) { rs->step += k; }

struct ShapeEntry {
    int rows, warps;
    void (*fn)(const TubeDev*, const Tile*, int, RunState*, int);
};

const ShapeEntry kShapes[] = {
    {8, 4, strip_kernel<8>},   {16, 4, strip_kernel<16>}, {32, 4, strip_kernel<32>}, {64, 4, strip_kernel<64>},
    {8, 8, strip_kernel<8>},   {16, 8, strip_kernel<16>}, {32, 8, strip_kernel<32>}, {64, 8, strip_kernel<64>},
};
constexpr int kNumShapes = sizeof(kShapes) / sizeof(kShapes[0]);

}  // namespace

int tile_shape_count() { return kNumShapes; }

TileShape tile_shape(int i) { return {kShapes[i].rows, kStride, kShapes[i].warps}; }

cudaError_t launch_step(int shape, const TubeDev* tubes, const Tile* tiles, int ntiles,
                        RunState* rs, int local, cudaStream_t stream) {
    if (shape < 0 || shape >= kNumShapes) return cudaErrorInvalidValue;
    if (ntiles <= 0) return cudaSuccess;
    const int wpb = kShapes[shape].warps;
    const int blocks = (ntiles + wpb - 1) / wpb;
    kShapes[shape].fn<<<blocks, wpb * 32, 0, stream>>>(tubes, tiles, ntiles, rs, local);
    return cudaGetLastError();
}

cudaError_t launch_advance(RunState* rs, int k, cudaStream_t stream) {
    advance_kernel<<<1, 1, 0, stream>>>(rs, k);
    return cudaGetLastError();
}

}  // namespace vsb
