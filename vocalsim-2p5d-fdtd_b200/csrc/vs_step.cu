// vs_step.cu -- fused FDTD time step for sm_100a.
//
// One launch advances every tile of every tube by one time step of the
// reference loop (FDTDEngineCPU.cpp:257-288):
//   exeV (table or on-device two-mass model) -> pressure pass with the 2.5D
//   depth fluxes, PML sigma and Dirichlet column -> listener readout -> wall
//   oscillator (when coupled) -> velocity pass with PML, boundary admittance
//   and source injection.
// The outer ring is never written, so it keeps the zeros that
// update_border_cells (:412-433) re-imposes each step, and the ping-pong by
// step parity replaces the PV_N = PV_Nplus1 copy (:287).
//
// Layout: one CTA per TR x TC tile; the tile plus a one-cell halo is staged in
// shared memory (depth-weighted velocities Ux = Vx*dX, Uy = Vy*dY, the code
// bytes), P' is computed on the tile plus its right column and top row, and
// V' of the tile reads P' neighbours from shared memory, so P and V of a step
// are fused in one pass.  All arithmetic uses round-to-nearest intrinsics in
// the reference's operand order (no FMA contraction), so results are
// identical to the reference FP32 engine on the same maps.
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

constexpr int kNT = 256;

// betaLookUpTable (FDTDSolver.cu:1047-1056) for beta in {0, 1}:
// (air, air) -> 0, (air, wall) -> 1, (wall, air) -> 2, (wall, wall) -> 3.
__device__ __forceinline__ int beta_lut(float br, float bt) {
    return (br == 0.0f ? 2 : 0) + (bt == 0.0f ? 1 : 0);
}

// One step of the Ishizaka-Flanagan two-mass model, TwoMassModel.cpp:90-232,
// in the reference's mixed float/double precision and operand order.  The
// reference's host build (g++) forms (rho/2)*fabs(ug) in double.
__device__ float tmm_step(const TmmConsts& k, TmmState& s, float p1) {
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

template <int TR, int TC>
__global__ void __launch_bounds__(kNT)
step_kernel(const TubeDev* __restrict__ tubes, const Tile* __restrict__ tiles,
            RunState* __restrict__ rs, int local) {
    __shared__ float sUx[TR + 1][TC + 2];   // rows r0-1.., cols c0-1..c0+TC
    __shared__ float sUy[TR + 2][TC + 1];   // rows r0-1..r0+TR, cols c0..c0+TC
    __shared__ float sPn[TR + 1][TC + 1];   // rows r0-1.., cols c0..c0+TC
    __shared__ uint8_t sCode[TR + 1][TC + 1];
    __shared__ float sSig[16];
    __shared__ float sExe;

    const Tile tile = tiles[blockIdx.x];
    const TubeDev& T = tubes[tile.tube];
    const int64_t n = rs->step + local;
    const int par = (int)(n & 1);
    const int H = T.H, W = T.W, pitch = T.pitch, flags = T.flags;
    const int r0 = tile.r0, c0 = tile.c0;
    const float* __restrict__ Pin = T.P[par];
    const float* __restrict__ Vxin = T.Vx[par];
    const float* __restrict__ Vyin = T.Vy[par];
    float* __restrict__ Pout = T.P[par ^ 1];
    float* __restrict__ Vxout = T.Vx[par ^ 1];
    float* __restrict__ Vyout = T.Vy[par ^ 1];
    const float* __restrict__ dPp = T.dP;
    const float* __restrict__ dXp = T.dX;
    const float* __restrict__ dYp = T.dY;
    const uint8_t* __restrict__ code = T.code;

    if (threadIdx.x < 16) sSig[threadIdx.x] = threadIdx.x < 13 ? T.sigma[threadIdx.x] : 0.0f;
    if (threadIdx.x == 0) {
        float e = 0.0f;
        if (tile.has_exc) {
            if (flags & TUBE_TMM) {
                // every tile of the excitation column advances the same state
                // from the same input; only the tile owning the excitation
                // cell stores it for the next step
                TmmState s = T.tmm[par];
                e = tmm_step(T.tmmc, s, Pin[(size_t)T.exc_y * pitch + T.exc_x]);
                if (T.exc_y >= r0 && T.exc_y < r0 + TR && T.exc_x >= c0 && T.exc_x < c0 + TC)
                    T.tmm[par ^ 1] = s;
            } else {
                e = n < T.src_len ? T.src[n] : 0.0f;
            }
        }
        sExe = e;
    }
    // ---- stage depth-weighted velocities and codes (one-cell halo) ----
    for (int i = threadIdx.x; i < (TR + 1) * (TC + 2); i += kNT) {
        const int rr = i / (TC + 2), cc = i - rr * (TC + 2);
        const int r = r0 - 1 + rr, c = c0 - 1 + cc;
        float u = 0.0f;
        if (r >= 0 && r < H && c >= 0 && c < W) {
            const size_t o = (size_t)r * pitch + c;
            u = fmul(Vxin[o], dXp[o]);
        }
        sUx[rr][cc] = u;
    }
    for (int i = threadIdx.x; i < (TR + 2) * (TC + 1); i += kNT) {
        const int rr = i / (TC + 1), cc = i - rr * (TC + 1);
        const int r = r0 - 1 + rr, c = c0 + cc;
        float u = 0.0f;
        if (r >= 0 && r < H && c < W) {
            const size_t o = (size_t)r * pitch + c;
            u = fmul(Vyin[o], dYp[o]);
        }
        sUy[rr][cc] = u;
    }
    for (int i = threadIdx.x; i < (TR + 1) * (TC + 1); i += kNT) {
        const int rr = i / (TC + 1), cc = i - rr * (TC + 1);
        const int r = r0 - 1 + rr, c = c0 + cc;
        sCode[rr][cc] = (r >= 0 && r < H && c < W) ? code[(size_t)r * pitch + c] : (uint8_t)VS_CELL_DEAD;
    }
    __syncthreads();

    // ---- pressure on the tile + right column + top row (FDTDEngineCPU.cpp:316-339)
    const float K1 = T.K1, K2 = T.K2;
    const bool eigen = flags & TUBE_EIGEN, dirichlet = flags & TUBE_DIRICHLET;
    const bool wall = flags & TUBE_WALL_ODE;
    for (int i = threadIdx.x; i < (TR + 1) * (TC + 1); i += kNT) {
        const int rr = i / (TC + 1), cc = i - rr * (TC + 1);
        const int r = r0 - 1 + rr, c = c0 + cc;
        float pn = 0.0f;
        if (r >= 1 && r <= H - 2 && c >= 1 && c <= W - 2) {
            const size_t o = (size_t)r * pitch + c;
            const int type = sCode[rr][cc] & CODE_TYPE_MASK;
            const float sig = sSig[type];
            const float cx = fsub(sUx[rr][cc + 1], sUx[rr][cc]);
            const float cy = fsub(sUy[rr][cc], sUy[rr + 1][cc]);
            const float dp = dPp[o];
            float num = fsub(fmul(Pin[o], dp), fmul(K1, fadd(cx, cy)));
            const bool mine = rr >= 1 && cc < TC;
            float w = 0.0f;
            if (wall) {
                w = T.w[par][o];
                num = fsub(num, fmul(K2, w));
            }
            const float den = eigen ? fadd(fmul(sig, dp), dp) : fmul(fadd(1.0f, sig), dp);
            pn = fdiv(num, den);
            if (dirichlet && type == VS_CELL_NOPRESSURE) pn = 0.0f;
            if (mine) {
                Pout[o] = pn;
                if (r == T.lis_y && c == T.lis_x)
                    rs->trace[(int64_t)tile.tube * rs->trace_stride + (n - rs->run_start)] = pn;
                if (wall) {
                    // wall oscillator, FDTDEngineCPU.cpp:345-361
                    const float dt = T.dt;
                    const float zn = fadd(T.z[par][o], fmul(w, dt));
                    const float wn = fdiv(fsub(fadd(fmul(T.Mw, w), fmul(fmul(T.cpl, dt), pn)),
                                              fmul(fmul(dt, T.Kw), zn)),
                                         fadd(T.Mw, fmul(dt, T.Bw)));
                    T.z[par ^ 1][o] = zn;
                    T.w[par ^ 1][o] = wn;
                }
            }
        }
        sPn[rr][cc] = pn;
    }
    __syncthreads();

    // ---- velocity on the tile (FDTDEngineCPU.cpp:364-410) ----
    const float exeV = sExe;
    const float zval = T.zinv, bco = T.bcoef;
    const float dir0 = T.dir0, dir1 = T.dir1, dir2 = T.dir2, dir3 = T.dir3;
    for (int i = threadIdx.x; i < TR * TC; i += kNT) {
        const int ri = i / TC, cc = i - ri * TC;
        const int rr = ri + 1;
        const int r = r0 + ri, c = c0 + cc;
        if (r < 1 || r > H - 2 || c < 1 || c > W - 2) continue;
        const size_t o = (size_t)r * pitch + c;
        const uint8_t kc = sCode[rr][cc];
        const int tc = kc & CODE_TYPE_MASK;
        const int tr = sCode[rr][cc + 1] & CODE_TYPE_MASK;
        const int tt = sCode[rr - 1][cc] & CODE_TYPE_MASK;
        const float bc = c_beta[tc], br = c_beta[tr], bt = c_beta[tt];
        const int lut = beta_lut(br, bt);
        const float Nout = fmul(c_airN[lut], bc);
        const float Nin = fmul(c_wallN[lut], fsub(1.0f, bc));
        const float sc = sSig[tc], sr = sSig[tr], st = sSig[tt];
        const int ec = tc == VS_CELL_EXCITATION, er = tr == VS_CELL_EXCITATION,
                  et = tt == VS_CELL_EXCITATION;
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
        const float pc = sPn[rr][cc], pr = sPn[rr][cc + 1], pt = sPn[rr - 1][cc];
        const float CxP = fsub(pr, pc), CyP = fsub(pt, pc);
        float vx = fsub(fmul(mBx, Vxin[o]), fmul(bX, CxP));
        float vy = fsub(fmul(mBy, Vyin[o]), fmul(bY, CyP));
        vx = fadd(vx, fmul(fmul(exeV, ewX), mSx));
        vy = fadd(vy, fmul(fmul(exeV, ewY), mSy));
        float vbx = fsub(fmul(fmul(x2, pc), Nout), fmul(fmul(x1, pr), Nin));
        float vby = fsub(fmul(fmul(x4, pc), Nout), fmul(fmul(x3, pt), Nin));
        vbx = fmul(fmul(vbx, nX), zinv);
        vby = fmul(fmul(vby, nY), zinv);
        vx = fadd(vx, fmul(mSx, vbx));
        vy = fadd(vy, fmul(mSy, vby));
        Vxout[o] = fdiv(vx, fadd(mBx, mSx));
        Vyout[o] = fdiv(vy, fadd(mBy, mSy));
    }
}

__global__ void advance_kernel(RunState* rs, int k) { rs->step += k; }

struct ShapeEntry {
    int rows, cols;
    void (*fn)(const TubeDev*, const Tile*, RunState*, int);
};

const ShapeEntry kShapes[] = {
    {4, 64, step_kernel<4, 64>},   {8, 32, step_kernel<8, 32>},   {8, 64, step_kernel<8, 64>},
    {16, 32, step_kernel<16, 32>}, {8, 128, step_kernel<8, 128>}, {16, 64, step_kernel<16, 64>},
    {32, 32, step_kernel<32, 32>}, {16, 128, step_kernel<16, 128>},
};
constexpr int kNumShapes = sizeof(kShapes) / sizeof(kShapes[0]);

}  // namespace

int tile_shape_count() { return kNumShapes; }

TileShape tile_shape(int i) { return {kShapes[i].rows, kShapes[i].cols}; }

cudaError_t launch_step(int shape, const TubeDev* tubes, const Tile* tiles, int ntiles,
                        RunState* rs, int local, cudaStream_t stream) {
    if (shape < 0 || shape >= kNumShapes) return cudaErrorInvalidValue;
    if (ntiles <= 0) return cudaSuccess;
    kShapes[shape].fn<<<ntiles, kNT, 0, stream>>>(tubes, tiles, rs, local);
    return cudaGetLastError();
}

cudaError_t launch_advance(RunState* rs, int k, cudaStream_t stream) {
    advance_kernel<<<1, 1, 0, stream>>>(rs, k);
    return cudaGetLastError();
}

}  // namespace vsb
