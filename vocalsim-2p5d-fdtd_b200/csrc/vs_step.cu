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

#include "vs_cellmath.cuh"
#include "vs_mbarrier.cuh"

namespace vsb {
namespace {


// Row-marching strip kernel.  One warp owns a strip of 32 columns x TR rows:
// lane i holds column c0 + i, strips overlap by two columns (stride 30), so
// lane 0 only supplies the left depth flux and lane 31 only the right P'
// neighbour, and lanes 1..30 commit.  Vertical neighbours (P' above, Vy*dY
// below) stay in registers, horizontal ones move by shuffles: no shared
// memory and no block barrier.  Each row's loads are issued one iteration
// before their use.  The strip's row masks (Tile) pick, uniformly per row,
// the pressure path (sigma = 0 or general) and the velocity class:
//   V_PLAIN    air cell with air right and top neighbours: beta = 1,
//              sigma = 0, no source, no boundary term; the reference's full
//              expression reduces exactly to V - dt/(rho ds) * dP'
//   V_BETA1    air / PML / no-pressure cells only: the source and boundary
//              terms add exact zeros, leaving the PML division
//   V_GENERIC  walls, excitation cells, admittance: the full expression
// Every shortened path drops only operations whose operands are exact 0 / 1
// (x*1, x+0, x/1), so values equal the full reference expression.
// Scalar row loads of the strip kernel: read once per warp, so they bypass
// L1 (no_allocate) and leave it to the tube descriptors and tables.
__device__ __forceinline__ float ld1(const float* p) {
    float v;
    asm("ld.global.nc.L1::no_allocate.f32 %0, [%1];" : "=f"(v) : "l"(p));
    return v;
}

__device__ __forceinline__ int ldcode(const uint8_t* p) {
    uint32_t v;
    asm("ld.global.nc.L1::no_allocate.u8 %0, [%1];" : "=r"(v) : "l"(p));
    return (int)v;
}

template <int TR, int MINB, bool WALL, bool HIST = false>
__global__ void __launch_bounds__(256, MINB)
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
    const bool col_in = x >= 1 && x <= W - 2;
    const bool lane_calc = col_in && lane >= 1;
    const bool lane_commit = lane_calc && lane <= kStripCommit;
    // planes are laid out P0 P1 Vx0 Vx1 Vy0 Vy1 and dP dX dY, `plane` apart.
    // Lanes read columns -1 .. W+28 of rows 0 .. H-1 without predicates: the
    // arena keeps guard bytes around every tube, and values read outside the
    // frame only reach lanes that neither compute nor commit them.
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
    const float* __restrict__ sig = T->sigma;
    const float K1 = T->K1, bco = T->bcoef;
    const bool eigen = flags & TUBE_EIGEN, dirichlet = flags & TUBE_DIRICHLET;
    const int lis_y = T->lis_y, lis_x = T->lis_x;
    const uint64_t pmask = it.p_rows, vb1 = it.v_beta1, vgen = it.v_generic;

    // excitation velocity of this step (only strips holding excitation cells need it)
    float exeV = 0.0f;
    if (it.has_exc) {
        if (flags & TUBE_TMM) {
            if (lane == 0) {
                // every strip holding excitation cells advances the same state from
                // the same input; the strip that commits the excitation cell stores it
                const int ex = T->exc_x - it.c0;
                const bool owner =
                    T->exc_y >= r0 && T->exc_y < r0 + TR && ex >= kStripLead && ex < kStripLead + kStripCommit;
                exeV = glottal_step(T, par, Pin[(size_t)T->exc_y * pitch + T->exc_x], owner,
                                    HIST ? T->tmm_hist + 6 * (n + 1 - rs->run_start) : nullptr);
            }
            exeV = __shfl_sync(kFull, exeV, 0);
        } else {
            exeV = n < T->src_len ? T->src[n] : 0.0f;
        }
    }
    const int rlast = min(r0 + TR - 1, H - 2);

    // Row pipeline: iteration j (row r = r0 - 1 + j) computes P' of row r
    // and, from row r0 on, commits it with V' of row r; it issues the loads
    // of row r+1 (Vx, dX, P, dP, code) and row r+2 (Vy, dY).  The row above
    // the strip supplies P' and codes for the top neighbours of row r0; its
    // own P' is recomputed, not committed.
    int r = r0 - 1;
    int o = r * pitch + x;
    float vx_c = ld1(Vxin + o);
    float ux_c = fmul(vx_c, ld1(dXp + o));
    float p_c = ld1(Pin + o), dp_c = ld1(dPp + o);
    int k_c = ldcode(code + o);
    float vy_c = ld1(Vyin + o);
    float uy_c = fmul(vy_c, ld1(dYp + o));
    float vy_n = ld1(Vyin + o + pitch);
    float uy_n = fmul(vy_n, ld1(dYp + o + pitch));
    float p_above = 0.0f;
    int k_above = VS_CELL_DEAD;

    for (int j = 0; r <= rlast; ++j, ++r) {
        // ---- loads for the next iterations
        const int o1 = o + pitch;
        // (read-only this step: the input planes are not the ones written)
        const float vx_1 = ld1(Vxin + o1), dx_1 = ld1(dXp + o1);
        const float p_1 = ld1(Pin + o1), dp_1 = ld1(dPp + o1);
        const int k_1 = ldcode(code + o1);
        float vy_2 = 0.0f, dy_2 = 0.0f;
        if (r + 2 <= H - 1) { vy_2 = ld1(Vyin + o1 + pitch); dy_2 = ld1(dYp + o1 + pitch); }

        // ---- pressure of row r (FDTDEngineCPU.cpp:316-339)
        const float ux_l = __shfl_up_sync(kFull, ux_c, 1);
        const bool calc = lane_calc && r >= 1;
        const int tc = k_c & CODE_TYPE_MASK;
        float num = fsub(fmul(p_c, dp_c), fmul(K1, fadd(fsub(ux_c, ux_l), fsub(uy_c, uy_n))));
        float w = 0.0f;
        if (WALL) {
            if (calc) w = T->w[par][o];
            num = fsub(num, fmul(T->K2, w));
        }
        const bool pgen = (pmask >> j) & 1;
        float den = dp_c;                  // sigma = 0: (1 + 0) * dP == 0 * dP + dP == dP
        if (pgen && tc != VS_CELL_AIR) {
            const float s = sig[tc];
            den = eigen ? fadd(fmul(s, dp_c), dp_c) : fmul(fadd(1.0f, s), dp_c);
        }
        float pn = 0.0f;
        if (calc) {
            pn = fdiv_z(num, den);
            if (pgen && dirichlet && tc == VS_CELL_NOPRESSURE) pn = 0.0f;
        }
        // ---- commit row r and its velocity (FDTDEngineCPU.cpp:364-410)
        const float p_right = __shfl_down_sync(kFull, pn, 1);
        const int k_right = __shfl_down_sync(kFull, k_c, 1);
        if (j >= 1) {
            const int jv = j - 1;
            if (lane_commit) {
                Pout[o] = pn;
                if (r == lis_y && x == lis_x)
                    store_trace(rs, rs->trace + (int64_t)it.tube * rs->trace_stride + (n - rs->run_start), pn);
                if (WALL) {
                    // wall oscillator, FDTDEngineCPU.cpp:345-361
                    const float dt = T->dt;
                    const float zn = fadd(T->z[par][o], fmul(w, dt));
                    T->z[par ^ 1][o] = zn;
                    T->w[par ^ 1][o] = fdiv_z(fsub(fadd(fmul(T->Mw, w), fmul(fmul(T->cpl, dt), pn)),
                                                   fmul(fmul(dt, T->Kw), zn)),
                                              fadd(T->Mw, fmul(dt, T->Bw)));
                }
            }
            float vx, vy;
            if ((vgen >> jv) & 1) {
                vx = 0.0f;
                vy = 0.0f;
                if (lane_commit) {
                    const VelocityOut v = velocity_generic(k_c, k_right, k_above, pn, p_right, p_above, vx_c, vy_c,
                                                           exeV, sig, T->zinv, bco, T->dir0, T->dir1, T->dir2,
                                                           T->dir3);
                    vx = v.vx;
                    vy = v.vy;
                }
            } else {
                vx = fsub(vx_c, fmul(bco, fsub(p_right, pn)));
                vy = fsub(vy_c, fmul(bco, fsub(p_above, pn)));
                if ((vb1 >> jv) & 1) {
                    const float sc = sig[tc];
                    vx = fdiv_z(vx, fadd(1.0f, fmaxf(sc, sig[k_right & CODE_TYPE_MASK])));
                    vy = fdiv_z(vy, fadd(1.0f, fmaxf(sc, sig[k_above & CODE_TYPE_MASK])));
                }
            }
            if (lane_commit) {
                Vxout[o] = vx;
                Vyout[o] = vy;
                if (HIST) {
                    float* h = T->hist + (n + 1 - rs->run_start) * 3 * pl;
                    h[o] = pn;
                    h[pl + o] = vx;
                    h[2 * pl + o] = vy;
                }
            }
        }
        // ---- shift the row pipeline
        p_above = pn; k_above = k_c;
        vy_c = vy_n; uy_c = uy_n;
        vy_n = vy_2; uy_n = fmul(vy_2, dy_2);
        vx_c = vx_1; ux_c = fmul(vx_1, dx_1); p_c = p_1; dp_c = dp_1; k_c = k_1;
        o = o1;
    }
}

// ---------------------------------------------------------------------------
// Quad-strip kernel: the strip kernel's row pipeline with four consecutive
// columns per lane.  A warp covers the 128 columns c0 .. c0 + 127, lane i
// holding x0 = c0 + 4i .. x0 + 3; c0 is a multiple of 4, so each lane's
// share of a plane row is one aligned 16-byte piece.  Lane 0 only supplies
// the left depth flux of column c0 + 4 and lane 31 only the P' right of
// column c0 + 123; lanes 1..30 commit the 120 columns between.  Per row and
// lane: seven 16-byte reads, three shuffles and four cells.  Same arithmetic
// as the strip kernel, cell by cell; no wall oscillator and no history
// capture (those batches use the strip kernel).
//
// Row supply.  STAGES = 0: each row's loads are issued into registers one
// row ahead.  STAGES > 0: lane 0 streams the strip's rows into a per-warp
// ring of STAGES shared-memory stages with bulk copies (cp.async.bulk, one
// per plane row, completion on the stage's mbarrier), keeping up to STAGES
// rows in flight without holding registers; a stage is refilled as soon as
// the warp has read it.  Waits are bounded: a stage that does not arrive
// sets RunState::error, and the warp waits (bounded) for its remaining
// copies before it leaves.
// ---------------------------------------------------------------------------
// Streamed rows are read once per warp: they bypass L1 (no_allocate), which
// keeps the descriptor tables resident there.
template <int NC>
__device__ __forceinline__ void ldn(float (&d)[NC], const float* p) {
    if constexpr (NC == 4) {
        asm("ld.global.nc.L1::no_allocate.v4.f32 {%0, %1, %2, %3}, [%4];"
            : "=f"(d[0]), "=f"(d[1]), "=f"(d[2]), "=f"(d[3]) : "l"(p));
    } else {
        asm("ld.global.nc.L1::no_allocate.v2.f32 {%0, %1}, [%2];" : "=f"(d[0]), "=f"(d[1]) : "l"(p));
    }
}

__device__ __forceinline__ uint32_t ld_desc2(const uint8_t* p) {
    unsigned short v;
    asm("ld.global.nc.L1::no_allocate.u16 %0, [%1];" : "=h"(v) : "l"(p));
    return v;
}

__device__ __forceinline__ uint32_t ld_desc4(const uint8_t* p) {
    uint32_t v;
    asm("ld.global.nc.L1::no_allocate.u32 %0, [%1];" : "=r"(v) : "l"(p));
    return v;
}

__device__ __forceinline__ void ld4(float (&d)[4], const float* p) { ldn<4>(d, p); }

__device__ __forceinline__ void lds4(float (&d)[4], const unsigned char* p) {
    const float4 v = *reinterpret_cast<const float4*>(p);
    d[0] = v.x; d[1] = v.y; d[2] = v.z; d[3] = v.w;
}

// Store the masked columns of a lane's four; partial masks only occur at a
// frame's left and right edges, so interior warps issue the vector store only.
__device__ __forceinline__ void st4(float* p, const float (&v)[4], unsigned mask) {
    if (mask == 0xfu) {
        *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
    } else if (mask != 0u) {
#pragma unroll
        for (int q = 0; q < 4; ++q)
            if ((mask >> q) & 1u) p[q] = v[q];
    }
}

__device__ __forceinline__ int code_byte(uint32_t k, int q) { return (int)((k >> (8 * q)) & 0xffu); }

// Stage layout: Vx, dX, P, dP, Vy, dY row pieces (512 B each), then 144 code
// bytes from the 16-byte boundary at or below column c0.
constexpr uint32_t kQSeg = 512;
constexpr uint32_t kQCode = 144;
constexpr uint32_t kQStage = 6 * kQSeg + 160;
constexpr uint32_t kQBars = 128;                 // per-warp mbarrier area (up to 16 stages)

__host__ __device__ constexpr uint32_t quad_warp_smem(int stages) {
    return stages > 0 ? kQBars + (uint32_t)stages * kQStage : 0;
}

template <int TR, int WARPS, int MINB, int STAGES, bool FAST, bool HIST = false>
__global__ void __launch_bounds__(WARPS * 32, MINB)
quad_kernel(const TubeDev* __restrict__ tubes, const Tile* __restrict__ items, int nitems,
            RunState* __restrict__ rs, int local) {
    extern __shared__ __align__(128) unsigned char q_smem[];
    const int lane = threadIdx.x & 31;
    const int wi = blockIdx.x * WARPS + (threadIdx.x >> 5);
    if (wi >= nitems) return;
    const Tile it = items[wi];
    const TubeDev* __restrict__ T = tubes + it.tube;
    const int64_t n = rs->step + local;
    const int par = (int)(n & 1);
    const int H = T->H, W = T->W, pitch = T->pitch, flags = T->flags;
    const int r0 = it.r0, c0 = it.c0, x0 = c0 + 4 * lane;
    // columns of this lane that compute P' / commit
    unsigned calc_m = 0, commit_m = 0;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const bool c = lane >= 1 && x0 + q >= 1 && x0 + q <= W - 2;
        calc_m |= (unsigned)c << q;
        commit_m |= (unsigned)(c && lane <= 30) << q;
    }
    // planes P0 P1 Vx0 Vx1 Vy0 Vy1 and dP dX dY, `plane` apart.  Rows
    // r0-1 .. r0+TR of columns c0-12 .. c0+127 are read without predicates:
    // the arena keeps guard bytes around every tube, and values read outside
    // the frame only reach columns that neither compute nor commit them.
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
    // reference arithmetic: cell codes; fast_math: per-cell descriptors
    const uint8_t* __restrict__ code = FAST ? T->desc : T->code;
    const float* __restrict__ sig = T->sigma;
    const float K1 = T->K1, bco = T->bcoef;
    const bool eigen = flags & TUBE_EIGEN, dirichlet = flags & TUBE_DIRICHLET;
    const int lis_y = T->lis_y, lis_q = T->lis_x - x0;
    const uint64_t pmask = it.p_rows, vb1 = it.v_beta1, vgen = it.v_generic;
    const int rlast = min(r0 + TR - 1, H - 2);

    // ---- row supply
    constexpr int kS = STAGES > 0 ? STAGES : 1;
    uint64_t* bars = nullptr;
    unsigned char* stages = nullptr;
    const int nrows = rlast - r0 + 3;                 // rows r0-1 .. rlast+1
    const int cshift = c0 & 15;                        // code bytes ahead of column c0 in a stage
    if constexpr (STAGES > 0) {
        unsigned char* wbase = q_smem + (threadIdx.x >> 5) * quad_warp_smem(STAGES);
        bars = reinterpret_cast<uint64_t*>(wbase);
        stages = wbase + kQBars;
        if (lane == 0) {
            for (int s2 = 0; s2 < STAGES; ++s2) mbar_init(bars + s2, 1);
            mbar_fence_init();
        }
        __syncwarp();
    }
    auto issue = [&](int i) {                           // lane 0: stage row r0 - 1 + i
        const int s2 = i % kS;
        uint64_t* bar = bars + s2;
        unsigned char* st = stages + s2 * kQStage;
        const int64_t off = (int64_t)(r0 - 1 + i) * pitch + c0;
        mbar_expect_tx(bar, 6 * kQSeg + kQCode);
        bulk_g2s(st + 0 * kQSeg, Vxin + off, kQSeg, bar);
        bulk_g2s(st + 1 * kQSeg, dXp + off, kQSeg, bar);
        bulk_g2s(st + 2 * kQSeg, Pin + off, kQSeg, bar);
        bulk_g2s(st + 3 * kQSeg, dPp + off, kQSeg, bar);
        bulk_g2s(st + 4 * kQSeg, Vyin + off, kQSeg, bar);
        bulk_g2s(st + 5 * kQSeg, dYp + off, kQSeg, bar);
        bulk_g2s(st + 6 * kQSeg, code + (off & ~(int64_t)15), kQCode, bar);
    };
    auto wait_row = [&](int i) -> bool {
        const bool ok = mbar_wait_parity_bounded(bars + i % kS, (uint32_t)(i / kS) & 1u, first_wait_limit(rs));
        return __all_sync(kFull, ok);
    };
    auto drain = [&](int from, int issued) {            // after a timeout: bounded wait for copies in flight
        if (lane == 0) {
            atomicExch(&rs->error, VS_ERR_TIMEOUT);
            for (int i = from; i < issued; ++i)
                mbar_wait_parity_bounded(bars + i % kS, (uint32_t)(i / kS) & 1u, kWaitPolls);
        }
        __syncwarp();
    };
    int issued = 0;
    if constexpr (STAGES > 0) {
        if (lane == 0)
            for (int i = 0; i < STAGES && i < nrows; ++i) issue(i);
        issued = min(STAGES, nrows);
    }

    float exeV = 0.0f;
    if (it.has_exc) {
        if (flags & TUBE_TMM) {
            if (lane == 0) {
                const int ex = T->exc_x - c0;
                const bool owner =
                    T->exc_y >= r0 && T->exc_y < r0 + TR && ex >= kQuadLead && ex < kQuadLead + kQuadCommit;
                exeV = glottal_step(T, par, Pin[(size_t)T->exc_y * pitch + T->exc_x], owner,
                                    HIST ? T->tmm_hist + 6 * (n + 1 - rs->run_start) : nullptr);
            }
            exeV = __shfl_sync(kFull, exeV, 0);
        } else {
            exeV = n < T->src_len ? T->src[n] : 0.0f;
        }
    }

    int r = r0 - 1;
    int o = r * pitch + x0;
    float vx_c[4], ux_c[4], p_c[4], dp_c[4], vy_c[4], uy_c[4], vy_n[4], uy_n[4], p_above[4], t4[4];
    uint32_t k_c;
    if constexpr (STAGES > 0) {
        if (!wait_row(0)) { drain(0, issued); return; }
        const unsigned char* st = stages;
        lds4(vy_c, st + 4 * kQSeg + 16 * lane);
        lds4(t4, st + 5 * kQSeg + 16 * lane);
    } else {
        ld4(vx_c, Vxin + o);
        ld4(t4, dXp + o);
#pragma unroll
        for (int q = 0; q < 4; ++q) ux_c[q] = fmul(vx_c[q], t4[q]);
        ld4(p_c, Pin + o);
        ld4(dp_c, dPp + o);
        k_c = ld_desc4(code + o);
        ld4(vy_c, Vyin + o);
        ld4(t4, dYp + o);
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        uy_c[q] = fmul(vy_c[q], t4[q]);
        p_above[q] = 0.0f;
    }
    if constexpr (STAGES == 0) {
        ld4(vy_n, Vyin + o + pitch);
        ld4(t4, dYp + o + pitch);
#pragma unroll
        for (int q = 0; q < 4; ++q) uy_n[q] = fmul(vy_n[q], t4[q]);
    }
    uint32_t k_above = 0;

    for (int j = 0; r <= rlast; ++j, ++r) {
        const int o1 = o + pitch;
        float vx_1[4], dx_1[4], p_1[4], dp_1[4], vy_2[4], dy_2[4];
        uint32_t k_1 = 0;
        if constexpr (STAGES > 0) {
            // row r from stage j (waited last iteration), Vy dY of row r+1 from stage j+1
            if (!wait_row(j + 1)) { drain(j + 1, issued); return; }
            const unsigned char* st = stages + (j % kS) * kQStage;
            const unsigned char* sn = stages + ((j + 1) % kS) * kQStage;
            lds4(vx_c, st + 0 * kQSeg + 16 * lane);
            lds4(t4, st + 1 * kQSeg + 16 * lane);
#pragma unroll
            for (int q = 0; q < 4; ++q) ux_c[q] = fmul(vx_c[q], t4[q]);
            lds4(p_c, st + 2 * kQSeg + 16 * lane);
            lds4(dp_c, st + 3 * kQSeg + 16 * lane);
            k_c = *reinterpret_cast<const uint32_t*>(st + 6 * kQSeg + cshift + 4 * lane);
            lds4(vy_n, sn + 4 * kQSeg + 16 * lane);
            lds4(t4, sn + 5 * kQSeg + 16 * lane);
#pragma unroll
            for (int q = 0; q < 4; ++q) uy_n[q] = fmul(vy_n[q], t4[q]);
            __syncwarp();
            if (lane == 0 && issued < nrows) {
                // the warp has read stage j: refill it
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                issue(issued);
            }
            issued = min(issued + 1, nrows);
        } else {
            // loads for the next iterations (input planes are read-only this step)
            ld4(vx_1, Vxin + o1);
            ld4(dx_1, dXp + o1);
            ld4(p_1, Pin + o1);
            ld4(dp_1, dPp + o1);
            k_1 = ld_desc4(code + o1);
            if (r + 2 <= H - 1) {
                ld4(vy_2, Vyin + o1 + pitch);
                ld4(dy_2, dYp + o1 + pitch);
            } else {
#pragma unroll
                for (int q = 0; q < 4; ++q) { vy_2[q] = 0.0f; dy_2[q] = 0.0f; }
            }
        }

        // ---- pressure of row r (FDTDEngineCPU.cpp:316-339)
        const float ux_l = __shfl_up_sync(kFull, ux_c[3], 1);
        const bool pgen = (pmask >> j) & 1;
        const unsigned cm = r >= 1 ? calc_m : 0u;
        float pn[4];
        // fast_math: rows with any non-air cell read the descriptors' coefficients
        const bool rowd = FAST && (pgen || (j >= 1 && (((vb1 | vgen) >> (j - 1)) & 1)));
        float4 da[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const float uxl = q == 0 ? ux_l : ux_c[q - 1];
            const int tc = code_byte(k_c, q) & CODE_TYPE_MASK;
            if constexpr (FAST) {
                // (P dP - K1 S) / ((1 + s) dP) = (P - K1 S / dP) g,  g = 1 / (1 + s)
                // (0 on the no-pressure cells of a Dirichlet mouth)
                const float ks = fmul(K1, fadd(fsub(ux_c[q], uxl), fsub(uy_c[q], uy_n[q])));
                float v = __fmaf_rn(-ks, rcp_approx(dp_c[q]), p_c[q]);
                if (rowd) {
                    da[q] = __ldg(T->desc_a + code_byte(k_c, q));
                    v = fmul(v, da[q].z);
                }
                pn[q] = ((cm >> q) & 1u) ? v : 0.0f;
            } else {
                const float num =
                    fsub(fmul(p_c[q], dp_c[q]), fmul(K1, fadd(fsub(ux_c[q], uxl), fsub(uy_c[q], uy_n[q]))));
                float den = dp_c[q];
                if (pgen && tc != VS_CELL_AIR) {
                    const float s = sig[tc];
                    den = eigen ? fadd(fmul(s, dp_c[q]), dp_c[q]) : fmul(fadd(1.0f, s), dp_c[q]);
                }
                pn[q] = 0.0f;
                if ((cm >> q) & 1u) {
                    pn[q] = fdiv_z(num, den);
                    if (pgen && dirichlet && tc == VS_CELL_NOPRESSURE) pn[q] = 0.0f;
                }
            }
        }
        // ---- commit row r and its velocity (FDTDEngineCPU.cpp:364-410)
        const float p_r3 = __shfl_down_sync(kFull, pn[0], 1);
        const int k_r3 = code_byte(__shfl_down_sync(kFull, k_c, 1), 0);
        if (j >= 1) {
            const int jv = j - 1;
            st4(Pout + o, pn, commit_m);
            if (r == lis_y && lis_q >= 0 && lis_q < 4 && ((commit_m >> lis_q) & 1u)) {
                float pv = pn[0];
#pragma unroll
                for (int q = 1; q < 4; ++q) if (lis_q == q) pv = pn[q];
                store_trace(rs, rs->trace + (int64_t)it.tube * rs->trace_stride + (n - rs->run_start), pv);
            }
            float vx[4], vy[4];
            if constexpr (FAST) {
                // V' = al (V - bco (P'n - P'c)) + zo P'c - zi P'n + ce exeV
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const float pr = q < 3 ? pn[q + 1] : p_r3;
                    vx[q] = fsub(vx_c[q], fmul(bco, fsub(pr, pn[q])));
                    vy[q] = fsub(vy_c[q], fmul(bco, fsub(p_above[q], pn[q])));
                    if (rowd) {
                        vx[q] = fmul(vx[q], da[q].x);
                        vy[q] = fmul(vy[q], da[q].y);
                    }
                }
                if ((vgen >> jv) & 1) {
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const float pr = q < 3 ? pn[q + 1] : p_r3;
                        const float4 db = __ldg(T->desc_b + code_byte(k_c, q));
                        vx[q] = __fmaf_rn(da[q].w, exeV, __fmaf_rn(-db.y, pr, __fmaf_rn(db.x, pn[q], vx[q])));
                        vy[q] = __fmaf_rn(-db.w, p_above[q], __fmaf_rn(db.z, pn[q], vy[q]));
                    }
                }
            } else if ((vgen >> jv) & 1) {
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    vx[q] = 0.0f;
                    vy[q] = 0.0f;
                    if ((commit_m >> q) & 1u) {
                        const int kr = q < 3 ? code_byte(k_c, q + 1) : k_r3;
                        const float pr = q < 3 ? pn[q + 1] : p_r3;
                        const VelocityOut v =
                            velocity_generic(code_byte(k_c, q), kr, code_byte(k_above, q), pn[q], pr, p_above[q],
                                             vx_c[q], vy_c[q], exeV, sig, T->zinv, bco, T->dir0, T->dir1, T->dir2,
                                             T->dir3);
                        vx[q] = v.vx;
                        vy[q] = v.vy;
                    }
                }
            } else {
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const float pr = q < 3 ? pn[q + 1] : p_r3;
                    vx[q] = fsub(vx_c[q], fmul(bco, fsub(pr, pn[q])));
                    vy[q] = fsub(vy_c[q], fmul(bco, fsub(p_above[q], pn[q])));
                }
                if ((vb1 >> jv) & 1) {
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const int kr = q < 3 ? code_byte(k_c, q + 1) : k_r3;
                        const float sc = sig[code_byte(k_c, q) & CODE_TYPE_MASK];
                        vx[q] = fdiv_z(vx[q], fadd(1.0f, fmaxf(sc, sig[kr & CODE_TYPE_MASK])));
                        vy[q] = fdiv_z(vy[q], fadd(1.0f, fmaxf(sc, sig[code_byte(k_above, q) & CODE_TYPE_MASK])));
                    }
                }
            }
            st4(Vxout + o, vx, commit_m);
            st4(Vyout + o, vy, commit_m);
            if constexpr (HIST) {
                // the state after step n, for the adjoint's segment recomputation
                float* h = T->hist + (n + 1 - rs->run_start) * 3 * pl;
                st4(h + o, pn, commit_m);
                st4(h + pl + o, vx, commit_m);
                st4(h + 2 * pl + o, vy, commit_m);
            }
        }
        // ---- shift the row pipeline
        k_above = k_c;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            p_above[q] = pn[q];
            vy_c[q] = vy_n[q];
            uy_c[q] = uy_n[q];
        }
        if constexpr (STAGES == 0) {
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                vy_n[q] = vy_2[q];
                uy_n[q] = fmul(vy_2[q], dy_2[q]);
                vx_c[q] = vx_1[q];
                ux_c[q] = fmul(vx_1[q], dx_1[q]);
                p_c[q] = p_1[q];
                dp_c[q] = dp_1[q];
            }
            k_c = k_1;
        }
        o = o1;
    }
}

// ---------------------------------------------------------------------------
// Two-step quad-strip kernel (no coupled wall; fast_math, and with EXACT the
// reference arithmetic): every strip advances TWO time steps per launch.  A
// lane holds NC adjacent
// columns (NC = 4 or 2), a warp 32 NC columns, of which lanes 1..30 commit.
// Step n runs the quad-strip row pipeline over rows r0-2 .. rlast+1 and all
// columns of the warp; step n+1 follows one row behind on the values step n
// just produced in registers, and only step n+1 is stored.  The halo this
// needs -- two columns on each side (lanes 0 and 31) and two rows above /
// one below -- is recomputed by the neighbouring strips, so the state of
// step n+1 is never written or read back: per two steps the planes are read
// and written once.  The step n+2 state goes to the other of two buffer sets
// (the parity set of step n and a third set TubeDev::X, alternating per
// launch); per cell and step the arithmetic is that of the quad-strip kernel
// in the reciprocal form, or with EXACT that of the strip kernel (the IEEE
// divides, the neighbourhood's factors from the descriptor tables, on the
// rows the tile's p_rows / v_beta1 masks mark), so the values are those of
// two single steps.
// Tile masks classify the extended region (rows from r0-2 / r0-1, columns
// c0 + NC/2 .. c0 + 32 NC - NC/2 - 1): bit j of v_generic = row r0-1+j.
// HIST: the adjoint's segment recomputation; the committed cells' state
// after step n and after step n+1 also go to the history slots n+1 and n+2
// (and the two-mass states to the two-mass history).
// ---------------------------------------------------------------------------


template <int NC>
__device__ __forceinline__ void stn(float* p, const float (&v)[NC], unsigned mask) {
    if constexpr (NC == 4) {
        st4(p, v, mask);
    } else if (mask == 0x3u) {
        *reinterpret_cast<float2*>(p) = make_float2(v[0], v[1]);
    } else if (mask != 0u) {
        if (mask & 1u) p[0] = v[0];
        if (mask & 2u) p[1] = v[1];
    }
}

template <int TR, int WARPS, int MINB, int NC, bool HIST = false, bool EXACT = false>
__global__ void __launch_bounds__(WARPS * 32, MINB)
quad2_kernel(const TubeDev* __restrict__ tubes, const Tile* __restrict__ items, int nitems,
             RunState* __restrict__ rs, int local) {
    const int lane = threadIdx.x & 31;
    const int wi = blockIdx.x * WARPS + (threadIdx.x >> 5);
    if (wi >= nitems) return;
    const Tile it = items[wi];
    const TubeDev* __restrict__ T = tubes + it.tube;
    // each warp copies the descriptors its tube uses (desc_a, then desc_b at
    // kDescEntries) into its own shared-memory slot, where the rows' lookups
    // go; up to 4 warps per CTA (32 KB), wider CTAs read through L1
    constexpr bool kSmemTab = WARPS <= 4;
    __shared__ float4 s_tab[kSmemTab ? WARPS : 1][kSmemTab ? 2 * kDescEntries : 1];
    float4* wtab = s_tab[kSmemTab ? (threadIdx.x >> 5) : 0];
    if constexpr (kSmemTab) {
        const float4* __restrict__ src = T->desc_a;
        for (int j = lane; j < T->ndesc; j += 32) {
            wtab[j] = __ldg(src + j);
            wtab[kDescEntries + j] = __ldg(src + kDescEntries + j);
        }
        __syncwarp();
    }
    auto tab = [&](int i) -> float4 {
        if constexpr (kSmemTab) return wtab[i];
        else return __ldg(T->desc_a + i);
    };
    const int64_t n = rs->step + 2 * (int64_t)local;
    const int par = (int)(n & 1);
    const bool from_x = ((rs->bsel ^ local) & 1) != 0;
    const int H = T->H, W = T->W, pitch = T->pitch;
    const int r0 = it.r0, c0 = it.c0, x0 = c0 + NC * lane;
    unsigned int_m = 0, commit_m = 0;
#pragma unroll
    for (int q = 0; q < NC; ++q) {
        const bool in = x0 + q >= 1 && x0 + q <= W - 2;
        int_m |= (unsigned)in << q;
        commit_m |= (unsigned)(in && lane >= 1 && lane <= 30) << q;
    }
    const int64_t pl = T->plane;
    float* __restrict__ Bp = T->P[0] + par * pl;          // P, Vx, Vy of step n's parity: +0, +2pl, +4pl
    float* __restrict__ Xp = T->X;                        // third set: +0, +pl, +2pl
    const float* __restrict__ Pin = from_x ? Xp : Bp;
    const float* __restrict__ Vxin = from_x ? Xp + pl : Bp + 2 * pl;
    const float* __restrict__ Vyin = from_x ? Xp + 2 * pl : Bp + 4 * pl;
    float* __restrict__ Pout = from_x ? Bp : Xp;
    float* __restrict__ Vxout = from_x ? Bp + 2 * pl : Xp + pl;
    float* __restrict__ Vyout = from_x ? Bp + 4 * pl : Xp + 2 * pl;
    const float* __restrict__ dPp = T->dP;
    const float* __restrict__ dXp = dPp + pl;
    const float* __restrict__ dYp = dPp + 2 * pl;
    const uint8_t* __restrict__ desc = T->desc;
    const float4* __restrict__ ta = T->desc_a;
    // desc_b follows desc_a (kDescEntries entries each): one base, immediate offsets
    const float K1 = T->K1, bco = T->bcoef;
    const bool eigen = (T->flags & TUBE_EIGEN) != 0;
    const float zval = T->zinv;
    const int lis_y = T->lis_y, lis_q = T->lis_x - x0;
    const bool lis_here = lis_q >= 0 && lis_q < NC && ((commit_m >> lis_q) & 1u);
    // bit 1 of gm = velocity class of step n's row r (v_generic bit j-1; in
    // the reference arithmetic v_beta1, every row with a velocity division),
    // bit 0 = that of step n+1's row r-1 (bit j-2); bit 1 of pm = step n's
    // row r holds a cell other than air (p_rows bit j), bit 0 = step n+1's
    // row r-1; both shifted once per row
    uint64_t gm = (EXACT ? it.v_beta1 : it.v_generic) << 2;
    uint64_t pm = it.p_rows << 1;
    float exe1 = 0.0f, exe2 = 0.0f;
    const int rlast = min(r0 + TR - 1, H - 2);
    if (it.has_exc) {
        if (T->flags & TUBE_TMM) {
            // two-mass source: exe of step n from P(n) at the glottis cell, that
            // of step n+1 from P'(n) there, evaluated from the input planes
            // with the strip's own arithmetic; the strip that commits the
            // cell stores the state of step n+2 in the other slot
            if (lane == 0) {
                const int64_t e = (int64_t)T->exc_y * pitch + T->exc_x;
                const float p1 = Pin[e];
                const float ks = fmul(K1, fadd(fsub(fmul(Vxin[e], dXp[e]), fmul(Vxin[e - 1], dXp[e - 1])),
                                               fsub(fmul(Vyin[e], dYp[e]), fmul(Vyin[e + pitch], dYp[e + pitch]))));
                float p2;
                if constexpr (EXACT)
                    p2 = fdiv_z(fsub(fmul(p1, dPp[e]), ks), pressure_den(__ldg(ta + desc[e]).x, dPp[e], eigen));
                else
                    p2 = fmul(__fmaf_rn(-ks, rcp_approx(dPp[e]), p1), __ldg(ta + desc[e]).z);
                const bool owner = T->exc_y >= r0 && T->exc_y <= rlast && T->exc_x >= c0 + NC &&
                                   T->exc_x < c0 + 31 * NC;
                const float2 ee = glottal_two_steps(T, par, from_x, p1, p2, owner,
                                                    HIST ? T->tmm_hist + 6 * (n + 1 - rs->run_start) : nullptr);
                exe1 = ee.x;
                exe2 = ee.y;
            }
            exe1 = __shfl_sync(kFull, exe1, 0);
            exe2 = __shfl_sync(kFull, exe2, 0);
        } else {
            exe1 = n < T->src_len ? T->src[n] : 0.0f;
            exe2 = n + 1 < T->src_len ? T->src[n + 1] : 0.0f;
        }
    }
    float* __restrict__ trace = rs->trace + (int64_t)it.tube * rs->trace_stride + (n - rs->run_start);
    float* __restrict__ hist1 = HIST ? T->hist + (n + 1 - rs->run_start) * 3 * pl : nullptr;   // after step n

    // rows outside the frame read as zeros (they only feed values that are not used)
    auto ldr = [&](float (&d)[NC], const float* base, int row) {
        if (row >= 0 && row <= H - 1) {
            ldn<NC>(d, base + (int64_t)row * pitch + x0);
        } else {
#pragma unroll
            for (int q = 0; q < NC; ++q) d[q] = 0.0f;
        }
    };
    auto ldk = [&](int row) -> uint32_t {
        if (row < 0 || row > H - 1) return 0u;
        const uint8_t* p = desc + (int64_t)row * pitch + x0;
        if constexpr (NC == 4) return ld_desc4(p);
        else return ld_desc2(p);
    };

    // step-n pipeline at row r: state and maps of row r, Vy dY of row r+1
    int r = r0 - 2;
    float vx_c[NC], dx_c[NC], p_c[NC], dp_c[NC], vy_c[NC], dy_c[NC], vy_n[NC], dy_n[NC];
    ldr(vx_c, Vxin, r);
    ldr(dx_c, dXp, r);
    ldr(p_c, Pin, r);
    ldr(dp_c, dPp, r);
    uint32_t k_c = ldk(r);
    ldr(vy_c, Vyin, r);
    ldr(dy_c, dYp, r);
    ldr(vy_n, Vyin, r + 1);
    ldr(dy_n, dYp, r + 1);
    // step-n results of the previous row (r-1) for step n+1, and P'' of the row above it
    float pn1_p[NC], v1x_p[NC], v1y_p[NC], u1_p[NC], w1_p[NC], dp_p[NC], pn2_p[NC];
    uint32_t k_p = 0;
#pragma unroll
    for (int q = 0; q < NC; ++q) {
        pn1_p[q] = 0.0f; v1x_p[q] = 0.0f; v1y_p[q] = 0.0f; u1_p[q] = 0.0f; w1_p[q] = 0.0f;
        dp_p[q] = 1.0f; pn2_p[q] = 0.0f;
    }

    for (int j = 0; r <= rlast + 1; ++j, ++r) {
        // ---- loads for the next row (read-only this launch)
        float vx_1[NC], dx_1[NC], p_1[NC], dp_1[NC], vy_2[NC], dy_2[NC];
        ldr(vx_1, Vxin, r + 1);
        ldr(dx_1, dXp, r + 1);
        ldr(p_1, Pin, r + 1);
        ldr(dp_1, dPp, r + 1);
        const uint32_t k_1 = ldk(r + 1);
        ldr(vy_2, Vyin, r + 2);
        ldr(dy_2, dYp, r + 2);

        // ---- step n, pressure of row r (FDTDEngineCPU.cpp:316-339, reciprocal form)
        const bool prow1 = r >= 1 && r <= H - 2;
        const unsigned cm1 = prow1 ? int_m : 0u;
        float ux_c[NC];
#pragma unroll
        for (int q = 0; q < NC; ++q) ux_c[q] = fmul(vx_c[q], dx_c[q]);
        const float ux_l = __shfl_up_sync(kFull, ux_c[NC - 1], 1);
        float4 da[NC];
        float pn1[NC];
        const bool pg1 = (pm & 2u) != 0;
#pragma unroll
        for (int q = 0; q < NC; ++q) {
            const float uxl = q == 0 ? ux_l : ux_c[q - 1];
            const float ks = fmul(K1, fadd(fsub(ux_c[q], uxl), fsub(fmul(vy_c[q], dy_c[q]), fmul(vy_n[q], dy_n[q]))));
            float v;
            if constexpr (EXACT) {
                // (P dP - K1 S) / ((1 + sigma) dP), the denominator dP on rows of air
                float den = dp_c[q];
                bool pz = false;
                if (pg1) {
                    const float4 a = tab(code_byte(k_c, q));
                    den = pressure_den(a.x, dp_c[q], eigen);
                    pz = (__float_as_uint(a.w) & EXD_PZERO) != 0u;
                }
                v = fdiv_z(fsub(fmul(p_c[q], dp_c[q]), ks), den);
                if (pz) v = 0.0f;
            } else {
                da[q] = tab(code_byte(k_c, q));
                v = fmul(__fmaf_rn(-ks, rcp_approx(dp_c[q]), p_c[q]), da[q].z);
            }
            pn1[q] = ((cm1 >> q) & 1u) ? v : 0.0f;
        }
        const float p_r = __shfl_down_sync(kFull, pn1[0], 1);
        // ---- step n, velocity of row r (FDTDEngineCPU.cpp:364-410)
        const bool vrow1 = r >= r0 - 1 && prow1;
        const unsigned vm1 = vrow1 ? int_m : 0u;
        const bool gen1 = (gm & 2u) != 0;
        float v1x[NC], v1y[NC], u1[NC], w1[NC];
#pragma unroll
        for (int q = 0; q < NC; ++q) {
            const float pr = q < NC - 1 ? pn1[q + 1] : p_r;
            float vx, vy;
            if constexpr (EXACT) {
                if (gen1) {
                    const int d = code_byte(k_c, q);
                    const float4 a = tab(d), bt = tab(kDescEntries + d);
                    const unsigned bits = __float_as_uint(a.w);
                    vx = velocity_tab(bits, a.y, bt.x, bt.y, vx_c[q], pn1[q], pr, exe1, zval, bco);
                    vy = velocity_tab(bits >> EXD_Y_SHIFT, a.z, bt.z, bt.w, vy_c[q], pn1[q], pn1_p[q], exe1, zval,
                                      bco);
                } else {
                    vx = fsub(vx_c[q], fmul(bco, fsub(pr, pn1[q])));
                    vy = fsub(vy_c[q], fmul(bco, fsub(pn1_p[q], pn1[q])));
                }
            } else {
                vx = fmul(fsub(vx_c[q], fmul(bco, fsub(pr, pn1[q]))), da[q].x);
                vy = fmul(fsub(vy_c[q], fmul(bco, fsub(pn1_p[q], pn1[q]))), da[q].y);
                if (gen1) {
                    const float4 db = tab(kDescEntries + code_byte(k_c, q));
                    vx = __fmaf_rn(da[q].w, exe1, __fmaf_rn(-db.y, pr, __fmaf_rn(db.x, pn1[q], vx)));
                    vy = __fmaf_rn(-db.w, pn1_p[q], __fmaf_rn(db.z, pn1[q], vy));
                }
            }
            v1x[q] = ((vm1 >> q) & 1u) ? vx : 0.0f;
            v1y[q] = ((vm1 >> q) & 1u) ? vy : 0.0f;
            u1[q] = fmul(v1x[q], dx_c[q]);
            w1[q] = fmul(v1y[q], dy_c[q]);
        }
        if (HIST && r >= r0 && r <= rlast) {
            const int64_t o = (int64_t)r * pitch + x0;
            stn<NC>(hist1 + o, pn1, commit_m);
            stn<NC>(hist1 + pl + o, v1x, commit_m);
            stn<NC>(hist1 + 2 * pl + o, v1y, commit_m);
        }
        if (r == lis_y && r >= r0 && r <= rlast && lis_here) {
            float pv = pn1[0];
#pragma unroll
            for (int q = 1; q < NC; ++q) if (lis_q == q) pv = pn1[q];
            store_trace(rs, trace, pv);
        }

        // ---- step n+1 at row s = r - 1
        const int s = r - 1;
        if (s >= r0 - 1) {
            const bool prow2 = s >= 1 && s <= H - 2;
            const unsigned cm2 = prow2 ? int_m : 0u;
            const float ul = __shfl_up_sync(kFull, u1_p[NC - 1], 1);
            float pn2[NC];
            float4 da_p[NC];
            const bool pg2 = (pm & 1u) != 0;
#pragma unroll
            for (int q = 0; q < NC; ++q) {
                const float uxl = q == 0 ? ul : u1_p[q - 1];
                const float ks = fmul(K1, fadd(fsub(u1_p[q], uxl), fsub(w1_p[q], w1[q])));
                float v;
                if constexpr (EXACT) {
                    float den = dp_p[q];
                    bool pz = false;
                    if (pg2) {
                        const float4 a = tab(code_byte(k_p, q));
                        den = pressure_den(a.x, dp_p[q], eigen);
                        pz = (__float_as_uint(a.w) & EXD_PZERO) != 0u;
                    }
                    v = fdiv_z(fsub(fmul(pn1_p[q], dp_p[q]), ks), den);
                    if (pz) v = 0.0f;
                } else {
                    da_p[q] = tab(code_byte(k_p, q));
                    v = fmul(__fmaf_rn(-ks, rcp_approx(dp_p[q]), pn1_p[q]), da_p[q].z);
                }
                pn2[q] = ((cm2 >> q) & 1u) ? v : 0.0f;
            }
            const float p2_r = __shfl_down_sync(kFull, pn2[0], 1);
            if (s >= r0 && s <= rlast) {
                const bool gen2 = (gm & 1u) != 0;
                float vx2[NC], vy2[NC];
#pragma unroll
                for (int q = 0; q < NC; ++q) {
                    const float pr = q < NC - 1 ? pn2[q + 1] : p2_r;
                    float vx, vy;
                    if constexpr (EXACT) {
                        if (gen2) {
                            const int d = code_byte(k_p, q);
                            const float4 a = tab(d), bt = tab(kDescEntries + d);
                            const unsigned bits = __float_as_uint(a.w);
                            vx = velocity_tab(bits, a.y, bt.x, bt.y, v1x_p[q], pn2[q], pr, exe2, zval, bco);
                            vy = velocity_tab(bits >> EXD_Y_SHIFT, a.z, bt.z, bt.w, v1y_p[q], pn2[q], pn2_p[q], exe2,
                                              zval, bco);
                        } else {
                            vx = fsub(v1x_p[q], fmul(bco, fsub(pr, pn2[q])));
                            vy = fsub(v1y_p[q], fmul(bco, fsub(pn2_p[q], pn2[q])));
                        }
                    } else {
                        vx = fmul(fsub(v1x_p[q], fmul(bco, fsub(pr, pn2[q]))), da_p[q].x);
                        vy = fmul(fsub(v1y_p[q], fmul(bco, fsub(pn2_p[q], pn2[q]))), da_p[q].y);
                        if (gen2) {
                            const float4 db = tab(kDescEntries + code_byte(k_p, q));
                            vx = __fmaf_rn(da_p[q].w, exe2, __fmaf_rn(-db.y, pr, __fmaf_rn(db.x, pn2[q], vx)));
                            vy = __fmaf_rn(-db.w, pn2_p[q], __fmaf_rn(db.z, pn2[q], vy));
                        }
                    }
                    vx2[q] = vx;
                    vy2[q] = vy;
                }
                const int64_t o = (int64_t)s * pitch + x0;
                stn<NC>(Pout + o, pn2, commit_m);
                stn<NC>(Vxout + o, vx2, commit_m);
                stn<NC>(Vyout + o, vy2, commit_m);
                if (HIST) {
                    float* hist2 = hist1 + 3 * pl;                // after step n+1
                    stn<NC>(hist2 + o, pn2, commit_m);
                    stn<NC>(hist2 + pl + o, vx2, commit_m);
                    stn<NC>(hist2 + 2 * pl + o, vy2, commit_m);
                }
                if (s == lis_y && lis_here) {
                    float pv = pn2[0];
#pragma unroll
                    for (int q = 1; q < NC; ++q) if (lis_q == q) pv = pn2[q];
                    store_trace(rs, trace + 1, pv);
                }
            }
#pragma unroll
            for (int q = 0; q < NC; ++q) pn2_p[q] = pn2[q];
        }

        // ---- shift the row pipelines
#pragma unroll
        for (int q = 0; q < NC; ++q) {
            pn1_p[q] = pn1[q];
            v1x_p[q] = v1x[q];
            v1y_p[q] = v1y[q];
            u1_p[q] = u1[q];
            w1_p[q] = w1[q];
            dp_p[q] = dp_c[q];
            vx_c[q] = vx_1[q];
            dx_c[q] = dx_1[q];
            p_c[q] = p_1[q];
            dp_c[q] = dp_1[q];
            vy_c[q] = vy_n[q];
            dy_c[q] = dy_n[q];
            vy_n[q] = vy_2[q];
            dy_n[q] = dy_2[q];
        }
        k_p = k_c;
        k_c = k_1;
        gm >>= 1;
        pm >>= 1;
    }
}

// After an odd number of two-step launches the state sits in TubeDev::X:
// copy it back to the parity set of the current step.
__global__ void copy_back_kernel(const TubeDev* __restrict__ tubes, const RunState* __restrict__ rs) {
    const TubeDev& T = tubes[blockIdx.y];
    const int64_t n = (int64_t)T.H * T.pitch;
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int par = (int)(rs->step & 1);
    const int64_t pl = T.plane;
    float* B = T.P[0] + par * pl;
    B[i] = T.X[i];
    B[2 * pl + i] = T.X[pl + i];
    B[4 * pl + i] = T.X[2 * pl + i];
    if (i == 0 && (T.flags & TUBE_TMM)) {
        T.tmm[par] = *T.tmm_x;
        T.tmm64[par] = *T.tmm64_x;
    }
}

__global__ void advance2_kernel(RunState* rs, int k, int toggle) {
    rs->step += k;
    rs->bsel ^= toggle;
}

// ---------------------------------------------------------------------------
// Band kernel: one CTA per band of R rows of a tube.  A band's rows are
// contiguous in every plane (rows are `pitch` apart), so the rows r0-1 ..
// r0+R of P, Vx, Vy, dP, dX, dY and the codes arrive with one bulk copy per
// plane (cp.async.bulk, completion on an mbarrier) and no registers held in
// flight.  The CTA then computes P' for rows r0-1 .. r0+R-1 into shared
// memory and V' for rows r0 .. r0+R-1, with the same arithmetic as the
// strip kernel (value-identical to the reference expressions), and stores
// both to global memory.
// ---------------------------------------------------------------------------
constexpr int kBandThreads = 256;

// Shared-memory bytes of a band kernel with R rows for a row pitch.
__host__ __device__ inline size_t band_smem_bytes(int R, int pitch) {
    const size_t plane = (size_t)(R + 2) * pitch * sizeof(float);
    const size_t codes = ((size_t)(R + 2) * pitch + 127) / 128 * 128;
    return 6 * plane + codes + (size_t)(R + 1) * pitch * sizeof(float);
}

template <int R, bool WALL>
__global__ void __launch_bounds__(kBandThreads)
band_kernel(const TubeDev* __restrict__ tubes, const Tile* __restrict__ bands, int nbands,
            RunState* __restrict__ rs, int local) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ uint64_t bar;
    __shared__ float s_exe;
    if ((int)blockIdx.x >= nbands) return;
    const Tile bd = bands[blockIdx.x];
    const TubeDev* __restrict__ T = tubes + bd.tube;
    const int64_t n = rs->step + local;
    const int par = (int)(n & 1);
    const int H = T->H, W = T->W, pitch = T->pitch, flags = T->flags;
    const int r0 = bd.r0;
    const int rfirst = r0 - 1;                          // first row held in shared memory
    const int rload = min(r0 + R, H - 1);               // last row held
    const int nload = rload - rfirst + 1;
    const int rcommit = min(r0 + R - 1, H - 2);         // last row this band commits
    const int64_t pl = T->plane;
    const float* __restrict__ Pin = T->P[0] + par * pl;
    float* __restrict__ Pout = T->P[0] + (par ^ 1) * pl;
    const float* __restrict__ Vxin = Pin + 2 * pl;
    const float* __restrict__ Vyin = Pin + 4 * pl;
    float* __restrict__ Vxout = Pout + 2 * pl;
    float* __restrict__ Vyout = Pout + 4 * pl;
    const float* __restrict__ dPp = T->dP;
    const size_t plane_sm = (size_t)(R + 2) * pitch;
    float* sP = reinterpret_cast<float*>(smem);
    float* sVx = sP + plane_sm;
    float* sVy = sVx + plane_sm;
    float* sdP = sVy + plane_sm;
    float* sdX = sdP + plane_sm;
    float* sdY = sdX + plane_sm;
    uint8_t* sK = reinterpret_cast<uint8_t*>(sdY + plane_sm);
    float* sPn = reinterpret_cast<float*>(sK + (plane_sm + 127) / 128 * 128);

    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        mbar_fence_init();
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const size_t off = (size_t)rfirst * pitch;
        const uint32_t fbytes = (uint32_t)(nload * pitch * sizeof(float));
        const uint32_t kbytes = (uint32_t)(((size_t)nload * pitch + 15) / 16 * 16);
        mbar_expect_tx(&bar, 6 * fbytes + kbytes);
        bulk_g2s(sP, Pin + off, fbytes, &bar);
        bulk_g2s(sVx, Vxin + off, fbytes, &bar);
        bulk_g2s(sVy, Vyin + off, fbytes, &bar);
        bulk_g2s(sdP, dPp + off, fbytes, &bar);
        bulk_g2s(sdX, dPp + pl + off, fbytes, &bar);
        bulk_g2s(sdY, dPp + 2 * pl + off, fbytes, &bar);
        bulk_g2s(sK, T->code + off, kbytes, &bar);
        // excitation velocity of this step, while the copies are in flight
        float e = 0.0f;
        if (bd.has_exc) {
            if (flags & TUBE_TMM) {
                e = glottal_step(T, par, Pin[(size_t)T->exc_y * pitch + T->exc_x],
                                 T->exc_y >= r0 && T->exc_y <= rcommit, nullptr);
            } else {
                e = n < T->src_len ? T->src[n] : 0.0f;
            }
        }
        s_exe = e;
    }
    // one thread decides whether the copies landed, so the whole CTA leaves or
    // stays together; the others then observe the completed phase themselves
    __shared__ int s_landed;
    if (threadIdx.x == 0) s_landed = mbar_wait_bounded(&bar, first_wait_limit(rs)) ? 1 : 0;
    __syncthreads();
    if (!s_landed) {
        // the copies did not land in time: flag the run, let them finish, and leave
        if (threadIdx.x == 0) {
            atomicExch(&rs->error, VS_ERR_TIMEOUT);
            mbar_wait_bounded(&bar, kWaitPolls);
        }
        return;
    }
    mbar_wait_bounded(&bar, kWaitPolls);       // completed: returns on the first poll
    __syncthreads();
    const float exeV = s_exe;
    const float* __restrict__ sig = T->sigma;
    const float K1 = T->K1, bco = T->bcoef;
    const bool eigen = flags & TUBE_EIGEN, dirichlet = flags & TUBE_DIRICHLET;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nseg = (W + 31) >> 5;

    // ---- P' of rows rfirst .. rcommit (row index i = r - rfirst)
    const int prow = rcommit - rfirst + 1;
    for (int q = warp; q < prow * nseg; q += kBandThreads / 32) {
        const int i = q / nseg;
        const int c = (q - i * nseg) * 32 + lane;
        const int r = rfirst + i;
        float pn = 0.0f;
        float w = 0.0f;
        const int k = i * pitch + c;
        if (r >= 1 && c >= 1 && c <= W - 2) {
            const int tc = sK[k] & CODE_TYPE_MASK;
            const float dp = sdP[k];
            const float cx = fsub(fmul(sVx[k], sdX[k]), fmul(sVx[k - 1], sdX[k - 1]));
            const float cy = fsub(fmul(sVy[k], sdY[k]), fmul(sVy[k + pitch], sdY[k + pitch]));
            float num = fsub(fmul(sP[k], dp), fmul(K1, fadd(cx, cy)));
            const int64_t o = (int64_t)r * pitch + c;
            if (WALL) {
                w = T->w[par][o];
                num = fsub(num, fmul(T->K2, w));
            }
            float den = dp;                       // sigma = 0: (1 + 0) * dP == dP
            if (tc != VS_CELL_AIR) {
                const float s = sig[tc];
                den = eigen ? fadd(fmul(s, dp), dp) : fmul(fadd(1.0f, s), dp);
            }
            pn = fdiv_z(num, den);
            if (dirichlet && tc == VS_CELL_NOPRESSURE) pn = 0.0f;
            if (r >= r0) {
                Pout[o] = pn;
                if (r == T->lis_y && c == T->lis_x)
                    store_trace(rs, rs->trace + (int64_t)bd.tube * rs->trace_stride + (n - rs->run_start), pn);
                if (WALL) {
                    // wall oscillator, FDTDEngineCPU.cpp:345-361
                    const float dt = T->dt;
                    const float zn = fadd(T->z[par][o], fmul(w, dt));
                    T->z[par ^ 1][o] = zn;
                    T->w[par ^ 1][o] = fdiv_z(fsub(fadd(fmul(T->Mw, w), fmul(fmul(T->cpl, dt), pn)),
                                                   fmul(fmul(dt, T->Kw), zn)),
                                              fadd(T->Mw, fmul(dt, T->Bw)));
                }
            }
        }
        if (c < pitch) sPn[k] = pn;
    }
    __syncthreads();

    // ---- V' of rows r0 .. rcommit
    const int vrow = rcommit - r0 + 1;
    for (int q = warp; q < vrow * nseg; q += kBandThreads / 32) {
        const int i = 1 + q / nseg;
        const int c = (q - (i - 1) * nseg) * 32 + lane;
        if (c < 1 || c > W - 2) continue;
        const int r = rfirst + i;
        const int k = i * pitch + c;
        const int kc = sK[k], kr = sK[k + 1], kt = sK[k - pitch];
        const float pc = sPn[k], pr = sPn[k + 1], pt = sPn[k - pitch];
        const float vx0 = sVx[k], vy0 = sVy[k];
        const int cls = velocity_class(kc, kr, kt);
        float vx, vy;
        if (cls == V_GENERIC) {
            const VelocityOut v = velocity_generic(kc, kr, kt, pc, pr, pt, vx0, vy0, exeV, sig, T->zinv, bco,
                                                   T->dir0, T->dir1, T->dir2, T->dir3);
            vx = v.vx;
            vy = v.vy;
        } else {
            vx = fsub(vx0, fmul(bco, fsub(pr, pc)));
            vy = fsub(vy0, fmul(bco, fsub(pt, pc)));
            if (cls == V_BETA1) {
                const float sc = sig[kc & CODE_TYPE_MASK];
                vx = fdiv_z(vx, fadd(1.0f, fmaxf(sc, sig[kr & CODE_TYPE_MASK])));
                vy = fdiv_z(vy, fadd(1.0f, fmaxf(sc, sig[kt & CODE_TYPE_MASK])));
            }
        }
        const int64_t o = (int64_t)r * pitch + c;
        Vxout[o] = vx;
        Vyout[o] = vy;
    }
}

__global__ void advance_kernel(RunState* rs, int k) { rs->step += k; }

using StepFn = void (*)(const TubeDev*, const Tile*, int, RunState*, int);

struct ShapeEntry {
    int kind, rows, warps;
    StepFn plain, wall;   // wall = nullptr: no wall-oscillator variant
    int stages;           // quad strips: shared-memory row stages per warp (0 = register prefetch)
    StepFn fast;          // reciprocal-form arithmetic (fast_math); nullptr: none
    int lane_cols = 4;    // two-step quad strips: columns per lane
};

#define VS_STRIP(R, WARPS, MINB) \
    {SHAPE_STRIP, R, WARPS, strip_kernel<R, MINB, false>, strip_kernel<R, MINB, true>, 0, nullptr}
#define VS_BAND(R) {SHAPE_BAND, R, kBandThreads / 32, band_kernel<R, false>, band_kernel<R, true>, 0, nullptr}
#define VS_QUAD(R, WARPS, MINB)                                                                          \
    {SHAPE_QUAD, R, WARPS, quad_kernel<R, WARPS, MINB, 0, false>, nullptr, 0, quad_kernel<R, WARPS, MINB, 0, true>}
#define VS_QUAD2(R, WARPS, MINB, NC) \
    {SHAPE_QUAD2, R, WARPS, quad2_exact<R, WARPS, MINB, NC>(), nullptr, 0, quad2_kernel<R, WARPS, MINB, NC>, NC}
#define VS_QPIPE(R, WARPS, MINB, ST)                                                                     \
    {SHAPE_QUAD, R, WARPS, quad_kernel<R, WARPS, MINB, ST, false>, nullptr, ST,                          \
     quad_kernel<R, WARPS, MINB, ST, true>}

// the two-step kernel in the reference arithmetic: the 2-column shapes
template <int R, int WARPS, int MINB, int NC>
constexpr StepFn quad2_exact() {
    if constexpr (NC == 2) return quad2_kernel<R, WARPS, MINB, NC, false, true>;
    else return nullptr;
}

// strips: (rows per strip, warps per CTA, CTAs per SM the register budget
// targets); bands: rows per band (one CTA of 256 threads each)
const ShapeEntry kShapes[] = {
    VS_STRIP(4, 4, 4),  VS_STRIP(16, 4, 4), VS_STRIP(8, 4, 4),  VS_STRIP(32, 4, 4),
    VS_STRIP(8, 8, 4),  VS_STRIP(16, 8, 4), VS_STRIP(32, 8, 4), VS_STRIP(2, 2, 4),
    VS_STRIP(4, 2, 4),  VS_STRIP(8, 2, 4),  VS_STRIP(16, 4, 3), VS_STRIP(8, 4, 3),
    VS_BAND(4),         VS_BAND(8),         VS_BAND(12),        VS_BAND(16),
    VS_QUAD(8, 4, 4),   VS_QUAD(16, 4, 4),  VS_QUAD(4, 4, 4),   VS_QUAD(8, 2, 8),
    VS_QUAD(16, 2, 8),  VS_QUAD(2, 2, 8),   VS_QUAD(8, 8, 2),   VS_QUAD(32, 4, 4),
    VS_QPIPE(16, 4, 4, 4), VS_QPIPE(32, 4, 4, 4), VS_QPIPE(16, 2, 8, 4), VS_QPIPE(32, 2, 8, 4),
    VS_QPIPE(16, 4, 2, 6), VS_QPIPE(32, 4, 2, 6), VS_QPIPE(8, 4, 4, 4), VS_QPIPE(48, 4, 4, 4),
    VS_QUAD2(16, 2, 4, 4), VS_QUAD2(32, 2, 4, 4), VS_QUAD2(16, 4, 4, 2), VS_QUAD2(24, 4, 4, 2),
    VS_QUAD2(32, 4, 4, 2), VS_QUAD2(32, 2, 8, 2), VS_QUAD2(48, 4, 4, 2), VS_QUAD2(24, 2, 8, 2),
    VS_QUAD2(32, 8, 2, 2), VS_QUAD2(40, 4, 4, 2), VS_QUAD2(2, 2, 8, 2), VS_QUAD2(4, 2, 8, 2),
    VS_QUAD2(8, 2, 8, 2), VS_QUAD2(4, 1, 16, 2),
};
#undef VS_QUAD2
#undef VS_STRIP
#undef VS_BAND
#undef VS_QUAD
#undef VS_QPIPE
constexpr int kNumShapes = sizeof(kShapes) / sizeof(kShapes[0]);

}  // namespace

int tile_shape_count() { return kNumShapes + 1; }

int cluster_shape() { return kNumShapes; }

TileShape tile_shape(int i) {
    if (i == kNumShapes) return {0, 0, 0, SHAPE_CLUSTER, 0};
    const ShapeEntry& e = kShapes[i];
    const int cols = e.kind == SHAPE_STRIP ? kStripCommit
                     : e.kind == SHAPE_BAND ? 0
                     : e.kind == SHAPE_QUAD2 ? 30 * e.lane_cols
                                             : kQuadCommit;
    return {e.rows, cols, e.warps, e.kind, e.kind == SHAPE_QUAD2 ? e.lane_cols : 4};
}

size_t shape_smem_bytes(int shape, int max_pitch) {
    if (shape < 0 || shape >= kNumShapes) return 0;
    const ShapeEntry& e = kShapes[shape];
    if (e.kind == SHAPE_QUAD) return (size_t)e.warps * quad_warp_smem(e.stages);
    if (e.kind != SHAPE_BAND) return 0;
    return band_smem_bytes(e.rows, max_pitch);
}

cudaError_t prepare_shape(int shape, int max_pitch) {
    const size_t bytes = shape_smem_bytes(shape, max_pitch);
    if (bytes == 0) return cudaSuccess;
    cudaError_t e = cudaFuncSetAttribute(kShapes[shape].plain, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e == cudaSuccess && kShapes[shape].wall)
        e = cudaFuncSetAttribute(kShapes[shape].wall, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e == cudaSuccess && kShapes[shape].fast)
        e = cudaFuncSetAttribute(kShapes[shape].fast, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    return e;
}

bool shape_has_plain(int shape) { return shape >= 0 && shape < kNumShapes && kShapes[shape].plain != nullptr; }

bool shape_has_fast(int shape) {
    return shape == kNumShapes || (shape >= 0 && shape < kNumShapes && kShapes[shape].fast != nullptr);
}

cudaError_t launch_step(int shape, bool wall, bool fast, const TubeDev* tubes, const Tile* tiles, int ntiles,
                        RunState* rs, int local, cudaStream_t stream, int max_pitch) {
    if (shape < 0 || shape >= kNumShapes) return cudaErrorInvalidValue;
    if (ntiles <= 0) return cudaSuccess;
    const ShapeEntry& e = kShapes[shape];
    if (fast && wall) return cudaErrorInvalidValue;
    const StepFn fn = fast ? e.fast : (wall ? e.wall : e.plain);
    if (!fn) return cudaErrorInvalidValue;
    if (e.kind == SHAPE_BAND) {
        fn<<<ntiles, kBandThreads, band_smem_bytes(e.rows, max_pitch), stream>>>(tubes, tiles, ntiles, rs, local);
    } else {
        const int wpb = e.warps;
        const size_t smem = e.kind == SHAPE_QUAD ? (size_t)wpb * quad_warp_smem(e.stages) : 0;   // QUAD2: none
        fn<<<(ntiles + wpb - 1) / wpb, wpb * 32, smem, stream>>>(tubes, tiles, ntiles, rs, local);
    }
    return cudaGetLastError();
}

int history_shape(int64_t cells, bool fast) {
    if (fast) return cells < 200000 ? 21 : 17;
    return cells < 200000 ? 7 : 2;
}

cudaError_t launch_step_history(int shape, const TubeDev* tubes, const Tile* tiles, int ntiles, RunState* rs,
                                int local, cudaStream_t stream) {
    // shape 7 of the table (2-row strips, 2 warps per CTA) for small grids,
    // whose step time is the latency of a strip; shape 2 (8-row strips, 4
    // warps per CTA) otherwise
    if (ntiles <= 0) return cudaSuccess;
    // with fast_math the quad strips of shapes 21 (2 rows, 2 warps) and 17
    // (16 rows, 4 warps), in the reciprocal form
    if (shape == 7)
        strip_kernel<2, 4, false, true><<<(ntiles + 1) / 2, 64, 0, stream>>>(tubes, tiles, ntiles, rs, local);
    else if (shape == 2)
        strip_kernel<8, 4, false, true><<<(ntiles + 3) / 4, 128, 0, stream>>>(tubes, tiles, ntiles, rs, local);
    else if (shape == 21)
        quad_kernel<2, 2, 8, 0, true, true><<<(ntiles + 1) / 2, 64, 0, stream>>>(tubes, tiles, ntiles, rs, local);
    else if (shape == 17)
        quad_kernel<16, 4, 4, 0, true, true><<<(ntiles + 3) / 4, 128, 0, stream>>>(tubes, tiles, ntiles, rs, local);
    else
        return cudaErrorInvalidValue;
    return cudaGetLastError();
}

// Strip height of the two-step kernels (forward and history) by batch size,
// measured on fs x 1 / x 15 / x 30 batches (B200, forward, us per step):
// taller strips waste fewer halo rows, shorter ones give the row march more
// warps per SM.  0.38 M interior cells: 4 rows 4.03, 8 rows 4.44, 32 rows 9.18;
// 0.67 M: 8 rows 4.99, 16 rows 6.50, 32 rows 9.32; 1.55 M: 16 rows 9.01,
// 32 rows 12.45; 2.55 M: 32 rows 15.4, 16 rows 16.4.
int two_step_shape(int64_t cells) {
    if (cells < 200000) return 42;       // 2 rows, 2 warps
    if (cells < 600000) return 43;       // 4 rows, 2 warps
    if (cells < 1000000) return 44;      // 8 rows, 2 warps
    if (cells < 2000000) return 34;      // 16 rows, 4 warps
    return 36;                           // 32 rows, 4 warps
}

int history2_shape(int64_t cells) { return two_step_shape(cells); }

cudaError_t launch_step_history2(int shape, const TubeDev* tubes, const Tile* tiles, int ntiles, RunState* rs,
                                 int local, cudaStream_t stream) {
    // the two-step shapes of two_step_shape() (36, 34, 44, 43, 42), storing
    // the history of both steps
    if (ntiles <= 0) return cudaSuccess;
    if (shape == 36)
        quad2_kernel<32, 4, 4, 2, true><<<(ntiles + 3) / 4, 128, 0, stream>>>(tubes, tiles, ntiles, rs, local);
    else if (shape == 34)
        quad2_kernel<16, 4, 4, 2, true><<<(ntiles + 3) / 4, 128, 0, stream>>>(tubes, tiles, ntiles, rs, local);
    else if (shape == 44)
        quad2_kernel<8, 2, 8, 2, true><<<(ntiles + 1) / 2, 64, 0, stream>>>(tubes, tiles, ntiles, rs, local);
    else if (shape == 43)
        quad2_kernel<4, 2, 8, 2, true><<<(ntiles + 1) / 2, 64, 0, stream>>>(tubes, tiles, ntiles, rs, local);
    else if (shape == 42)
        quad2_kernel<2, 2, 8, 2, true><<<(ntiles + 1) / 2, 64, 0, stream>>>(tubes, tiles, ntiles, rs, local);
    else
        return cudaErrorInvalidValue;
    return cudaGetLastError();
}

cudaError_t launch_advance2(RunState* rs, int k, int toggle, cudaStream_t stream) {
    advance2_kernel<<<1, 1, 0, stream>>>(rs, k, toggle);
    return cudaGetLastError();
}

cudaError_t launch_copy_back(const TubeDev* tubes, int ntubes, int max_plane_cells, const RunState* rs,
                             cudaStream_t stream) {
    const dim3 grid((max_plane_cells + 255) / 256, ntubes);
    copy_back_kernel<<<grid, 256, 0, stream>>>(tubes, rs);
    return cudaGetLastError();
}

cudaError_t launch_advance(RunState* rs, int k, cudaStream_t stream) {
    advance_kernel<<<1, 1, 0, stream>>>(rs, k);
    return cudaGetLastError();
}

}  // namespace vsb
