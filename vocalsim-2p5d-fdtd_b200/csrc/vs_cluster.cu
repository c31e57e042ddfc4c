// vs_cluster.cu -- one tube on one thread-block cluster, a whole run per launch.
//
// A single tube is too small to fill the GPU with one launch per step: the
// graph-replayed step kernels spend most of each step in launch and memory
// latency.  This kernel keeps the tube's state on chip for the whole run.
// The interior rows are split into C contiguous bands, one CTA of a cluster
// of C (up to 16) per band; each CTA holds in shared memory the P, Vx and Vy
// of its rows, the maps and codes it needs, and two ghost rows:
//   top    (row r0 - 1): P, Vx, Vy; its P' is recomputed locally each step
//          with the same inputs and expressions as its owner uses, so only
//          its velocities arrive from the CTA above
//   bottom (row r1 + 1): Vy, from the CTA below
// One step of the reference loop (FDTDEngineCPU.cpp:257-288):
//   P' of rows r0 - 1 .. r1 (in place; the listener sample is stored)
//   __syncthreads
//   V' of rows r0 .. r1 (in place); the threads of the first and last row
//   store their new velocities into the neighbours' ghost rows (distributed
//   shared memory); the excitation velocity of the next step is prepared
//   (table value, or the two-mass step on the new pressure, finished by one
//   thread of the CTA that owns the excitation cell and sent to every CTA)
//   cluster barrier (arrive.release / wait.acquire; the two-mass thread
//   prepares the state-only part of a later step between the two)
// Ghost rows and the excitation slot are double-buffered by step parity, so a
// CTA that runs ahead into the next step never overwrites values a neighbour
// still reads.  At the end every CTA writes its rows back to the parity set
// of the final step; the other set is not touched.
//
// Arithmetic per cell is that of the strip and quad-strip kernels
// (vs_cellmath.cuh): reference rounding (fast_math = 0), or the reciprocal
// form with the per-cell descriptor tables (fast_math = 1).  The row masks of
// the strip kernels are replaced by each cell's own velocity class; where a
// strip kernel applies a shortened or a full form, both give the same value
// (they differ only by operations with exact 0 / 1 operands).
//
// No wall oscillator and no history capture (those runs use the step
// kernels).  Every thread executes the same barrier sequence; there are no
// spin waits.
#include <cooperative_groups.h>

#include <algorithm>
#include <type_traits>

#include "vs_cellmath.cuh"
#include "vs_mbarrier.cuh"

namespace cg = cooperative_groups;

namespace vsb {
namespace {

// Shared-memory layout of one CTA (rows of `pitch` elements).
struct ClusterLayout {
    int pitch, R;           // R = rows of the tallest band
    // float row offsets
    int P, Vx, gVx, Vy, gVyT, gVyB, dP, dX, dY;
    int nfloat_rows;
    // byte rows: code, velocity class, descriptor (fast_math)
    int nbyte_rows;
    size_t bytes;
};

__host__ __device__ inline ClusterLayout cluster_layout(int pitch, int R, bool fast) {
    ClusterLayout L{};
    L.pitch = pitch;
    L.R = R;
    int o = 0;
    L.P = o;    o += R + 1;     // rows r0-1 .. r1
    L.Vx = o;   o += R;         // rows r0 .. r1
    L.gVx = o;  o += 2;         // ghost top row, two slots
    L.Vy = o;   o += R;
    L.gVyT = o; o += 2;
    L.gVyB = o; o += 2;         // ghost bottom row, two slots
    L.dP = o;   o += R + 1;     // rows r0-1 .. r1
    L.dX = o;   o += R + 1;
    L.dY = o;   o += R + 2;     // rows r0-1 .. r1+1
    L.nfloat_rows = o;
    L.nbyte_rows = 3 * (R + 1);
    // floats, then 2 x 256 float4 descriptor tables (fast_math), sigma[16],
    // the two excitation slots, then the byte rows
    size_t b = (size_t)o * pitch * sizeof(float);
    b += fast ? 2 * kDescEntries * sizeof(float4) : 0;
    b += 16 * sizeof(float) + 2 * sizeof(float) + 8;
    b += (size_t)L.nbyte_rows * pitch;
    L.bytes = (b + 127) / 128 * 128;
    return L;
}

template <bool FAST>
__global__ void __launch_bounds__(512, 1)
cluster_kernel(const TubeDev* __restrict__ Tp, RunState* __restrict__ rs, int64_t nsteps, int R) {
    extern __shared__ __align__(16) unsigned char c_smem[];
    cg::cluster_group cluster = cg::this_cluster();
    const int C = (int)cluster.num_blocks();
    const int k = (int)cluster.block_rank();
    const TubeDev* __restrict__ T = Tp + blockIdx.y;          // one cluster per tube of the batch
    const int H = T->H, W = T->W, pitch = T->pitch, flags = T->flags;
    const ClusterLayout L = cluster_layout(pitch, R, FAST);
    float* sf = reinterpret_cast<float*>(c_smem);
    float4* tabA = reinterpret_cast<float4*>(sf + (size_t)L.nfloat_rows * pitch);
    float4* tabB = tabA + (FAST ? kDescEntries : 0);
    float* sSig = reinterpret_cast<float*>(tabB + (FAST ? kDescEntries : 0));
    float* sExe = sSig + 16;
    unsigned char* sb = reinterpret_cast<unsigned char*>(sExe + 4);
    auto row = [&](int base, int i) { return sf + (size_t)(base + i) * pitch; };
    unsigned char* sCode = sb;                          // rows i = 0..R (r0-1 .. r1)
    unsigned char* sCls = sb + (size_t)(R + 1) * pitch;
    unsigned char* sDesc = sb + (size_t)2 * (R + 1) * pitch;

    // band of this CTA
    const int NR = H - 2;
    const int r0 = 1 + (int)(((int64_t)k * NR) / C);
    const int r1 = (int)(((int64_t)(k + 1) * NR) / C);      // inclusive
    const int Rk = r1 - r0 + 1;
    const int64_t n0 = rs->step;
    const int64_t run_start = rs->run_start;
    float* __restrict__ trace = rs->trace + (int64_t)blockIdx.y * rs->trace_stride;
    const int par0 = (int)(n0 & 1);
    const int64_t pl = T->plane;
    const float* __restrict__ gP = T->P[0] + par0 * pl;
    const float* __restrict__ gVx = gP + 2 * pl;
    const float* __restrict__ gVy = gP + 4 * pl;
    const float* __restrict__ gdP = T->dP;
    const float* __restrict__ gdX = gdP + pl;
    const float* __restrict__ gdY = gdP + 2 * pl;
    const int tid = threadIdx.x, nthr = blockDim.x;

    // ---- load the band, its ghost rows and the maps
    for (int c = tid; c < pitch; c += nthr) {
        for (int i = 0; i <= Rk + 1; ++i) {
            const int r = r0 - 1 + i;                     // 0 .. H-1
            const int64_t o = (int64_t)r * pitch + c;
            const float p = gP[o], vx = gVx[o], vy = gVy[o];
            if (i <= Rk) {
                row(L.P, i)[c] = p;
                row(L.dP, i)[c] = gdP[o];
                row(L.dX, i)[c] = gdX[o];
                const int kc = T->code[o];
                sCode[(size_t)i * pitch + c] = (unsigned char)kc;
                if (FAST) sDesc[(size_t)i * pitch + c] = T->desc[o];
                const int kr = c + 1 < pitch ? T->code[o + 1] : VS_CELL_DEAD;
                const int kt = r >= 1 ? T->code[o - pitch] : VS_CELL_DEAD;
                sCls[(size_t)i * pitch + c] = (unsigned char)velocity_class(kc, kr, kt);
            }
            row(L.dY, i)[c] = gdY[o];
            if (i == 0) {
                row(L.gVx, par0)[c] = vx;
                row(L.gVyT, par0)[c] = vy;
                row(L.gVx, par0 ^ 1)[c] = 0.0f;
                row(L.gVyT, par0 ^ 1)[c] = 0.0f;
            } else if (i <= Rk) {
                row(L.Vx, i - 1)[c] = vx;
                row(L.Vy, i - 1)[c] = vy;
            } else {
                row(L.gVyB, par0)[c] = vy;
                row(L.gVyB, par0 ^ 1)[c] = 0.0f;
            }
        }
    }
    if (FAST)
        for (int j = tid; j < 2 * kDescEntries; j += nthr) tabA[j] = T->desc_a[j];   // desc_b = desc_a + 256
    if (tid < 16) sSig[tid] = tid < 13 ? T->sigma[tid] : 0.0f;

    const bool tmm = flags & TUBE_TMM, tmm64 = flags & TUBE_TMM64;
    const bool exc_owner = tmm && T->exc_y >= r0 && T->exc_y <= r1;
    const int exc_i = T->exc_y - (r0 - 1), exc_x = T->exc_x;
    // The two-mass model runs in the last thread of the CTA that owns the
    // excitation cell (a thread with few or no cells).  Its step is split at
    // the one use of the pressure (tmm_prepare / tmm_finish): the state-only
    // part for step n + 2 is computed between this thread's arrival at the
    // cluster barrier of step n and its wait, beside the other CTAs' work, and
    // only the last division waits for the new pressure.
    const bool tmm_thread = exc_owner && tid == nthr - 1;
    TmmState s32{};
    TmmState64 s64{};
    TmmPrep prep32{};
    TmmPrep64 prep64{};
    if (tmm_thread) {
        if (tmm64) s64 = T->tmm64[par0];
        else s32 = T->tmm[par0];
    }
    auto tmm_prepare_next = [&]() {
        if (tmm64) prep64 = tmm_prepare64(T->tmmd, T->tmmx, s64);
        else prep32 = tmm_prepare(T->tmmc, s32);
    };
    auto tmm_finish_next = [&](float p1) -> float {
        return tmm64 ? tmm_finish64(prep64, s64, p1) : tmm_finish(prep32, s32, p1);
    };
    auto send_exe = [&](int slot, float e) {
        for (int q = 0; q < C; ++q) *cluster.map_shared_rank(sExe + slot, q) = e;
    };
    __syncthreads();
    cluster.sync();                                       // every CTA of the cluster is running
    if (tmm_thread) {
        tmm_prepare_next();
        send_exe(par0, tmm_finish_next(row(L.P, exc_i)[exc_x]));
        tmm_prepare_next();
    } else if (!tmm && tid == 0) {
        sExe[par0] = n0 < T->src_len ? T->src[n0] : 0.0f;
    }
    cluster.sync();

    // neighbours' ghost rows (distributed shared memory)
    float* up_gVyB = k > 0 ? cluster.map_shared_rank(row(L.gVyB, 0), k - 1) : nullptr;
    float* dn_gVx = k + 1 < C ? cluster.map_shared_rank(row(L.gVx, 0), k + 1) : nullptr;
    float* dn_gVyT = k + 1 < C ? cluster.map_shared_rank(row(L.gVyT, 0), k + 1) : nullptr;

    const float K1 = T->K1, bco = T->bcoef;
    const bool eigen = flags & TUBE_EIGEN, dirichlet = flags & TUBE_DIRICHLET;
    const float zval = T->zinv, dir0 = T->dir0, dir1 = T->dir1, dir2 = T->dir2, dir3 = T->dir3;
    const int lis_y = T->lis_y, lis_x = T->lis_x;
    const bool lis_here = lis_y >= r0 && lis_y <= r1;
    const int64_t n_end = n0 + nsteps;

    for (int64_t n = n0; n < n_end; ++n) {
        const int p = (int)(n & 1), q = p ^ 1;
        // ---- P' of rows r0-1 .. r1 (FDTDEngineCPU.cpp:316-339)
        for (int c = 1 + tid; c <= W - 2; c += nthr) {
            for (int i = (r0 == 1 ? 1 : 0); i <= Rk; ++i) {
                const float vx = i == 0 ? row(L.gVx, p)[c] : row(L.Vx, i - 1)[c];
                const float vxl = i == 0 ? row(L.gVx, p)[c - 1] : row(L.Vx, i - 1)[c - 1];
                const float vy = i == 0 ? row(L.gVyT, p)[c] : row(L.Vy, i - 1)[c];
                const float vyb = i == Rk ? row(L.gVyB, p)[c] : row(L.Vy, i)[c];
                const float* dXr = row(L.dX, i);
                const float ux = fmul(vx, dXr[c]), uxl = fmul(vxl, dXr[c - 1]);
                const float uy = fmul(vy, row(L.dY, i)[c]), uyb = fmul(vyb, row(L.dY, i + 1)[c]);
                const float dp = row(L.dP, i)[c];
                float* Pr = row(L.P, i);
                float pn;
                if constexpr (FAST) {
                    // (P dP - K1 S) / ((1 + s) dP) = (P - K1 S / dP) g
                    const float ks = fmul(K1, fadd(fsub(ux, uxl), fsub(uy, uyb)));
                    pn = __fmaf_rn(-ks, rcp_approx(dp), Pr[c]);
                    const int d = sDesc[(size_t)i * pitch + c];
                    if (d) pn = fmul(pn, tabA[d].z);
                } else {
                    const float num = fsub(fmul(Pr[c], dp), fmul(K1, fadd(fsub(ux, uxl), fsub(uy, uyb))));
                    const int tc = sCode[(size_t)i * pitch + c] & CODE_TYPE_MASK;
                    float den = dp;                       // sigma = 0: (1 + 0) dP == dP
                    if (tc != VS_CELL_AIR) {
                        const float s = sSig[tc];
                        den = eigen ? fadd(fmul(s, dp), dp) : fmul(fadd(1.0f, s), dp);
                    }
                    pn = fdiv_z(num, den);
                    if (dirichlet && tc == VS_CELL_NOPRESSURE) pn = 0.0f;
                }
                Pr[c] = pn;
                if (i >= 1 && lis_here && r0 - 1 + i == lis_y && c == lis_x) store_trace(rs, trace + (n - run_start), pn);
            }
        }
        __syncthreads();
        // ---- excitation velocity of the next step
        if (n + 1 < n_end) {
            if (tmm_thread) send_exe(q, tmm_finish_next(row(L.P, exc_i)[exc_x]));
            else if (!tmm && tid == 0) sExe[q] = n + 1 < T->src_len ? T->src[n + 1] : 0.0f;
        }
        const float exeV = sExe[p];
        // ---- V' of rows r0 .. r1 (FDTDEngineCPU.cpp:364-410)
        for (int c = 1 + tid; c <= W - 2; c += nthr) {
            for (int i = 1; i <= Rk; ++i) {
                const float* Pr = row(L.P, i);
                const float pc = Pr[c], pr = Pr[c + 1], pt = row(L.P, i - 1)[c];
                float* Vxr = row(L.Vx, i - 1);
                float* Vyr = row(L.Vy, i - 1);
                float vx = Vxr[c], vy = Vyr[c];
                const int cls = sCls[(size_t)i * pitch + c];
                if constexpr (FAST) {
                    // V' = al (V - bco (P'n - P'c)) + zo P'c - zi P'n + ce exeV
                    vx = fsub(vx, fmul(bco, fsub(pr, pc)));
                    vy = fsub(vy, fmul(bco, fsub(pt, pc)));
                    const int d = sDesc[(size_t)i * pitch + c];
                    if (d) {
                        const float4 da = tabA[d];
                        vx = fmul(vx, da.x);
                        vy = fmul(vy, da.y);
                        if (cls == V_GENERIC) {
                            const float4 db = tabB[d];
                            vx = __fmaf_rn(da.w, exeV, __fmaf_rn(-db.y, pr, __fmaf_rn(db.x, pc, vx)));
                            vy = __fmaf_rn(-db.w, pt, __fmaf_rn(db.z, pc, vy));
                        }
                    }
                } else if (cls == V_GENERIC) {
                    const int kc = sCode[(size_t)i * pitch + c], kr = sCode[(size_t)i * pitch + c + 1];
                    const int kt = sCode[(size_t)(i - 1) * pitch + c];
                    const VelocityOut v = velocity_generic(kc, kr, kt, pc, pr, pt, vx, vy, exeV, sSig, zval, bco,
                                                           dir0, dir1, dir2, dir3);
                    vx = v.vx;
                    vy = v.vy;
                } else {
                    vx = fsub(vx, fmul(bco, fsub(pr, pc)));
                    vy = fsub(vy, fmul(bco, fsub(pt, pc)));
                    if (cls == V_BETA1) {
                        const float sc = sSig[sCode[(size_t)i * pitch + c] & CODE_TYPE_MASK];
                        vx = fdiv_z(vx, fadd(1.0f, fmaxf(sc, sSig[sCode[(size_t)i * pitch + c + 1] & CODE_TYPE_MASK])));
                        vy = fdiv_z(vy, fadd(1.0f, fmaxf(sc, sSig[sCode[(size_t)(i - 1) * pitch + c] & CODE_TYPE_MASK])));
                    }
                }
                Vxr[c] = vx;
                Vyr[c] = vy;
                if (i == Rk && dn_gVx) {
                    dn_gVx[(size_t)q * pitch + c] = vx;
                    dn_gVyT[(size_t)q * pitch + c] = vy;
                }
                if (i == 1 && up_gVyB) up_gVyB[(size_t)q * pitch + c] = vy;
            }
        }
        // cluster barrier, split: the two-mass thread prepares step n + 2 in between
        asm volatile("barrier.cluster.arrive.release;" ::: "memory");
        if (tmm_thread && n + 2 < n_end) tmm_prepare_next();
        asm volatile("barrier.cluster.wait.acquire;" ::: "memory");
    }

    // ---- the state of step n_end back to its parity set
    const int pe = (int)(n_end & 1);
    float* __restrict__ oP = T->P[0] + pe * pl;
    float* __restrict__ oVx = oP + 2 * pl;
    float* __restrict__ oVy = oP + 4 * pl;
    for (int c = 1 + tid; c <= W - 2; c += nthr)
        for (int i = 1; i <= Rk; ++i) {
            const int64_t o = (int64_t)(r0 - 1 + i) * pitch + c;
            oP[o] = row(L.P, i)[c];
            oVx[o] = row(L.Vx, i - 1)[c];
            oVy[o] = row(L.Vy, i - 1)[c];
        }
    if (tmm_thread) {
        if (tmm64) T->tmm64[pe] = s64;
        else T->tmm[pe] = s32;
    }
}

// ---------------------------------------------------------------------------
// Register-resident form (frames of at most RMAX rows per CTA and 512
// columns).  Thread t owns column c = t + 1 of its band for the whole run: the
// P, Vx, Vy of its rows (and of the top ghost row) and every per-cell
// coefficient (depths, codes or descriptor) live in its registers, with the
// rows unrolled so the cells of a column are independent instruction
// streams.  Horizontal neighbours move by warp shuffles; only the two warp-edge
// values of each row go through shared memory (eUX: Vx dX of the column left of
// a warp, for its lane 0; eP: P' of the column right of a warp, for its lane
// 31), and the ghost rows arrive in shared memory as in the first form.  The
// step sequence and the per-cell arithmetic are those of the first form.
//
// Step synchronisation, two variants:
//   P2P = false  the first form's cluster barrier after every step (its
//                release fence waits for every thread's stores into the
//                neighbours' ghost rows)
//   P2P = true   point to point: a thread sends its boundary velocities with
//                st.async, whose bytes count against the receiving CTA's
//                mbarrier for that ghost parity; at the end of a step one
//                thread arrives on the barrier of the next step's ghosts
//                (expecting the bytes both neighbours send) and waits for it,
//                and the block barrier that follows publishes the ghosts and
//                the warp-edge values to the CTA.  A CTA then waits only for
//                its two neighbours, never for the whole cluster.  Ghost slots
//                stay double-buffered: a neighbour writes parity q again only
//                after it received this CTA's ghosts of the step in between,
//                which this CTA sends after it has read parity q.  The
//                two-mass excitation value, which every CTA needs, travels in a
//                ring of kExeRing tagged slots (the value and its step in one
//                8-byte store); a CTA lags the owner of the excitation cell by
//                at most its distance in CTAs, so a slot is never reused while
//                a CTA may still read it.  Waits are bounded; a CTA that gives
//                up reports VS_ERR_TIMEOUT, and every CTA meets at a final
//                cluster barrier before any exits.
// The two-mass model's state and its prepared step, kept in shared memory by
// the one thread that runs it, so that the model's registers do not count
// against every thread's budget (the helpers are not inlined).
struct TmmSlot {
    TmmState64 s64;
    TmmPrep64 prep64;
    TmmState s32;
    TmmPrep prep32;
};

__device__ __noinline__ void tmm_slot_prepare(const TubeDev* __restrict__ T, TmmSlot* slot, bool tmm64) {
    if (tmm64) slot->prep64 = tmm_prepare64(T->tmmd, T->tmmx, slot->s64);
    else slot->prep32 = tmm_prepare(T->tmmc, slot->s32);
}

__device__ __noinline__ float tmm_slot_finish(TmmSlot* slot, bool tmm64, float p1) {
    return tmm64 ? tmm_finish64(slot->prep64, slot->s64, p1) : tmm_finish(slot->prep32, slot->s32, p1);
}

// The model's current state as the adjoint's two-mass history keeps it.
__device__ __noinline__ void tmm_slot_hist(const TmmSlot* slot, bool tmm64, double* h) {
    if (tmm64) tmm_to_hist(slot->s64, h);
    else tmm_to_hist(slot->s32, h);
}

struct RegLayout {
    int pitch, nw, rmax;
    size_t gT, gVyB, dX0, eUX, eP, tab, sig, exe, tmm, bar, exr, bytes;   // byte offsets
};

constexpr int kExeRing = 32;        // excitation values in flight (> the largest cluster)

// f(integral_constant<int, I>) for I = B .. E-1, unrolled at compile time
template <int B, int E, class F>
__device__ __forceinline__ void static_for(F&& f) {
    if constexpr (B < E) {
        f(std::integral_constant<int, B>{});
        static_for<B + 1, E>(f);
    }
}

__host__ __device__ inline RegLayout reg_layout(int pitch, int nthreads, int rmax, bool fast) {
    RegLayout L{};
    L.pitch = pitch;
    L.nw = nthreads / 32;
    L.rmax = rmax;
    size_t o = 0;
    auto take = [&](size_t bytes) { const size_t at = o; o += (bytes + 15) / 16 * 16; return at; };
    L.gT = take(2 * (size_t)pitch * sizeof(float2));
    L.gVyB = take(2 * (size_t)pitch * sizeof(float));
    L.dX0 = take((size_t)pitch * sizeof(float));
    L.eUX = take((size_t)(L.nw + 1) * (rmax + 1) * sizeof(float));
    L.eP = take((size_t)(L.nw + 1) * (rmax + 1) * sizeof(float));
    L.tab = take(fast ? 2 * kDescEntries * sizeof(float4) : 0);
    L.sig = take(16 * sizeof(float));
    L.exe = take(8 * sizeof(float));
    L.tmm = take(sizeof(TmmSlot));
    L.bar = take(2 * sizeof(uint64_t));
    L.exr = take(kExeRing * sizeof(float2));
    L.bytes = (o + 127) / 128 * 128;
    return L;
}

// Named barrier 1 over the first `count` threads of the CTA (the column
// warps), plain and with an OR reduction.
__device__ __forceinline__ void cols_sync(int count) { asm volatile("bar.sync 1, %0;" ::"r"(count) : "memory"); }

__device__ __forceinline__ int cols_sync_or(int count, int pred) {
    int r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.s32 p, %2, 0;\n\t"
        "bar.red.or.pred q, 1, %1, p;\n\t"
        "selp.s32 %0, 1, 0, q;\n\t}"
        : "=r"(r)
        : "r"(count), "r"(pred)
        : "memory");
    return r;
}

// SYNC: 0 = cluster barrier per step, 1 = point to point, 2 = point to point
// with the two-mass model in an extra warp (launched with MAXT + 32 threads;
// the extra warp's registers come out of every thread's budget, so this
// variant is only used for two-mass tubes)
template <bool FAST, int RMAX, int MAXT, int SYNC>
__global__ void __launch_bounds__(SYNC == 2 ? MAXT + 32 : MAXT, 1)
cluster_reg_kernel(const TubeDev* __restrict__ Tp, RunState* __restrict__ rs, int64_t nsteps) {
    constexpr bool P2P = SYNC >= 1;
    extern __shared__ __align__(16) unsigned char r_smem[];
    cg::cluster_group cluster = cg::this_cluster();
    const int C = (int)cluster.num_blocks();
    const int k = (int)cluster.block_rank();
    const TubeDev* __restrict__ T = Tp + blockIdx.y;          // one cluster per tube of the batch
    const int H = T->H, W = T->W, pitch = T->pitch, flags = T->flags;
    const int tid = threadIdx.x, nthr = blockDim.x, lane = tid & 31, warp = tid >> 5;
    // point to point with the two-mass source: the last warp runs the model
    // (two_mass_warp); the column warps are the ones before it
    const bool two_mass_warp = SYNC == 2 && (T->flags & TUBE_TMM);
    const int ncols = two_mass_warp ? nthr - 32 : nthr;
    const RegLayout L = reg_layout(pitch, nthr, RMAX, FAST);
    float2* gT = reinterpret_cast<float2*>(r_smem + L.gT);     // [2][pitch] ghost top (Vx, Vy)
    float* gVyB = reinterpret_cast<float*>(r_smem + L.gVyB);   // [2][pitch] ghost bottom Vy
    uint64_t* bar = reinterpret_cast<uint64_t*>(r_smem + L.bar);   // [2] ghost arrival, by parity
    // [kExeRing] excitation slots: value bits | step << 32, one 8-byte (single-copy atomic) word each
    unsigned long long* exr = reinterpret_cast<unsigned long long*>(r_smem + L.exr);
    float* sdX0 = reinterpret_cast<float*>(r_smem + L.dX0);    // dX of the top ghost row
    float* eUX = reinterpret_cast<float*>(r_smem + L.eUX);     // [nw + 1][RMAX + 1]
    float* eP = reinterpret_cast<float*>(r_smem + L.eP);       // [nw + 1][RMAX + 1]
    float4* tabA = reinterpret_cast<float4*>(r_smem + L.tab);
    float4* tabB = tabA + kDescEntries;
    float* sSig = reinterpret_cast<float*>(r_smem + L.sig);
    float* sExe = reinterpret_cast<float*>(r_smem + L.exe);

    const int NR = H - 2;
    const int r0 = 1 + (int)(((int64_t)k * NR) / C);
    const int r1 = (int)(((int64_t)(k + 1) * NR) / C);
    const int Rk = r1 - r0 + 1;                               // 1 .. RMAX
    const int64_t n0 = rs->step;
    const int64_t run_start = rs->run_start;
    float* __restrict__ trace = rs->trace + (int64_t)blockIdx.y * rs->trace_stride;
    const int par0 = (int)(n0 & 1);
    const int64_t pl = T->plane;
    const float* __restrict__ gP = T->P[0] + par0 * pl;
    const float* __restrict__ gdP = T->dP;
    const int c = tid + 1;                                     // this thread's column
    const bool mine = c <= W - 2 && tid < ncols;               // an interior column
    const int cc = c < pitch ? c : pitch - 1;                  // clamped for the loads

    // ---- state, maps and codes of this column (rows r0-1 .. r1, and r1+1 for Vy / dY)
    float P[RMAX + 1], VX[RMAX + 1], VY[RMAX + 1], dP[RMAX + 1], dX[RMAX + 1], dY[RMAX + 2];
    uint32_t cw[RMAX + 1];      // code | right code << 8 | top code << 16 | velocity class << 24 (| desc in FAST: << 8 replaced)
    uint32_t dsc[RMAX + 1];
    float vyb = 0.0f;
#pragma unroll
    for (int i = 0; i <= RMAX; ++i) {
        P[i] = VX[i] = VY[i] = 0.0f;
        dP[i] = dX[i] = 1.0f;
        dY[i] = 1.0f;
        cw[i] = VS_CELL_DEAD;
        dsc[i] = 0;
        if (i <= Rk) {
            const int r = r0 - 1 + i;
            const int64_t o = (int64_t)r * pitch + cc;
            P[i] = gP[o];
            VX[i] = gP[2 * pl + o];
            VY[i] = gP[4 * pl + o];
            dP[i] = gdP[o];
            dX[i] = gdP[pl + o];
            dY[i] = gdP[2 * pl + o];
            const int kc = T->code[o];
            const int kr = cc + 1 < pitch ? T->code[o + 1] : VS_CELL_DEAD;
            const int kt = r >= 1 ? T->code[o - pitch] : VS_CELL_DEAD;
            cw[i] = (uint32_t)kc | ((uint32_t)kr << 8) | ((uint32_t)kt << 16) |
                    ((uint32_t)velocity_class(kc, kr, kt) << 24);
            if (FAST) dsc[i] = T->desc[o];
        }
    }
    dY[RMAX + 1] = 1.0f;
    {
        const int64_t o = (int64_t)(r0 + Rk) * pitch + cc;   // row r1 + 1
#pragma unroll
        for (int i = 1; i <= RMAX + 1; ++i)
            if (i == Rk + 1) dY[i] = gdP[2 * pl + o];
        vyb = gP[4 * pl + o];
    }
    // ghost slots, edge buffers, tables
    for (int x = tid; x < pitch; x += nthr) {
        const int64_t o = (int64_t)(r0 - 1) * pitch + x;
        gT[par0 * pitch + x] = make_float2(gP[2 * pl + o], gP[4 * pl + o]);
        gT[(par0 ^ 1) * pitch + x] = make_float2(0.0f, 0.0f);
        const int64_t ob = (int64_t)(r0 + Rk) * pitch + x;
        gVyB[par0 * pitch + x] = gP[4 * pl + ob];
        gVyB[(par0 ^ 1) * pitch + x] = 0.0f;
        sdX0[x] = gdP[pl + o];
    }
    for (int j = tid; j < (L.nw + 1) * (RMAX + 1); j += nthr) {
        eUX[j] = 0.0f;
        eP[j] = 0.0f;
    }
    if (FAST)
        for (int j = tid; j < 2 * kDescEntries; j += nthr) tabA[j] = T->desc_a[j];
    if (tid < 16) sSig[tid] = tid < 13 ? T->sigma[tid] : 0.0f;
    if (P2P) {
        if (tid == 0) {
            mbar_init(bar, 1);
            mbar_init(bar + 1, 1);
            mbar_fence_init();            // visible to the cluster before its first remote arrival
        }
        for (int j = tid; j < kExeRing; j += nthr) exr[j] = 0xffffffff00000000ull;   // tag: no step
    }
    __syncthreads();
    // left-edge values of every warp for the first step (lane 31 of the warp before)
    if (lane == 31 && warp + 1 <= L.nw) {
#pragma unroll
        for (int i = 1; i <= RMAX; ++i)
            if (i <= Rk) eUX[(warp + 1) * (RMAX + 1) + i] = fmul(VX[i], dX[i]);
    }

    const bool tmm = flags & TUBE_TMM, tmm64 = flags & TUBE_TMM64;
    const bool exc_owner = tmm && T->exc_y >= r0 && T->exc_y <= r1;
    const int exc_i = T->exc_y - (r0 - 1), exc_x = T->exc_x;
    const bool tmm_thread = exc_owner && tid == (two_mass_warp ? ncols : nthr - 1);
    // the adjoint's segment recomputation: every step's state (and the
    // two-mass state) also goes to the history slots
    float* __restrict__ hist = T->hist;
    double* __restrict__ thist = T->tmm_hist;
    // the excitation cell's column owner publishes its P' for the two-mass thread;
    // for the two-mass warp as tagged words (P bits | step << 32) by step parity
    // in sExe[4..7] (the owner writes step n + 2 only after the warp sent the
    // excitation value of step n + 1, which needed the word of step n)
    float* sPexc = sExe + 2;
    volatile unsigned long long* pexw = reinterpret_cast<volatile unsigned long long*>(sExe + 4);
    TmmSlot* slot = reinterpret_cast<TmmSlot*>(r_smem + L.tmm);
    if (tmm_thread) {
        if (tmm64) slot->s64 = T->tmm64[par0];
        else slot->s32 = T->tmm[par0];
    }
    auto tmm_prepare_next = [&]() { tmm_slot_prepare(T, slot, tmm64); };
    auto tmm_finish_next = [&](float p1) -> float { return tmm_slot_finish(slot, tmm64, p1); };
    auto send_exe = [&](int slot, float e) {
        for (int q = 0; q < C; ++q) *cluster.map_shared_rank(sExe + slot, q) = e;
    };
    // P at the excitation cell, from its column owner
    auto publish_pexc = [&]() {
        if (exc_owner && c == exc_x && tid < ncols) {
#pragma unroll
            for (int i = 1; i <= RMAX; ++i)
                if (i == exc_i) *sPexc = P[i];
        }
    };
    auto publish_pexc_tagged = [&](int64_t m) {
        if (exc_owner && c == exc_x && tid < ncols) {
#pragma unroll
            for (int i = 1; i <= RMAX; ++i)
                if (i == exc_i) pexw[m & 1] = ((unsigned long long)(uint32_t)m << 32) | __float_as_uint(P[i]);
        }
    };
    if (tid < 2) pexw[tid] = 0xffffffff00000000ull;               // tag: no step
    // the two-mass value of step m into every CTA's ring slot, tagged with m
    auto send_exe_ring = [&](int64_t m, float e) {
        const unsigned long long v = ((unsigned long long)(uint32_t)m << 32) | __float_as_uint(e);
        for (int j = 0; j < C; ++j) {
            volatile unsigned long long* d = cluster.map_shared_rank(exr + (m & (kExeRing - 1)), j);
            *d = v;
        }
    };
    publish_pexc();
    __syncthreads();
    cluster.sync();
    if (tmm_thread) {
        tmm_prepare_next();
        const float e0 = tmm_finish_next(*sPexc);
        if (thist) tmm_slot_hist(slot, tmm64, thist + 6 * (n0 + 1 - run_start));
        if (P2P) send_exe_ring(n0, e0);
        else send_exe(par0, e0);
        tmm_prepare_next();
    } else if (!tmm && tid == 0) {
        sExe[par0] = n0 < T->src_len ? T->src[n0] : 0.0f;
    }
    cluster.sync();

    float* up_gVyB = k > 0 ? cluster.map_shared_rank(gVyB, k - 1) : nullptr;
    float2* dn_gT = k + 1 < C ? cluster.map_shared_rank(gT, k + 1) : nullptr;
    // point to point: cluster addresses of the neighbours' ghost slots and barriers,
    // and the bytes both neighbours send into this CTA per step
    const uint32_t up_gVyB_a = P2P && k > 0 ? cluster_addr(gVyB, k - 1) : 0u;
    const uint32_t up_bar_a = P2P && k > 0 ? cluster_addr(bar, k - 1) : 0u;
    const uint32_t dn_gT_a = P2P && k + 1 < C ? cluster_addr(gT, k + 1) : 0u;
    const uint32_t dn_bar_a = P2P && k + 1 < C ? cluster_addr(bar, k + 1) : 0u;
    const uint32_t expect = (k > 0 ? 8u * (uint32_t)(W - 2) : 0u) + (k + 1 < C ? 4u * (uint32_t)(W - 2) : 0u);
    const uint32_t limit = first_wait_limit(rs);
    uint32_t phase = 0;                          // bit b: parity of the next phase of bar[b]
    bool fail = false;

    const float K1 = T->K1, bco = T->bcoef;
    const bool eigen = flags & TUBE_EIGEN, dirichlet = flags & TUBE_DIRICHLET;
    const float zval = T->zinv, dir0 = T->dir0, dir1 = T->dir1, dir2 = T->dir2, dir3 = T->dir3;
    const int lis_y = T->lis_y, lis_x = T->lis_x;
    const int lis_i = (lis_y >= r0 && lis_y <= r1 && c == lis_x) ? lis_y - (r0 - 1) : -1;
    const int64_t n_end = n0 + nsteps;
    const int ifirst = r0 == 1 ? 1 : 0;          // the ring row above the first band is never computed
    constexpr unsigned kAll = 0xffffffffu;

    for (int64_t n = n0; n < n_end && tid < ncols; ++n) {
        const int p = (int)(n & 1), q = p ^ 1;
        // the table value of the next step, loaded while this step runs
        const float src_next = (P2P && !tmm && tid == 0 && n + 1 < n_end && n + 1 < T->src_len) ? T->src[n + 1]
                                                                                               : 0.0f;
        // ---- P' of rows r0-1 .. r1 (FDTDEngineCPU.cpp:316-339); row i of the
        // band takes its lower Vy from vyd (the bottom ghost for row Rk)
        float uxl_ghost = 0.0f;
        auto prow = [&](auto ic, float vyd) {
            constexpr int i = decltype(ic)::value;
            const float ux = fmul(VX[i], dX[i]);
            float uxl = __shfl_up_sync(kAll, ux, 1);
            if (i == 0) uxl = uxl_ghost;
            else if (lane == 0) uxl = eUX[warp * (RMAX + 1) + i];
            const float uy = fmul(VY[i], dY[i]), uyb = fmul(vyd, dY[i + 1]);
            float pn;
            if constexpr (FAST) {
                const float ks = fmul(K1, fadd(fsub(ux, uxl), fsub(uy, uyb)));
                pn = __fmaf_rn(-ks, rcp_approx(dP[i]), P[i]);
                if (dsc[i]) pn = fmul(pn, tabA[dsc[i]].z);
            } else {
                const float num = fsub(fmul(P[i], dP[i]), fmul(K1, fadd(fsub(ux, uxl), fsub(uy, uyb))));
                const int tc = cw[i] & CODE_TYPE_MASK;
                float den = dP[i];
                if (tc != VS_CELL_AIR) {
                    const float sg = sSig[tc];
                    den = eigen ? fadd(fmul(sg, dP[i]), dP[i]) : fmul(fadd(1.0f, sg), dP[i]);
                }
                pn = fdiv_z(num, den);
                if (dirichlet && tc == VS_CELL_NOPRESSURE) pn = 0.0f;
            }
            if (mine && !(i == 0 && ifirst == 1)) P[i] = pn;
            if (i == lis_i && i >= 1) store_trace(rs, trace + (n - run_start), pn);
            if (lane == 0 && i >= 1) eP[warp * (RMAX + 1) + i] = P[i];
        };
        int bad = 0;
        if (P2P) {
            // rows 1 .. Rk-1 need no ghost value: they run while the neighbours' rows arrive
            static_for<1, RMAX>([&](auto ic) {
                constexpr int i = decltype(ic)::value;
                if (i < Rk) prow(ic, VY[i + 1]);
            });
            if (n > n0) {
                // every thread polls the arrival of this step's ghosts (bounded)
                const uint32_t par = (phase >> p) & 1u;
                phase ^= 1u << p;
                if (!mbar_wait_parity_bounded(bar + p, par, limit)) bad = 1;
            }
        }
        // ghost values of this step
        const float2 gt = gT[p * pitch + cc];
        VX[0] = gt.x;
        VY[0] = gt.y;
        vyb = gVyB[p * pitch + cc];
        uxl_ghost = c - 1 >= 0 ? fmul(gT[p * pitch + c - 1].x, sdX0[c - 1]) : 0.0f;
        if (P2P) {
            prow(std::integral_constant<int, 0>{}, VY[1]);
            static_for<1, RMAX + 1>([&](auto ic) {
                if (decltype(ic)::value == Rk) prow(ic, vyb);
            });
        } else {
            static_for<0, RMAX + 1>([&](auto ic) {
                constexpr int i = decltype(ic)::value;
                if (i <= Rk) prow(ic, i == Rk ? vyb : VY[i + 1 <= RMAX ? i + 1 : RMAX]);
            });
        }
        if (two_mass_warp) publish_pexc_tagged(n);
        else publish_pexc();
        if (P2P) {
            // this step's two-mass value from the ring slot its warp filled
            if (tid == 0 && tmm) {
                const volatile unsigned long long* e = exr + (n & (kExeRing - 1));
                unsigned long long v = *e;
                for (uint32_t i = 1; (uint32_t)(v >> 32) != (uint32_t)n && i < limit; ++i) v = *e;
                if ((uint32_t)(v >> 32) == (uint32_t)n) sExe[p] = __uint_as_float((uint32_t)v);
                else bad = 1;
            }
            if (cols_sync_or(ncols, bad)) {
                fail = true;
                break;
            }
            if (n + 1 < n_end && !tmm && tid == 0) sExe[q] = src_next;
        } else {
            __syncthreads();
            if (n + 1 < n_end) {
                if (tmm_thread) {
                    send_exe(q, tmm_finish_next(*sPexc));
                    if (thist) tmm_slot_hist(slot, tmm64, thist + 6 * (n + 2 - run_start));
                } else if (!tmm && tid == 0) {
                    sExe[q] = n + 1 < T->src_len ? T->src[n + 1] : 0.0f;
                }
            }
        }
        const float exeV = sExe[p];
        // ---- V' of rows r0 .. r1 (FDTDEngineCPU.cpp:364-410)
#pragma unroll
        for (int i = 1; i <= RMAX; ++i) {
            if (i > Rk) break;
            float pr = __shfl_down_sync(kAll, P[i], 1);
            if (lane == 31) pr = eP[(warp + 1) * (RMAX + 1) + i];
            if (c + 1 > W - 2) pr = 0.0f;                    // the ring column
            const float pc = P[i], pt = P[i - 1];
            float vx = VX[i], vy = VY[i];
            const uint32_t w = cw[i];
            const int cls = (int)(w >> 24);
            if constexpr (FAST) {
                vx = fsub(vx, fmul(bco, fsub(pr, pc)));
                vy = fsub(vy, fmul(bco, fsub(pt, pc)));
                const int d = (int)dsc[i];
                if (d) {
                    const float4 da = tabA[d];
                    vx = fmul(vx, da.x);
                    vy = fmul(vy, da.y);
                    if (cls == V_GENERIC) {
                        const float4 db = tabB[d];
                        vx = __fmaf_rn(da.w, exeV, __fmaf_rn(-db.y, pr, __fmaf_rn(db.x, pc, vx)));
                        vy = __fmaf_rn(-db.w, pt, __fmaf_rn(db.z, pc, vy));
                    }
                }
            } else if (cls == V_GENERIC) {
                const VelocityOut v = velocity_generic((int)(w & 0xff), (int)((w >> 8) & 0xff), (int)((w >> 16) & 0xff),
                                                       pc, pr, pt, vx, vy, exeV, sSig, zval, bco, dir0, dir1, dir2, dir3);
                vx = v.vx;
                vy = v.vy;
            } else {
                vx = fsub(vx, fmul(bco, fsub(pr, pc)));
                vy = fsub(vy, fmul(bco, fsub(pt, pc)));
                if (cls == V_BETA1) {
                    const float sc = sSig[w & CODE_TYPE_MASK];
                    vx = fdiv_z(vx, fadd(1.0f, fmaxf(sc, sSig[(w >> 8) & CODE_TYPE_MASK])));
                    vy = fdiv_z(vy, fadd(1.0f, fmaxf(sc, sSig[(w >> 16) & CODE_TYPE_MASK])));
                }
            }
            if (mine) {
                VX[i] = vx;
                VY[i] = vy;
                if (P2P) {
                    if (n + 1 < n_end) {
                        if (i == Rk && dn_gT_a)
                            st_async_v2(dn_gT_a + 8u * (uint32_t)(q * pitch + c), vx, vy, dn_bar_a + 8u * q);
                        if (i == 1 && up_gVyB_a)
                            st_async_b32(up_gVyB_a + 4u * (uint32_t)(q * pitch + c), vy, up_bar_a + 8u * q);
                    }
                } else {
                    if (i == Rk && dn_gT) dn_gT[(size_t)q * pitch + c] = make_float2(vx, vy);
                    if (i == 1 && up_gVyB) up_gVyB[(size_t)q * pitch + c] = vy;
                }
            }
            if (lane == 31) eUX[(warp + 1) * (RMAX + 1) + i] = fmul(VX[i], dX[i]);
        }
        if (hist && mine) {
            float* h = hist + (n + 1 - run_start) * 3 * pl;
#pragma unroll
            for (int i = 1; i <= RMAX; ++i) {
                if (i > Rk) break;
                const int64_t o = (int64_t)(r0 - 1 + i) * pitch + c;
                h[o] = P[i];
                h[pl + o] = VX[i];
                h[2 * pl + o] = VY[i];
            }
        }
        if (P2P) {
            // one thread arrives on the barrier of the next step's ghosts, expecting
            // the bytes both neighbours send; the block barrier publishes the edges
            if (n + 1 < n_end && tid == 0) mbar_expect_tx(bar + q, expect);
            cols_sync(ncols);
        } else {
            asm volatile("barrier.cluster.arrive.release;" ::: "memory");
            if (tmm_thread && n + 2 < n_end) tmm_prepare_next();
            asm volatile("barrier.cluster.wait.acquire;" ::: "memory");
        }
    }
    if (two_mass_warp && tmm_thread) {
        // the two-mass warp: the excitation value of step n + 1 from the
        // owner's P' of step n, then the state-only part of the next step
        for (int64_t n = n0; n + 1 < n_end; ++n) {
            unsigned long long v = pexw[n & 1];
            for (uint32_t i = 1; (uint32_t)(v >> 32) != (uint32_t)n && i < limit; ++i) v = pexw[n & 1];
            if ((uint32_t)(v >> 32) != (uint32_t)n) {
                fail = true;
                break;
            }
            send_exe_ring(n + 1, tmm_finish_next(__uint_as_float((uint32_t)v)));
            if (thist) tmm_slot_hist(slot, tmm64, thist + 6 * (n + 2 - run_start));
            if (n + 2 < n_end) tmm_prepare_next();
        }
    }
    if (P2P) {
        if (fail) {
            // a neighbour may still be sending: give its stores time to land
            // before the CTAs meet, and leave the state as it is
            if (tid == 0 || tmm_thread) atomicExch(&rs->error, VS_ERR_TIMEOUT);
            for (int i = 0; i < 64; ++i) __nanosleep(1000);
        }
        cluster.sync();                          // no CTA exits while another may store into it
        if (fail) return;
    }

    // ---- the state of step n_end back to its parity set
    const int pe = (int)(n_end & 1);
    float* __restrict__ oP = T->P[0] + pe * pl;
    if (mine) {
#pragma unroll
        for (int i = 1; i <= RMAX; ++i) {
            if (i > Rk) break;
            const int64_t o = (int64_t)(r0 - 1 + i) * pitch + c;
            oP[o] = P[i];
            oP[2 * pl + o] = VX[i];
            oP[4 * pl + o] = VY[i];
        }
    }
    if (tmm_thread) {
        if (tmm64) T->tmm64[pe] = slot->s64;
        else T->tmm[pe] = slot->s32;
    }
}

}  // namespace

size_t cluster_smem_bytes(int pitch, int rows_max, bool fast) { return cluster_layout(pitch, rows_max, fast).bytes; }

// Cluster size, threads and shared memory for one tube of H x W (pitch), or
// false when no cluster of at least 4 CTAs fits on this device.
namespace {

// The register form is compiled for at most 4 or 8 rows per band and 256 or
// 512 threads per CTA (a thread per column; 256 threads leave 255 registers
// per thread).
template <bool FAST, int SYNC>
const void* reg_fn(int rmax, int cols) {
    if (rmax <= 4) return cols <= 256 ? (const void*)cluster_reg_kernel<FAST, 4, 256, SYNC>
                                      : (const void*)cluster_reg_kernel<FAST, 4, 512, SYNC>;
    return cols <= 256 ? (const void*)cluster_reg_kernel<FAST, 8, 256, SYNC>
                       : (const void*)cluster_reg_kernel<FAST, 8, 512, SYNC>;
}

// form 0: shared-memory bands; register form with 1: a cluster barrier per
// step, 2: the point-to-point neighbour exchange, 3: the exchange and the
// two-mass model in its own warp
const void* cluster_fn(bool fast, int form, int rmax, int cols) {
    if (form == 0) return fast ? (const void*)cluster_kernel<true> : (const void*)cluster_kernel<false>;
    if (form == 1) return fast ? reg_fn<true, 0>(rmax, cols) : reg_fn<false, 0>(rmax, cols);
    if (form == 2) return fast ? reg_fn<true, 1>(rmax, cols) : reg_fn<false, 1>(rmax, cols);
    return fast ? reg_fn<true, 2>(rmax, cols) : reg_fn<false, 2>(rmax, cols);
}

template <bool FAST, int SYNC>
cudaError_t launch_reg(const cudaLaunchConfig_t& cfg, int rmax, int cols, const TubeDev* tube, RunState* rs,
                       int64_t steps) {
    if (rmax <= 4)
        return cols <= 256 ? cudaLaunchKernelEx(&cfg, cluster_reg_kernel<FAST, 4, 256, SYNC>, tube, rs, steps)
                           : cudaLaunchKernelEx(&cfg, cluster_reg_kernel<FAST, 4, 512, SYNC>, tube, rs, steps);
    return cols <= 256 ? cudaLaunchKernelEx(&cfg, cluster_reg_kernel<FAST, 8, 256, SYNC>, tube, rs, steps)
                       : cudaLaunchKernelEx(&cfg, cluster_reg_kernel<FAST, 8, 512, SYNC>, tube, rs, steps);
}

// The register form's step synchronisation: point to point (form 2), or for
// two-mass tubes point to point with the model in its own warp (form 3, up
// to 256 columns: the extra warp lowers every thread's register budget), else
// the cluster barrier (form 1).  The exact arithmetic's 512-column variants
// spill and measured slower point to point.
int reg_form(bool fast, bool tmm, int cols) {
    if (tmm) return cols <= 256 ? 3 : 1;
    return fast || cols <= 256 ? 2 : 1;
}

}  // namespace

bool cluster_config(int H, int W, int pitch, bool fast, bool tmm, ClusterConfig* out) {
    const int NR = H - 2;
    if (NR < 4) return false;
    int dev = 0, optin = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return false;
    if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) return false;
    const int cols = std::min(512, (W + 31) / 32 * 32);     // a thread per column
    for (int C : {16, 8, 4}) {
        if (C > NR) continue;
        const int R = (NR + C - 1) / C;
        // the register-resident form where a band has at most 8 rows and a
        // thread per column fits a CTA, the shared-memory form otherwise
        const int form = (R <= 8 && W <= 512) ? reg_form(fast, tmm, cols) : 0;
        const int rmax = R <= 4 ? 4 : 8;
        const int threads = cols + (form == 3 ? 32 : 0);         // + the two-mass warp
        const void* fn = cluster_fn(fast, form, rmax, cols);
        const size_t smem = form ? reg_layout(pitch, threads, rmax, fast).bytes : cluster_layout(pitch, R, fast).bytes;
        if (smem > (size_t)optin) continue;
        if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) continue;
        if (C > 8 && cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess)
            continue;
        cudaLaunchConfig_t cfg{};
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = C;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.gridDim = dim3(C);
        cfg.blockDim = dim3(threads);
        cfg.dynamicSmemBytes = smem;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        int nclusters = 0;
        if (cudaOccupancyMaxActiveClusters(&nclusters, fn, &cfg) != cudaSuccess || nclusters < 1) {
            cudaGetLastError();
            continue;
        }
        out->ctas = C;
        out->threads = threads;
        out->cols = cols;
        out->rows_max = R;
        out->smem = smem;
        out->form = form;
        out->rmax = rmax;
        out->nclusters = nclusters;
        return true;
    }
    cudaGetLastError();
    return false;
}

cudaError_t launch_cluster_run(const TubeDev* tube, RunState* rs, int64_t steps, bool fast, const ClusterConfig& c,
                               cudaStream_t stream, int ntubes) {
    if (steps <= 0 || ntubes <= 0) return cudaSuccess;
    cudaLaunchConfig_t cfg{};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = c.ctas;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3(c.ctas, ntubes);                      // clusters along x, a tube per grid row
    cfg.blockDim = dim3(c.threads);
    cfg.dynamicSmemBytes = c.smem;
    cfg.stream = stream;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaError_t e;
    if (c.form == 1)
        e = fast ? launch_reg<true, 0>(cfg, c.rmax, c.cols, tube, rs, steps)
                 : launch_reg<false, 0>(cfg, c.rmax, c.cols, tube, rs, steps);
    else if (c.form == 2)
        e = fast ? launch_reg<true, 1>(cfg, c.rmax, c.cols, tube, rs, steps)
                 : launch_reg<false, 1>(cfg, c.rmax, c.cols, tube, rs, steps);
    else if (c.form == 3)
        e = fast ? launch_reg<true, 2>(cfg, c.rmax, c.cols, tube, rs, steps)
                 : launch_reg<false, 2>(cfg, c.rmax, c.cols, tube, rs, steps);
    else if (fast)
        e = cudaLaunchKernelEx(&cfg, cluster_kernel<true>, tube, rs, steps, c.rows_max);
    else
        e = cudaLaunchKernelEx(&cfg, cluster_kernel<false>, tube, rs, steps, c.rows_max);
    // the step counter advances after every cluster has run: a cluster of a
    // later wave reads RunState::step when it starts
    for (int64_t left = steps; e == cudaSuccess && left > 0; left -= INT32_MAX)
        e = launch_advance(rs, (int)std::min<int64_t>(left, INT32_MAX), stream);
    return e;
}

}  // namespace vsb
