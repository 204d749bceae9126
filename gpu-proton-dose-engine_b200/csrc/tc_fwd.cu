// tc_fwd.cu -- forward dose on the 5th-generation tensor cores (tcgen05, TMEM accumulators),
// warp-specialised and software-pipelined across (layer, slice) steps.
//
// For every active (layer l, slice z) and 128 x 128 lateral tile:
//
//   stage 1   U[x, j]  = sum_i Gx[x, i] W[j, i]        M = 128 (x), N = N1 (j), K = K1 (i)
//   stage 2   D[y, x] += sum_j Gy[y, j] (s U)[x, j]     M = 128 (y), N = 128 (x), K = N1 (j)
//
// with s = IDD_l(z) / (2 pi sigma^2) and unnormalised Gaussians exp(-d^2 / (2 sigma^2))
// (engines.py:191-197 contracted in the cheap order).  Nothing Gaussian is stored in HBM:
// the factors of each (layer, slice) are regenerated on the chip.
//
// CTA = 8 math warps, 1 scheduler warp, 1 MMA warp; one CTA per SM (persistent).
//  * Scheduler warp: pulls work units (slice z, chunk c of <= C active layers, tile) from an
//    atomic counter in z-major order -- the shallow slices, which see the most layers, come
//    first -- reads the slice's column of the IDD table and pushes one step per active layer
//    of its chunk (layer, exponent scale, dose scale, first / last flags) into an 8-deep ring
//    of shared-memory slots guarded by full / empty mbarriers.
//  * Math warps (each on its own, no block barrier in the steady state):
//      at a unit's first step: squared distances (x - xs)^2, (y - ys)^2 of the tile, formed
//          in FP64 and kept in FP32 in a per-thread shared-memory table (padding = +inf)
//      G   Gy -> A2[n & 1] (smem, two buffers), Gx -> TMEM (stage 1's A operand), W -> B1
//          (smem; its loads are issued first), each Gaussian = ex2(-d^2 * a2); then arrive
//          on `ops1`
//      DR  previous step's stage-2 result: D from TMEM into registers; at the end of a unit
//          the unit's small accumulator too, and the unit's output (below)
//      E1  stage-1 result: U from TMEM, scaled by s, split, stored as stage 2's B; arrive
//          on `ops2`
//  * MMA warp: waits for `ops1` / `ops2` and issues stage 1 (A from TMEM, "TS" form) and
//    stage 2 (both operands in smem), each followed by a tcgen05.commit to `mma1` / `mma2`.
//  Stage 2 of step n-1 runs under G of step n, stage 1 of step n under DR.
//
// Accumulation.  The tensor core's FP32 accumulation aligns and truncates, so its error
// grows with the MMA steps into one accumulator.  The large hi*hi products of each step go
// to a fresh accumulator (6 steps at K = 48) that is read back and added in FP32 registers
// (IEEE round to nearest); the two small cross products (~2^-11 of the large ones) stay in
// one TMEM accumulator for the whole unit and are read once at its end.
//
// Output.  Each math warp owns 32 rows x 64 columns of the tile.  A unit whose chunk holds
// every active layer of its slice writes its dose rows directly.  Otherwise the warp writes
// its partial rows, and the warp that completes the last chunk of those rows (per-(slice,
// tile, warp) arrival counter) sums the partials in chunk order -- deterministic whichever
// CTA gets there -- and writes the dose.  With the masked quadratic loss the same writer
// forms dL/dD = 2 m (D - P) and an FP64 partial sum of m (D - P)^2 for its rows.
// Per-layer maps (a job with layer_stride > 0, no loss): every step is its own output --
// the layer's dose rows go to dose + l * layer_stride -- while the unit's steps still share
// its squared-distance tables (kTab on the first step only); slices no layer reaches are
// not written.
//
// Every wait is bounded (2 s of %globaltimer, or a test limit).  A warp whose wait runs out
// sets the error word and leaves its loop; the waits of the others then run out in turn.
// The dose is invalid after that and the callers poison the results (NaN) from the error
// word.  A warp leaves only after the MMAs it issued have completed (or its wait for them ran
// out), and the block frees its TMEM after a final barrier of all warps.
//
// Precision modes (accumulation always FP32):
//   TF32X3  a b ~ ah bh + ah bl + al bh with ah = tf32(a), al = tf32(a - ah)  (~1e-7)
//   TF32    ah bh
//   BF16X3  the same split with bf16 hi / lo parts
//   BF16    ah bh in bf16
#include <algorithm>
#include <math.h>

#include "pbd_internal.cuh"
#include "tc_common.cuh"

namespace pbd {
namespace {
using namespace tcc;

constexpr int kMathWarps = kTcFwdWarps;
constexpr int kMath = 32 * kMathWarps;     // 256 math threads: warpgroups 0 and 1
constexpr int kSchedWarp = kMathWarps;     // warpgroup 2: warp 8 schedules, warps 9-11 issue
constexpr int kMmaWarp = kMathWarps + 1;   // the MMAs of one accumulator chain each (below)
constexpr int kThreads = kMath + 128;
// Register split (setmaxnreg): the block launches with 168 registers per thread (12 warps,
// three per SM sub-partition); the control warpgroup gives registers back and the math
// warpgroups take them: 8 * 32 * 208 + 4 * 32 * 80 = 63,488 <= 384 * 168 = 64,512.
constexpr int kMathRegs = 208, kCtrlRegs = 80;
constexpr int kLaunchRegsNeeded = (kMath * kMathRegs + 128 * kCtrlRegs + kThreads - 1) / kThreads;
constexpr int kRing = 8;                   // step slots
constexpr uint32_t kCols = 512;
// TMEM columns: stage-2 big [0,128), unit small [128,256), stage-1 big / small
// [256, 256 + N1) / [320, 320 + N1), stage-1 A operand hi / lo [384, +K1) / [448, +K1)
constexpr uint32_t kColD = 0, kColS = 128, kColUb = 256, kColUs = 320, kColAh = 384, kColAl = 448;

// kFirst / kLast: the step opens / closes an accumulation (and its output); kTab: the step
// builds the unit's squared-distance tables.
enum : int { kFirst = 1, kLast = 2, kEnd = 4, kZero = 8, kTab = 16 };

struct Step {
    int job, z, tile, l;
    int chunk, nch, flags, nsx;
    float a2, scale;
    const float* w;     // W_l (nsy, nsx): the math warps load it at the top of the step
    int nsy, pad;
};

struct Params {
    const JobDev* jobs;
    int n_jobs, chunk, cmax, tmax, n_units;
    int* counter;       // [0] unit counter
    int* err;           // error word: set when a bounded wait ran out
    unsigned long long wait_ns;   // limit of every bounded wait
    int hold;           // test of the timeout path: the scheduler publishes no step
    int with_loss;
    int K1, N1, na2;    // operand dims; A2 buffers (1 or 2)
    int ty4, tx4;       // float4 groups of the per-thread distance table: y part, x part
};

// ------------------------------------------------------------------------------------------
// Scheduler warp: units -> steps.
// ------------------------------------------------------------------------------------------
template <bool MAPS>
__device__ __forceinline__ void scheduler_warp(const Params& P, Step* ring, uint64_t* full, uint64_t* empty) {
    const int lane = threadIdx.x & 31;
    const unsigned FULL = 0xffffffffu;
    int k = 0;
    bool ok = true;

    // Wait for slot k to be free; lane `src` writes it and arrives on `full`.
    auto push = [&](int src, const Step& st) -> bool {
        const int slot = k % kRing, n = k / kRing;
        const bool w = wait_bar(&empty[slot], (uint32_t)((n & 1) ^ 1), P.wait_ns);
        if (!__all_sync(FULL, w)) return false;
        if (lane == src) {
            ring[slot] = st;
            tc::mbar_arrive(&full[slot]);
        }
        __syncwarp();
        ++k;
        return true;
    };

    // timeout-path test: publish nothing, so that every consumer's first wait runs out
    if (P.hold) return;
    for (;;) {
        int u = 0;
        if (lane == 0) u = atomicAdd(P.counter, 1);
        u = __shfl_sync(FULL, u, 0);
        if (u >= P.n_units) break;
        int v = u;
        const int tile = v % P.tmax; v /= P.tmax;
        const int job = v % P.n_jobs; v /= P.n_jobs;
        const int c = v % P.cmax;
        const int z = v / P.cmax;
        const JobDev& J = P.jobs[job];
        const int nz = J.nz, nl = J.nl;
        if (z >= nz || tile >= J.ntx * J.nty) continue;
        const double* idd = J.idd;
        int tot = 0;   // active layers of slice z
        for (int b = 0; b < nl; b += 32) {
            const int l = b + lane;
            const bool a = l < nl && idd[(size_t)l * nz + z] != 0.0;
            tot += __popc(__ballot_sync(FULL, a));
        }
        if (tot == 0) {
            // a slice no layer reaches: the math warps write zeros (and loss); per-layer
            // maps have nothing to write
            if (c == 0 && !MAPS) {
                Step st{};
                st.job = job; st.z = z; st.tile = tile;
                st.nch = 1; st.flags = kFirst | kLast | kZero;
                if (!push(0, st)) { ok = false; break; }
            }
            continue;
        }
        const int nch = (tot + P.chunk - 1) / P.chunk;
        if (c >= nch) continue;
        const int r0 = c * P.chunk, r1 = min(tot, r0 + P.chunk);
        int rank = 0;
        for (int b = 0; b < nl && rank < r1 && ok; b += 32) {
            const int l = b + lane;
            const double iv = l < nl ? idd[(size_t)l * nz + z] : 0.0;
            const bool a = iv != 0.0;
            const unsigned bal = __ballot_sync(FULL, a);
            const int my = rank + __popc(bal & ((1u << lane) - 1u));
            const bool mine = a && my >= r0 && my < r1;
            Step st{};
            if (mine) {
                const double s = fmax(J.sigma[(size_t)l * nz + z], 1e-9);
                st.job = job; st.z = z; st.tile = tile; st.l = l;
                st.chunk = c; st.nch = nch;
                st.nsx = J.nsx; st.nsy = J.nsy;
                st.w = J.w + (size_t)l * J.nsy * J.nsx;
                st.flags = MAPS ? (kFirst | kLast | (my == r0 ? kTab : 0))
                                : ((my == r0 ? kFirst | kTab : 0) | (my == r1 - 1 ? kLast : 0));
                st.a2 = (float)(kLog2e / (2.0 * s * s));
                st.scale = (float)(iv * kInv2Pi / (s * s));
            }
            unsigned emit = __ballot_sync(FULL, mine);
            while (emit) {
                const int src = __ffs(emit) - 1;
                emit &= emit - 1u;
                if (!push(src, st)) { ok = false; break; }
            }
            rank += __popc(bal);
        }
        if (!ok) break;
    }
    if (ok) {
        Step st{};
        st.flags = kEnd;
        (void)push(0, st);
    }
}

// ------------------------------------------------------------------------------------------
// MMA warp.
// ------------------------------------------------------------------------------------------
template <int MODE>
struct Issue {
    using Pr = Prec<MODE>;
    __device__ static void mma_ss(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
        if (Pr::EB == 4) tc::mma_tf32(d, a, b, idesc, acc);
        else tc::mma_bf16(d, a, b, idesc, acc);
    }
    __device__ static void mma_ts(uint32_t d, uint32_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
        if (Pr::EB == 4) tc::mma_tf32_ts(d, a, b, idesc, acc);
        else tc::mma_bf16_ts(d, a, b, idesc, acc);
    }
    // Each MMA costs an issuing thread ~100+ cycles whatever its N, so the products go to
    // independent accumulators issued by different warps: chain 0 = the hi*hi products of
    // both stages, chain 1 = stage 1's two cross products, chain 2 = stage 2's.
    // Operand descriptors are built from shared-memory addresses at every k-step.

    // stage 1 (U = Gx (TMEM, K1) x W^T (smem B1, N1 rows, chunk planes plane_n1 apart))
    __device__ static void stage1_big(uint32_t tb, uint32_t b1h, uint32_t plane_n1, int steps,
                                      uint32_t idesc) {
        for (int st = 0; st < steps; ++st) {
            const uint32_t ob = (uint32_t)st * 2u * plane_n1;
            mma_ts(tb + kColUb, tb + kColAh + (uint32_t)st * 8u,
                   tc::smem_desc(b1h + ob, plane_n1, 128), idesc, st > 0 ? 1u : 0u);
        }
    }
    __device__ static void stage1_small(uint32_t tb, uint32_t b1h, uint32_t b1l, uint32_t plane_n1,
                                        int steps, uint32_t idesc) {
        for (int st = 0; st < steps; ++st) {
            const uint32_t ob = (uint32_t)st * 2u * plane_n1;
            mma_ts(tb + kColUs, tb + kColAh + (uint32_t)st * 8u,
                   tc::smem_desc(b1l + ob, plane_n1, 128), idesc, st > 0 ? 1u : 0u);
            mma_ts(tb + kColUs, tb + kColAl + (uint32_t)st * 8u,
                   tc::smem_desc(b1h + ob, plane_n1, 128), idesc, 1u);
        }
    }
    // stage 2 (D = Gy (smem A2) x (sU)^T (smem B2), chunk planes of 128 rows): big fresh,
    // small continues the unit's sum
    __device__ static void stage2_big(uint32_t tb, uint32_t a2h, uint32_t b2h, int steps,
                                      uint32_t idesc) {
        constexpr uint32_t plane = 128u * 16u;
        for (int st = 0; st < steps; ++st) {
            const uint32_t o = (uint32_t)st * 2u * plane;
            mma_ss(tb + kColD, tc::smem_desc(a2h + o, plane, 128), tc::smem_desc(b2h + o, plane, 128),
                   idesc, st > 0 ? 1u : 0u);
        }
    }
    __device__ static void stage2_small(uint32_t tb, uint32_t a2h, uint32_t a2l, uint32_t b2h,
                                        uint32_t b2l, int steps, uint32_t idesc, bool first) {
        constexpr uint32_t plane = 128u * 16u;
        for (int st = 0; st < steps; ++st) {
            const uint32_t o = (uint32_t)st * 2u * plane;
            mma_ss(tb + kColS, tc::smem_desc(a2h + o, plane, 128), tc::smem_desc(b2l + o, plane, 128),
                   idesc, (first && st == 0) ? 0u : 1u);
            mma_ss(tb + kColS, tc::smem_desc(a2l + o, plane, 128), tc::smem_desc(b2h + o, plane, 128),
                   idesc, 1u);
        }
    }
};

// Shared-memory layout (byte offsets from the dynamic base).
struct Layout {
    uint32_t b1h, b1l, b2h, b2l, a2, a2_lo, a2_stride, tab;
};

template <int MODE>
__device__ __forceinline__ Layout make_layout(int K1, int N1, int na2) {
    using Pr = Prec<MODE>;
    constexpr uint32_t NARR = Pr::NPROD == 3 ? 2 : 1;
    const uint32_t b1 = (uint32_t)N1 * K1 * Pr::EB, op = 128u * N1 * Pr::EB;
    Layout L;
    L.b1h = 0;
    L.b1l = L.b1h + (NARR == 2 ? b1 : 0u);
    L.b2h = L.b1l + b1;
    L.b2l = L.b2h + (NARR == 2 ? op : 0u);
    L.a2 = L.b2l + op;
    L.a2_lo = NARR == 2 ? op : 0u;
    L.a2_stride = NARR * op;
    L.tab = L.a2 + (uint32_t)na2 * L.a2_stride;
    return L;
}

// One MMA issuer warp.  role 0: hi*hi chains of both stages (commits to mma1 and mma2);
// role 1: stage 1's cross products (mma1); role 2: stage 2's cross products (mma2).
template <int MODE>
__device__ __forceinline__ void mma_warp(const Params& P, const Layout& L, uint32_t sbase, uint32_t tb, int role,
                         const Step* ring, uint64_t* full, uint64_t* empty, uint64_t* bars) {
    using Pr = Prec<MODE>;
    using I = Issue<MODE>;
    const int lane = threadIdx.x & 31;
    uint64_t* ops1 = bars + 0;
    uint64_t* ops2 = bars + 1;
    uint64_t* mma1 = bars + 2;
    uint64_t* mma2 = bars + 3;
    const uint32_t idesc1 = tc::instr_desc(128, P.N1, Pr::FMT);
    const uint32_t idesc2 = tc::instr_desc(128, 128, Pr::FMT);
    const uint32_t plane_n1 = (uint32_t)P.N1 * 16u;
    const int steps1 = P.K1 / Pr::KSTEP, steps2 = P.N1 / Pr::KSTEP;
    const bool do1 = role != 2, do2 = role != 1;
    int k = 0, n = 0;
    bool ok = true;
    for (;;) {
        const int slot = k % kRing;
        ok = wait_bar(&full[slot], (uint32_t)((k / kRing) & 1), P.wait_ns);
        const int flags = ring[slot].flags;
        __syncwarp();
        if (lane == 0) tc::mbar_arrive(&empty[slot]);
        ++k;
        if (!__all_sync(0xffffffffu, ok)) break;
        if (flags & kEnd) break;
        if (flags & kZero) continue;
        const uint32_t par = (uint32_t)(n & 1);
        const uint32_t a2h = sbase + L.a2 + (P.na2 == 2 ? (uint32_t)(n & 1) * L.a2_stride : 0u);
        if (do1) {
            ok = wait_bar(ops1, par, P.wait_ns);
            if (!__all_sync(0xffffffffu, ok)) break;
            tc::fence_after_sync();
            if (lane == 0) {
                if (role == 0) I::stage1_big(tb, sbase + L.b1h, plane_n1, steps1, idesc1);
                else I::stage1_small(tb, sbase + L.b1h, sbase + L.b1l, plane_n1, steps1, idesc1);
                tc::commit(mma1);
            }
            __syncwarp();
        }
        if (do2) {
            ok = wait_bar(ops2, par, P.wait_ns);
            if (!__all_sync(0xffffffffu, ok)) break;
            tc::fence_after_sync();
            if (lane == 0) {
                if (role == 0)
                    I::stage2_big(tb, a2h, sbase + L.b2h, steps2, idesc2);
                else
                    I::stage2_small(tb, a2h, a2h + L.a2_lo, sbase + L.b2h, sbase + L.b2l, steps2,
                                    idesc2, (flags & kFirst) != 0);
                tc::commit(mma2);
            }
            __syncwarp();
        }
        ++n;
    }
    if (!ok && lane == 0) atomicExch(P.err, 1);
    // this warp's last MMAs must be complete before the block frees its TMEM
    if (n > 0) {
        if (do1) (void)wait_bar(mma1, (uint32_t)((n - 1) & 1), P.wait_ns);
        if (do2) (void)wait_bar(mma2, (uint32_t)((n - 1) & 1), P.wait_ns);
    }
}

// ------------------------------------------------------------------------------------------
// Math warps.
// ------------------------------------------------------------------------------------------
// Dose (and loss) of 64 voxels of row y from column xb (v = null: zeros); returns the FP64
// sum of m (D - P)^2.  The mask and prescription are loaded four float4s at a time before any
// store, so their round trips overlap (the stores could alias the loads otherwise).
__device__ __forceinline__ double write_final(const JobDev& J, int z, int y, int xb,
                                              const float* v, int with_loss) {
    double lsum = 0.0;
    if (y >= J.ny) return lsum;
    const size_t o = ((size_t)z * J.ny + y) * J.nx + xb;
    float* __restrict__ d = J.dose + o;
    const bool vec = xb + 64 <= J.nx && (J.nx & 3) == 0;
    if (!with_loss) {
#pragma unroll
        for (int q = 0; q < 64; q += 4) {
            float x4[4];
#pragma unroll
            for (int r = 0; r < 4; ++r) x4[r] = v ? v[q + r] : 0.f;
            if (vec) {
                *reinterpret_cast<float4*>(d + q) = make_float4(x4[0], x4[1], x4[2], x4[3]);
            } else {
#pragma unroll
                for (int r = 0; r < 4; ++r)
                    if (xb + q + r < J.nx) d[q + r] = x4[r];
            }
        }
        return lsum;
    }
    const float* __restrict__ mk = J.mask + o;
    const float* __restrict__ pr = J.presc + o;
    float* __restrict__ g = J.grad_dose + o;
#pragma unroll
    for (int h = 0; h < 64; h += 16) {
        float m8[16], p8[16];
#pragma unroll
        for (int q = 0; q < 16; q += 4) {
            if (vec) {
                const float4 a = __ldg(reinterpret_cast<const float4*>(mk + h + q));
                const float4 b = __ldg(reinterpret_cast<const float4*>(pr + h + q));
                m8[q] = a.x; m8[q + 1] = a.y; m8[q + 2] = a.z; m8[q + 3] = a.w;
                p8[q] = b.x; p8[q + 1] = b.y; p8[q + 2] = b.z; p8[q + 3] = b.w;
            } else {
#pragma unroll
                for (int r = 0; r < 4; ++r) {
                    const bool in = xb + h + q + r < J.nx;
                    m8[q + r] = in ? mk[h + q + r] : 0.f;
                    p8[q + r] = in ? pr[h + q + r] : 0.f;
                }
            }
        }
#pragma unroll
        for (int q = 0; q < 16; q += 4) {
            float x4[4], r4[4];
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                x4[r] = v ? v[h + q + r] : 0.f;
                r4[r] = x4[r] - p8[q + r];
                lsum += (double)m8[q + r] * (double)r4[r] * (double)r4[r];
            }
            if (vec) {
                *reinterpret_cast<float4*>(d + h + q) = make_float4(x4[0], x4[1], x4[2], x4[3]);
                *reinterpret_cast<float4*>(g + h + q) =
                    make_float4(2.f * m8[q] * r4[0], 2.f * m8[q + 1] * r4[1], 2.f * m8[q + 2] * r4[2],
                                2.f * m8[q + 3] * r4[3]);
            } else {
#pragma unroll
                for (int r = 0; r < 4; ++r)
                    if (xb + h + q + r < J.nx) {
                        d[h + q + r] = x4[r];
                        g[h + q + r] = 2.f * m8[q + r] * r4[r];
                    }
            }
        }
    }
    return lsum;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

template <int MODE, bool MAPS>
__device__ __forceinline__ void math_warps(const Params& P, const Layout& L, uint8_t* smem, uint32_t tb,
                           const Step* ring, uint64_t* full, uint64_t* empty, uint64_t* bars) {
    using Pr = Prec<MODE>;
    constexpr int NARR = Pr::NPROD == 3 ? 2 : 1;
    constexpr int EPC = Pr::EPC;                    // elements per 16-byte operand chunk
    constexpr int EPG = Pr::EB == 4 ? 8 : 16;       // elements per 8 TMEM columns
    constexpr int kWReg = 4;                        // B1 chunks per thread (<= 64 x 64 lattice)
    uint64_t* ops1 = bars + 0;
    uint64_t* ops2 = bars + 1;
    uint64_t* mma1 = bars + 2;
    uint64_t* mma2 = bars + 3;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int K1 = P.K1, N1 = P.N1, K2 = P.N1;
    const int sp = warp & 3, half = warp >> 2;
    const uint32_t lane_base = (uint32_t)(32 * sp) << 16;
    const int trow = 32 * sp + lane;                // TMEM lane = tile row of this thread
    const uint32_t plane128 = 128u * 16u, plane_n1 = (uint32_t)N1 * 16u;
    const int nb1 = N1 * (K1 / EPC);                // B1 chunks
    const int ny_chunks = 128 * (K2 / EPC);          // A2 chunks
    const int nxg = K1 / EPG;                        // stage-1 A column groups
    const int nyr = ny_chunks / kMath;               // A2 chunks of every thread
    // per-thread maxima for K, N <= 64 (loops unrolled to these bounds, predicated)
    constexpr int kYR = 128 * (64 / EPC) / kMath;    // A2 chunks per thread
    constexpr int kXG = (64 / EPG) / 2;              // stage-1 A groups per thread
    // per-thread distance table: float4 groups [g][tid]; y part first, then x part
    float4* tab = reinterpret_cast<float4*>(smem + L.tab);

    // this thread's B1 chunks (row j, K group) -- fixed for the launch, so the divisions by
    // N1 are done once here rather than in every step
    int wrg[kWReg];                                 // row | group << 16, or -1
#pragma unroll
    for (int r = 0; r < kWReg; ++r) {
        const int e = tid + r * kMath;
        wrg[r] = e < nb1 ? (e % N1) | ((e / N1) << 16) : -1;
    }

    uint32_t ph1 = 0, ph2 = 0;
    bool ok = true;
    float dsum[64];
#pragma unroll
    for (int q = 0; q < 64; ++q) dsum[q] = 0.f;
    Step prev{};
    bool have_prev = false;
    int k = 0, n = 0;

    // D of the previous step into the registers (+ the unit's small sum when it ended it).
    auto drain = [&]() {
        ok = ok && wait_bar(mma2, ph2, P.wait_ns);
        if (ok) ph2 ^= 1;
        tc::fence_after_sync();
        uint32_t r[4][16];
#pragma unroll
        for (int c = 0; c < 4; ++c)
            tc::tmem_ld16(tb + kColD + lane_base + (uint32_t)(half * 64 + c * 16), r[c]);
        tc::tmem_wait_ld();
#pragma unroll
        for (int c = 0; c < 4; ++c)
#pragma unroll
            for (int q = 0; q < 16; ++q) dsum[c * 16 + q] += __uint_as_float(r[c][q]);
        if (Pr::NPROD == 3 && (prev.flags & kLast)) {
#pragma unroll
            for (int c = 0; c < 4; ++c)
                tc::tmem_ld16(tb + kColS + lane_base + (uint32_t)(half * 64 + c * 16), r[c]);
            tc::tmem_wait_ld();
#pragma unroll
            for (int c = 0; c < 4; ++c)
#pragma unroll
                for (int q = 0; q < 16; ++q) dsum[c * 16 + q] += __uint_as_float(r[c][q]);
        }
    };

    // Output of this warp's rows of a finished unit (dsum = its dose), then dsum = 0.
    auto output = [&](const Step& st) {
        const JobDev& J = P.jobs[st.job];
        const int ty = st.tile / J.ntx, tx = st.tile % J.ntx;
        const int y = ty * kTile + trow, xb = tx * kTile + half * 64;
        const int slot = (st.z * (J.ntx * J.nty) + st.tile) * kMathWarps + warp;
        if constexpr (MAPS) {
            // per-layer maps: this step's layer, written whole
            if (y < J.ny) {
                float* d = J.dose + (size_t)st.l * J.layer_stride +
                           ((size_t)st.z * J.ny + y) * J.nx + xb;
                const bool vec = xb + 64 <= J.nx && (J.nx & 3) == 0;
#pragma unroll
                for (int q = 0; q < 64; q += 4) {
                    if (vec) {
                        *reinterpret_cast<float4*>(d + q) =
                            make_float4(dsum[q], dsum[q + 1], dsum[q + 2], dsum[q + 3]);
                    } else {
#pragma unroll
                        for (int r = 0; r < 4; ++r)
                            if (xb + q + r < J.nx) d[q + r] = dsum[q + r];
                    }
                }
            }
        } else if (st.nch == 1) {
            const double ls = warp_sum(write_final(J, st.z, y, xb, dsum, P.with_loss));
            if (P.with_loss && lane == 0) J.loss_part[slot] = ls;
        } else {
            const size_t n3 = (size_t)J.nz * J.ny * J.nx;
            const bool vec = xb + 64 <= J.nx && (J.nx & 3) == 0;
            if (y < J.ny) {
                float* o = J.partial + (size_t)st.chunk * n3 + ((size_t)st.z * J.ny + y) * J.nx + xb;
#pragma unroll
                for (int q = 0; q < 64; q += 4) {
                    if (vec) {
                        *reinterpret_cast<float4*>(o + q) =
                            make_float4(dsum[q], dsum[q + 1], dsum[q + 2], dsum[q + 3]);
                    } else {
#pragma unroll
                        for (int r = 0; r < 4; ++r)
                            if (xb + q + r < J.nx) o[q + r] = dsum[q + r];
                    }
                }
            }
            __threadfence();
            __syncwarp();
            int last = 0;
            if (lane == 0) last = atomicAdd(&J.arrive[slot], 1) == st.nch - 1;
            last = __shfl_sync(0xffffffffu, last, 0);
            if (last) {
                // the partials of every chunk (this one's included) summed in chunk order;
                // dsum is free again once this chunk's partial is written
                __threadfence();
                float* v = dsum;
#pragma unroll
                for (int q = 0; q < 64; ++q) v[q] = 0.f;
                if (y < J.ny) {
                    const float* base = J.partial + ((size_t)st.z * J.ny + y) * J.nx + xb;
                    for (int c = 0; c < st.nch; ++c) {
                        const float* pc = base + (size_t)c * n3;
#pragma unroll
                        for (int q = 0; q < 64; q += 4) {
                            if (vec) {
                                const float4 a = __ldcg(reinterpret_cast<const float4*>(pc + q));
                                v[q] += a.x; v[q + 1] += a.y; v[q + 2] += a.z; v[q + 3] += a.w;
                            } else {
#pragma unroll
                                for (int r = 0; r < 4; ++r)
                                    if (xb + q + r < J.nx) v[q + r] += __ldcg(pc + q + r);
                            }
                        }
                    }
                }
                const double ls = warp_sum(write_final(J, st.z, y, xb, v, P.with_loss));
                if (P.with_loss && lane == 0) J.loss_part[slot] = ls;
            }
        }
#pragma unroll
        for (int q = 0; q < 64; ++q) dsum[q] = 0.f;
    };

    for (;;) {
        // ---- next step ----
        const int slot = k % kRing;
        ok = wait_bar(&full[slot], (uint32_t)((k / kRing) & 1), P.wait_ns);
        const Step cur = ring[slot];
        if (cur.flags != kEnd && (cur.job < 0 || cur.job >= P.n_jobs)) ok = false;
        __syncwarp();
        if (lane == 0) tc::mbar_arrive(&empty[slot]);
        ++k;
        if (!__all_sync(0xffffffffu, ok)) break;
        if (cur.flags & kEnd) break;
        if (cur.flags & kZero) {
            if (have_prev) {
                drain();
                if (!__all_sync(0xffffffffu, ok)) break;
                output(prev);   // a zero unit always follows the last step of a unit
            }
            have_prev = false;
            output(cur);        // dsum is zero here
            continue;
        }
        const JobDev& J = P.jobs[cur.job];
        const int nsx = cur.nsx, nsy = cur.nsy;
        const float a2 = cur.a2;

        // With one Gy buffer (lattices too wide for two), the previous step's stage 2 reads the
        // buffer this step's G overwrites: drain that step (its completion) first.
        bool drained = false;
        if (P.na2 == 1 && have_prev) {
            drain();
            if (!__all_sync(0xffffffffu, ok)) break;
            if (prev.flags & kLast) output(prev);
            drained = true;
        }

        // ---- W_l loads, consumed after the Gaussian generation ----
        float wv[kWReg][EPC];
        {
            const float* wl = cur.w;
#pragma unroll
            for (int r = 0; r < kWReg; ++r) {
                const int row = wrg[r] & 0xFFFF, g = wrg[r] >> 16;
#pragma unroll
                for (int q = 0; q < EPC; ++q) {
                    const int i = g * EPC + q;
                    wv[r][q] = (wrg[r] >= 0 && row < nsy && i < nsx) ? __ldg(wl + (size_t)row * nsx + i) : 0.f;
                }
            }
        }
        // ---- unit start: the mask and prescription of this warp's output rows into L2 ahead
        // of the unit's output (two 128-byte lines of each) ----
        if ((cur.flags & kFirst) && P.with_loss) {
            const int ty = cur.tile / J.ntx, tx = cur.tile % J.ntx;
            const int y = ty * kTile + trow, xb = tx * kTile + half * 64;
            if (y < J.ny && xb < J.nx) {
                const size_t o = ((size_t)cur.z * J.ny + y) * J.nx + xb;
                const int last = min(63, J.nx - 1 - xb);
                asm volatile("prefetch.global.L2 [%0];" ::"l"(J.mask + o));
                asm volatile("prefetch.global.L2 [%0];" ::"l"(J.mask + o + last));
                asm volatile("prefetch.global.L2 [%0];" ::"l"(J.presc + o));
                asm volatile("prefetch.global.L2 [%0];" ::"l"(J.presc + o + last));
            }
        }
        // ---- unit start: this thread's squared distances (FP64 differences) ----
        if (cur.flags & kTab) {
            const int ty = cur.tile / J.ntx, tx = cur.tile % J.ntx;
            const double cx = 0.5 * (double)(nsx - 1), cy = 0.5 * (double)(nsy - 1);
#pragma unroll
            for (int r = 0; r < kYR; ++r) {
                const int e = tid + r * kMath;
                if (e < ny_chunks) {
                    const int row = e & 127, g = e >> 7;
                    const double yv = J.oy + (double)(ty * kTile + row) * J.dy;
                    float d2[EPC];
#pragma unroll
                    for (int q = 0; q < EPC; ++q) {
                        const int j = g * EPC + q;
                        const float d = (float)(yv - (J.sy0 + ((double)j - cy) * J.dsy));
                        d2[q] = j < nsy ? d * d : INFINITY;
                    }
#pragma unroll
                    for (int q = 0; q < EPC; q += 4)
                        tab[(r * (EPC / 4) + q / 4) * kMath + tid] =
                            make_float4(d2[q], d2[q + 1], d2[q + 2], d2[q + 3]);
                }
            }
            const double xv = J.ox + (double)(tx * kTile + trow) * J.dx;
#pragma unroll
            for (int m = 0; m < kXG; ++m) {
                const int g = half + 2 * m;
                if (g < nxg) {
#pragma unroll
                    for (int q = 0; q < EPG; q += 4) {
                        float d2[4];
#pragma unroll
                        for (int r = 0; r < 4; ++r) {
                            const int i = g * EPG + q + r;
                            const float d = (float)(xv - (J.sx0 + ((double)i - cx) * J.dsx));
                            d2[r] = i < nsx ? d * d : INFINITY;
                        }
                        tab[(P.ty4 + m * (EPG / 4) + q / 4) * kMath + tid] =
                            make_float4(d2[0], d2[1], d2[2], d2[3]);
                    }
                }
            }
        }
        // ---- G: A2 = Gy (y rows, K2 = j) ----
        const uint32_t oA2h = L.a2 + (P.na2 == 2 ? (uint32_t)(n & 1) * L.a2_stride : 0u);
        const uint32_t oA2l = oA2h + L.a2_lo;
        // Every thread owns nyr chunks of row tid & 127 (128 * N1 / EPC is a multiple of 256).
        {
            constexpr int Q4 = EPC / 4;
            const uint32_t rowoff = (uint32_t)(tid & 127) * 16u;
            for (int r = 0; r < nyr; ++r) {
                {
                    float v[EPC];
#pragma unroll
                    for (int q = 0; q < Q4; ++q) {
                        const float4 dd = tab[(r * Q4 + q) * kMath + tid];
                        v[4 * q] = ex2_approx(-dd.x * a2);
                        v[4 * q + 1] = ex2_approx(-dd.y * a2);
                        v[4 * q + 2] = ex2_approx(-dd.z * a2);
                        v[4 * q + 3] = ex2_approx(-dd.w * a2);
                    }
                    uint4 hi, lo;
                    split_chunk<MODE>(v, hi, lo);
                    const uint32_t off = (uint32_t)((tid >> 7) + 2 * r) * plane128 + rowoff;
                    *reinterpret_cast<uint4*>(smem + oA2h + off) = hi;
                    if (NARR == 2) *reinterpret_cast<uint4*>(smem + oA2l + off) = lo;
                }
            }
        }
        // ---- G: Gx -> TMEM (stage-1 A operand; lane = x row, K1 columns) ----
        for (int m = 0; m < kXG; ++m) {
            const int g = half + 2 * m;
            if (g < nxg) {
                float v[EPG];
#pragma unroll
                for (int q = 0; q < EPG / 4; ++q) {
                    const float4 dd = tab[(P.ty4 + m * (EPG / 4) + q) * kMath + tid];
                    v[4 * q] = ex2_approx(-dd.x * a2);
                    v[4 * q + 1] = ex2_approx(-dd.y * a2);
                    v[4 * q + 2] = ex2_approx(-dd.z * a2);
                    v[4 * q + 3] = ex2_approx(-dd.w * a2);
                }
                uint32_t hi[8], lo[8];
                if constexpr (Pr::EB == 4) {
#pragma unroll
                    for (int q = 0; q < 8; ++q) {
                        hi[q] = tc::to_tf32(v[q]);
                        lo[q] = NARR == 2 ? tc::to_tf32(v[q] - __uint_as_float(hi[q])) : 0u;
                    }
                } else {
#pragma unroll
                    for (int q = 0; q < 8; ++q) {
                        const uint32_t ha = bf16_bits(v[2 * q]), hb = bf16_bits(v[2 * q + 1]);
                        hi[q] = ha | (hb << 16);
                        if (NARR == 2) {
                            const float ra = v[2 * q] - __uint_as_float(ha << 16);
                            const float rb = v[2 * q + 1] - __uint_as_float(hb << 16);
                            lo[q] = bf16_bits(ra) | (bf16_bits(rb) << 16);
                        } else {
                            lo[q] = 0u;
                        }
                    }
                }
                tc::tmem_st8(tb + kColAh + lane_base + (uint32_t)(g * 8), hi);
                if (NARR == 2) tc::tmem_st8(tb + kColAl + lane_base + (uint32_t)(g * 8), lo);
            }
        }
        // ---- G: B1 = W (N1 rows j, K1 = i) from the registers ----
#pragma unroll
        for (int r = 0; r < kWReg; ++r) {
            if (wrg[r] >= 0) {
                const int row = wrg[r] & 0xFFFF, g = wrg[r] >> 16;
                uint4 hi, lo;
                split_chunk<MODE>(wv[r], hi, lo);
                const uint32_t off = (uint32_t)g * plane_n1 + (uint32_t)row * 16u;
                *reinterpret_cast<uint4*>(smem + L.b1h + off) = hi;
                if (NARR == 2) *reinterpret_cast<uint4*>(smem + L.b1l + off) = lo;
            }
        }
        tc::tmem_wait_st();
        tc::fence_async_smem();
        tc::fence_before_sync();
        __syncwarp();
        if (lane == 0) tc::mbar_arrive(ops1);

        // ---- DR: previous step's D; its unit's output when it was the unit's last step ----
        if (have_prev && !drained) {
            drain();
            if (!__all_sync(0xffffffffu, ok)) break;
            if (prev.flags & kLast) output(prev);
        }

        // ---- E1: U = stage-1 result, scaled and split -> B2 (x rows, K2 = j) ----
        ok = ok && wait_bar(mma1, ph1, P.wait_ns);
        if (ok) ph1 ^= 1;
        if (!__all_sync(0xffffffffu, ok)) break;
        tc::fence_after_sync();
        {
            // this warp's N1 / 2 columns (<= 32) of U: every load first, then one wait
            const float scale = cur.scale;
            const int ncol = N1 / 2, c00 = half * ncol;
            uint32_t rb[4][8], rs[4][8];
#pragma unroll
            for (int m = 0; m < 4; ++m) {
                if (m * 8 < ncol) {
                    tc::tmem_ld8(tb + kColUb + lane_base + (uint32_t)(c00 + m * 8), rb[m]);
                    if (Pr::NPROD == 3) tc::tmem_ld8(tb + kColUs + lane_base + (uint32_t)(c00 + m * 8), rs[m]);
                }
            }
            tc::tmem_wait_ld();
#pragma unroll
            for (int m = 0; m < 4; ++m) {
                if (m * 8 < ncol) {
                    float v[8];
#pragma unroll
                    for (int q = 0; q < 8; ++q) {
                        float uu = __uint_as_float(rb[m][q]);
                        if (Pr::NPROD == 3) uu += __uint_as_float(rs[m][q]);
                        v[q] = uu * scale;
                    }
#pragma unroll
                    for (int part = 0; part < 8 / EPC; ++part) {
                        uint4 hi, lo;
                        split_chunk<MODE>(v + part * EPC, hi, lo);
                        const int g = (c00 + m * 8 + part * EPC) / EPC;
                        const uint32_t off = (uint32_t)g * plane128 + (uint32_t)trow * 16u;
                        *reinterpret_cast<uint4*>(smem + L.b2h + off) = hi;
                        if (NARR == 2) *reinterpret_cast<uint4*>(smem + L.b2l + off) = lo;
                    }
                }
            }
        }
        tc::fence_async_smem();
        tc::fence_before_sync();
        __syncwarp();
        if (lane == 0) tc::mbar_arrive(ops2);
        prev = cur;
        have_prev = true;
        ++n;
    }
    if (ok && have_prev) {
        drain();
        if (__all_sync(0xffffffffu, ok)) output(prev);
    }
    if (!ok && lane == 0) atomicExch(P.err, 1);
}

// MAPS: the per-layer-maps mode, a separate instantiation so that the dose kernel's code and
// registers are those of the plain build.
template <int MODE, bool MAPS>
__global__ void __launch_bounds__(kThreads, 1) fwd_tc_kernel(Params P) {
    extern __shared__ __align__(1024) uint8_t smem[];
    __shared__ __align__(8) uint64_t full[kRing];
    __shared__ __align__(8) uint64_t empty[kRing];
    __shared__ __align__(8) uint64_t bars[4];   // ops1, ops2, mma1, mma2
    __shared__ Step ring[kRing];
    __shared__ uint32_t tmem_base_s;

    const int warp = threadIdx.x >> 5;
    constexpr int kIssuers = Prec<MODE>::NPROD == 3 ? 3 : 1;
    if (warp == 0) {
        tc::tmem_alloc(&tmem_base_s, kCols);
        tc::tmem_relinquish();
    }
    if (threadIdx.x == 0) {
        for (int i = 0; i < kRing; ++i) {
            tc::mbar_init(&full[i], 1);
            tc::mbar_init(&empty[i], kMathWarps + kIssuers);   // math warps + MMA issuers
        }
        tc::mbar_init(&bars[0], kMathWarps);
        tc::mbar_init(&bars[1], kMathWarps);
        tc::mbar_init(&bars[2], kIssuers == 3 ? 2 : 1);   // stage-1 chains
        tc::mbar_init(&bars[3], kIssuers == 3 ? 2 : 1);   // stage-2 chains
        tc::fence_mbar_init();
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();

    // Roles.  Each computes what it needs after its register change, so that no value
    // lives across the split.
    if (warp >= kMathWarps) {
        asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;" ::"n"(kCtrlRegs));
        if (warp == kSchedWarp) {
            scheduler_warp<MAPS>(P, ring, full, empty);
        } else if (warp - kMmaWarp < kIssuers) {
            const Layout L = make_layout<MODE>(P.K1, P.N1, P.na2);
            mma_warp<MODE>(P, L, tc::smem_u32(smem), tmem_base_s, warp - kMmaWarp, ring, full,
                           empty, bars);
        }
    } else {
        asm volatile("setmaxnreg.inc.sync.aligned.u32 %0;" ::"n"(kMathRegs));
        const Layout L = make_layout<MODE>(P.K1, P.N1, P.na2);
        math_warps<MODE, MAPS>(P, L, smem, tmem_base_s, ring, full, empty, bars);
    }

    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    if (warp == 0) tc::tmem_dealloc(tmem_base_s, kCols);
}

// Dose of every job NaN when a device wait ran out (a no-op otherwise).
__global__ void fwd_poison_kernel(const JobDev* __restrict__ jobs, int n_jobs, const int* err) {
    if (*err == 0) return;
    for (int j = 0; j < n_jobs; ++j) {
        const JobDev& J = jobs[j];
        const size_t n = (size_t)J.nx * J.ny * J.nz;
        for (size_t v = (size_t)blockIdx.x * blockDim.x + threadIdx.x; v < n;
             v += (size_t)gridDim.x * blockDim.x)
            J.dose[v] = __int_as_float(0x7fc00000);
    }
}

// Table groups (float4 per thread): y part = chunks per thread * EPC / 4, x part = groups
// per thread * EPG / 4.
template <int MODE>
void table_groups(int K1, int N1, int* ty4, int* tx4) {
    using Pr = Prec<MODE>;
    constexpr int EPG = Pr::EB == 4 ? 8 : 16;
    const int ych = (128 * (N1 / Pr::EPC) + kMath - 1) / kMath;
    const int xg = (K1 / EPG + 1) / 2;
    *ty4 = ych * Pr::EPC / 4;
    *tx4 = xg * EPG / 4;
}

template <int MODE>
size_t smem_bytes(int K1, int N1, int na2) {
    using Pr = Prec<MODE>;
    const size_t narr = Pr::NPROD == 3 ? 2 : 1;
    int ty4 = 0, tx4 = 0;
    table_groups<MODE>(K1, N1, &ty4, &tx4);
    return narr * Pr::EB * ((size_t)N1 * K1 + 128u * N1 * (1u + (size_t)na2)) +
           (size_t)(ty4 + tx4) * kMath * 16u;
}

template <int MODE, bool MAPS>
int launch_mode(const Params& P0, cudaStream_t s) {
    // the setmaxnreg split needs the full launch allotment, or its increase never returns
    int max_dyn = 0;
    PBD_TRY(smem_optin((const void*)fwd_tc_kernel<MODE, MAPS>, -1, kLaunchRegsNeeded, &max_dyn));
    Params P = P0;
    table_groups<MODE>(P.K1, P.N1, &P.ty4, &P.tx4);
    P.na2 = 2;
    size_t smem = smem_bytes<MODE>(P.K1, P.N1, 2);
    if (smem > (size_t)max_dyn) {
        P.na2 = 1;
        smem = smem_bytes<MODE>(P.K1, P.N1, 1);
    }
    // At least 116 KiB so that one CTA (and its 512 TMEM columns) occupies an SM: a second
    // resident CTA would only wait in tcgen05.alloc for the first to finish.
    smem = std::max<size_t>(smem, 116u * 1024u);
    if (smem > (size_t)max_dyn) return PBD_ERR_NO_SMEM;
    const int grid = std::max(1, std::min(P.n_units, num_sms()));
    prof_mark(kProfFwd, 0, s);
    fwd_tc_kernel<MODE, MAPS><<<grid, kThreads, smem, s>>>(P);
    PBD_LAUNCH_CHECK();
    prof_mark(kProfFwd, 1, s);
    return PBD_OK;
}

}  // namespace

int tc_operand_dims(int precision, int nsx, int nsy, int* K1, int* N1) {
    const int kstep = (precision == PBD_PREC_BF16X3 || precision == PBD_PREC_BF16 ||
                       precision == PBD_PREC_FP16X3) ? 16 : 8;
    *K1 = (nsx + kstep - 1) / kstep * kstep;
    *N1 = (nsy + 15) / 16 * 16;
    if (*K1 > 64 || *N1 > 64) return PBD_ERR_UNSUPPORTED;
    return PBD_OK;
}

int tc_forward_units(const JobDev* jobs_host, int n_jobs, int chunk, int* cmax, int* tmax,
                     int* n_units) {
    int cm = 1, tm = 1, nzm = 1;
    for (int j = 0; j < n_jobs; ++j) {
        const JobDev& J = jobs_host[j];
        cm = std::max(cm, (J.nl + chunk - 1) / chunk);
        tm = std::max(tm, ((J.nx + kTile - 1) / kTile) * ((J.ny + kTile - 1) / kTile));
        nzm = std::max(nzm, J.nz);
    }
    const long long u = (long long)nzm * cm * n_jobs * tm;
    if (u > (1LL << 30)) return PBD_ERR_UNSUPPORTED;
    *cmax = cm; *tmax = tm; *n_units = (int)u;
    return PBD_OK;
}

int launch_forward_tc(int precision, JobDev* jobs_dev, const JobDev* jobs_host, int n_jobs,
                      int* counter, int* err, int chunk, int with_loss, int poison,
                      cudaStream_t s) {
    Params P{};
    P.jobs = jobs_dev;
    P.n_jobs = n_jobs;
    P.chunk = chunk;
    P.counter = counter;
    P.err = err;
    P.wait_ns = wait_limit_ns();
    P.hold = test_hold();
    P.with_loss = with_loss;
    for (int j = 0; j < n_jobs; ++j) {
        int k1 = 0, n1 = 0;
        PBD_TRY(tc_operand_dims(precision, jobs_host[j].nsx, jobs_host[j].nsy, &k1, &n1));
        P.K1 = std::max(P.K1, k1);
        P.N1 = std::max(P.N1, n1);
    }
    PBD_TRY(tc_forward_units(jobs_host, n_jobs, chunk, &P.cmax, &P.tmax, &P.n_units));
    // per-layer maps (layer_stride > 0, no loss) or the dose: every job of a launch alike
    const bool maps = jobs_host[0].layer_stride != 0;
    for (int j = 1; j < n_jobs; ++j)
        if ((jobs_host[j].layer_stride != 0) != maps) return PBD_ERR_UNSUPPORTED;
    if (maps && with_loss) return PBD_ERR_UNSUPPORTED;
    // the split-FP16 kernel has no per-layer-maps mode: its accuracy class is TF32x3's
    if (precision == PBD_PREC_FP16X3) precision = PBD_PREC_TF32X3;
    int rc = PBD_ERR_BAD_VALUE;
    switch (precision) {
        case PBD_PREC_TF32X3:
            rc = maps ? launch_mode<PBD_PREC_TF32X3, true>(P, s) : launch_mode<PBD_PREC_TF32X3, false>(P, s);
            break;
        case PBD_PREC_TF32:
            rc = maps ? launch_mode<PBD_PREC_TF32, true>(P, s) : launch_mode<PBD_PREC_TF32, false>(P, s);
            break;
        case PBD_PREC_BF16X3:
            rc = maps ? launch_mode<PBD_PREC_BF16X3, true>(P, s) : launch_mode<PBD_PREC_BF16X3, false>(P, s);
            break;
        case PBD_PREC_BF16:
            rc = maps ? launch_mode<PBD_PREC_BF16, true>(P, s) : launch_mode<PBD_PREC_BF16, false>(P, s);
            break;
        default: break;
    }
    PBD_TRY(rc);
    count_launch(1);
    if (poison) {
        fwd_poison_kernel<<<num_sms(), 256, 0, s>>>(jobs_dev, n_jobs, err);
        PBD_LAUNCH_CHECK();
        count_launch(1);
    }
    return PBD_OK;
}

}  // namespace pbd
