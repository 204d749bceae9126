// adj_tc.cu -- adjoint of the separable dose on the tensor cores (tcgen05), warp-specialised
// and software-pipelined across (layer, slice) pairs.
//
// Same mathematics as adj_simt.cu.  With G = dL/dD[z] and unnormalised Gaussians of width
// s = sigma_l(z), for every active (layer l, slice z):
//
//   stage 1   Y[m, x] = sum_y A[m, y] G[y, x]        A = [Gy | Gy']^T, m = 2 j: j, m = 2 j + 1: j'
//             M = 128 (m), N = 128 (x), K = 128 (y); A generated into TMEM, G^T in smem
//   stage 2   Q[m, n] = sum_x Y[m, x] B[n, x]        B = [Gx | Gx'], n < N1: i, n >= N1: i'
//             M = 128 (m), N = 2 N1 (n), K = 128 (x); Y split back into TMEM, B in smem
//
// P = Q[j, i] gives dL/dW_l += IDD P / (2 pi s^2) and dL/dIDD = <P, W> / (2 pi s^2);
// Q[j, i'] + Q[j', i] gives dL/dsigma = IDD <., W> / (2 pi s^2) (G' = dG/ds).  The
// Gaussian factors are regenerated per pair; nothing Gaussian is stored in HBM.
//
// Precision.  The contraction runs in split BF16 (hi + lo, three products, FP32
// accumulation) for every split or TF32 mode and in plain BF16 for the BF16 mode: the
// gradients need 1e-4 and the split form keeps ~16 mantissa bits (measured ~1e-6 of the
// largest gradient), and BF16 operands halve the MMA count and the on-chip footprint
// against TF32, which is what lets the pipeline below double-buffer.
//
// CTA = 8 math warps, a scheduler warp, two MMA warps (one per stage); one CTA per SM.
//  * Scheduler warp: units (slice z, chunk of <= C active layers) from an atomic counter
//    in z-major order; one step per active layer into an 8-slot ring (full / empty
//    mbarriers).
//  * Math warps, per pair n (buffer b = n & 1), without block barriers:
//      at a unit's first pair: G^T of the slice, split, into smem (the previous unit's last
//          stage 1 is complete: it was waited for before this pair)
//      G   A = [Gy | Gy']^T -> TMEM A[b] (tcgen05.st); arrive on ops1.  Rows j and j' of a
//          spot are adjacent lanes of one warp: each lane evaluates the exponentials of half
//          the row's columns and the pair swaps them (one shuffle per value), so every
//          exponential of Gy serves Gy' too
//      DR  pair n-1's Q from TMEM: P = Q[j, i] / (2 pi s^2) into the (layer, slice) slot,
//          stored transposed ([i][j]) so that the j lanes of a warp write 64 contiguous
//          bytes; the dot products <P, W> and <S, W>, S = (Q[j, i'] + Q[j', i]) / (2 pi s^2)
//          (the j' lane's value moved to the j lane by shuffle), summed over the warp
//      B   [Gx | Gx'] -> smem (read by stage 2 only, whose previous use DR waited for);
//          each Gaussian value and its derivative come from one exp
//      E1  Y of pair n from TMEM, split, back into TMEM A[b]; arrive on ops2
//  * MMA warp 1: stage 1 after ops1 (A from TMEM, "TS" form), commit to mma1.
//    MMA warp 2: stage 2 after ops2 (A = split Y from TMEM), commit to mma2.
//  Stage 2 of pair n-1 runs under G of pair n; stage 1 of pair n under DR and B.
//
// dL/dW_l = sum over active slices of IDD * slot P in slice order, and the sums of the warps'
// dot-product partials (dL/dIDD, dL/dsigma), are formed by one follow-up kernel in a fixed
// order (deterministic).  Every wait is bounded (2 s of %globaltimer, or a test limit); a warp
// whose wait runs out sets the error word and leaves, the others' waits then run out in
// turn, and the finalize pass turns the gradients into NaN.
// Grids of at most 128 x 128 voxels per slice; lattices up to 64 x 64 spots.
#include <algorithm>
#include <math.h>

#include "pbd_internal.cuh"
#include "tc_common.cuh"

namespace pbd {
namespace {
using namespace tcc;

constexpr int kMathWarps = 8;
constexpr int kMath = 32 * kMathWarps;     // 256 math threads: warpgroups 0 and 1
constexpr int kSchedWarp = kMathWarps;     // warpgroup 2: warp 8 schedules, warp 9 issues
constexpr int kS1Warp = kMathWarps + 1;    // stage 1, warp 10 stage 2, warp 11 idle
constexpr int kS2Warp = kMathWarps + 2;
constexpr int kThreads = kMath + 128;
constexpr int kRing = 8;
constexpr uint32_t kCols = 512;
// Register split (setmaxnreg) as in the forward: 8 * 32 * 208 + 4 * 32 * 80 <= 384 * 168.
constexpr int kMathRegs = 208, kCtrlRegs = 80;
constexpr int kLaunchRegsNeeded = (kMath * kMathRegs + 128 * kCtrlRegs + kThreads - 1) / kThreads;
// TMEM columns: A[0] [0,128), A[1] [128,256) (bf16 pairs: hi [0,64), lo [64,128) of each),
// Y [256,384), Q [384, 384 + 2 N1)
constexpr uint32_t kColA = 0, kColY = 256, kColQ = 384;
constexpr uint32_t kLoOff = 64;

enum : int { kFirst = 1, kLast = 2, kEnd = 4 };

struct Step {
    int job, z, l, flags;
    float a2, inv_s, inv_s3, nrm;   // exponent scale, 1/s, 1/s^3, 1/(2 pi s^2)
};

struct Params {
    const JobDev* jobs;
    int n_jobs, chunk, cmax, n_units;
    int* counter;        // [0] unit counter
    int* err;            // error word: set when a bounded wait ran out
    unsigned long long wait_ns;   // limit of every bounded wait
    int hold;            // test of the timeout path: the scheduler publishes no step
    int N1;              // x-lattice padded to 16
    int stage;           // 1: each unit's dL/dD slice arrives by bulk copy into a staging buffer
                         //    (every job's slice is contiguous, 16-byte aligned, nx ny % 4 == 0)
    uint32_t o_stage;    // its shared-memory offset
    int sym;             // 1: every job is symmetric in x and y (grid, lattice, origins), so the
                         //    stage-2 operand [Gx | Gx'] equals the [Gy | Gy'] rows G evaluates
    int adapt;           // 1 (one job, no explicit schedule): every CTA counts the active pairs T
                         //    and uses units of ceil(T / grid) + 1 layers (chunk, cmax, n_units
                         //    then describe that unit size)
};

// The adjoint's unit decomposition in force (P's, or the one the CTA derived).
struct Units {
    int chunk, cmax, n_units;
};

struct Layout {
    uint32_t gth, gtl, b2, b2_lo;
};

template <int NARR>
__device__ __forceinline__ Layout make_layout(int N1) {
    const uint32_t gt = 128u * 128u * 2u, b2 = 2u * (uint32_t)N1 * 128u * 2u;
    Layout L;
    L.gth = 0;
    L.gtl = NARR == 2 ? gt : 0u;
    L.b2 = (uint32_t)NARR * gt;
    L.b2_lo = NARR == 2 ? b2 : 0u;
    return L;
}

// Two adjacent K elements as packed bf16 {a in the low half, b in the high half}: hi, and for
// split modes lo = bf16 of the remainders (the hi values back in FP32 are exact bit shifts).  One
// packed conversion per word.
template <int NARR>
__device__ __forceinline__ void split2(float a, float b, uint32_t& hi, uint32_t& lo) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    hi = *reinterpret_cast<const uint32_t*>(&h);
    if (NARR == 2) {
        const __nv_bfloat162 l = __floats2bfloat162_rn(a - __uint_as_float(hi << 16),
                                                       b - __uint_as_float(hi & 0xFFFF0000u));
        lo = *reinterpret_cast<const uint32_t*>(&l);
    } else {
        lo = 0u;
    }
}

// Split 8 floats into packed bf16 hi / lo words (lo = bf16 of the remainder).
template <int NARR>
__device__ __forceinline__ void split8(const float* v, uint4& hi, uint4& lo) {
    uint32_t h[4], l[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) split2<NARR>(v[2 * q], v[2 * q + 1], h[q], l[q]);
    hi = make_uint4(h[0], h[1], h[2], h[3]);
    lo = make_uint4(l[0], l[1], l[2], l[3]);
}

// ------------------------------------------------------------------------------------------
// Scheduler warp: units (z, chunk) -> one step per active layer.
// ------------------------------------------------------------------------------------------
__device__ __forceinline__ void scheduler_warp(const Params& P, const Units U, Step* ring,
                                               uint64_t* full, uint64_t* empty, uint8_t* smem,
                                               uint64_t* sfull, uint64_t* sfree) {
    const int lane = threadIdx.x & 31;
    const unsigned FULL = 0xffffffffu;
    int k = 0, nu = 0;       // ring pushes; units whose slice was copied into the staging buffer
    bool ok = true;
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
        if (u >= U.n_units) break;
        int v = u;
        const int job = v % P.n_jobs; v /= P.n_jobs;
        const int c = v % U.cmax;
        const int z = v / U.cmax;
        const JobDev& J = P.jobs[job];
        const int nz = J.nz, nl = J.nl;
        if (z >= nz) continue;
        const double* idd = J.idd;
        int tot = 0;
        for (int b = 0; b < nl; b += 32) {
            const int l = b + lane;
            const bool a = l < nl && idd[(size_t)l * nz + z] != 0.0;
            tot += __popc(__ballot_sync(FULL, a));
        }
        const int r0 = c * U.chunk;
        if (r0 >= tot) continue;   // no chunk c here (slices no layer reaches carry no gradient)
        const int r1 = min(tot, r0 + U.chunk);
        if (P.stage) {
            // the unit's dL/dD slice into the staging buffer, once the math warps have converted
            // the previous unit's copy
            bool w = true;
            if (nu > 0) w = wait_bar(sfree, (uint32_t)((nu - 1) & 1), P.wait_ns);
            if (!__all_sync(FULL, w)) { ok = false; break; }
            if (lane == 0) {
                const uint32_t bytes = (uint32_t)J.nx * (uint32_t)J.ny * 4u;
                const uint32_t dst = tc::smem_u32(smem) + P.o_stage;
                asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(
                                 tc::smem_u32(sfull)), "r"(bytes)
                             : "memory");
                asm volatile(
                    "cp.async.bulk.shared::cta.global.mbarrier::complete_tx::bytes [%0], [%1], %2, "
                    "[%3];" ::"r"(dst),
                    "l"(J.grad_dose + (size_t)z * J.ny * J.nx), "r"(bytes), "r"(tc::smem_u32(sfull))
                    : "memory");
            }
            __syncwarp();
            ++nu;
        }
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
                st.job = job; st.z = z; st.l = l;
                st.flags = (my == r0 ? kFirst : 0) | (my == r1 - 1 ? kLast : 0);
                st.a2 = (float)(kLog2e / (2.0 * s * s));
                st.inv_s = (float)(1.0 / s);
                st.inv_s3 = (float)(1.0 / (s * s * s));
                st.nrm = (float)(kInv2Pi / (s * s));
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
    // the last staging copy lands before the block exits
    if (nu > 0) (void)wait_bar(sfull, (uint32_t)((nu - 1) & 1), P.wait_ns);
    if (!ok && lane == 0) atomicExch(P.err, 1);
}

// ------------------------------------------------------------------------------------------
// MMA warps.  stage 1: Y = A[b] (TMEM, K = y) x G^T (smem rows x); stage 2: Q = Y split
// (TMEM A[b], K = x) x B2^T (smem rows n).  One accumulator per stage (gradients carry a
// 1e-4 tolerance), the three products of a k-step issued back to back.
// ------------------------------------------------------------------------------------------
template <int MODE>
__device__ __forceinline__ void mma_warp(const Params& P, const Layout& L, uint32_t sbase,
                                         uint32_t tb, int stage, const Step* ring,
                                         uint64_t* full, uint64_t* empty, uint64_t* bars) {
    using Pr = Prec<MODE>;
    const int lane = threadIdx.x & 31;
    uint64_t* ops = bars + (stage == 1 ? 0 : 1);
    uint64_t* done = bars + (stage == 1 ? 2 : 3);
    const uint32_t R2 = 2u * (uint32_t)P.N1;
    const uint32_t idesc = tc::instr_desc(128, stage == 1 ? 128 : (int)R2, Pr::FMT);
    const uint32_t plane_b = stage == 1 ? 128u * 16u : R2 * 16u;
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
        ok = wait_bar(ops, (uint32_t)(n & 1), P.wait_ns);
        if (!__all_sync(0xffffffffu, ok)) break;
        tc::fence_after_sync();
        if (lane == 0) {
            const uint32_t a = tb + kColA + (uint32_t)(n & 1) * 128u;
            const uint32_t d = tb + (stage == 1 ? kColY : kColQ);
            uint32_t bh, bl;
            if (stage == 1) {
                bh = sbase + L.gth;
                bl = sbase + L.gtl;
            } else {
                bh = sbase + L.b2;
                bl = bh + L.b2_lo;
            }
            for (int st = 0; st < 128 / 16; ++st) {
                const uint32_t ob = (uint32_t)st * 2u * plane_b;
                const uint32_t ac = a + (uint32_t)st * 8u;
                const uint64_t dh = tc::smem_desc(bh + ob, plane_b, 128);
                if (Pr::NPROD == 3) {
                    const uint64_t dl = tc::smem_desc(bl + ob, plane_b, 128);
                    tc::mma_bf16_ts(d, ac, dl, idesc, st > 0 ? 1u : 0u);
                    tc::mma_bf16_ts(d, ac + kLoOff, dh, idesc, 1u);
                    tc::mma_bf16_ts(d, ac, dh, idesc, 1u);
                } else {
                    tc::mma_bf16_ts(d, ac, dh, idesc, st > 0 ? 1u : 0u);
                }
            }
            tc::commit(done);
        }
        __syncwarp();
        ++n;
    }
    if (!ok && lane == 0) atomicExch(P.err, 1);
    if (n > 0) (void)wait_bar(done, (uint32_t)((n - 1) & 1), P.wait_ns);
}

// ------------------------------------------------------------------------------------------
// DR: a pair's Q (TMEM columns from tq: Q[., i] at i, Q[., i'] at N1 + i) -> the pair's P slot
// and this warp's share of the pair's two dot products.
//  * Slot layout: P[j][i] = Q[j, i] / (2 pi s^2), rows of n1 = nsx rounded up to 16 floats
//    (columns i >= nsx hold 0), so that a j lane writes its 8 columns as two 16-byte stores.
//  * A thread's columns: 8-column chunks c0 = 8 half + 16 t, so that both halves of a lane
//    quadrant drain the same number of chunks.
//  * <P, W> is summed by the j lanes; <S, W>, S = (Q[j, i'] + Q[j', i]) / (2 pi s^2), by the
//    j lane (Q[j, i'] W[j, i]) and the j' lane (Q[j', i] W[j, i]) together, and a butterfly
//    over the warp adds all of them; the follow-up kernel adds the eight warps' partials in
//    warp order.  Padding rows (j >= nsy) and columns (i >= nsx) hold products of unset
//    operand rows and are never read into a sum.
// ------------------------------------------------------------------------------------------
// This thread's W entries for pr's DR (W_l[j, c0 + q], zero where it owns no entry).  Loaded a
// phase ahead of the DR, so that the load latency is hidden.
__device__ __forceinline__ void load_w_rows(const Params& P, const Step& pr, int half, int jrow,
                                            float (&wv)[4][8]) {
    const JobDev& Jp = P.jobs[pr.job];
    const int pnsx = Jp.nsx, pnsy = Jp.nsy;
    const bool row_ok = jrow < pnsy;
    const float* wrow = Jp.w + (size_t)pr.l * pnsy * pnsx + (size_t)(row_ok ? jrow : 0) * pnsx;
#pragma unroll
    for (int t = 0; t < 4; ++t) {
        const int c0 = 8 * half + 16 * t;
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int i = c0 + q;
            wv[t][q] = (row_ok && i < pnsx) ? __ldg(wrow + i) : 0.f;
        }
    }
}

__device__ __forceinline__ void drain_q(const Params& P, const Step& pr, uint32_t tq, int half,
                                        int jrow, bool deriv, int warp, int lane,
                                        const float (&wv)[4][8]) {
    const JobDev& Jp = P.jobs[pr.job];
    const int pnsx = Jp.nsx, pnsy = Jp.nsy, nz = Jp.nz, N1 = P.N1;
    const int n1 = (pnsx + 15) / 16 * 16;
    const size_t per = (size_t)pnsy * n1;
    const size_t pair = (size_t)pr.l * nz + pr.z;
    const bool row_ok = jrow < pnsy;
    float* slot_row = Jp.partial + pair * per + (size_t)(row_ok ? jrow : 0) * n1;
    float dp = 0.f, ds = 0.f;
    // a warp whose 32 rows are all padding (its first row 16 sp >= nsy) owns no entry: it skips
    // the TMEM loads and stores zero partials
    const bool pad = __shfl_sync(0xffffffffu, jrow, 0) >= pnsy;
    if (!pad) {
#pragma unroll
        for (int t = 0; t < 4; ++t) {
            const int c0 = 8 * half + 16 * t;
            if (c0 >= n1) break;
            uint32_t ri[8], rd[8];
            tc::tmem_ld8(tq + (uint32_t)c0, ri);
            tc::tmem_ld8(tq + (uint32_t)(N1 + c0), rd);
            tc::tmem_wait_ld();
            float pv[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const bool in = row_ok && c0 + q < pnsx;
                const float vi = __uint_as_float(ri[q]);   // Q[j, i] (j lane) or Q[j', i] (j' lane)
                const float vd = __uint_as_float(rd[q]);   // Q[j, i'] (j lane)
                if (in) {
                    if (!deriv) dp = fmaf(vi, wv[t][q], dp);
                    ds = fmaf(deriv ? vi : vd, wv[t][q], ds);
                }
                pv[q] = in ? pr.nrm * vi : 0.f;
            }
            if (!deriv && row_ok) {
                float4* o = reinterpret_cast<float4*>(slot_row + c0);
                o[0] = make_float4(pv[0], pv[1], pv[2], pv[3]);
                o[1] = make_float4(pv[4], pv[5], pv[6], pv[7]);
            }
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        dp += __shfl_xor_sync(0xffffffffu, dp, o);
        ds += __shfl_xor_sync(0xffffffffu, ds, o);
    }
    if (lane == 0) {
        float* dots = Jp.partial + (size_t)Jp.nl * nz * per;   // (2, nl, nz, kMathWarps)
        dots[pair * kMathWarps + warp] = pr.nrm * dp;
        dots[((size_t)Jp.nl * nz + pair) * kMathWarps + warp] = pr.nrm * ds;
    }
}

// Symmetric fields: this lane's G row (row j of Gy, or of Gy' on the j' lane; K columns
// [64 half, +64) as packed bf16 pairs) stored as B2 row j (or N1 + j), K chunks 8 half + cc.
template <int NARR>
__device__ __forceinline__ void store_b2_sym(uint8_t* smem, const Layout& L, int N1, int half,
                                             int jrow, bool deriv, const uint32_t (&hi)[2][16],
                                             const uint32_t (&lo)[2][16]) {
    const uint32_t planeR2 = (uint32_t)(2 * N1) * 16u;
    const uint32_t row = (uint32_t)(deriv ? N1 + jrow : jrow);
#pragma unroll
    for (int cc = 0; cc < 8; ++cc) {
        const uint32_t off = L.b2 + (uint32_t)(8 * half + cc) * planeR2 + row * 16u;
        const int a = cc >> 2, w = 4 * (cc & 3);
        *reinterpret_cast<uint4*>(smem + off) = make_uint4(hi[a][w], hi[a][w + 1], hi[a][w + 2], hi[a][w + 3]);
        if (NARR == 2)
            *reinterpret_cast<uint4*>(smem + off + L.b2_lo) =
                make_uint4(lo[a][w], lo[a][w + 1], lo[a][w + 2], lo[a][w + 3]);
    }
}

// ------------------------------------------------------------------------------------------
// Math warps.
// ------------------------------------------------------------------------------------------
template <int MODE>
__device__ __forceinline__ void math_warps(const Params& P, const Layout& L, uint8_t* smem,
                                           uint32_t tb, const Step* ring, uint64_t* full,
                                           uint64_t* empty, uint64_t* bars, uint64_t* sfull,
                                           uint64_t* sfree) {
    using Pr = Prec<MODE>;
    constexpr int NARR = Pr::NPROD == 3 ? 2 : 1;
    uint64_t* ops1 = bars + 0;
    uint64_t* ops2 = bars + 1;
    uint64_t* mma1 = bars + 2;
    uint64_t* mma2 = bars + 3;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int sp = warp & 3, half = warp >> 2;
    const uint32_t lane_base = (uint32_t)(32 * sp) << 16;
    const int m = 32 * sp + lane;          // TMEM lane: row m of A, Y, Q
    const int jrow = m >> 1;               // rows 2 j (Gy) and 2 j + 1 (Gy') of spot row j
    const bool deriv = (m & 1) != 0;
    const int N1 = P.N1, R2 = 2 * N1;
    const uint32_t planeR2 = (uint32_t)R2 * 16u;

    uint32_t ph1 = 0, ph2 = 0;
    bool ok = true;
    Step prev{};
    bool have_prev = false;
    int k = 0, n = 0, nu = 0;
    float ybase = 0.f;                     // (y0 of this thread's columns) - ys_j, per unit

    for (;;) {
        const int slot = k % kRing;
        ok = wait_bar(&full[slot], (uint32_t)((k / kRing) & 1), P.wait_ns);
        const Step cur = ring[slot];
        if (cur.flags != kEnd && (cur.job < 0 || cur.job >= P.n_jobs)) ok = false;
        __syncwarp();
        if (lane == 0) tc::mbar_arrive(&empty[slot]);
        ++k;
        if (!__all_sync(0xffffffffu, ok)) break;
        if (cur.flags & kEnd) break;
        // W of the pair this iteration drains, in flight while G runs
        float wpre[4][8];
        if (have_prev) load_w_rows(P, prev, half, jrow, wpre);
        const JobDev& J = P.jobs[cur.job];
        const int nx = J.nx, ny = J.ny, nsx = J.nsx, nsy = J.nsy;
        const int b = n & 1;
        const float a2 = cur.a2, inv_s = cur.inv_s, inv_s3 = cur.inv_s3;

        // ---- unit start: G^T of the slice (rows x, K = y; zero outside the grid) ----
        if (cur.flags & kFirst) {
            // the slice from the staging buffer (bulk copy issued by the scheduler when it
            // claimed the unit) or, for slices that cannot be bulk copied, from global memory
            const float* g = J.grad_dose + (size_t)cur.z * ny * nx;
            if (P.stage) {
                ok = wait_bar(sfull, (uint32_t)(nu & 1), P.wait_ns);
                if (!__all_sync(0xffffffffu, ok)) break;
                g = reinterpret_cast<const float*>(smem + P.o_stage);
            }
#pragma unroll 1
            for (int r = 0; r < 8; ++r) {
                const int e = tid + r * kMath;
                const int x = e & 127, c = e >> 7;
                float v[8];
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    const int y = c * 8 + q;
                    v[q] = (y < ny && x < nx) ? g[(size_t)y * nx + x] : 0.f;
                }
                uint4 hi, lo;
                split8<NARR>(v, hi, lo);
                const uint32_t off = (uint32_t)c * 2048u + (uint32_t)x * 16u;
                *reinterpret_cast<uint4*>(smem + L.gth + off) = hi;
                if (NARR == 2) *reinterpret_cast<uint4*>(smem + L.gtl + off) = lo;
            }
            if (P.stage) {
                __syncwarp();
                if (lane == 0) tc::mbar_arrive(sfree);   // the staging buffer is free again
                ++nu;
            }
            const double cy = 0.5 * (double)(nsy - 1);
            ybase = (float)((J.oy + (double)(64 * half) * J.dy) - (J.sy0 + ((double)jrow - cy) * J.dsy));
        }

        // ---- G: A = [Gy | Gy']^T -> TMEM A[b] (row m, y columns [64 half, +64)) ----
        // The j lane evaluates the exponentials of columns c < 32 of the two rows, the j'
        // lane those of columns 32 + c; a shuffle swaps them.  Each column's value is the
        // same FP32 computation as evaluating it in place.
        // a warp whose 32 TMEM rows are all padding (m >= 2 nsy) skips G and E1: those rows of
        // every product only ever feed rows of Q that are never read
        const bool pad_warp = 32 * sp >= 2 * nsy;
        uint32_t hi[2][16], lo[2][16];   // this lane's G row, kept for B2 on symmetric fields
        if (!pad_warp) {
            const float dyf = (float)J.dy;
            const bool valid = jrow < nsy;
            const float cself = deriv ? 32.f : 0.f;   // first column of this lane's exponentials
#pragma unroll
            for (int kp = 0; kp < 16; ++kp) {
                float vl[2], vh[2];                     // columns 2 kp + t and 32 + 2 kp + t
#pragma unroll
                for (int t = 0; t < 2; ++t) {
                    const float c = (float)(2 * kp + t);
                    const float ds = fmaf(cself + c, dyf, ybase);
                    const float own = ex2_approx(-(ds * ds) * a2);
                    const float oth = __shfl_xor_sync(0xffffffffu, own, 1);
                    const float el = deriv ? oth : own, eh = deriv ? own : oth;
                    const float dl = fmaf(c, dyf, ybase), ddl = dl * dl;
                    const float dh = fmaf(32.f + c, dyf, ybase), ddh = dh * dh;
                    vl[t] = valid ? (deriv ? el * fmaf(ddl, inv_s3, -inv_s) : el) : 0.f;
                    vh[t] = valid ? (deriv ? eh * fmaf(ddh, inv_s3, -inv_s) : eh) : 0.f;
                }
                split2<NARR>(vl[0], vl[1], hi[0][kp], lo[0][kp]);
                split2<NARR>(vh[0], vh[1], hi[1][kp], lo[1][kp]);
            }
            const uint32_t col = kColA + (uint32_t)b * 128u + (uint32_t)(32 * half);
            tc::tmem_st16(tb + lane_base + col, hi[0]);
            tc::tmem_st16(tb + lane_base + col + 16u, hi[1]);
            if (NARR == 2) {
                tc::tmem_st16(tb + lane_base + col + kLoOff, lo[0]);
                tc::tmem_st16(tb + lane_base + col + kLoOff + 16u, lo[1]);
            }
        }
        tc::tmem_wait_st();
        tc::fence_async_smem();
        tc::fence_before_sync();
        __syncwarp();
        if (lane == 0) tc::mbar_arrive(ops1);

        // ---- DR: Q of the previous pair -> its P slot and dot products ----
        if (have_prev) {
            ok = ok && wait_bar(mma2, ph2, P.wait_ns);
            if (ok) ph2 ^= 1;
            if (!__all_sync(0xffffffffu, ok)) break;
            tc::fence_after_sync();
        }
        // symmetric fields: B2 = the G rows just evaluated.  Stage 2 of the previous pair, the
        // only reader of B2, is complete (waited for above, or there is none).  Pad warps hold
        // only rows j >= N1, which B2 does not have.
        if (P.sym && !pad_warp && jrow < N1) store_b2_sym<NARR>(smem, L, N1, half, jrow, deriv, hi, lo);
        if (have_prev) drain_q(P, prev, tb + lane_base + kColQ, half, jrow, deriv, warp, lane, wpre);

        // ---- B2 = [Gx | Gx'] -> smem (rows i and N1 + i, K = x).  Only stage 2 reads it,
        // and the previous pair's stage 2 is complete (DR waited), so one buffer serves. ----
        if (!P.sym) {
            const uint32_t ob2 = L.b2;
            const double cx = 0.5 * (double)(nsx - 1);
            const float dxf = (float)J.dx;
            const int items = N1 * 16;   // (i, x-chunk of 8)
            for (int e = tid; e < items; e += kMath) {
                const int i = e % N1, c = e / N1;
                const float base = (float)((J.ox + (double)(8 * c) * J.dx) - (J.sx0 + ((double)i - cx) * J.dsx));
                float g0[8], g1[8];
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    const float d = fmaf((float)q, dxf, base), dd = d * d;
                    const float ev = i < nsx ? ex2_approx(-dd * a2) : 0.f;
                    g0[q] = ev;
                    g1[q] = ev * fmaf(dd, inv_s3, -inv_s);
                }
                uint4 h0, l0, h1, l1;
                split8<NARR>(g0, h0, l0);
                split8<NARR>(g1, h1, l1);
                const uint32_t o0 = ob2 + (uint32_t)c * planeR2 + (uint32_t)i * 16u;
                const uint32_t o1 = o0 + (uint32_t)N1 * 16u;
                *reinterpret_cast<uint4*>(smem + o0) = h0;
                *reinterpret_cast<uint4*>(smem + o1) = h1;
                if (NARR == 2) {
                    *reinterpret_cast<uint4*>(smem + o0 + L.b2_lo) = l0;
                    *reinterpret_cast<uint4*>(smem + o1 + L.b2_lo) = l1;
                }
            }
        }
        // ---- E1: Y of this pair -> split -> TMEM A[b] (row m, x columns [64 half, +64)) ----
        ok = ok && wait_bar(mma1, ph1, P.wait_ns);
        if (ok) ph1 ^= 1;
        if (!__all_sync(0xffffffffu, ok)) break;
        tc::fence_after_sync();
        if (!pad_warp) {
            uint32_t r[4][16];
#pragma unroll
            for (int c = 0; c < 4; ++c)
                tc::tmem_ld16(tb + lane_base + kColY + (uint32_t)(64 * half + 16 * c), r[c]);
            tc::tmem_wait_ld();
            uint32_t hi[2][16], lo[2][16];
#pragma unroll
            for (int q = 0; q < 32; ++q) {
                const float va = __uint_as_float(r[q >> 3][(2 * q) & 15]);
                const float vb = __uint_as_float(r[q >> 3][(2 * q + 1) & 15]);
                split2<NARR>(va, vb, hi[q >> 4][q & 15], lo[q >> 4][q & 15]);
            }
            const uint32_t col = kColA + (uint32_t)b * 128u + (uint32_t)(32 * half);
            tc::tmem_st16(tb + lane_base + col, hi[0]);
            tc::tmem_st16(tb + lane_base + col + 16u, hi[1]);
            if (NARR == 2) {
                tc::tmem_st16(tb + lane_base + col + kLoOff, lo[0]);
                tc::tmem_st16(tb + lane_base + col + kLoOff + 16u, lo[1]);
            }
        }
        tc::tmem_wait_st();
        tc::fence_async_smem();
        tc::fence_before_sync();
        __syncwarp();
        if (lane == 0) tc::mbar_arrive(ops2);
        prev = cur;
        have_prev = true;
        ++n;
    }
    // last pair's Q
    if (ok && have_prev) {
        ok = wait_bar(mma2, ph2, P.wait_ns);
        if (__all_sync(0xffffffffu, ok)) {
            tc::fence_after_sync();
            float wl[4][8];
            load_w_rows(P, prev, half, jrow, wl);
            drain_q(P, prev, tb + lane_base + kColQ, half, jrow, deriv, warp, lane, wl);
        }
    }
    if (!ok && lane == 0) atomicExch(P.err, 1);
}

template <int MODE>
__global__ void __launch_bounds__(kThreads, 1) adj_tc_kernel(Params P) {
    constexpr int NARR = Prec<MODE>::NPROD == 3 ? 2 : 1;
    extern __shared__ __align__(1024) uint8_t smem[];
    __shared__ __align__(8) uint64_t full[kRing];
    __shared__ __align__(8) uint64_t empty[kRing];
    __shared__ __align__(8) uint64_t bars[4];   // ops1, ops2, mma1, mma2
    __shared__ __align__(8) uint64_t sbars[2];  // staging buffer full, free
    __shared__ Step ring[kRing];
    __shared__ uint32_t tmem_base_s;

    const int warp = threadIdx.x >> 5;
    if (warp == 0) {
        tc::tmem_alloc(&tmem_base_s, kCols);
        tc::tmem_relinquish();
    }
    if (threadIdx.x == 0) {
        for (int i = 0; i < kRing; ++i) {
            tc::mbar_init(&full[i], 1);
            tc::mbar_init(&empty[i], kMathWarps + 2);   // math warps + both MMA warps
        }
        tc::mbar_init(&sbars[0], 1);                    // the scheduler's expect_tx + bytes
        tc::mbar_init(&sbars[1], kMathWarps);
        tc::mbar_init(&bars[0], kMathWarps);
        tc::mbar_init(&bars[1], kMathWarps);
        tc::mbar_init(&bars[2], 1);
        tc::mbar_init(&bars[3], 1);
        tc::fence_mbar_init();
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    // Launched as a programmatic dependent of the forward: everything above overlaps the
    // forward's last CTAs; nothing below runs before the forward has completed (no-op when
    // there is no such predecessor).
    asm volatile("griddepcontrol.wait;" ::: "memory");
    // the reduce (a programmatic dependent) may be scheduled onto the SMs this grid frees; one
    // CTA per SM here, so it takes no SM that a CTA of this grid still needs
    asm volatile("griddepcontrol.launch_dependents;");
    // Units: the largest unit bounds the balance of the persistent grid (a slice with exactly
    // C active layers is one unit, claimed late), so units just above the mean load per CTA,
    // ceil(T / grid) + 1 layers, balance best (a scheduling model and measurements agree); the
    // job views are visible from here on.
    __shared__ Units s_units;
    __shared__ int s_pairs;
    Units U{P.chunk, P.cmax, P.n_units};
    if (P.adapt) {
        if (threadIdx.x == 0) s_pairs = 0;
        __syncthreads();
        const JobDev& J = P.jobs[0];
        const int ne = J.nz * J.nl;
        int cnt = 0;
        for (int e = threadIdx.x; e < ne; e += kThreads) cnt += J.idd[e] != 0.0 ? 1 : 0;
        cnt = __reduce_add_sync(0xffffffffu, cnt);
        if ((threadIdx.x & 31) == 0) atomicAdd(&s_pairs, cnt);
        __syncthreads();
        if (threadIdx.x == 0) {
            const int g = (int)gridDim.x;
            int c = (s_pairs + g - 1) / g + 1;
            c = c < 1 ? 1 : (c > kMaxChunkCost ? kMaxChunkCost : c);
            const int cm = (J.nl + c - 1) / c;
            s_units = Units{c, cm, J.nz * cm};
        }
        __syncthreads();
        U = s_units;
    }

    if (warp >= kMathWarps) {
        asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;" ::"n"(kCtrlRegs));
        if (warp == kSchedWarp) {
            scheduler_warp(P, U, ring, full, empty, smem, &sbars[0], &sbars[1]);
        } else if (warp == kS1Warp || warp == kS2Warp) {
            const Layout L = make_layout<NARR>(P.N1);
            mma_warp<MODE>(P, L, tc::smem_u32(smem), tmem_base_s, warp == kS1Warp ? 1 : 2, ring,
                           full, empty, bars);
        }
    } else {
        asm volatile("setmaxnreg.inc.sync.aligned.u32 %0;" ::"n"(kMathRegs));
        const Layout L = make_layout<NARR>(P.N1);
        math_warps<MODE>(P, L, smem, tmem_base_s, ring, full, empty, bars, &sbars[0], &sbars[1]);
    }

    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    if (warp == 0) tc::tmem_dealloc(tmem_base_s, kCols);
}

// After the main kernel: dL/dW, the per-pair dot products and dL/dR from the slots, with no
// block waiting on another.  Block (entry chunk, layer l, job): kRedEnt slot entries
// e = j * n1 + i of layer l (n1 = nsx rounded up to 16) times kRedSeg depth segments.  The
// layer's IDD column is staged in shared memory with its last active slice ze; segment s of an
// entry sums IDD * P slot over its quarter of [0, ze) in slice order, its slot values arriving
// by asynchronous 4-byte copies (cp.async: kRedB slices per batch, every copy of a batch in
// flight together; inactive slices copy nothing and read 0); the segments' sums are then added
// in segment order and written as dL/dW[l, j, i] (i < nsx).  One more block per layer (the
// last in x) adds, per active slice, the eight warp partials of <P, W> (dL/dIDD) and <S, W>
// (dL/dsigma, times IDD) in warp order and forms dL/dR_l in FP64 (a fixed tree over the
// block); that block of layer 0 sums the loss partials the same way.  Every sum is in a fixed
// order: deterministic.
constexpr int kRedThreads = 256;
constexpr int kRedEnt = 64;                        // entries per block
constexpr int kRedSeg = kRedThreads / kRedEnt;     // depth segments per entry
constexpr int kRedTile = 1024;                     // slices staged per pass
constexpr int kRedB = 16;                          // slices per copy batch

__device__ __forceinline__ double block_sum_fixed(double v, double* red) {
    const int tid = threadIdx.x;
    red[tid] = v;
    __syncthreads();
    for (int w = kRedThreads / 2; w > 0; w >>= 1) {
        if (tid < w) red[tid] += red[tid + w];
        __syncthreads();
    }
    const double r = red[0];
    __syncthreads();
    return r;
}

__global__ void __launch_bounds__(kRedThreads) adj_tc_reduce_kernel(
    const JobDev* __restrict__ jobs, int with_range, int finalize_loss, const int* __restrict__ err) {
    // a programmatic dependent of the adjoint kernel: wait for its slots (no-op otherwise)
    asm volatile("griddepcontrol.wait;" ::: "memory");
    const JobDev& J = jobs[blockIdx.z];
    const int ec = blockIdx.x, l = blockIdx.y;
    if (l >= J.nl) return;
    const int nz = J.nz, nsx = J.nsx, nsy = J.nsy;
    const int n1 = (nsx + 15) / 16 * 16, per = nsy * n1;
    const int nchunk = (per + kRedEnt - 1) / kRedEnt;   // entry blocks; block nchunk: the dots
    if (ec > nchunk) return;
    const int tid = threadIdx.x, el = tid % kRedEnt, sg = tid / kRedEnt;
    const int e = ec * kRedEnt + el;
    const int ej = e / n1, ei = e - ej * n1;
    const bool own = e < per && ei < nsx;
    const size_t ndots = (size_t)J.nl * nz * kMathWarps;
    const float* slots = J.partial + (size_t)l * nz * per;           // (nz, per) of layer l
    const float* dots = J.partial + (size_t)J.nl * nz * per;          // (2, nl, nz, kMathWarps)
    const double* idd = J.idd + (size_t)l * nz;
    const bool bad = *err != 0 || (J.fwd_err != nullptr && *J.fwd_err != 0);
    const float nan = __int_as_float(0x7fc00000);
    __shared__ double red[kRedThreads];
    if (ec == nchunk) {
        // per job: no dL/dR output, or a missing derivative table, contributes nothing (the
        // heterogeneous range gradient's two job sets use one table each)
        const bool rng = with_range && J.grad_range != nullptr;
        double a = 0.0;
        for (int z = tid; z < nz; z += kRedThreads) {
            const double c = idd[z];
            if (c == 0.0) continue;
            const size_t o = (size_t)l * nz + z;
            const float* pa = dots + o * kMathWarps;
            const float* pb = pa + ndots;
            float sa = 0.f, sb = 0.f;
#pragma unroll
            for (int w = 0; w < kMathWarps; ++w) { sa += pa[w]; sb += pb[w]; }
            const float dsg = (float)c * sb;
            J.dc[o] = sa;
            J.dsg[o] = dsg;
            if (rng)
                a += (J.didd_dr ? (double)sa * J.didd_dr[o] : 0.0) +
                     (J.dsig_dr ? (double)dsg * J.dsig_dr[o] : 0.0);
        }
        if (rng) {
            const double r = block_sum_fixed(a, red);
            if (tid == 0) J.grad_range[l] = bad ? nan : (float)r;
        }
        if (finalize_loss && l == 0) {
            double t = 0.0;
            for (int b = tid; b < J.n_loss_part; b += kRedThreads) t += J.loss_part[b];
            const double sum = block_sum_fixed(t, red);
            if (tid == 0) *J.loss = bad ? (double)nan : sum;
        }
        return;
    }

    __shared__ float s_c[kRedTile];
    __shared__ int s_end;
    __shared__ float sbuf[kRedB][kRedThreads];
    __shared__ float s_part[kRedSeg][kRedEnt];
    float acc = 0.f;
    const float* se = slots + (own ? e : 0);
    for (int zt = 0; zt < nz; zt += kRedTile) {
        const int zn = min(kRedTile, nz - zt);
        __syncthreads();   // the previous pass's reads of s_c and s_end are done
        if (tid == 0) s_end = 0;
        for (int z = tid; z < zn; z += kRedThreads) s_c[z] = (float)idd[zt + z];
        __syncthreads();
        for (int z = tid; z < zn; z += kRedThreads)
            if (s_c[z] != 0.f) atomicMax(&s_end, z + 1);
        __syncthreads();
        const int ze = s_end;   // slices [0, ze) of the pass hold every active one
        const int q = (ze + kRedSeg - 1) / kRedSeg;
        const int zb = sg * q, zf = min(ze, zb + q);
        for (int z0 = zb; z0 < zf; z0 += kRedB) {
#pragma unroll
            for (int h = 0; h < kRedB; ++h) {
                const int z = z0 + h;
                const bool rd = own && z < zf && s_c[z < zf ? z : zb] != 0.f;
                asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(
                                 tc::smem_u32(&sbuf[h][tid])),
                             "l"(se + (size_t)(zt + (rd ? z : 0)) * per), "r"(rd ? 4 : 0)
                             : "memory");
            }
            asm volatile("cp.async.commit_group;" ::: "memory");
            asm volatile("cp.async.wait_group 0;" ::: "memory");
#pragma unroll
            for (int h = 0; h < kRedB; ++h) {
                const int z = z0 + h;
                const float cf = z < zf ? s_c[z] : 0.f;
                acc = fmaf(cf, sbuf[h][tid], acc);
            }
        }
    }
    s_part[sg][el] = acc;
    __syncthreads();
    if (sg == 0 && own) {
        float g = s_part[0][el];
#pragma unroll
        for (int k = 1; k < kRedSeg; ++k) g += s_part[k][el];
        J.grad_w[((size_t)l * nsy + ej) * nsx + ei] = bad ? nan : g;
    }
}

template <int MODE>
size_t adj_smem_bytes(int N1) {
    using Pr = Prec<MODE>;
    const size_t narr = Pr::NPROD == 3 ? 2 : 1;
    return narr * 2u * (128u * 128u + 2u * (size_t)N1 * 128u);
}

template <int MODE>
int launch_mode(const Params& P0, cudaStream_t s) {
    // the setmaxnreg split needs the full launch allotment, or its increase never returns
    int max_dyn = 0;
    PBD_TRY(smem_optin((const void*)adj_tc_kernel<MODE>, -1, kLaunchRegsNeeded, &max_dyn));
    Params P = P0;
    size_t smem = adj_smem_bytes<MODE>(P.N1);
    // the staging buffer (one 128 x 128 FP32 slice) after the operands, when it fits
    P.o_stage = (uint32_t)align_up(smem, 1024);
    if (P.stage && P.o_stage + 65536u > (size_t)max_dyn) P.stage = 0;
    if (P.stage) smem = P.o_stage + 65536u;
    // >= 116 KiB: one CTA, and its 512 TMEM columns, per SM
    smem = std::max<size_t>(smem, 116u * 1024u);
    if (smem > (size_t)max_dyn) return PBD_ERR_NO_SMEM;
    const int grid = std::max(1, std::min(P.n_units, num_sms()));
    prof_mark(kProfAdj, 0, s);
    PBD_TRY(launch_dependent(adj_tc_kernel<MODE>, dim3(grid), dim3(kThreads), smem, s, P));
    prof_mark(kProfAdj, 1, s);
    return PBD_OK;
}

}  // namespace

int tc_adjoint_dims(int precision, const pbd_field* f, int* N1) {
    if (precision == PBD_PREC_FP32) return PBD_ERR_UNSUPPORTED;
    if (f->nx > kTile || f->ny > kTile || f->n_sy > 64 || f->n_sx > 64) return PBD_ERR_UNSUPPORTED;
    *N1 = (f->n_sx + 15) / 16 * 16;
    return PBD_OK;
}

size_t tc_adjoint_counter_ints(int n_jobs, int max_layers) {
    (void)n_jobs;
    (void)max_layers;
    return 2u;
}

size_t tc_adjoint_slot_elems(const pbd_field* f) {
    // slot rows of nsx rounded up to 16 floats: every job's slots start on a 64-byte boundary
    const size_t per = (size_t)f->n_sy * (size_t)((f->n_sx + 15) / 16 * 16);
    const size_t pairs = (size_t)f->n_layers * f->nz;
    return pairs * per + 2u * pairs * kMathWarps;
}

int launch_adjoint_tc(int precision, JobDev* jobs_dev, const JobDev* jobs_host, int n_jobs,
                      int* counter, int* err, int chunk, int with_range, int finalize_loss,
                      int counters_zeroed, cudaStream_t s) {
    Params P{};
    P.jobs = jobs_dev;
    P.n_jobs = n_jobs;
    P.chunk = chunk;
    P.counter = counter;
    P.err = err;
    P.wait_ns = wait_limit_ns();
    P.hold = test_hold();
    // bulk copies of the dL/dD slices need them contiguous and 16-byte aligned
    P.stage = 1;
    for (int j = 0; j < n_jobs; ++j) {
        const JobDev& J = jobs_host[j];
        if (((size_t)J.nx * J.ny) % 4 != 0 ||
            (reinterpret_cast<uintptr_t>(J.grad_dose) & 15u) != 0)
            P.stage = 0;
    }
    int cm = 1, nzm = 1, max_l = 1, max_per = 1;
    for (int j = 0; j < n_jobs; ++j) {
        pbd_field f{};
        f.nx = jobs_host[j].nx; f.ny = jobs_host[j].ny;
        f.n_sx = jobs_host[j].nsx; f.n_sy = jobs_host[j].nsy;
        int n1 = 0;
        PBD_TRY(tc_adjoint_dims(precision, &f, &n1));
        P.N1 = std::max(P.N1, n1);
        cm = std::max(cm, (jobs_host[j].nl + chunk - 1) / chunk);
        nzm = std::max(nzm, jobs_host[j].nz);
        max_l = std::max(max_l, jobs_host[j].nl);
        max_per = std::max(max_per, jobs_host[j].nsy * ((jobs_host[j].nsx + 15) / 16 * 16));
    }
    P.cmax = cm;
    // one job and no explicit schedule: the CTAs derive the unit size from the active pairs
    P.adapt = (n_jobs == 1 && schedule_adj_override() == 0) ? 1 : 0;
    P.sym = 1;
    for (int j = 0; j < n_jobs; ++j) {
        const JobDev& J = jobs_host[j];
        if (!(J.nx == J.ny && J.ox == J.oy && J.dx == J.dy && J.nsx == J.nsy && J.sx0 == J.sy0 &&
              J.dsx == J.dsy))
            P.sym = 0;
    }
    const long long units = (long long)nzm * cm * n_jobs;
    if (units > (1LL << 30)) return PBD_ERR_UNSUPPORTED;
    P.n_units = (int)units;
    if (!counters_zeroed)
        PBD_TRY(cuda_rc(cudaMemsetAsync(counter, 0,
                                        tc_adjoint_counter_ints(n_jobs, max_l) * sizeof(int), s)));
    int rc = PBD_OK;
    if (precision == PBD_PREC_BF16) rc = launch_mode<PBD_PREC_BF16>(P, s);
    else rc = launch_mode<PBD_PREC_BF16X3>(P, s);
    PBD_TRY(rc);
    PBD_TRY(launch_dependent(adj_tc_reduce_kernel,
                             dim3((max_per + kRedEnt - 1) / kRedEnt + 1, max_l, n_jobs),
                             dim3(kRedThreads), 0, s, (const JobDev*)jobs_dev, with_range,
                             finalize_loss, (const int*)err));
    count_launch(2);
    return PBD_OK;
}

}  // namespace pbd
