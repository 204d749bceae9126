// tc_fwd16.cu -- forward dose on the 5th-generation tensor cores in split FP16 (hi + lo halves,
// three products, FP32 accumulation): PBD_PREC_FP16X3.
//
// For every active (layer l, slice z) and 128 x 128 lateral tile ("step"):
//
//   stage 1   U[x, n]  = sum_i Gx[x, i] [Wh; Wl][n, i]     M = 128 (x), N = 2 N1, K = K1
//             U[x, N1 + j] += sum_i Gxl[x, i] Wh[j, i]      M = 128, N = N1 (cross products)
//   stage 2   Db[y, x]  = sum_j Gyh[y, j] sUh[x, j]         M = N = 128, K = N1 (hi * hi, per step)
//             Dc[y, x] += sum_j Gyh sUl + Gyl sUh           (cross products, per unit)
//
// with unnormalised Gaussians exp(-d^2 / (2 s^2)) generated on the chip, s U = IDD / (2 pi s^2)
// (U big + U cross), and every operand split a = hi + lo, hi = fp16(a), lo = fp16(a - hi)
// (11 + 11 significant bits; the dropped lo * lo term is ~2^-22 of a product).  FP16 has a 5-bit
// exponent, so every operand is scaled by a power of two into [2^-14, 2^15]: the Gaussians by
// 2^14 (folded into the exponent), each layer's W by 2^e_l (its largest |W| lands in
// [2^14, 2^15)), and s U by 2^k with k chosen per unit from a bound on |s U|
// (max|W_l| (1 + sqrt(2 pi) s / dx_spot) s); the drain divides by the unit's power of two
// exactly.  Values that still fall below the FP16 normal range are at most 2^-38 of the
// operand's scale.  kind::f16 takes K = 16 per MMA (twice TF32's 8) at twice the TF32 rate.
//
// CTA = 8 math warps, 1 scheduler / producer warp, 3 MMA warps; one CTA per SM (persistent).
//  * Scheduler warp: units (slice z, chunk c of <= C active layers, tile) from an atomic
//    counter in z-major order (the shallow slices, which see the most layers, first); per unit
//    the scale exponent; one step per active layer into an 8-deep ring.  As producer it also brings each step's spot map into a shared-memory ring
//    with one bulk copy (cp.async.bulk, mbarrier transaction count): the maps are packed once
//    per call by pack_w16_kernel into the exact operand image (hi rows then lo rows, K-major
//    8 x 16-byte core matrices), so the math warps never load W.
//  * Math warps, software-pipelined by one step: G(n+1) (Gy, Gx of the next step into
//    double-buffered shared memory, from per-thread squared-distance tables formed in FP64 at
//    a unit's first step), then E1(n) (U from TMEM, scaled, split into stage 2's B operand),
//    then DR(n-1) (the hi * hi product of the step before from TMEM into FP32 registers, and
//    at a unit's end its cross products and the output).
//  * MMA warps: stage 1 (waits for the spot map, Gx and a free U), stage 2 hi * hi into one of
//    two D accumulators, stage 2 cross products into the unit's accumulator; each commits to
//    the barriers that release its operands and publish its result.
//
// Accumulation as in the TF32 forward: the large products of a step go to a fresh accumulator
// that the math warps add in FP32 registers (the tensor core truncates when it accumulates),
// the cross products (~2^-11 of them) stay in one accumulator per unit.
//
// Output (per math warp: 32 rows x 64 columns of the tile): plain stores of the unit's partial
// slice (or, where every unit holds all layers of its slice, of the dose itself); a finalize
// pass then sums each voxel's partials in chunk order -- deterministic -- and, with the loss,
// forms dL/dD = 2 m (D - P) and FP64 partial sums of the loss: the persistent kernel never
// waits on memory for its outputs.  Every wait is bounded (2 s of %globaltimer, or the test
// limit): a warp whose wait runs out sets the error word and leaves, after the MMAs and bulk
// copies it issued have completed (bounded), and the finalize (or poison) pass turns the
// results into NaN.
#include <algorithm>
#include <cuda_fp16.h>
#include <math.h>
#include <string.h>

#include "pbd_internal.cuh"
#include "tc_common.cuh"

namespace pbd {
namespace {
using namespace tcc;

constexpr int kMathWarps = kTcFwdWarps;
constexpr int kMath = 32 * kMathWarps;     // 256 math threads: warpgroups 0 and 1
constexpr int kSchedWarp = kMathWarps;     // warpgroup 2: scheduler / producer, then 3 MMA warps
constexpr int kS1Warp = kMathWarps + 1;
constexpr int kS2Warp = kMathWarps + 2;
constexpr int kS3Warp = kMathWarps + 3;
constexpr int kThreads = kMath + 128;
constexpr int kMathRegs = 208, kCtrlRegs = 80;
constexpr int kLaunchRegsNeeded = (kMath * kMathRegs + 128 * kCtrlRegs + kThreads - 1) / kThreads;
constexpr int kRing = 8;                   // step slots
constexpr uint32_t kCols = 512;
// TMEM columns: D big [0,128) and [128,256) (alternating steps), D cross [256,384), U [384, +2 N1)
constexpr uint32_t kColDb = 0, kColDc = 256, kColU = 384;
constexpr float kGScale = 14.0f;           // log2 of the Gaussians' scale
constexpr int kGExp = 14;

// kSym: Gx == Gy bit for bit (same grid and lattice along x and y, a diagonal tile): G writes
// Gy only and stage 1 reads it as its A operand
enum : int { kFirst = 1, kLast = 2, kEnd = 4, kZero = 8, kTab = 16, kSym = 32 };

struct Step {
    int job, z, tile, l;
    int chunk, nch, flags, kd;   // kd: D = accumulator * 2^-kd
    float a2, f1;                // exponent scale (log2 e / (2 s^2)); U -> s U factor
    const uint8_t* wimg;         // packed spot map of (job, layer)
};

struct Params {
    const JobDev* jobs;
    int n_jobs, chunk, cmax, tmax, n_units;
    int* counter;                // [0] unit counter
    int* err;                    // error word
    unsigned long long wait_ns;
    int hold;
    int with_loss;
    int sym;                     // every job symmetric in x and y (see kSym)
    int K1, N1;
    int nR, nA1, nA2, nB2;       // buffers: spot-map ring slots, Gx, Gy (>= 2), sU
    uint32_t img;                // bytes of one packed spot map (= ring slot)
    uint32_t oW, oA1, oA2, oB2, oTab;   // shared-memory offsets
    int ty4, tx4;                // float4 groups of the per-thread distance table
    const uint8_t* wpack;        // (n_jobs, lmax) packed spot maps
    const float* wmax;           // (n_jobs, lmax) max |W_l|
    const int* wexp;             // (n_jobs, lmax) e_l
    int lmax;
};

__device__ __forceinline__ uint32_t h2bits(__half2 h) { return *reinterpret_cast<uint32_t*>(&h); }

// a = hi + lo for two adjacent K elements (already scaled into FP16's range), packed as
// {element 0 in the low half, element 1 in the high half}.  hi = a rounded to 11 significant
// bits in FP32 with integer operations (half an ulp added to the magnitude, low 13 bits
// cleared), so a - hi is exact and hi converts to FP16 exactly (in FP16's normal range; below it
// the conversion's rounding is at most 2^-25 of the operand's scale); lo = fp16(a - hi).
__device__ __forceinline__ float round11(float a) {
    return __uint_as_float((__float_as_uint(a) + 0x1000u) & 0xFFFFE000u);
}
__device__ __forceinline__ void split2(float a, float b, uint32_t& hi, uint32_t& lo) {
    const float ha = round11(a), hb = round11(b);
    hi = h2bits(__floats2half2_rn(ha, hb));
    lo = h2bits(__floats2half2_rn(a - ha, b - hb));
}

__device__ __forceinline__ void split8(const float* v, uint4& hi, uint4& lo) {
    uint32_t h[4], l[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) split2(v[2 * q], v[2 * q + 1], h[q], l[q]);
    hi = make_uint4(h[0], h[1], h[2], h[3]);
    lo = make_uint4(l[0], l[1], l[2], l[3]);
}

__device__ __forceinline__ void bulk_copy(uint32_t dst, const void* src, uint32_t bytes,
                                          uint64_t* bar) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(tc::smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
    asm volatile(
        "cp.async.bulk.shared::cta.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            dst),
        "l"(src), "r"(bytes), "r"(tc::smem_u32(bar))
        : "memory");
}

// ------------------------------------------------------------------------------------------
// Spot maps -> packed FP16 operand images, one block per (layer, job).  Image of layer l:
// K1 / 8 planes of 2 N1 rows x 16 bytes (8 halves of K); rows j < N1 hold hi(W[j, i] 2^e),
// rows N1 + j hold lo; zero outside the lattice.
// ------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(256) pack_w16_kernel(const JobDev* __restrict__ jobs, int K1,
                                                       int N1, int lmax, uint32_t img,
                                                       uint8_t* wpack, float* wmax, int* wexp,
                                                       int* unit_counter, JobPair inst,
                                                       int has_inst, JobDev* inst_dst,
                                                       int* inst_status) {
    // the dose kernel (a programmatic dependent) may start its prologue now; it reads the packed
    // maps, the unit counter and the job views only after griddepcontrol.wait, i.e. after this
    // grid has completed
    asm volatile("griddepcontrol.launch_dependents;");
    // launched as a programmatic dependent of the kernel before it (the job install, or the
    // previous call's last kernel when this grid installs the views itself)
    asm volatile("griddepcontrol.wait;" ::: "memory");
    if (blockIdx.x == 0 && blockIdx.y == 0) {
        if (threadIdx.x == 0) *unit_counter = 0;
        if (has_inst) {
            // the call's job views, status header and cleared counters (install_jobs_kernel's work)
            if ((int)threadIdx.x < inst.n) inst_dst[threadIdx.x] = inst.j[threadIdx.x];
            if (inst_status && (int)threadIdx.x < kStatusInts) inst_status[threadIdx.x] = 0;
            if (inst.zero && (int)threadIdx.x < inst.nzero) inst.zero[threadIdx.x] = 0;
        }
    }
    const JobDev& J = has_inst ? inst.j[blockIdx.y] : jobs[blockIdx.y];
    const int l = blockIdx.x;
    if (l >= J.nl) return;
    const int nsx = J.nsx, nsy = J.nsy, per = nsx * nsy;   // <= 64 x 64
    const float* w = J.w + (size_t)l * per;
    __shared__ float red[8];
    __shared__ float ws[64 * 64];
    // the layer's weights into shared memory, every load of a thread issued together
    float m = 0.f;
    bool nonfinite = false;
    {
        float v[16];
#pragma unroll
        for (int q = 0; q < 16; ++q) {
            const int e = threadIdx.x + q * 256;
            v[q] = e < per ? __ldg(w + e) : 0.f;
        }
#pragma unroll
        for (int q = 0; q < 16; ++q) {
            const int e = threadIdx.x + q * 256;
            if (e < per) ws[e] = v[q];
            const float a = fabsf(v[q]);
            if (!(a <= 3.0e38f)) nonfinite = true;   // NaN or inf: leave the layer unscaled
            m = fmaxf(m, a);
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    nonfinite = __syncthreads_or(nonfinite);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    m = red[0];
#pragma unroll
    for (int k = 1; k < 8; ++k) m = fmaxf(m, red[k]);
    int q = 0;
    (void)frexpf(m, &q);                        // m = f 2^q, f in [0.5, 1)
    const int e = (m > 0.f && !nonfinite) ? 15 - q : 0;   // m 2^e in [2^14, 2^15)
    uint8_t* out = wpack + ((size_t)blockIdx.y * lmax + l) * img;
    const int rows = 2 * N1, items = (K1 / 8) * rows;
    for (int it = threadIdx.x; it < items; it += blockDim.x) {
        const int g = it / rows, r = it % rows;
        const int j = r < N1 ? r : r - N1;
        float v[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const int i = 8 * g + k;
            v[k] = (i < nsx && j < nsy) ? ldexpf(ws[j * nsx + i], e) : 0.f;
        }
        uint4 hi, lo;
        split8(v, hi, lo);
        *reinterpret_cast<uint4*>(out + (size_t)g * rows * 16 + (size_t)r * 16) = r < N1 ? hi : lo;
    }
    if (threadIdx.x == 0) {
        wmax[(size_t)blockIdx.y * lmax + l] = m;
        wexp[(size_t)blockIdx.y * lmax + l] = e;
    }
}

// ------------------------------------------------------------------------------------------
// Scheduler / producer warp.
// ------------------------------------------------------------------------------------------
__device__ __forceinline__ void scheduler_warp(const Params& P, uint8_t* smem, Step* ring,
                                               uint64_t* full, uint64_t* empty, uint64_t* wfull,
                                               uint64_t* wempty) {
    const int lane = threadIdx.x & 31;
    const unsigned FULL = 0xffffffffu;
    const uint32_t sW = tc::smem_u32(smem) + P.oW;
    int k = 0, n = 0;          // ring pushes; steps with a spot map (bulk copies issued)
    bool ok = true;

    auto push = [&](int src, const Step& st) -> bool {
        const int slot = k % kRing, u = k / kRing;
        bool w = wait_bar(&empty[slot], (uint32_t)((u & 1) ^ 1), P.wait_ns);
        const bool mapped = !(st.flags & (kZero | kEnd));
        if (mapped && n >= P.nR) {   // the ring slot of the spot map is free again
            const int ws = n % P.nR;
            w = w && wait_bar(&wempty[ws], (uint32_t)(((n / P.nR) - 1) & 1), P.wait_ns);
        }
        if (!__all_sync(FULL, w)) return false;
        if (lane == src) {
            if (mapped) bulk_copy(sW + (uint32_t)(n % P.nR) * P.img, st.wimg, P.img, &wfull[n % P.nR]);
            ring[slot] = st;
            tc::mbar_arrive(&full[slot]);
        }
        __syncwarp();
        ++k;
        if (__shfl_sync(FULL, mapped ? 1 : 0, src)) ++n;
        return true;
    };

    if (!P.hold) {
        // The unit's data (depth dose, width, spot-map scale of each of its slice's layers) is
        // loaded in one batch per 32 layers: every load of a unit in flight together.
        constexpr int kG = 2;                       // layer groups kept in registers (<= 64 layers)
        // A unit is claimed once the one before is pushed (dynamic balance); its loads then
        // overlap the steps still queued in the rings.
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
            double ivg[kG], sg[kG];
            float wmg[kG];
            int ewg[kG];
            auto load = [&](int b, double& iv, double& sv, float& wm, int& ew) {
                const int l = b + lane;
                const bool in = l < nl;
                iv = in ? idd[(size_t)l * nz + z] : 0.0;
                sv = in ? J.sigma[(size_t)l * nz + z] : 1.0;
                wm = in ? P.wmax[(size_t)job * P.lmax + l] : 0.f;
                ew = in ? P.wexp[(size_t)job * P.lmax + l] : 0;
            };
            const bool cached = nl <= 32 * kG;
            if (cached) {
#pragma unroll
                for (int g = 0; g < kG; ++g) load(32 * g, ivg[g], sg[g], wmg[g], ewg[g]);
            }
            auto group = [&](int b, double& iv, double& sv, float& wm, int& ew) {
                if (cached) {
                    const int g = b >> 5;
                    iv = g == 0 ? ivg[0] : ivg[1];
                    sv = g == 0 ? sg[0] : sg[1];
                    wm = g == 0 ? wmg[0] : wmg[1];
                    ew = g == 0 ? ewg[0] : ewg[1];
                } else {
                    load(b, iv, sv, wm, ew);
                }
            };
            int tot = 0;
            for (int b = 0; b < nl; b += 32) {
                double iv, sv; float wm; int ew;
                group(b, iv, sv, wm, ew);
                tot += __popc(__ballot_sync(FULL, iv != 0.0));
            }
            const int nch = (tot + P.chunk - 1) / P.chunk;
            // the finalize pass sums nch partial slices of slice z (every unit of the slice
            // writes the same count)
            if (!J.direct && c == 0 && tile == 0 && lane == 0) J.nchunks[z] = nch;
            if (tot == 0) {
                // a slice no layer reaches: zeros written here when the output is the dose
                // itself, else by the finalize pass (zero partial slices)
                if (c == 0 && J.direct) {
                    Step st{};
                    st.job = job; st.z = z; st.tile = tile;
                    st.nch = 1; st.flags = kFirst | kLast | kZero;
                    if (!push(0, st)) { ok = false; break; }
                }
                continue;
            }
            if (c >= nch) continue;
            const int r0 = c * P.chunk, r1 = min(tot, r0 + P.chunk);
            // the unit's scale exponent: the smallest over its layers of
            // 14 - ceil(log2(bound on |s U|)), so that every s U of the unit fits FP16
            int ks = 127;
            {
                int rank = 0;
                for (int b = 0; b < nl && rank < r1; b += 32) {
                    double iv, sv; float wm; int ew;
                    group(b, iv, sv, wm, ew);
                    const unsigned bal = __ballot_sync(FULL, iv != 0.0);
                    const int my = rank + __popc(bal & ((1u << lane) - 1u));
                    if (iv != 0.0 && my >= r0 && my < r1) {
                        const double s = fmax(sv, 1e-9);
                        const double bnd = fabs(iv) * kInv2Pi / (s * s) * (double)wm *
                                           (1.0 + 2.5066282746310002 * s / J.dsx);
                        int q = 0;
                        if (bnd > 0.0 && bnd < 1e300) {
                            (void)frexp(bnd, &q);          // bnd < 2^q
                            ks = min(ks, 14 - q);
                        }
                    }
                    rank += __popc(bal);
                }
                ks = __reduce_min_sync(FULL, ks);
                ks = ks > 100 ? 100 : (ks < -100 ? -100 : ks);
            }
            const int tyy = tile / J.ntx, txx = tile % J.ntx;
            const int sym = (P.sym && tyy == txx) ? kSym : 0;
            int rank = 0;
            for (int b = 0; b < nl && rank < r1 && ok; b += 32) {
                double iv, sv; float wm; int ew;
                group(b, iv, sv, wm, ew);
                const bool a = iv != 0.0;
                const unsigned bal = __ballot_sync(FULL, a);
                const int my = rank + __popc(bal & ((1u << lane) - 1u));
                const bool mine = a && my >= r0 && my < r1;
                Step st{};
                if (mine) {
                    const int l = b + lane;
                    const double s = fmax(sv, 1e-9);
                    st.job = job; st.z = z; st.tile = tile; st.l = l;
                    st.chunk = c; st.nch = nch;
                    st.flags = (my == r0 ? kFirst | kTab : 0) | (my == r1 - 1 ? kLast : 0) | sym;
                    // U = 2^(14 + e_l) U_true; s U enters stage 2 as 2^ks s U_true, so
                    // D = 2^(14 + ks) D_true
                    st.kd = kGExp + ks;
                    st.a2 = (float)(kLog2e / (2.0 * s * s));
                    st.f1 = (float)ldexp(iv * kInv2Pi / (s * s), ks - ew - kGExp);
                    st.wimg = P.wpack + ((size_t)job * P.lmax + l) * P.img;
                }
                unsigned emit = __ballot_sync(FULL, mine);
                while (emit) {
                    const int src = __ffs(emit) - 1;
                    emit &= emit - 1u;
                    Step sb;
                    // every lane passes the emitting lane's step (push reads its flags)
                    sb.flags = __shfl_sync(FULL, st.flags, src);
                    if (lane == src) sb = st;
                    if (!push(src, sb)) { ok = false; break; }
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
    // the spot-map copies still in flight land before the block exits
    const int first = n > P.nR ? n - P.nR : 0;
    for (int m = first; m < n; ++m)
        (void)wait_bar(&wfull[m % P.nR], (uint32_t)((m / P.nR) & 1), P.wait_ns);
    if (!ok && lane == 0) atomicExch(P.err, 1);
}

// ------------------------------------------------------------------------------------------
// MMA warps.  role 1: stage 1; role 2: stage 2 hi * hi; role 3: stage 2 cross products.
// bars: [0,4) wfull, [4,8) wempty (ring slots), then
//   a1r[2], a1f[2], a2r[3], a2f[3], b2r[2], b2f[2], uf (U full), uu (U free),
//   df[2] (D big full), du[2] (D big free), cf (cross full), cu (cross free)
// ------------------------------------------------------------------------------------------
struct Bars {
    uint64_t *wfull, *wempty, *a1r, *a1f, *a2r, *a2f, *b2r, *b2f, *uf, *uu, *df, *du, *cf, *cu;
};

__device__ __forceinline__ Bars make_bars(uint64_t* b) {
    Bars B;
    B.wfull = b; B.wempty = b + 4;
    B.a1r = b + 8; B.a1f = b + 10; B.a2r = b + 12; B.a2f = b + 15; B.b2r = b + 18; B.b2f = b + 20;
    B.uf = b + 22; B.uu = b + 23; B.df = b + 24; B.du = b + 26; B.cf = b + 28; B.cu = b + 29;
    return B;
}
constexpr int kNumBars = 30;

__device__ __forceinline__ void mma_warp(const Params& P, uint32_t sbase, uint32_t tb, int role,
                                         const Step* ring, uint64_t* full, uint64_t* empty,
                                         const Bars& B) {
    const int lane = threadIdx.x & 31;
    const int K1 = P.K1, N1 = P.N1;
    const uint32_t plA = 128u * 16u;                 // plane of a 128-row operand
    const uint32_t plW = 2u * (uint32_t)N1 * 16u;    // plane of the spot map (2 N1 rows)
    const uint32_t aBytes1 = (uint32_t)K1 * 256u;    // one half (hi or lo) of a Gx buffer
    const uint32_t aBytes2 = (uint32_t)N1 * 256u;    // one half of a Gy / sU buffer
    const uint32_t id1w = tc::instr_desc(128, 2 * N1, 0u);
    const uint32_t id1n = tc::instr_desc(128, N1, 0u);
    const uint32_t id2 = tc::instr_desc(128, 128, 0u);
    int k = 0, n = 0, seg = 0;
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
        if (role == 1) {
            const int ws = n % P.nR, ia = n % P.nA1, ia2 = n % P.nA2;
            ok = wait_bar(&B.wfull[ws], (uint32_t)((n / P.nR) & 1), P.wait_ns);
            ok = ok && wait_bar(&B.a1r[ia], (uint32_t)((n / P.nA1) & 1), P.wait_ns);
            if (n > 0) ok = ok && wait_bar(B.uu, (uint32_t)((n - 1) & 1), P.wait_ns);
            if (!__all_sync(0xffffffffu, ok)) break;
            tc::fence_after_sync();
            if (lane == 0) {
                // symmetric step: Gx is the Gy buffer (same bits, same layout; K1 == N1)
                const bool sym = (flags & kSym) != 0;
                const uint32_t a = sym ? sbase + P.oA2 + (uint32_t)ia2 * 2u * aBytes2
                                       : sbase + P.oA1 + (uint32_t)ia * 2u * aBytes1;
                const uint32_t alo = sym ? aBytes2 : aBytes1;
                const uint32_t w = sbase + P.oW + (uint32_t)ws * P.img;
                for (int st = 0; st < K1 / 16; ++st) {
                    const uint32_t oa = (uint32_t)st * 2u * plA, ow = (uint32_t)st * 2u * plW;
                    tc::mma_bf16(tb + kColU, tc::smem_desc(a + oa, plA, 128),
                                 tc::smem_desc(w + ow, plW, 128), id1w, st > 0 ? 1u : 0u);
                    tc::mma_bf16(tb + kColU + (uint32_t)N1, tc::smem_desc(a + alo + oa, plA, 128),
                                 tc::smem_desc(w + ow, plW, 128), id1n, 1u);
                }
                tc::commit(B.uf);
                tc::commit(&B.a1f[ia]);
                tc::commit(&B.wempty[ws]);
                tc::commit(&B.a2f[ia2]);   // Gy buffers are released by stage 1 as well
            }
            __syncwarp();
        } else {
            const int ia = n % P.nA2, ib = n % P.nB2, db = n & 1;
            ok = wait_bar(&B.a2r[ia], (uint32_t)((n / P.nA2) & 1), P.wait_ns);
            ok = ok && wait_bar(&B.b2r[ib], (uint32_t)((n / P.nB2) & 1), P.wait_ns);
            const bool first = (flags & kFirst) != 0;
            if (role == 2 && n >= 2)
                ok = ok && wait_bar(&B.du[db], (uint32_t)(((n >> 1) - 1) & 1), P.wait_ns);
            if (role == 3 && first && seg > 0)
                ok = ok && wait_bar(B.cu, (uint32_t)((seg - 1) & 1), P.wait_ns);
            if (!__all_sync(0xffffffffu, ok)) break;
            tc::fence_after_sync();
            if (lane == 0) {
                const uint32_t a = sbase + P.oA2 + (uint32_t)ia * 2u * aBytes2;
                const uint32_t b = sbase + P.oB2 + (uint32_t)ib * 2u * aBytes2;
                for (int st = 0; st < N1 / 16; ++st) {
                    const uint32_t o = (uint32_t)st * 2u * plA;
                    if (role == 2) {
                        tc::mma_bf16(tb + kColDb + (uint32_t)db * 128u, tc::smem_desc(a + o, plA, 128),
                                     tc::smem_desc(b + o, plA, 128), id2, st > 0 ? 1u : 0u);
                    } else {
                        tc::mma_bf16(tb + kColDc, tc::smem_desc(a + o, plA, 128),
                                     tc::smem_desc(b + aBytes2 + o, plA, 128), id2,
                                     (first && st == 0) ? 0u : 1u);
                        tc::mma_bf16(tb + kColDc, tc::smem_desc(a + aBytes2 + o, plA, 128),
                                     tc::smem_desc(b + o, plA, 128), id2, 1u);
                    }
                }
                if (role == 2) tc::commit(&B.df[db]);
                tc::commit(&B.a2f[ia]);
                tc::commit(&B.b2f[ib]);
                if (role == 3 && (flags & kLast)) tc::commit(B.cf);
            }
            __syncwarp();
            if (role == 3 && (flags & kLast)) ++seg;
        }
        ++n;
    }
    if (!ok && lane == 0) atomicExch(P.err, 1);
    // this warp's last MMAs are complete before the block frees its TMEM
    if (n > 0) {
        const int m = n - 1;
        if (role == 1) (void)wait_bar(&B.a1f[m % P.nA1], (uint32_t)((m / P.nA1) & 1), P.wait_ns);
        else (void)wait_bar(&B.b2f[m % P.nB2], (uint32_t)((m / P.nB2) & 1), P.wait_ns);
    }
}

// ------------------------------------------------------------------------------------------
// Math warps.
// ------------------------------------------------------------------------------------------
__device__ __forceinline__ void math_warps(const Params& P, uint8_t* smem, uint32_t tb,
                                           const Step* ring, uint64_t* full, uint64_t* empty,
                                           const Bars& B) {
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int K1 = P.K1, N1 = P.N1;
    const int sp = warp & 3, half = warp >> 2;
    const uint32_t lane_base = (uint32_t)(32 * sp) << 16;
    const int trow = 32 * sp + lane;                 // TMEM lane = tile row of this thread
    const int grow = tid & 127, ghalf = tid >> 7;    // operand row and chunk parity generated
    const uint32_t aBytes1 = (uint32_t)K1 * 256u, aBytes2 = (uint32_t)N1 * 256u;
    float4* tab = reinterpret_cast<float4*>(smem + P.oTab);
    constexpr int kMaxR = 64 / 16;                   // chunk pairs per thread (K <= 64)

    float dsum[64];
#pragma unroll
    for (int q = 0; q < 64; ++q) dsum[q] = 0.f;
    bool ok = true;
    int k = 0;         // ring reads
    int ng = 0;        // steps generated (G done)
    int useg = 0;      // units whose cross accumulator was drained
    Step s1{}, s2{};   // step ng - 1 (awaiting E1) and ng - 2 (awaiting DR), when pending

    // Output of this warp's rows of a finished unit: its dose rows when the unit holds every
    // layer of a slice whose output is the dose itself (or zeros, for a slice no layer
    // reaches), else its partial slice (chunk); the finalize pass sums the partials in chunk
    // order and forms the loss.  Plain stores: nothing here waits.
    auto output = [&](const Step& st, bool zero) {
        const JobDev& J = P.jobs[st.job];
        const int ty = st.tile / J.ntx, tx = st.tile % J.ntx;
        const int y = ty * kTile + trow, xb = tx * kTile + half * 64;
        if (y < J.ny) {
            const size_t n3 = (size_t)J.nz * J.ny * J.nx;
            float* o = (J.direct ? J.dose : J.partial + (size_t)st.chunk * n3) +
                       ((size_t)st.z * J.ny + y) * J.nx + xb;
            const bool vec = xb + 64 <= J.nx && (J.nx & 3) == 0;
            if (zero) {
                for (int q = 0; q < 64; ++q)
                    if (xb + q < J.nx) o[q] = 0.f;
            } else {
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
        }
        if (!zero) {
#pragma unroll
            for (int q = 0; q < 64; ++q) dsum[q] = 0.f;
        }
    };

    // G: the Gaussian operands of step m (= ng) into buffers A1[m % nA1], A2[m % nA2].  Stage 2
    // of step m - 2 becomes ready only in this iteration (E1 of step m - 1 precedes it), so with
    // three Gy buffers G never waits for it.
    auto gen = [&](const Step& st, int m) -> bool {
        const int ia = m % P.nA1, ia2 = m % P.nA2;
        bool w = true;
        if (m >= P.nA1) w = wait_bar(&B.a1f[ia], (uint32_t)(((m / P.nA1) - 1) & 1), P.wait_ns);
        if (m >= P.nA2)
            w = w && wait_bar(&B.a2f[ia2], (uint32_t)(((m / P.nA2) - 1) & 1), P.wait_ns);
        if (!__all_sync(0xffffffffu, w)) return false;
        const JobDev& J = P.jobs[st.job];
        if (st.flags & kTab) {
            // this thread's squared distances (FP64 differences), +inf outside the lattice
            const int ty = st.tile / J.ntx, tx = st.tile % J.ntx;
            const double cx = 0.5 * (double)(J.nsx - 1), cy = 0.5 * (double)(J.nsy - 1);
            const double yv = J.oy + (double)(ty * kTile + grow) * J.dy;
            const double xv = J.ox + (double)(tx * kTile + grow) * J.dx;
#pragma unroll 1
            for (int r = 0; r < kMaxR; ++r) {
                const int g = ghalf + 2 * r;
                if (r < N1 / 16) {
                    float d2[8];
#pragma unroll
                    for (int q = 0; q < 8; ++q) {
                        const int j = 8 * g + q;
                        const float d = (float)(yv - (J.sy0 + ((double)j - cy) * J.dsy));
                        d2[q] = j < J.nsy ? d * d : INFINITY;
                    }
                    tab[(2 * r) * kMath + tid] = make_float4(d2[0], d2[1], d2[2], d2[3]);
                    tab[(2 * r + 1) * kMath + tid] = make_float4(d2[4], d2[5], d2[6], d2[7]);
                }
                if (r < K1 / 16) {
                    float d2[8];
#pragma unroll
                    for (int q = 0; q < 8; ++q) {
                        const int i = 8 * g + q;
                        const float d = (float)(xv - (J.sx0 + ((double)i - cx) * J.dsx));
                        d2[q] = i < J.nsx ? d * d : INFINITY;
                    }
                    tab[(P.ty4 + 2 * r) * kMath + tid] = make_float4(d2[0], d2[1], d2[2], d2[3]);
                    tab[(P.ty4 + 2 * r + 1) * kMath + tid] = make_float4(d2[4], d2[5], d2[6], d2[7]);
                }
            }
        }
        const float a2 = st.a2;
        uint8_t* a2h = smem + P.oA2 + (uint32_t)ia2 * 2u * aBytes2;
        uint8_t* a1h = smem + P.oA1 + (uint32_t)ia * 2u * aBytes1;
        auto operand = [&](int tab0, int nc, uint8_t* dst, uint32_t lo_off) {
#pragma unroll 1
            for (int r = 0; r < kMaxR; ++r) {
                if (r < nc) {
                    const float4 p = tab[(tab0 + 2 * r) * kMath + tid];
                    const float4 q4 = tab[(tab0 + 2 * r + 1) * kMath + tid];
                    float v[8] = {p.x, p.y, p.z, p.w, q4.x, q4.y, q4.z, q4.w};
#pragma unroll
                    for (int e = 0; e < 8; ++e) v[e] = ex2_approx(fmaf(-v[e], a2, kGScale));
                    uint4 hi, lo;
                    split8(v, hi, lo);
                    const uint32_t off = (uint32_t)(ghalf + 2 * r) * 2048u + (uint32_t)grow * 16u;
                    *reinterpret_cast<uint4*>(dst + off) = hi;
                    *reinterpret_cast<uint4*>(dst + lo_off + off) = lo;
                }
            }
        };
        operand(0, N1 / 16, a2h, aBytes2);
        if (!(st.flags & kSym)) operand(P.ty4, K1 / 16, a1h, aBytes1);
        tc::fence_async_smem();
        __syncwarp();
        if (lane == 0) {
            tc::mbar_arrive(&B.a1r[ia]);
            tc::mbar_arrive(&B.a2r[ia2]);
        }
        return true;
    };

    // E1: U of step m from TMEM, times f1, split -> B2[m % nB2] (x rows, K = j).
    // E1 in two parts: the TMEM loads of U are issued before the next step's G, which hides
    // their latency, and waited for after it (G issues no TMEM load of its own).
    const int ncol = N1 / 2, c0 = half * ncol;   // this warp's columns j: multiple of 8
    uint32_t rb[4][8], rc[4][8];
    auto e1_issue = [&](int m) -> bool {
        bool w = wait_bar(B.uf, (uint32_t)(m & 1), P.wait_ns);
        if (!__all_sync(0xffffffffu, w)) return false;
        tc::fence_after_sync();
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            if (q * 8 < ncol) {
                tc::tmem_ld8(tb + kColU + lane_base + (uint32_t)(c0 + 8 * q), rb[q]);
                tc::tmem_ld8(tb + kColU + lane_base + (uint32_t)(N1 + c0 + 8 * q), rc[q]);
            }
        }
        return true;
    };
    auto e1 = [&](const Step& st, int m) -> bool {
        bool w = true;
        tc::tmem_wait_ld();
        tc::fence_before_sync();
        __syncwarp();
        if (lane == 0) tc::mbar_arrive(B.uu);
        const int ib = m % P.nB2;
        if (m >= P.nB2) w = wait_bar(&B.b2f[ib], (uint32_t)(((m / P.nB2) - 1) & 1), P.wait_ns);
        if (!__all_sync(0xffffffffu, w)) return false;
        uint8_t* bh = smem + P.oB2 + (uint32_t)ib * 2u * aBytes2;
        const float f1 = st.f1;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            if (q * 8 < ncol) {
                float v[8];
#pragma unroll
                for (int e = 0; e < 8; ++e)
                    v[e] = (__uint_as_float(rb[q][e]) + __uint_as_float(rc[q][e])) * f1;
                uint4 hi, lo;
                split8(v, hi, lo);
                const uint32_t off = (uint32_t)((c0 >> 3) + q) * 2048u + (uint32_t)trow * 16u;
                *reinterpret_cast<uint4*>(bh + off) = hi;
                *reinterpret_cast<uint4*>(bh + aBytes2 + off) = lo;
            }
        }
        tc::fence_async_smem();
        __syncwarp();
        if (lane == 0) tc::mbar_arrive(&B.b2r[ib]);
        return true;
    };

    // DR: step m's hi * hi product into dsum; at its unit's end the cross products and output.
    auto dr = [&](const Step& st, int m) -> bool {
        const int db = m & 1;
        bool w = wait_bar(&B.df[db], (uint32_t)((m >> 1) & 1), P.wait_ns);
        if (!__all_sync(0xffffffffu, w)) return false;
        tc::fence_after_sync();
        const float sc = __int_as_float((127 - st.kd) << 23);   // 2^-kd, exact (|kd| <= 114)
        uint32_t r[4][16];
#pragma unroll
        for (int c = 0; c < 4; ++c)
            tc::tmem_ld16(tb + kColDb + (uint32_t)db * 128u + lane_base + (uint32_t)(half * 64 + c * 16), r[c]);
        tc::tmem_wait_ld();
        tc::fence_before_sync();
        __syncwarp();
        if (lane == 0) tc::mbar_arrive(&B.du[db]);
#pragma unroll
        for (int c = 0; c < 4; ++c)
#pragma unroll
            for (int q = 0; q < 16; ++q) dsum[c * 16 + q] = fmaf(__uint_as_float(r[c][q]), sc, dsum[c * 16 + q]);
        if (st.flags & kLast) {
            w = wait_bar(B.cf, (uint32_t)(useg & 1), P.wait_ns);
            if (!__all_sync(0xffffffffu, w)) return false;
            tc::fence_after_sync();
#pragma unroll
            for (int c = 0; c < 4; ++c)
                tc::tmem_ld16(tb + kColDc + lane_base + (uint32_t)(half * 64 + c * 16), r[c]);
            tc::tmem_wait_ld();
            tc::fence_before_sync();
            __syncwarp();
            if (lane == 0) tc::mbar_arrive(B.cu);
            ++useg;
#pragma unroll
            for (int c = 0; c < 4; ++c)
#pragma unroll
                for (int q = 0; q < 16; ++q) dsum[c * 16 + q] = fmaf(__uint_as_float(r[c][q]), sc, dsum[c * 16 + q]);
            output(st, false);
        }
        return true;
    };

    // Each iteration: G of the step read (if it has work), E1 of the step before, DR of the one
    // before that -- one call site each.  A slice no layer reaches, or the end, is handled after
    // the pending steps are finished (iterations without G): E1 of a step otherwise waits for
    // the next step with work, which a run of such slices could keep out of the ring.
    bool p1 = false, p2 = false;   // s1 pending (awaiting E1), s2 pending (awaiting DR)
    int i1 = 0, i2 = 0;            // their step indices
    bool flushing = false, at_end = false, zero_pending = false;
    Step zs{};
    for (;;) {
        Step cur{};
        bool have = false;
        if (!flushing) {
            const int slot = k % kRing;
            ok = wait_bar(&full[slot], (uint32_t)((k / kRing) & 1), P.wait_ns);
            cur = ring[slot];
            if (cur.flags != kEnd && (cur.job < 0 || cur.job >= P.n_jobs)) ok = false;
            __syncwarp();
            if (lane == 0) tc::mbar_arrive(&empty[slot]);
            ++k;
            if (!__all_sync(0xffffffffu, ok)) break;
            if (cur.flags & kEnd) {
                flushing = at_end = true;
            } else if (cur.flags & kZero) {
                flushing = zero_pending = true;
                zs = cur;
            } else {
                have = true;
            }
        }
        if (p1) {
            ok = e1_issue(i1);
            if (!ok) break;
        }
        if (have) {
            ok = gen(cur, ng);
            if (!ok) {
                tc::tmem_wait_ld();   // the E1 loads in flight land before the kernel leaves
                break;
            }
        }
        if (p1) {
            ok = e1(s1, i1);
            if (!ok) break;
        }
        if (p2) {
            ok = dr(s2, i2);
            if (!ok) break;
        }
        s2 = s1; i2 = i1; p2 = p1;
        if (have) {
            s1 = cur; i1 = ng; p1 = true;
            ++ng;
        } else {
            p1 = false;
        }
        if (flushing && !p1 && !p2) {
            if (zero_pending) output(zs, true);   // zeros (and the loss)
            zero_pending = flushing = false;
            if (at_end) break;
        }
    }
    if (!ok && lane == 0) atomicExch(P.err, 1);
}

__global__ void __launch_bounds__(kThreads, 1) fwd_tc16_kernel(Params P) {
    extern __shared__ __align__(1024) uint8_t smem[];
    __shared__ __align__(8) uint64_t full[kRing];
    __shared__ __align__(8) uint64_t empty[kRing];
    __shared__ __align__(8) uint64_t bars[kNumBars];
    __shared__ Step ring[kRing];
    __shared__ uint32_t tmem_base_s;

    const int warp = threadIdx.x >> 5;
    if (warp == 0) {
        tc::tmem_alloc(&tmem_base_s, kCols);
        tc::tmem_relinquish();
    }
    const Bars B = make_bars(bars);
    if (threadIdx.x == 0) {
        for (int i = 0; i < kRing; ++i) {
            tc::mbar_init(&full[i], 1);
            tc::mbar_init(&empty[i], kMathWarps + 3);   // math warps + the three MMA warps
        }
        for (int i = 0; i < 4; ++i) {
            tc::mbar_init(&B.wfull[i], 1);             // producer's expect_tx arrival + bytes
            tc::mbar_init(&B.wempty[i], 1);            // stage-1 commit
        }
        for (int i = 0; i < 3; ++i) {
            tc::mbar_init(&B.a2r[i], kMathWarps);
            tc::mbar_init(&B.a2f[i], 3);               // stage 1 and both stage-2 warps
        }
        for (int i = 0; i < 2; ++i) {
            tc::mbar_init(&B.a1r[i], kMathWarps);
            tc::mbar_init(&B.a1f[i], 1);
            tc::mbar_init(&B.b2r[i], kMathWarps);
            tc::mbar_init(&B.b2f[i], 2);
            tc::mbar_init(&B.df[i], 1);
            tc::mbar_init(&B.du[i], kMathWarps);
        }
        tc::mbar_init(B.uf, 1);
        tc::mbar_init(B.uu, kMathWarps);
        tc::mbar_init(B.cf, 1);
        tc::mbar_init(B.cu, kMathWarps);
        tc::fence_mbar_init();
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    // the spot maps are packed by the kernel before this one (a programmatic dependent launch:
    // everything above overlaps its end)
    asm volatile("griddepcontrol.wait;" ::: "memory");
    // the finalize pass (a programmatic dependent) may be scheduled onto the SMs this grid frees;
    // it reads the partial slices only after its griddepcontrol.wait.  One CTA per SM here, so an
    // early dependent takes no SM that a CTA of this grid still needs.
    asm volatile("griddepcontrol.launch_dependents;");

    if (warp >= kMathWarps) {
        asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;" ::"n"(kCtrlRegs));
        if (warp == kSchedWarp)
            scheduler_warp(P, smem, ring, full, empty, B.wfull, B.wempty);
        else
            mma_warp(P, tc::smem_u32(smem), tmem_base_s, warp - kSchedWarp, ring, full, empty, B);
    } else {
        asm volatile("setmaxnreg.inc.sync.aligned.u32 %0;" ::"n"(kMathRegs));
        math_warps(P, smem, tmem_base_s, ring, full, empty, B);
    }

    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    if (warp == 0) tc::tmem_dealloc(tmem_base_s, kCols);
}

// Finalize pass (grid (kLossBlocks or more, jobs)): each voxel's dose as the sum of its slice's
// partial slices in chunk order (or the dose itself, direct), NaN when a wait of the forward ran
// out; with the loss, dL/dD = 2 m (D - P) and per-block FP64 partial sums of m (D - P)^2 in a
// fixed order.  Four voxels per thread per step when every slice plane is a multiple of four.
constexpr int kFinMaxZ = 1024;   // slices whose partial-slice counts the finalize stages

__global__ void __launch_bounds__(256) fwd16_finalize_kernel(const JobDev* __restrict__ jobs,
                                                             int with_loss,
                                                             const int* __restrict__ err) {
    // a programmatic dependent of the dose kernel: its partial slices are visible after this
    asm volatile("griddepcontrol.wait;" ::: "memory");
    const JobDev& J = jobs[blockIdx.y];
    const size_t plane = (size_t)J.nx * J.ny, n = plane * J.nz;
    const bool bad = *err != 0;
    const float nan = __int_as_float(0x7fc00000);
    double lsum = 0.0;
    auto voxel4 = [&](size_t v, int cnt) {      // voxels v .. v + cnt - 1 of one slice
        const int z = (int)(v / plane);
        const int nch = J.direct ? 1 : J.nchunks[z];
        const float* src = J.direct ? J.dose : J.partial;
        float s4[4] = {0.f, 0.f, 0.f, 0.f};
        if (cnt == 4) {
            for (int k = 0; k < nch; ++k) {
                const float4 a = __ldcs(reinterpret_cast<const float4*>(src + (size_t)k * n + v));
                s4[0] += a.x; s4[1] += a.y; s4[2] += a.z; s4[3] += a.w;
            }
        } else {
            for (int k = 0; k < nch; ++k)
                for (int r = 0; r < cnt; ++r) s4[r] += __ldcs(src + (size_t)k * n + v + r);
        }
        if (bad)
            for (int r = 0; r < 4; ++r) s4[r] = nan;
        if (!J.direct || bad) {
            if (cnt == 4) *reinterpret_cast<float4*>(J.dose + v) = make_float4(s4[0], s4[1], s4[2], s4[3]);
            else for (int r = 0; r < cnt; ++r) J.dose[v + r] = s4[r];
        }
        if (with_loss) {
            float m4[4], p4[4], g4[4];
            if (cnt == 4) {
                const float4 a = __ldcs(reinterpret_cast<const float4*>(J.mask + v));
                const float4 b = __ldcs(reinterpret_cast<const float4*>(J.presc + v));
                m4[0] = a.x; m4[1] = a.y; m4[2] = a.z; m4[3] = a.w;
                p4[0] = b.x; p4[1] = b.y; p4[2] = b.z; p4[3] = b.w;
            } else {
                for (int r = 0; r < 4; ++r) {
                    m4[r] = r < cnt ? J.mask[v + r] : 0.f;
                    p4[r] = r < cnt ? J.presc[v + r] : 0.f;
                }
            }
            for (int r = 0; r < 4; ++r) {
                const float rr = s4[r] - p4[r];
                g4[r] = 2.f * m4[r] * rr;
                if (r < cnt) lsum += (double)m4[r] * (double)rr * (double)rr;
            }
            if (cnt == 4) *reinterpret_cast<float4*>(J.grad_dose + v) = make_float4(g4[0], g4[1], g4[2], g4[3]);
            else for (int r = 0; r < cnt; ++r) J.grad_dose[v + r] = g4[r];
        }
    };
    const size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const size_t nthr = (size_t)gridDim.x * blockDim.x;
    if ((plane & 3) == 0) {
        // Four voxels of one slice per group, two groups per step: the slices' partial-slice
        // counts are staged in shared memory and the mask and prescription loads issued first,
        // so that a step waits on one round of loads (the partial slices).  Sums in piece order,
        // the loss in group order: deterministic.
        __shared__ int s_nch[kFinMaxZ];
        const bool stage = !J.direct && J.nz <= kFinMaxZ;
        if (stage)
            for (int z = threadIdx.x; z < J.nz; z += blockDim.x) s_nch[z] = J.nchunks[z];
        __syncthreads();
        auto nch_of = [&](size_t v) -> int {
            if (J.direct) return 1;
            const int z = (int)(v / plane);
            return stage ? s_nch[z] : J.nchunks[z];
        };
        const float* src = J.direct ? J.dose : J.partial;
        const float4 zero4 = make_float4(0.f, 0.f, 0.f, 0.f);
        auto finish = [&](size_t v, float4 s, float4 m, float4 pr) {
            if (bad) s = make_float4(nan, nan, nan, nan);
            if (!J.direct || bad) *reinterpret_cast<float4*>(J.dose + v) = s;
            if (with_loss) {
                const float r0 = s.x - pr.x, r1 = s.y - pr.y, r2 = s.z - pr.z, r3 = s.w - pr.w;
                lsum += (double)m.x * (double)r0 * (double)r0;
                lsum += (double)m.y * (double)r1 * (double)r1;
                lsum += (double)m.z * (double)r2 * (double)r2;
                lsum += (double)m.w * (double)r3 * (double)r3;
                *reinterpret_cast<float4*>(J.grad_dose + v) =
                    make_float4(2.f * m.x * r0, 2.f * m.y * r1, 2.f * m.z * r2, 2.f * m.w * r3);
            }
        };
        for (size_t va = 4 * tid; va < n; va += 8 * nthr) {
            const size_t vb = va + 4 * nthr;
            const bool hb = vb < n;
            float4 ma = zero4, pa = zero4, mb = zero4, pb = zero4;
            if (with_loss) {
                ma = __ldcs(reinterpret_cast<const float4*>(J.mask + va));
                pa = __ldcs(reinterpret_cast<const float4*>(J.presc + va));
                if (hb) {
                    mb = __ldcs(reinterpret_cast<const float4*>(J.mask + vb));
                    pb = __ldcs(reinterpret_cast<const float4*>(J.presc + vb));
                }
            }
            const int na = nch_of(va), nb = hb ? nch_of(vb) : 0;
            float4 sa = zero4, sb = zero4;
            for (int k = 0; k < na || k < nb; ++k) {
                if (k < na) {
                    const float4 a = __ldcs(reinterpret_cast<const float4*>(src + (size_t)k * n + va));
                    sa.x += a.x; sa.y += a.y; sa.z += a.z; sa.w += a.w;
                }
                if (k < nb) {
                    const float4 b = __ldcs(reinterpret_cast<const float4*>(src + (size_t)k * n + vb));
                    sb.x += b.x; sb.y += b.y; sb.z += b.z; sb.w += b.w;
                }
            }
            finish(va, sa, ma, pa);
            if (hb) finish(vb, sb, mb, pb);
        }
    } else {
        for (size_t v = tid; v < n; v += nthr) voxel4(v, 1);
    }
    if (with_loss) {
        __shared__ double red[256];
        red[threadIdx.x] = lsum;
        __syncthreads();
        for (int w = blockDim.x / 2; w > 0; w >>= 1) {
            if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
            __syncthreads();
        }
        if (threadIdx.x == 0) J.loss_part[blockIdx.x] = red[0];
    }
}

__global__ void fwd16_poison_kernel(const JobDev* __restrict__ jobs, int n_jobs, const int* err) {
    if (*err == 0) return;
    for (int j = 0; j < n_jobs; ++j) {
        const JobDev& J = jobs[j];
        const size_t n = (size_t)J.nx * J.ny * J.nz;
        for (size_t v = (size_t)blockIdx.x * blockDim.x + threadIdx.x; v < n;
             v += (size_t)gridDim.x * blockDim.x)
            J.dose[v] = __int_as_float(0x7fc00000);
    }
}

// Shared-memory plan: buffer counts (largest first that fit) and offsets.
struct Plan16 {
    int nR, nA1, nA2, nB2;
    uint32_t img, oW, oA1, oA2, oB2, oTab, total;
    int ty4, tx4;
};

bool plan16(int K1, int N1, int max_dyn, Plan16* p) {
    p->img = 4u * (uint32_t)K1 * (uint32_t)N1;
    p->ty4 = N1 / 8;
    p->tx4 = K1 / 8;
    const uint32_t a1 = 2u * (uint32_t)K1 * 256u, a2 = 2u * (uint32_t)N1 * 256u;
    const uint32_t tab = (uint32_t)(p->ty4 + p->tx4) * (uint32_t)kMath * 16u;
    // (ring, Gx, Gy, sU) buffers, deepest first; Gy needs at least two (G of step m + 1 runs
    // before E1 of step m, which stage 2 of step m waits for)
    static const int cand[][4] = {{3, 2, 3, 1}, {2, 2, 3, 1}, {2, 1, 3, 1}, {2, 2, 2, 1},
                                  {2, 1, 2, 1}};
    for (const auto& c : cand) {
        p->nR = c[0]; p->nA1 = c[1]; p->nA2 = c[2]; p->nB2 = c[3];
        p->oW = 0;
        p->oA1 = p->oW + (uint32_t)p->nR * p->img;
        p->oA2 = p->oA1 + (uint32_t)p->nA1 * a1;
        p->oB2 = p->oA2 + (uint32_t)p->nA2 * a2;
        p->oTab = p->oB2 + (uint32_t)p->nB2 * a2;
        p->total = p->oTab + tab;
        if ((int)p->total <= max_dyn) return true;
    }
    return false;
}

}  // namespace

size_t tc16_pack_bytes(int n_jobs, int max_layers, int nsx, int nsy) {
    const size_t K1 = (size_t)(nsx + 15) / 16 * 16, N1 = (size_t)(nsy + 15) / 16 * 16;
    return (size_t)n_jobs * (size_t)max_layers * (4u * K1 * N1 + 8u);
}

int launch_forward_tc16(JobDev* jobs_dev, const JobDev* jobs_host, int n_jobs, int* counter,
                        int* err, int chunk, int with_loss, int poison, void* pack,
                        size_t pack_bytes, cudaStream_t s,
                        const JobPair* inst, JobDev* inst_dst, int* inst_status) {
    Params P{};
    P.jobs = jobs_dev;
    P.n_jobs = n_jobs;
    P.chunk = chunk;
    P.counter = counter;
    P.err = err;
    P.wait_ns = wait_limit_ns();
    P.hold = test_hold();
    P.with_loss = with_loss;
    int lmax = 1, nsx = 1, nsy = 1;
    for (int j = 0; j < n_jobs; ++j) {
        int k1 = 0, n1 = 0;
        PBD_TRY(tc_operand_dims(PBD_PREC_BF16X3, jobs_host[j].nsx, jobs_host[j].nsy, &k1, &n1));
        P.K1 = std::max(P.K1, k1);
        P.N1 = std::max(P.N1, n1);
        lmax = std::max(lmax, jobs_host[j].nl);
        nsx = std::max(nsx, jobs_host[j].nsx);
        nsy = std::max(nsy, jobs_host[j].nsy);
    }
    if (jobs_host[0].layer_stride != 0) return PBD_ERR_UNSUPPORTED;   // per-layer maps: TF32 kernel
    P.sym = 1;
    for (int j = 0; j < n_jobs; ++j) {
        const JobDev& J = jobs_host[j];
        if (!(J.nx == J.ny && J.ox == J.oy && J.dx == J.dy && J.nsx == J.nsy && J.sx0 == J.sy0 &&
              J.dsx == J.dsy))
            P.sym = 0;
    }
    PBD_TRY(tc_forward_units(jobs_host, n_jobs, chunk, &P.cmax, &P.tmax, &P.n_units));
    const size_t need = tc16_pack_bytes(n_jobs, lmax, P.K1, P.N1);
    if (!pack || pack_bytes < need) return PBD_ERR_WORKSPACE;
    P.lmax = lmax;
    P.img = 4u * (uint32_t)P.K1 * (uint32_t)P.N1;
    uint8_t* base = static_cast<uint8_t*>(pack);
    P.wpack = base;
    float* wmax = reinterpret_cast<float*>(base + (size_t)n_jobs * lmax * P.img);
    int* wexp = reinterpret_cast<int*>(wmax + (size_t)n_jobs * lmax);
    P.wmax = wmax;
    P.wexp = wexp;
    int max_dyn = 0;
    PBD_TRY(smem_optin((const void*)fwd_tc16_kernel, -1, kLaunchRegsNeeded, &max_dyn));
    Plan16 pl;
    if (!plan16(P.K1, P.N1, max_dyn, &pl)) return PBD_ERR_NO_SMEM;
    P.nR = pl.nR; P.nA1 = pl.nA1; P.nA2 = pl.nA2; P.nB2 = pl.nB2;
    P.oW = pl.oW; P.oA1 = pl.oA1; P.oA2 = pl.oA2; P.oB2 = pl.oB2; P.oTab = pl.oTab;
    P.ty4 = pl.ty4; P.tx4 = pl.tx4;
    // >= 116 KiB: one CTA (and its 512 TMEM columns) per SM
    const size_t smem = std::max<size_t>(pl.total, 116u * 1024u);
    if (smem > (size_t)max_dyn) return PBD_ERR_NO_SMEM;
    JobPair ip;
    memset(&ip, 0, sizeof(ip));
    if (inst) {
        if (n_jobs > inst->n || inst->n > 2) return PBD_ERR_UNSUPPORTED;
        ip = *inst;
    }
    PBD_TRY(launch_dependent(pack_w16_kernel, dim3(lmax, n_jobs), dim3(256), 0, s,
                             (const JobDev*)jobs_dev, P.K1, P.N1, lmax, P.img,
                             const_cast<uint8_t*>(P.wpack), wmax, wexp, counter, ip,
                             inst ? 1 : 0, inst_dst, inst_status));
    const int grid = std::max(1, std::min(P.n_units, num_sms()));
    prof_mark(kProfFwd, 0, s);
    PBD_TRY(launch_dependent(fwd_tc16_kernel, dim3(grid), dim3(kThreads), smem, s, P));
    prof_mark(kProfFwd, 1, s);
    count_launch(2);
    // every job of a launch shares its output mode (the callers set it per launch)
    if (!jobs_host[0].direct || with_loss) {
        size_t maxn = 1;
        for (int j = 0; j < n_jobs; ++j)
            maxn = std::max(maxn, (size_t)jobs_host[j].nx * jobs_host[j].ny * jobs_host[j].nz);
        // kLossBlocks16 blocks with the loss (the adjoint sums that many partials per job)
        const int blocks = with_loss ? kLossBlocks16
                                     : (int)std::min<size_t>((maxn / 8 + 255) / 256,
                                                             (size_t)num_sms() * 4);
        PBD_TRY(launch_dependent(fwd16_finalize_kernel, dim3(std::max(blocks, 1), n_jobs), dim3(256),
                                 0, s, (const JobDev*)jobs_dev, with_loss, (const int*)err));
        count_launch(1);
    } else if (poison) {
        fwd16_poison_kernel<<<num_sms(), 256, 0, s>>>(jobs_dev, n_jobs, err);
        PBD_LAUNCH_CHECK();
        count_launch(1);
    }
    return PBD_OK;
}

}  // namespace pbd
