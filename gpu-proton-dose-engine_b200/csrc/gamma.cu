// gamma.cu -- gamma index (Low et al. 1998) of an evaluated dose against a reference dose,
// with the reference's semantics (gamma.py:41-60 dta_offsets, 81-160 gamma_index, 213-261
// gamma_index_torch):
//
//   gamma(r)^2 = min over integer voxel offsets o with |o| <= DTA of
//                (|o| / DTA)^2 + ((E[r + o] - R[r]) / dose_crit(r))^2
//
// E is zero outside the grid; dose_crit = pct/100 * ref_max (global) or
// pct/100 * max(R[r], 1e-12) (local); the statistics run over the mask
// R >= thr/100 * ref_max (or R > 0 when that mask is empty).
//
// Arithmetic: FP64 with every operation rounded separately (no FMA contraction) in the order
// the reference's NumPy code evaluates it, so the gamma map, the mask, the counts, the
// maximum and the percentiles equal the reference's float64 results bit for bit (the mean is
// a fixed-order sum, within rounding of NumPy's pairwise sum).  The distance table is built
// on the host with libm pow() -- the call Python's float ** makes -- so the offsets and
// their weights (|o|/DTA)^2 are identical too.
//
// Kernels (all on `stream`, no host synchronisation):
//   gamma_refmax_kernel   max of the reference dose (skipped when a normalisation dose is given)
//   gamma_kernel          one thread per 4 voxels along z, the evaluated dose of a 32x8x4 brick
//                         plus its halo staged in shared memory as FP64; offsets visited in
//                         ascending (|o|/DTA)^2, stopping once that weight reaches the current
//                         minimum (exact: w + d^2 >= w after rounding); masked voxels' gamma
//                         appended to a key list; per-block partial sums and maxima
//   (same kernel, fallback pass: runs only when the threshold mask was empty)
//   gamma_finish_kernel   counts, mean, max, pass rate, percentile ranks (NumPy 'linear')
//   gamma_select_kernel   radix select of the four order statistics the percentiles need (one
//                         launch per digit; the last block to arrive picks the digits)
//   gamma_final_kernel    NumPy's interpolation between the order statistics
#include <math.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "pbd_internal.cuh"

namespace pbd {
namespace {

constexpr int kGR = 7;                 // table size per axis (radius <= 6 voxels)
constexpr int kGTab = kGR * kGR * kGR;
constexpr int kTX = 32, kTY = 8, kTZ = 4;
constexpr int kGThreads = kTX * kTY;
constexpr int kDigitBits = 11;
constexpr int kBins = 1 << kDigitBits;
constexpr int kSelPasses = 6;          // 6 x 11 bits cover the 64-bit keys
constexpr int kHistThreads = 512;
constexpr int kFinThreads = 1024;
constexpr int kSelPer = 16;            // keys per thread a select pass aims at
constexpr int kRowBatch = 4;           // staged rows per warp whose loads are issued together
// largest staged brick (radius 6 on every axis) and offset list (13^3 offsets)
constexpr int kGMaxOff = 13 * 13 * 13;
constexpr int kGMaxSmem = (kTX + 12) * (kTY + 12) * (kTZ + 12) * (int)sizeof(double) +
                          kGMaxOff * (int)(sizeof(double) + sizeof(int));

struct GammaParams {
    int nz, ny, nx;
    int hz, hy, hx;
    int n_entries;                     // distinct (|a|,|b|,|c|) inside the ball
    int n_off;                         // offsets (entries with their signs)
    int local;
    int use_ref_dose;
    int want_gamma, want_mask;
    double ref_dose;
    double crit_frac;                  // dose_crit_pct / 100
    double thr_frac;                   // threshold_pct / 100
    double q[2];                       // 95/100, 99/100
    double w[kGTab];                   // (|o|/DTA)^2, ascending
    unsigned char abc[kGTab][4];       // |a|, |b|, |c| of each entry
    short start[kGTab];                // first offset of each entry in the expanded list
};

// Device state in the workspace.
struct GammaState {
    unsigned long long ref_key;        // ordered key of max(reference)
    unsigned long long cnt[2][4];      // per pass: n_eval, n_pass, n_nan, n_keys (pass 0: the
                                       // threshold mask, pass 1: the R > 0 fallback)
    int fallback;                      // the statistics use the R > 0 mask
    int status;
    double ref_max;
    unsigned long long rank[4];        // wanted order statistics (0-based)
    unsigned long long prefix[4];      // key bits found so far
    unsigned long long rem[4];         // rank within the current prefix
    double vir[2];                     // NumPy virtual indexes of p95, p99 (-1: use max)
    double mean, maxv, pass_rate;
    unsigned long long n_eval, n_pass, n_nan;
    unsigned int sel_arrive;           // blocks of the current select pass that finished
    unsigned long long n_cand;         // keys copied to the candidate list
};

// Order-preserving map of a double to an unsigned key (NaN above +inf).
__device__ __forceinline__ unsigned long long dkey(double v) {
    unsigned long long b = (unsigned long long)__double_as_longlong(v);
    if (v != v) b = 0x7FF8000000000000ull;
    return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
__device__ __forceinline__ double dunkey(unsigned long long k) {
    const unsigned long long b = (k >> 63) ? (k & 0x7FFFFFFFFFFFFFFFull) : ~k;
    return __longlong_as_double((long long)b);
}
// NumPy's minimum: NaN if either is NaN.
__device__ __forceinline__ double nmin(double a, double b) {
    if (a != a || b != b) return __longlong_as_double(0x7FF8000000000000ll);
    return b < a ? b : a;
}
__device__ __forceinline__ bool finite_d(double v) { return v == v && v - v == 0.0; }

template <class T>
__device__ __forceinline__ double ld(const T* p, size_t i) { return (double)__ldg(p + i); }

template <class T>
__global__ void __launch_bounds__(kGThreads)
gamma_refmax_kernel(const T* __restrict__ ref, size_t n, GammaState* st) {
    unsigned long long best = 0ull;
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    for (; i + 3 * stride < n; i += 4 * stride) {          // four loads in flight
        const double a = ld(ref, i), b = ld(ref, i + stride), c = ld(ref, i + 2 * stride),
                     d = ld(ref, i + 3 * stride);
        best = max(max(best, dkey(a)), max(dkey(b), max(dkey(c), dkey(d))));
    }
    for (; i < n; i += stride) best = max(best, dkey(ld(ref, i)));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) best = max(best, __shfl_xor_sync(0xffffffffu, best, o));
    if ((threadIdx.x & 31) == 0 && best) atomicMax(&st->ref_key, best);
}

template <class T, bool kFallback>
__global__ void __launch_bounds__(kGThreads)
gamma_kernel(const GammaParams P, const T* __restrict__ ref, const T* __restrict__ ev,
             double* __restrict__ gmap, unsigned char* __restrict__ mmap, GammaState* st,
             unsigned long long* __restrict__ keys, double* __restrict__ part_sum,
             double* __restrict__ part_max, int gx, int gy, int n_bricks) {
    extern __shared__ double tile[];
    __shared__ double red_s[kGThreads / 32], red_m[kGThreads / 32];
    __shared__ unsigned long long red_c[kGThreads / 32][3];
    __shared__ unsigned int s_wcnt[kGThreads / 32], s_wpre[kGThreads / 32];
    __shared__ unsigned long long s_base;
    __shared__ int s_nonfinite;
    const int pass = kFallback ? 1 : 0;
    if (kFallback && __ldcg(&st->cnt[0][0]) != 0ull) return;   // the threshold mask is used
    const double ref_max = P.use_ref_dose ? P.ref_dose : dunkey(__ldcg(&st->ref_key));
    if (ref_max <= 0.0) {                                      // gamma.py:112-113
        if (blockIdx.x == 0 && threadIdx.x == 0) st->status = PBD_ERR_BAD_VALUE;
        return;
    }
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int TX = kTX + 2 * P.hx, TY = kTY + 2 * P.hy, TZ = kTZ + 2 * P.hz;
    const int plane = TX * TY;
    double* s_w = tile + (size_t)plane * TZ;                    // weight of each offset
    int* s_off = reinterpret_cast<int*>(s_w + P.n_off);         // its position in the tile
    // offsets of each (|a|,|b|,|c|) entry with their signs, in ascending weight
    for (int u = tid; u < P.n_entries; u += kGThreads) {
        const int ia = P.abc[u][0], ib = P.abc[u][1], ic = P.abc[u][2];
        int o = P.start[u];
        for (int sgn = 0; sgn < 8; ++sgn) {
            if (((sgn & 4) && ia == 0) || ((sgn & 2) && ib == 0) || ((sgn & 1) && ic == 0))
                continue;
            const int sa = (sgn & 4) ? -ia : ia, sb = (sgn & 2) ? -ib : ib, sc = (sgn & 1) ? -ic : ic;
            s_w[o] = P.w[u];
            s_off[o] = sa * plane + sb * TX + sc;
            ++o;
        }
    }
    const double crit_g = __dmul_rn(P.crit_frac, ref_max);     // global dose criterion
    const double thr_dose = __dmul_rn(P.thr_frac, ref_max);
    const bool ok_g = finite_d(crit_g) || P.local;
    const int tx = lane, ty = warp;
    double sum = 0.0, mx = -1.0;                 // gamma >= 0
    unsigned long long c_eval = 0, c_pass = 0, c_nan = 0;
    // bricks of 32 x 8 x 4 voxels, statically strided over the persistent blocks
    for (int brick = blockIdx.x; brick < n_bricks; brick += gridDim.x) {
        const int bx = brick % gx, rest = brick / gx, by = rest % gy, bz = rest / gy;
        const int x0 = bx * kTX, y0 = by * kTY, z0 = bz * kTZ;
        const int x = x0 + tx, y = y0 + ty;
        // this thread's reference doses, loaded before the staging barrier
        double rv[kTZ];
#pragma unroll
        for (int k = 0; k < kTZ; ++k) {
            const int z = z0 + k;
            rv[k] = (x < P.nx && y < P.ny && z < P.nz)
                        ? ld(ref, ((size_t)z * P.ny + y) * P.nx + x) : 0.0;
        }
        __syncthreads();                         // the previous brick is done with the tile
        if (tid == 0) s_nonfinite = 0;
        __syncthreads();
        // the evaluated dose of the brick and its halo: each warp takes rows of TX voxels,
        // kRowBatch rows' loads issued before their stores
        int nonfin = 0;
        const int n_rows = TY * TZ;
        for (int row0 = warp; row0 < n_rows; row0 += kRowBatch * (kGThreads / 32)) {
            for (int t0 = 0; t0 < TX; t0 += 32) {
                double v[kRowBatch];
#pragma unroll
                for (int q = 0; q < kRowBatch; ++q) {
                    const int row = row0 + q * (kGThreads / 32);
                    const int tz = row / TY, tyy = row - tz * TY;
                    const int z = z0 - P.hz + tz, yy = y0 - P.hy + tyy, xx = x0 - P.hx + t0 + lane;
                    const bool ok = row < n_rows && t0 + lane < TX && z >= 0 && z < P.nz &&
                                    yy >= 0 && yy < P.ny && xx >= 0 && xx < P.nx;
                    v[q] = ok ? ld(ev, ((size_t)z * P.ny + yy) * P.nx + xx) : 0.0;
                }
#pragma unroll
                for (int q = 0; q < kRowBatch; ++q) {
                    const int row = row0 + q * (kGThreads / 32);
                    if (row < n_rows && t0 + lane < TX) {
                        nonfin |= !finite_d(v[q]);
                        tile[row * TX + t0 + lane] = v[q];
                    }
                }
            }
        }
        if (nonfin) s_nonfinite = 1;
        __syncthreads();
        const bool tile_finite = s_nonfinite == 0;
        double gk[kTZ];
        unsigned int bal[kTZ];
        unsigned int wcnt = 0;
#pragma unroll
        for (int k = 0; k < kTZ; ++k) {
            const int z = z0 + k;
            const bool in = x < P.nx && y < P.ny && z < P.nz;
            double g = 0.0;
            bool masked = false;
            if (in) {
                const size_t v = ((size_t)z * P.ny + y) * P.nx + x;
                const double r = rv[k];
                masked = kFallback ? (r > 0.0) : (r >= thr_dose);
                // without a gamma map only masked voxels need their gamma
                if (masked || (!kFallback && P.want_gamma)) {
                    const double crit =
                        P.local ? __dmul_rn(P.crit_frac, r > 1e-12 || r != r ? r : 1e-12) : crit_g;
                    // early exit is exact when no NaN can appear later: finite doses, a finite
                    // non-zero criterion (NaN needs 0/0, inf - inf or inf/inf)
                    const bool fast =
                        tile_finite && finite_d(r) && finite_d(crit) && crit != 0.0 && ok_g;
                    const double* c0 =
                        tile + (size_t)(k + P.hz) * plane + (ty + P.hy) * TX + (tx + P.hx);
                    double best = __longlong_as_double(0x7FF0000000000000ll);    // +inf
                    for (int j = 0; j < P.n_off; ++j) {
                        const double w = s_w[j];
                        if (fast && w >= best) break;    // w + d^2 >= w >= best, here and later
                        const double dd = __ddiv_rn(__dsub_rn(c0[s_off[j]], r), crit);
                        best = nmin(best, __dadd_rn(w, __dmul_rn(dd, dd)));
                    }
                    g = __dsqrt_rn(best);
                    if (!kFallback && P.want_gamma) gmap[v] = g;
                }
                if (P.want_mask) mmap[v] = masked ? 1 : 0;
            }
            if (masked) {
                ++c_eval;
                c_pass += g <= 1.0;
                if (g != g) ++c_nan;
                else { sum = __dadd_rn(sum, g); mx = g > mx ? g : mx; }
            }
            gk[k] = g;
            bal[k] = __ballot_sync(0xffffffffu, masked);
            wcnt += __popc(bal[k]);
        }
        // masked voxels' keys for the percentiles: one atomic per brick
        if (lane == 0) s_wcnt[warp] = wcnt;
        __syncthreads();
        if (tid == 0) {
            unsigned int tot = 0;
            for (int w = 0; w < kGThreads / 32; ++w) { s_wpre[w] = tot; tot += s_wcnt[w]; }
            s_base = tot ? atomicAdd(&st->cnt[pass][3], (unsigned long long)tot) : 0ull;
        }
        __syncthreads();
        unsigned long long pos = s_base + s_wpre[warp];
        const unsigned int below = (1u << lane) - 1u;
#pragma unroll
        for (int k = 0; k < kTZ; ++k) {
            if (bal[k] & (1u << lane)) keys[pos + __popc(bal[k] & below)] = dkey(gk[k]);
            pos += __popc(bal[k]);
        }
    }
    // block reduction in a fixed order
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        sum = __dadd_rn(sum, __shfl_xor_sync(0xffffffffu, sum, o));
        const double om = __shfl_xor_sync(0xffffffffu, mx, o);
        mx = om > mx ? om : mx;
        c_eval += __shfl_xor_sync(0xffffffffu, c_eval, o);
        c_pass += __shfl_xor_sync(0xffffffffu, c_pass, o);
        c_nan += __shfl_xor_sync(0xffffffffu, c_nan, o);
    }
    if (lane == 0) {
        red_s[warp] = sum; red_m[warp] = mx;
        red_c[warp][0] = c_eval; red_c[warp][1] = c_pass; red_c[warp][2] = c_nan;
    }
    __syncthreads();
    if (tid == 0) {
        double s = 0.0, m = -1.0;
        unsigned long long a = 0, b = 0, c = 0;
        for (int w = 0; w < kGThreads / 32; ++w) {
            s = __dadd_rn(s, red_s[w]);
            m = red_m[w] > m ? red_m[w] : m;
            a += red_c[w][0]; b += red_c[w][1]; c += red_c[w][2];
        }
        part_sum[blockIdx.x] = s;
        part_max[blockIdx.x] = m;
        if (a) atomicAdd(&st->cnt[pass][0], a);
        if (b) atomicAdd(&st->cnt[pass][1], b);
        if (c) atomicAdd(&st->cnt[pass][2], c);
    }
}

// Statistics of the chosen mask and the ranks of the order statistics (one block).
__global__ void __launch_bounds__(kFinThreads)
gamma_finish_kernel(const GammaParams P, GammaState* st, const double* __restrict__ part_sum,
                    const double* __restrict__ part_max, int grid0, int grid1) {
    __shared__ double s_sum[kFinThreads / 32], s_max[kFinThreads / 32];
    if (st->status != 0) return;
    const int pass = st->cnt[0][0] != 0ull ? 0 : 1;
    const int n_blocks = pass ? grid1 : grid0;
    double s = 0.0, m = -1.0;
    // fixed order: thread t sums blocks t, t + T, ... then the warps, then the block
    for (int b = threadIdx.x; b < n_blocks; b += kFinThreads) {
        s = __dadd_rn(s, part_sum[b]);
        m = part_max[b] > m ? part_max[b] : m;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        s = __dadd_rn(s, __shfl_down_sync(0xffffffffu, s, o));
        const double om = __shfl_down_sync(0xffffffffu, m, o);
        m = om > m ? om : m;
    }
    if ((threadIdx.x & 31) == 0) { s_sum[threadIdx.x >> 5] = s; s_max[threadIdx.x >> 5] = m; }
    __syncthreads();
    if (threadIdx.x != 0) return;
    s = 0.0; m = -1.0;
    for (int w = 0; w < kFinThreads / 32; ++w) {
        s = __dadd_rn(s, s_sum[w]);
        m = s_max[w] > m ? s_max[w] : m;
    }
    const unsigned long long n = st->cnt[pass][0], np_ = st->cnt[pass][1], nn = st->cnt[pass][2];
    st->fallback = pass;
    st->n_eval = n; st->n_pass = np_; st->n_nan = nn;
    st->ref_max = P.use_ref_dose ? P.ref_dose : dunkey(st->ref_key);
    if (n == 0ull) { st->status = PBD_ERR_BAD_VALUE; return; }   // no voxel to evaluate
    const double nan = __longlong_as_double(0x7FF8000000000000ll);
    st->pass_rate = __dmul_rn(__ddiv_rn((double)np_, (double)n), 100.0);
    st->mean = nn ? nan : __ddiv_rn(s, (double)n);
    st->maxv = nn ? nan : m;
    // NumPy 'linear' percentiles: virtual index (n - 1) * q, the floor and the next element,
    // or the last element when the index is at or beyond n - 1
    for (int j = 0; j < 2; ++j) {
        const double vi = __dmul_rn((double)(n - 1ull), P.q[j]);
        unsigned long long lo;
        if (vi >= (double)(n - 1ull)) { lo = n - 1ull; st->vir[j] = -1.0; }
        else { lo = (unsigned long long)floor(vi); st->vir[j] = vi; }
        const unsigned long long hi = lo + 1ull < n ? lo + 1ull : n - 1ull;
        st->rank[2 * j] = lo;
        st->rank[2 * j + 1] = hi;
    }
    for (int j = 0; j < 4; ++j) { st->prefix[j] = 0ull; st->rem[j] = st->rank[j]; }
}

// One radix-select pass over key bits [shift, top) (digits of 11 bits from the top, the last
// one 9 bits).  The blocks histogram the keys whose bits above `top` equal a target's prefix
// (targets with equal prefixes share a histogram; runs of equal digits are counted in
// registers before one shared-memory atomic), add their histograms to the global one, and
// the last block to arrive picks each target's digit from the totals, updates its prefix and
// remaining rank, and clears the histogram and the arrival counter for the next pass.
// mode 0 reads every masked key; mode 1 also copies the keys that match any target's
// prefix into a candidate list; mode 2 reads only the candidates.  The grid is trimmed to
// about kSelPer keys per thread.
__global__ void __launch_bounds__(kHistThreads)
gamma_select_kernel(GammaState* st, const unsigned long long* __restrict__ keys,
                    unsigned long long* __restrict__ cand, int shift, int top, int mode,
                    unsigned int* __restrict__ hist) {
    __shared__ unsigned int h[4][kBins];
    __shared__ int s_last;
    if (st->status != 0) return;
    const unsigned long long n = mode == 2 ? st->n_cand : st->n_eval;
    const unsigned long long* src = mode == 2 ? cand : keys;
    const unsigned long long want = (n + (unsigned long long)kHistThreads * kSelPer - 1) /
                                    ((unsigned long long)kHistThreads * kSelPer);
    const unsigned int active = (unsigned int)(want < gridDim.x ? (want ? want : 1) : gridDim.x);
    if (blockIdx.x >= active) return;
    const unsigned long long himask = top >= 64 ? 0ull : ~((1ull << top) - 1ull);
    const unsigned int dmask = (1u << (top - shift)) - 1u;
    unsigned long long pre[4];
    int grp[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        pre[j] = st->prefix[j];
        grp[j] = j;
        for (int q = 0; q < j; ++q)
            if (grp[j] == j && pre[q] == pre[j]) grp[j] = grp[q];
    }
    for (int j = 0; j < 4; ++j)
        if (grp[j] == j)
            for (int i = threadIdx.x; i < kBins; i += kHistThreads) h[j][i] = 0u;
    __syncthreads();
    const int lane = threadIdx.x & 31;
    unsigned int rd[4] = {0u, 0u, 0u, 0u}, rc[4] = {0u, 0u, 0u, 0u};
    const unsigned long long stride = (unsigned long long)active * kHistThreads;
    // warp-uniform trip count (the candidate append is warp-collective); four keys per
    // thread loaded before they are counted
    for (unsigned long long b0 = (unsigned long long)blockIdx.x * kHistThreads + (threadIdx.x & ~31);
         b0 < n; b0 += 4 * stride) {
      unsigned long long kk[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const unsigned long long i = b0 + q * stride + lane;
        kk[q] = i < n ? __ldg(src + i) : 0ull;
      }
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const unsigned long long b = b0 + q * stride;
        if (b >= n) break;                                   // warp-uniform
        const bool valid = b + lane < n;
        const unsigned long long k = kk[q];
        const unsigned int d = (unsigned int)(k >> shift) & dmask;
        bool any = false;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            if (grp[j] != j || !valid || (k & himask) != pre[j]) continue;
            any = true;
            if (rc[j] && rd[j] == d) { ++rc[j]; continue; }
            if (rc[j]) atomicAdd(&h[j][rd[j]], rc[j]);
            rd[j] = d;
            rc[j] = 1u;
        }
        if (mode == 1) {
            const unsigned int bal = __ballot_sync(0xffffffffu, any);
            if (bal) {
                unsigned long long base = 0;
                if (lane == 0) base = atomicAdd(&st->n_cand, (unsigned long long)__popc(bal));
                base = __shfl_sync(0xffffffffu, base, 0);
                if (any) cand[base + __popc(bal & ((1u << lane) - 1u))] = k;
            }
        }
      }
    }
#pragma unroll
    for (int j = 0; j < 4; ++j)
        if (rc[j]) atomicAdd(&h[j][rd[j]], rc[j]);
    __syncthreads();
    for (int j = 0; j < 4; ++j)
        if (grp[j] == j)
            for (int i = threadIdx.x; i < kBins; i += kHistThreads) {
                const unsigned int c = h[j][i];
                if (c) atomicAdd(hist + j * kBins + i, c);
            }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) s_last = atomicAdd(&st->sel_arrive, 1u) == active - 1u;
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    for (int j = 0; j < 4; ++j)
        if (grp[j] == j) {
            unsigned int c[kBins / kHistThreads];
#pragma unroll
            for (int q = 0; q < kBins / kHistThreads; ++q)
                c[q] = __ldcg(hist + j * kBins + threadIdx.x + q * kHistThreads);
#pragma unroll
            for (int q = 0; q < kBins / kHistThreads; ++q) {
                h[j][threadIdx.x + q * kHistThreads] = c[q];
                hist[j * kBins + threadIdx.x + q * kHistThreads] = 0u;
            }
        }
    __syncthreads();
    const int j = threadIdx.x >> 5;
    if (j < 4) {
        const unsigned int* hj = h[grp[j]];
        constexpr int per = kBins / 32;
        unsigned long long loc = 0;
        for (int q = 0; q < per; ++q) loc += hj[lane * per + q];
        unsigned long long inc = loc;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned long long t = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += t;
        }
        const unsigned long long rem = st->rem[j];
        const unsigned int hit = __ballot_sync(0xffffffffu, inc > rem);
        const int srcl = hit ? __ffs(hit) - 1 : 31;
        if (lane == srcl) {
            unsigned long long before = inc - loc;
            int dsel = lane * per + per - 1;
            for (int q = 0; q < per; ++q) {
                const unsigned int c = hj[lane * per + q];
                if (before + c > rem) { dsel = lane * per + q; break; }
                before += c;
            }
            st->rem[j] = rem - before;
            st->prefix[j] |= (unsigned long long)dsel << shift;
        }
    }
    if (threadIdx.x == 0) st->sel_arrive = 0u;
}

// NumPy's _lerp between the order statistics; statistics out.
__global__ void gamma_final_kernel(const GammaParams P, GammaState* st, pbd_gamma_stats* out,
                                   int n_offsets) {
    pbd_gamma_stats r;
    memset(&r, 0, sizeof(r));
    r.status = st->status;
    r.n_dta_offsets = n_offsets;
    r.ref_max = P.use_ref_dose ? P.ref_dose : dunkey(st->ref_key);
    if (st->status == 0) {
        const double nan = __longlong_as_double(0x7FF8000000000000ll);
        r.n_eval = (long long)st->n_eval;
        r.n_pass = (long long)st->n_pass;
        r.pass_rate = st->pass_rate;
        r.gamma_mean = st->mean;
        r.gamma_max = st->maxv;
        r.mask_fallback = st->fallback;
        double pct[2];
        for (int j = 0; j < 2; ++j) {
            const double a = dunkey(st->prefix[2 * j]), b = dunkey(st->prefix[2 * j + 1]);
            const double vi = st->vir[j];
            double t;
            if (vi < 0.0) {
                // at or beyond the last index: NumPy sets the floor index to -1 and both
                // neighbours to the last element
                t = __dadd_rn(__dmul_rn((double)(st->n_eval - 1ull), P.q[j]), 1.0);
            } else {
                t = __dsub_rn(vi, floor(vi));
            }
            const double diff = __dsub_rn(b, a);
            double v = __dadd_rn(a, __dmul_rn(diff, t));
            if (t >= 0.5) v = __dsub_rn(b, __dmul_rn(diff, __dsub_rn(1.0, t)));
            pct[j] = st->n_nan ? nan : v;
        }
        r.gamma_p95 = pct[0];
        r.gamma_p99 = pct[1];
    }
    *out = r;
}

// ---- host ---------------------------------------------------------------------------------

// libm pow through a pointer the compiler cannot fold (Python's float ** calls pow(); a
// folded x*x differs from it in the last bit for some x).
double (*volatile g_pow)(double, double) = pow;

struct GammaTable {
    int hz, hy, hx, n_entries, n_offsets;
    double w[kGTab];
    unsigned char abc[kGTab][3];
};

int build_table(const pbd_gamma_spec* s, GammaTable* t) {
    const double dta_cm = s->dta_mm / 10.0;                        // gamma.py:113
    const double sp[3] = {s->dz, s->dy, s->dx};
    int h[3];
    for (int a = 0; a < 3; ++a) {                                  // gamma.py:48-51
        h[a] = (int)floor(dta_cm / sp[a] + 1e-9);
        h[a] = std::min(h[a], s->max_vox);
        if (h[a] < 0) h[a] = 0;
    }
    struct E { double w; int a, b, c; };
    std::vector<E> es;
    int n_off = 0;
    for (int a = 0; a <= h[0]; ++a)
        for (int b = 0; b <= h[1]; ++b)
            for (int c = 0; c <= h[2]; ++c) {
                const double xa = a * s->dz, xb = b * s->dy, xc = c * s->dx;
                const double d = sqrt(g_pow(xa, 2.0) + g_pow(xb, 2.0) + g_pow(xc, 2.0));
                if (!(d <= dta_cm + 1e-12)) continue;              // gamma.py:56
                const double dr = d / dta_cm;                      // gamma.py:129
                es.push_back({dr * dr, a, b, c});
                n_off += (a ? 2 : 1) * (b ? 2 : 1) * (c ? 2 : 1);
            }
    std::stable_sort(es.begin(), es.end(), [](const E& x, const E& y) { return x.w < y.w; });
    t->hz = h[0]; t->hy = h[1]; t->hx = h[2];
    t->n_entries = (int)es.size();
    t->n_offsets = n_off;
    for (size_t i = 0; i < es.size(); ++i) {
        t->w[i] = es[i].w;
        t->abc[i][0] = (unsigned char)es[i].a;
        t->abc[i][1] = (unsigned char)es[i].b;
        t->abc[i][2] = (unsigned char)es[i].c;
    }
    return PBD_OK;
}

bool finite_h(double v) { return std::isfinite(v); }

int validate(const pbd_gamma_spec* s, int nz, int ny, int nx) {
    if (!s) return PBD_ERR_NULL_ARG;
    if (nz <= 0 || ny <= 0 || nx <= 0) return PBD_ERR_BAD_DIM;
    if ((size_t)nz * ny * nx > ((size_t)1 << 40)) return PBD_ERR_BAD_DIM;
    if ((ny + kTY - 1) / kTY > 65535 || (nz + kTZ - 1) / kTZ > 65535) return PBD_ERR_BAD_DIM;
    if (!(finite_h(s->dz) && s->dz > 0 && finite_h(s->dy) && s->dy > 0 && finite_h(s->dx) &&
          s->dx > 0))
        return PBD_ERR_BAD_VALUE;
    if (!(finite_h(s->dta_mm) && s->dta_mm > 0)) return PBD_ERR_BAD_VALUE;
    if (!finite_h(s->dose_crit_pct) || !finite_h(s->threshold_pct)) return PBD_ERR_BAD_VALUE;
    if (s->max_vox < 0 || s->max_vox > kGR - 1) return PBD_ERR_BAD_VALUE;
    if (s->normalization != PBD_GAMMA_GLOBAL && s->normalization != PBD_GAMMA_LOCAL)
        return PBD_ERR_BAD_VALUE;
    if (s->use_ref_dose && s->ref_dose != s->ref_dose) return PBD_ERR_BAD_VALUE;
    return PBD_OK;
}

struct GammaWs {
    GammaState* st;
    unsigned long long* keys;
    unsigned long long* cand;
    double* psum;
    double* pmax;
    unsigned int* hist;
    int n_blocks;
};

int carve(void* base, int nz, int ny, int nx, GammaWs& w, size_t* bytes) {
    Carve c(base);
    const size_t n = (size_t)nz * ny * nx;
    const int gx = (nx + kTX - 1) / kTX, gy = (ny + kTY - 1) / kTY, gz = (nz + kTZ - 1) / kTZ;
    w.n_blocks = gx * gy * gz;
    w.st = c.take<GammaState>(1);
    w.hist = c.take<unsigned int>(4 * kBins);
    w.psum = c.take<double>(w.n_blocks);
    w.pmax = c.take<double>(w.n_blocks);
    w.keys = c.take<unsigned long long>(n);
    w.cand = c.take<unsigned long long>(n);
    *bytes = c.used + 256;       // slack for an unaligned workspace base
    return PBD_OK;
}

template <class T>
int launch_gamma(const GammaParams& P, const T* ref, const T* ev, double* gmap,
                 unsigned char* mmap, const GammaWs& w, pbd_gamma_stats* out, int n_offsets,
                 cudaStream_t s) {
    const size_t n = (size_t)P.nz * P.ny * P.nx;
    PBD_TRY(cuda_rc(cudaMemsetAsync(w.st, 0, sizeof(GammaState), s)));
    PBD_TRY(cuda_rc(cudaMemsetAsync(w.hist, 0, 4 * kBins * sizeof(unsigned int), s)));
    int launches = 0;
    if (!P.use_ref_dose) {
        const int blocks = (int)std::min<size_t>((n + kGThreads - 1) / kGThreads,
                                                 (size_t)num_sms() * 8);
        gamma_refmax_kernel<T><<<blocks, kGThreads, 0, s>>>(ref, n, w.st);
        PBD_LAUNCH_CHECK();
        ++launches;
    }
    const size_t smem = (size_t)(kTX + 2 * P.hx) * (kTY + 2 * P.hy) * (kTZ + 2 * P.hz) *
                            sizeof(double) +
                        (size_t)P.n_off * (sizeof(double) + sizeof(int));
    int set = 0;                                // once per (device, kernel)
    PBD_TRY(smem_optin((const void*)gamma_kernel<T, false>, kGMaxSmem, 0, &set));
    PBD_TRY(smem_optin((const void*)gamma_kernel<T, true>, kGMaxSmem, 0, &set));
    const int gx = (P.nx + kTX - 1) / kTX, gy = (P.ny + kTY - 1) / kTY;
    const int n_bricks = w.n_blocks;
    int occ = 0;
    PBD_TRY(cuda_rc(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, gamma_kernel<T, false>,
                                                                  kGThreads, smem)));
    const int grid0 = std::max(1, std::min(n_bricks, std::max(occ, 1) * num_sms()));
    const int grid1 = std::max(1, std::min(n_bricks, num_sms()));   // fallback: usually idle
    gamma_kernel<T, false><<<grid0, kGThreads, smem, s>>>(P, ref, ev, gmap, mmap, w.st, w.keys,
                                                          w.psum, w.pmax, gx, gy, n_bricks);
    PBD_LAUNCH_CHECK();
    gamma_kernel<T, true><<<grid1, kGThreads, smem, s>>>(P, ref, ev, gmap, mmap, w.st, w.keys,
                                                         w.psum, w.pmax, gx, gy, n_bricks);
    PBD_LAUNCH_CHECK();
    gamma_finish_kernel<<<1, kFinThreads, 0, s>>>(P, w.st, w.psum, w.pmax, grid0, grid1);
    PBD_LAUNCH_CHECK();
    const int hblocks = num_sms() * 2;
    for (int p = 0; p < kSelPasses; ++p) {
        const int top = 64 - kDigitBits * p;                       // 64, 53, 42, 31, 20, 9
        const int shift = top > kDigitBits ? top - kDigitBits : 0;
        const int mode = p < 2 ? 0 : (p == 2 ? 1 : 2);
        gamma_select_kernel<<<hblocks, kHistThreads, 0, s>>>(w.st, w.keys, w.cand, shift, top,
                                                             mode, w.hist);
        PBD_LAUNCH_CHECK();
    }
    gamma_final_kernel<<<1, 1, 0, s>>>(P, w.st, out, n_offsets);
    PBD_LAUNCH_CHECK();
    count_launch(launches + 4 + kSelPasses);
    return PBD_OK;
}

}  // namespace
}  // namespace pbd

using namespace pbd;

int pbd_gamma_offsets(const pbd_gamma_spec* spec, int* n_offsets, int* radii, double* weights) {
    if (!spec || !n_offsets) return PBD_ERR_NULL_ARG;
    PBD_TRY(validate(spec, 1, 1, 1));
    GammaTable t;
    PBD_TRY(build_table(spec, &t));
    *n_offsets = t.n_offsets;
    if (radii) { radii[0] = t.hz; radii[1] = t.hy; radii[2] = t.hx; }
    if (weights) {
        for (int i = 0; i < kGTab; ++i) weights[i] = -1.0;
        for (int i = 0; i < t.n_entries; ++i)
            weights[(t.abc[i][0] * kGR + t.abc[i][1]) * kGR + t.abc[i][2]] = t.w[i];
    }
    return PBD_OK;
}

int pbd_gamma_workspace(int nz, int ny, int nx, size_t* bytes) {
    if (!bytes) return PBD_ERR_NULL_ARG;
    if (nz <= 0 || ny <= 0 || nx <= 0) return PBD_ERR_BAD_DIM;
    GammaWs w;
    return carve(nullptr, nz, ny, nx, w, bytes);
}

int pbd_gamma_index(const pbd_gamma_spec* spec, int nz, int ny, int nx, const void* reference,
                    const void* evaluation, int dtype, double* gamma_map,
                    unsigned char* mask_map, pbd_gamma_stats* stats, void* workspace,
                    size_t workspace_bytes, void* stream) {
    PBD_TRY(validate(spec, nz, ny, nx));
    if (!reference || !evaluation || !stats) return PBD_ERR_NULL_ARG;
    if (dtype != PBD_DTYPE_F32 && dtype != PBD_DTYPE_F64) return PBD_ERR_BAD_VALUE;
    GammaWs w;
    size_t need = 0;
    PBD_TRY(carve(nullptr, nz, ny, nx, w, &need));
    if (!workspace || workspace_bytes < need) return PBD_ERR_WORKSPACE;
    PBD_TRY(carve(workspace, nz, ny, nx, w, &need));
    GammaTable t;
    PBD_TRY(build_table(spec, &t));
    GammaParams P;
    memset(&P, 0, sizeof(P));
    P.nz = nz; P.ny = ny; P.nx = nx;
    P.hz = t.hz; P.hy = t.hy; P.hx = t.hx;
    P.n_entries = t.n_entries;
    P.local = spec->normalization == PBD_GAMMA_LOCAL;
    P.use_ref_dose = spec->use_ref_dose != 0;
    P.ref_dose = spec->ref_dose;
    P.want_gamma = gamma_map != nullptr;
    P.want_mask = mask_map != nullptr;
    P.crit_frac = spec->dose_crit_pct / 100.0;                     // gamma.py:120, 123
    P.thr_frac = spec->threshold_pct / 100.0;                      // gamma.py:126
    P.q[0] = 95.0 / 100.0;
    P.q[1] = 99.0 / 100.0;
    int o = 0;
    for (int i = 0; i < t.n_entries; ++i) {
        P.w[i] = t.w[i];
        for (int a = 0; a < 3; ++a) P.abc[i][a] = t.abc[i][a];
        P.start[i] = (short)o;
        o += (t.abc[i][0] ? 2 : 1) * (t.abc[i][1] ? 2 : 1) * (t.abc[i][2] ? 2 : 1);
    }
    P.n_off = o;
    cudaStream_t s = (cudaStream_t)stream;
    if (dtype == PBD_DTYPE_F32)
        return launch_gamma<float>(P, (const float*)reference, (const float*)evaluation,
                                   gamma_map, mask_map, w, stats, t.n_offsets, s);
    return launch_gamma<double>(P, (const double*)reference, (const double*)evaluation,
                                gamma_map, mask_map, w, stats, t.n_offsets, s);
}
