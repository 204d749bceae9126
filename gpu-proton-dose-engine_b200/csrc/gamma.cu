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
//   gamma_hist/scan       radix select of the four order statistics the percentiles need
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
// largest staged brick: radius 6 on every axis
constexpr int kGMaxSmem = (kTX + 12) * (kTY + 12) * (kTZ + 12) * (int)sizeof(double);

struct GammaParams {
    int nz, ny, nx;
    int hz, hy, hx;
    int n_entries;                     // distinct (|a|,|b|,|c|) inside the ball
    int local;
    int use_ref_dose;
    int want_gamma, want_mask;
    double ref_dose;
    double crit_frac;                  // dose_crit_pct / 100
    double thr_frac;                   // threshold_pct / 100
    double q[2];                       // 95/100, 99/100
    double w[kGTab];                   // (|o|/DTA)^2, ascending
    unsigned char abc[kGTab][4];       // |a|, |b|, |c| of each entry
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
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x)
        best = max(best, dkey(ld(ref, i)));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) best = max(best, __shfl_xor_sync(0xffffffffu, best, o));
    if ((threadIdx.x & 31) == 0 && best) atomicMax(&st->ref_key, best);
}

template <class T, bool kFallback>
__global__ void __launch_bounds__(kGThreads)
gamma_kernel(const GammaParams P, const T* __restrict__ ref, const T* __restrict__ ev,
             double* __restrict__ gmap, unsigned char* __restrict__ mmap, GammaState* st,
             unsigned long long* __restrict__ keys, double* __restrict__ part_sum,
             double* __restrict__ part_max) {
    extern __shared__ double tile[];
    __shared__ double red_s[kGThreads / 32], red_m[kGThreads / 32];
    __shared__ unsigned long long red_c[kGThreads / 32][3];
    __shared__ int s_nonfinite;
    const int pass = kFallback ? 1 : 0;
    if (kFallback && __ldcg(&st->cnt[0][0]) != 0ull) return;   // the threshold mask is used
    const double ref_max = P.use_ref_dose ? P.ref_dose : dunkey(__ldcg(&st->ref_key));
    if (ref_max <= 0.0) {                                      // gamma.py:112-113
        if (blockIdx.x == 0 && blockIdx.y == 0 && blockIdx.z == 0 && threadIdx.x == 0)
            st->status = PBD_ERR_BAD_VALUE;
        return;
    }
    const int tid = threadIdx.x;
    const int x0 = blockIdx.x * kTX, y0 = blockIdx.y * kTY, z0 = blockIdx.z * kTZ;
    const int TX = kTX + 2 * P.hx, TY = kTY + 2 * P.hy, TZ = kTZ + 2 * P.hz;
    const int plane = TX * TY;
    if (tid == 0) s_nonfinite = 0;
    __syncthreads();
    int nonfin = 0;
    for (int i = tid; i < plane * TZ; i += kGThreads) {
        const int tz = i / plane, r = i - tz * plane, ty = r / TX, tx = r - ty * TX;
        const int z = z0 - P.hz + tz, y = y0 - P.hy + ty, x = x0 - P.hx + tx;
        double v = 0.0;
        if (z >= 0 && z < P.nz && y >= 0 && y < P.ny && x >= 0 && x < P.nx)
            v = ld(ev, ((size_t)z * P.ny + y) * P.nx + x);
        nonfin |= !finite_d(v);
        tile[i] = v;
    }
    if (nonfin) s_nonfinite = 1;
    __syncthreads();
    const bool tile_finite = s_nonfinite == 0;
    const double crit_g = __dmul_rn(P.crit_frac, ref_max);     // global dose criterion
    const double thr_dose = __dmul_rn(P.thr_frac, ref_max);
    const bool ok_g = finite_d(crit_g) || P.local;
    const int tx = tid & 31, ty = tid >> 5;
    const int x = x0 + tx, y = y0 + ty;
    double sum = 0.0, mx = -1.0;                 // gamma >= 0
    unsigned long long c_eval = 0, c_pass = 0, c_nan = 0;
    const int lane = tid & 31;
    for (int k = 0; k < kTZ; ++k) {
        const int z = z0 + k;
        const bool in = x < P.nx && y < P.ny && z < P.nz;
        double g = 0.0;
        bool masked = false;
        if (in) {
            const size_t v = ((size_t)z * P.ny + y) * P.nx + x;
            const double r = ld(ref, v);
            const double crit = P.local ? __dmul_rn(P.crit_frac, r > 1e-12 || r != r ? r : 1e-12)
                                        : crit_g;
            // early exit is exact when no NaN can appear later: finite doses, a finite
            // non-zero criterion (NaN needs 0/0, inf - inf or inf/inf)
            const bool fast = tile_finite && finite_d(r) && finite_d(crit) && crit != 0.0 && ok_g;
            const double* c0 = tile + (size_t)(k + P.hz) * plane + (ty + P.hy) * TX + (tx + P.hx);
            double best = __longlong_as_double(0x7FF0000000000000ll);    // +inf
            for (int u = 0; u < P.n_entries; ++u) {
                const double w = P.w[u];
                if (fast && w >= best) break;    // w + d^2 >= w >= best for this and later
                const int ia = P.abc[u][0], ib = P.abc[u][1], ic = P.abc[u][2];
                for (int s = 0; s < 8; ++s) {
                    const int sa = (s & 4) ? -ia : ia, sb = (s & 2) ? -ib : ib,
                              sc = (s & 1) ? -ic : ic;
                    if (((s & 4) && ia == 0) || ((s & 2) && ib == 0) || ((s & 1) && ic == 0))
                        continue;
                    const double e = c0[sa * plane + sb * TX + sc];
                    const double dd = __ddiv_rn(__dsub_rn(e, r), crit);
                    best = nmin(best, __dadd_rn(w, __dmul_rn(dd, dd)));
                }
            }
            g = __dsqrt_rn(best);
            masked = kFallback ? (r > 0.0) : (r >= thr_dose);
            if (!kFallback && P.want_gamma) gmap[v] = g;
            if (P.want_mask) mmap[v] = masked ? 1 : 0;
        }
        // masked voxels: counts, partial sum / max, and the key list for the percentiles
        if (masked) {
            ++c_eval;
            c_pass += g <= 1.0;
            if (g != g) ++c_nan;
            else { sum = __dadd_rn(sum, g); mx = g > mx ? g : mx; }
        }
        const unsigned int bal = __ballot_sync(0xffffffffu, masked);
        if (bal) {
            unsigned long long base = 0;
            if (lane == 0) base = atomicAdd(&st->cnt[pass][3], (unsigned long long)__popc(bal));
            base = __shfl_sync(0xffffffffu, base, 0);
            if (masked) keys[base + __popc(bal & ((1u << lane) - 1u))] = dkey(g);
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
    const int warp = tid >> 5;
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
        const size_t bid = ((size_t)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
        part_sum[bid] = s;
        part_max[bid] = m;
        if (a) atomicAdd(&st->cnt[pass][0], a);
        if (b) atomicAdd(&st->cnt[pass][1], b);
        if (c) atomicAdd(&st->cnt[pass][2], c);
    }
}

// Statistics of the chosen mask and the ranks of the order statistics (one block).
__global__ void __launch_bounds__(kFinThreads)
gamma_finish_kernel(const GammaParams P, GammaState* st, const double* __restrict__ part_sum,
                    const double* __restrict__ part_max, int n_blocks) {
    __shared__ double s_sum[kFinThreads / 32], s_max[kFinThreads / 32];
    if (st->status != 0) return;
    const int pass = st->cnt[0][0] != 0ull ? 0 : 1;
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

// One radix-select pass: histogram of key bits [shift, top) of the keys whose bits above
// `top` equal each target's prefix (digits of 11 bits from the top, the last one 9 bits).
__global__ void __launch_bounds__(kHistThreads)
gamma_hist_kernel(const GammaState* st, const unsigned long long* __restrict__ keys, int shift,
                  int top, unsigned int* __restrict__ hist) {
    __shared__ unsigned int h[4][kBins];
    if (st->status != 0) return;
    for (int i = threadIdx.x; i < 4 * kBins; i += kHistThreads) (&h[0][0])[i] = 0u;
    __syncthreads();
    const unsigned long long n = st->n_eval;
    const unsigned long long himask = top >= 64 ? 0ull : ~((1ull << top) - 1ull);
    const unsigned int dmask = (1u << (top - shift)) - 1u;
    unsigned long long pre[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) pre[j] = st->prefix[j];
    for (unsigned long long i = (unsigned long long)blockIdx.x * kHistThreads + threadIdx.x; i < n;
         i += (unsigned long long)gridDim.x * kHistThreads) {
        const unsigned long long k = __ldg(keys + i);
        const unsigned int d = (unsigned int)(k >> shift) & dmask;
#pragma unroll
        for (int j = 0; j < 4; ++j)
            if ((k & himask) == pre[j]) atomicAdd(&h[j][d], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 4 * kBins; i += kHistThreads) {
        const unsigned int c = (&h[0][0])[i];
        if (c) atomicAdd(hist + i, c);
    }
}

// Pick each target's digit from its histogram (one warp per target), then clear the histogram.
__global__ void __launch_bounds__(128)
gamma_scan_kernel(GammaState* st, int shift, unsigned int* __restrict__ hist) {
    if (st->status != 0) return;
    const int j = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned int* hj = hist + j * kBins;
    constexpr int per = kBins / 32;
    unsigned long long loc = 0;
    for (int i = 0; i < per; ++i) loc += hj[lane * per + i];
    unsigned long long inc = loc;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long t = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += t;
    }
    const unsigned long long rem = st->rem[j];
    const unsigned int hit = __ballot_sync(0xffffffffu, inc > rem);
    const int src = hit ? __ffs(hit) - 1 : 31;
    if (lane == src) {
        unsigned long long before = inc - loc;
        int d = lane * per;
        for (int i = 0; i < per; ++i) {
            const unsigned int c = hj[lane * per + i];
            if (before + c > rem) { d = lane * per + i; break; }
            before += c;
        }
        st->rem[j] = rem - before;
        st->prefix[j] |= (unsigned long long)d << shift;
    }
    __syncwarp();
    for (int i = lane; i < kBins; i += 32) hj[i] = 0u;
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
    *bytes = c.used;
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
                        sizeof(double);
    static bool attr_set = false;               // one per input type
    if (!attr_set) {
        PBD_TRY(cuda_rc(cudaFuncSetAttribute(gamma_kernel<T, false>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             kGMaxSmem)));
        PBD_TRY(cuda_rc(cudaFuncSetAttribute(gamma_kernel<T, true>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             kGMaxSmem)));
        attr_set = true;
    }
    const dim3 grid((P.nx + kTX - 1) / kTX, (P.ny + kTY - 1) / kTY, (P.nz + kTZ - 1) / kTZ);
    gamma_kernel<T, false><<<grid, kGThreads, smem, s>>>(P, ref, ev, gmap, mmap, w.st, w.keys,
                                                         w.psum, w.pmax);
    PBD_LAUNCH_CHECK();
    gamma_kernel<T, true><<<grid, kGThreads, smem, s>>>(P, ref, ev, gmap, mmap, w.st, w.keys,
                                                        w.psum, w.pmax);
    PBD_LAUNCH_CHECK();
    gamma_finish_kernel<<<1, kFinThreads, 0, s>>>(P, w.st, w.psum, w.pmax, w.n_blocks);
    PBD_LAUNCH_CHECK();
    const int hblocks = num_sms() * 2;
    for (int p = 0; p < kSelPasses; ++p) {
        const int top = 64 - kDigitBits * p;                       // 64, 53, 42, 31, 20, 9
        const int shift = top > kDigitBits ? top - kDigitBits : 0;
        gamma_hist_kernel<<<hblocks, kHistThreads, 0, s>>>(w.st, w.keys, shift, top, w.hist);
        PBD_LAUNCH_CHECK();
        gamma_scan_kernel<<<1, 128, 0, s>>>(w.st, shift, w.hist);
        PBD_LAUNCH_CHECK();
    }
    gamma_final_kernel<<<1, 1, 0, s>>>(P, w.st, out, n_offsets);
    PBD_LAUNCH_CHECK();
    count_launch(launches + 4 + 2 * kSelPasses);
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
    for (int i = 0; i < t.n_entries; ++i) {
        P.w[i] = t.w[i];
        for (int a = 0; a < 3; ++a) P.abc[i][a] = t.abc[i][a];
    }
    cudaStream_t s = (cudaStream_t)stream;
    if (dtype == PBD_DTYPE_F32)
        return launch_gamma<float>(P, (const float*)reference, (const float*)evaluation,
                                   gamma_map, mask_map, w, stats, t.n_offsets, s);
    return launch_gamma<double>(P, (const double*)reference, (const double*)evaluation,
                                gamma_map, mask_map, w, stats, t.n_offsets, s);
}
