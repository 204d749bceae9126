// tc_fwd.cu -- forward dose on the 5th-generation tensor cores (tcgen05, TMEM accumulators).
//
// Same work items and partial-slice output as the FP32 kernel (fwd_simt.cu); per active
// (layer l, slice z) of an item and per 128 x 128 lateral tile:
//
//   stage 1   U[x, j]  = sum_i Gx[x, i] W[j, i]          M = 128 (x), N = N1 (j), K = K1 (i)
//   stage 2   D[y, x] += sum_j Gy[y, j] (s U)[x, j]       M = 128 (y), N = 128 (x), K = N1 (j)
//
// with s = IDD_l(z) / (2 pi sigma^2) and unnormalised Gaussians exp(-d^2 / (2 sigma^2)).
// The Gaussian factors are generated by the CTA's 256 threads straight into shared memory
// in the UMMA canonical K-major layout (no swizzle; 16-byte chunk planes of all rows, so
// a warp's stores are 512 contiguous bytes); the stage-1 accumulator is read back from
// TMEM, scaled, rounded and stored as stage 2's B operand.  One thread issues the MMAs;
// completion is signalled through mbarriers by tcgen05.commit.  Every wait is bounded
// (2 s of %globaltimer): on expiry the CTA sets the workspace error word, drains, frees
// its TMEM and leaves, and the finalize pass turns the output into NaN.
//
// Accumulation.  The tensor core's FP32 accumulation aligns and truncates, so its error
// grows with the number of MMA steps into one accumulator.  Each (layer, slice) therefore
// starts fresh accumulators, and the large hi*hi products and the two small cross
// products go to separate ones (6 + 12 steps at K = 48; the small accumulator is ~2^-11 of
// the large one).  Big + small are added in FP32 registers, and the layers of an item are
// summed there too (IEEE round to nearest): D is read back from TMEM once per layer while
// the next layer's stage 1 runs.
//
// Precision modes (accumulation always FP32):
//   TF32X3  a b ~ ah bh + ah bl + al bh with ah = tf32(a), al = tf32(a - ah)  (~1e-7)
//   TF32    ah bh
//   BF16X3  the same split with bf16 hi / lo parts
//   BF16    ah bh in bf16
#include <algorithm>

#include "pbd_internal.cuh"
#include "tc_common.cuh"

namespace pbd {
namespace {
using namespace tcc;

constexpr int TNT = 256;
constexpr uint32_t kTmemCols = 512;   // stage 2 big/small 2 x 128, stage 1 big/small 2 x 64
struct Bufs {
    uint8_t *a1[2], *b1[2], *a2[2], *b2[2];
};

template <int MODE>
struct Ops {
    using P = Prec<MODE>;
    // One stage: big products (hi x hi) into t_big, the two cross products into t_small.
    // Each accumulator starts fresh (acc = 0) for every (layer, slice): the tensor core's
    // FP32 accumulation truncates, so its error grows with the steps per accumulator.
    __device__ static void issue(uint32_t t_big, uint32_t t_small, uint8_t* const* a,
                                 uint8_t* const* b, uint32_t plane_a, uint32_t plane_b,
                                 int ksteps, uint32_t idesc) {
        uint32_t acc_b = 0, acc_s = 0;
        for (int st = 0; st < ksteps; ++st) {
            const uint32_t oa = (uint32_t)st * 2u * plane_a, ob = (uint32_t)st * 2u * plane_b;
            const uint64_t da_hi = tc::smem_desc(tc::smem_u32(a[0]) + oa, plane_a, 128);
            const uint64_t db_hi = tc::smem_desc(tc::smem_u32(b[0]) + ob, plane_b, 128);
            mma(t_big, da_hi, db_hi, idesc, acc_b);
            acc_b = 1;
            if (P::NPROD == 3) {
                const uint64_t da_lo = tc::smem_desc(tc::smem_u32(a[1]) + oa, plane_a, 128);
                const uint64_t db_lo = tc::smem_desc(tc::smem_u32(b[1]) + ob, plane_b, 128);
                mma(t_small, da_hi, db_lo, idesc, acc_s);
                acc_s = 1;
                mma(t_small, da_lo, db_hi, idesc, 1u);
            }
        }
    }
    __device__ static void mma(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
        if (P::EB == 4) tc::mma_tf32(d, a, b, idesc, acc);
        else tc::mma_bf16(d, a, b, idesc, acc);
    }
};

template <int MODE>
__global__ void __launch_bounds__(TNT, 1)
fwd_tc_kernel(const JobDev* __restrict__ jobs, const FwdItem* __restrict__ items, int total,
              int* counter, int* err, int K1, int N1) {
    using P = Prec<MODE>;
    constexpr int NARR = P::NPROD == 3 ? 2 : 1;
    extern __shared__ __align__(1024) uint8_t smem[];
    __shared__ __align__(8) uint64_t bar[2];
    __shared__ uint32_t tmem_base_s;
    __shared__ int s_item;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int K2 = N1;
    const uint32_t a1_bytes = 128u * K1 * P::EB, b1_bytes = (uint32_t)N1 * K1 * P::EB;
    const uint32_t a2_bytes = 128u * K2 * P::EB;
    Bufs B;
    {
        uint8_t* p = smem;
        for (int k = 0; k < 2; ++k) { B.a1[k] = p; p += (k < NARR) ? a1_bytes : 0; }
        for (int k = 0; k < 2; ++k) { B.b1[k] = p; p += (k < NARR) ? b1_bytes : 0; }
        for (int k = 0; k < 2; ++k) { B.a2[k] = p; p += (k < NARR) ? a2_bytes : 0; }
        for (int k = 0; k < 2; ++k) { B.b2[k] = p; p += (k < NARR) ? a2_bytes : 0; }
    }

    if (warp == 0) {
        tc::tmem_alloc(&tmem_base_s, kTmemCols);
        tc::tmem_relinquish();
    }
    if (tid == 0) {
        tc::mbar_init(&bar[0], 1);
        tc::mbar_init(&bar[1], 1);
        tc::fence_mbar_init();
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    // TMEM columns: stage-2 big / small [0,128) [128,256); stage-1 big / small [256,320) [320,384)
    const uint32_t tDb = tmem_base_s, tDs = tmem_base_s + 128u;
    const uint32_t tUb = tmem_base_s + 256u, tUs = tmem_base_s + 320u;
    const uint32_t lane_base = (uint32_t)(32 * (warp & 3)) << 16;
    const uint32_t idesc1 = tc::instr_desc(128, N1, P::FMT);
    const uint32_t idesc2 = tc::instr_desc(128, 128, P::FMT);
    const uint32_t plane128 = 128u * 16u, plane_n1 = (uint32_t)N1 * 16u;
    const int half = warp >> 2;          // which 64 columns this warp reads back
    const int trow = 32 * (warp & 3) + lane;

    uint32_t ph1 = 0, ph2 = 0;
    bool mma1_pending = false, mma2_pending = false, failed = false;
    float dsum[64];

    // Wait for the stage-2 MMAs of the previous layer and add its D into the registers.
    auto drain_stage2 = [&]() -> bool {
        const bool ok = wait_bar(&bar[1], ph2);
        if (ok) { ph2 ^= 1; mma2_pending = false; }
        if (__syncthreads_or(!ok)) return false;
        tc::fence_after_sync();
        for (int c0 = 0; c0 < 64; c0 += 16) {
            uint32_t rb[16], rs[16];
            tc::tmem_ld16(tDb + lane_base + (uint32_t)(half * 64 + c0), rb);
            if (P::NPROD == 3) tc::tmem_ld16(tDs + lane_base + (uint32_t)(half * 64 + c0), rs);
            tc::tmem_wait_ld();
#pragma unroll
            for (int q = 0; q < 16; ++q) {
                float v = __uint_as_float(rb[q]);
                if (P::NPROD == 3) v += __uint_as_float(rs[q]);
                dsum[c0 + q] += v;
            }
        }
        return true;
    };

    for (;;) {
        if (tid == 0) s_item = atomicAdd(counter, 1);
        __syncthreads();
        const int it_idx = s_item;
        __syncthreads();
        if (it_idx >= total) break;
        const FwdItem it = items[it_idx];
        if (it.cost == 0) continue;
        const JobDev& J = jobs[it.job];
        const int nz = J.nz, nx = J.nx, ny = J.ny, nsx = J.nsx, nsy = J.nsy;
        const int z = it.z, y0 = it.ty * kTile, x0 = it.tx * kTile;
        const double cx = 0.5 * (double)(nsx - 1), cy = 0.5 * (double)(nsy - 1);
#pragma unroll
        for (int q = 0; q < 64; ++q) dsum[q] = 0.f;

        for (int l = it.lb; l < it.le && !failed; ++l) {
            const double c = J.idd[(size_t)l * nz + z];
            if (c == 0.0) continue;
            const double s = fmax(J.sigma[(size_t)l * nz + z], 1e-9);
            const float a2 = (float)(kLog2e / (2.0 * s * s));   // exponent scale, FP32
            const float scale = (float)(c * kInv2Pi / (s * s));
            const float* wl = J.w + (size_t)l * nsy * nsx;

            // ---- stage-1 operands: A1 = Gx (128 x-rows, K1), B1 = W (N1 j-rows, K1) ----
            const int g1 = K1 / P::EPC;
            for (int e = tid; e < 128 * g1; e += TNT) {
                const int row = e & 127, g = e >> 7;
                const double xv = J.ox + (double)(x0 + row) * J.dx;
                // one FP64 difference per chunk (taken at the chunk's middle spot, so that
                // |base - d| <= EPC/2 pitches), then one FP32 fma per spot: d is rounded
                // once, and base's own rounding stays below 1e-7 cm for nearby spots
                constexpr int MID = P::EPC / 2;
                const float base = (float)(xv - (J.sx0 + ((double)(g * P::EPC + MID) - cx) * J.dsx));
                const float dsf = (float)J.dsx;
                float v[P::EPC];
#pragma unroll
                for (int q = 0; q < P::EPC; ++q) {
                    const int i = g * P::EPC + q;
                    const float df = fmaf(-(float)(q - MID), dsf, base);
                    v[q] = i < nsx ? ex2_approx(-(df * df) * a2) : 0.f;
                }
                uint4 hi, lo;
                split_chunk<MODE>(v, hi, lo);
                const uint32_t off = (uint32_t)g * plane128 + (uint32_t)row * 16u;
                *reinterpret_cast<uint4*>(B.a1[0] + off) = hi;
                if (NARR == 2) *reinterpret_cast<uint4*>(B.a1[1] + off) = lo;
            }
            for (int e = tid; e < N1 * g1; e += TNT) {
                const int row = e % N1, g = e / N1;
                float v[P::EPC];
#pragma unroll
                for (int q = 0; q < P::EPC; ++q) {
                    const int i = g * P::EPC + q;
                    v[q] = (row < nsy && i < nsx) ? wl[(size_t)row * nsx + i] : 0.f;
                }
                uint4 hi, lo;
                split_chunk<MODE>(v, hi, lo);
                const uint32_t off = (uint32_t)g * plane_n1 + (uint32_t)row * 16u;
                *reinterpret_cast<uint4*>(B.b1[0] + off) = hi;
                if (NARR == 2) *reinterpret_cast<uint4*>(B.b1[1] + off) = lo;
            }
            tc::fence_async_smem();
            __syncthreads();
            if (tid == 0) {
                tc::fence_after_sync();
                Ops<MODE>::issue(tUb, tUs, B.a1, B.b1, plane128, plane_n1, K1 / P::KSTEP, idesc1);
                tc::commit(&bar[0]);
            }
            mma1_pending = true;

            // ---- previous layer's stage 2 done: D into registers, A2/B2 free ----
            if (mma2_pending && !drain_stage2()) { failed = true; break; }

            // ---- stage-2 A operand: Gy (128 y-rows, K2) ----
            const int g2 = K2 / P::EPC;
            for (int e = tid; e < 128 * g2; e += TNT) {
                const int row = e & 127, g = e >> 7;
                const double yv = J.oy + (double)(y0 + row) * J.dy;
                constexpr int MID = P::EPC / 2;
                const float base = (float)(yv - (J.sy0 + ((double)(g * P::EPC + MID) - cy) * J.dsy));
                const float dsf = (float)J.dsy;
                float v[P::EPC];
#pragma unroll
                for (int q = 0; q < P::EPC; ++q) {
                    const int j = g * P::EPC + q;
                    const float df = fmaf(-(float)(q - MID), dsf, base);
                    v[q] = j < nsy ? ex2_approx(-(df * df) * a2) : 0.f;
                }
                uint4 hi, lo;
                split_chunk<MODE>(v, hi, lo);
                const uint32_t off = (uint32_t)g * plane128 + (uint32_t)row * 16u;
                *reinterpret_cast<uint4*>(B.a2[0] + off) = hi;
                if (NARR == 2) *reinterpret_cast<uint4*>(B.a2[1] + off) = lo;
            }

            // ---- U = s * (stage-1 big + small) -> B2 (128 x-rows, K2) ----
            {
                const bool ok = wait_bar(&bar[0], ph1);
                if (ok) { ph1 ^= 1; mma1_pending = false; }
                if (__syncthreads_or(!ok)) { failed = true; break; }
            }
            tc::fence_after_sync();
            {
                const int ncol = N1 / 2;
                for (int c0 = half * ncol; c0 < (half + 1) * ncol; c0 += 8) {
                    uint32_t rb[8], rs[8];
                    tc::tmem_ld8(tUb + lane_base + (uint32_t)c0, rb);
                    if (P::NPROD == 3) tc::tmem_ld8(tUs + lane_base + (uint32_t)c0, rs);
                    tc::tmem_wait_ld();
                    float v[8];
#pragma unroll
                    for (int q = 0; q < 8; ++q) {
                        float u = __uint_as_float(rb[q]);
                        if (P::NPROD == 3) u += __uint_as_float(rs[q]);
                        v[q] = u * scale;
                    }
#pragma unroll
                    for (int part = 0; part < 8 / P::EPC; ++part) {
                        uint4 hi, lo;
                        split_chunk<MODE>(v + part * P::EPC, hi, lo);
                        const int g = (c0 + part * P::EPC) / P::EPC;
                        const uint32_t off = (uint32_t)g * plane128 + (uint32_t)trow * 16u;
                        *reinterpret_cast<uint4*>(B.b2[0] + off) = hi;
                        if (NARR == 2) *reinterpret_cast<uint4*>(B.b2[1] + off) = lo;
                    }
                }
            }
            tc::fence_async_smem();
            tc::fence_before_sync();
            __syncthreads();
            if (tid == 0) {
                tc::fence_after_sync();
                Ops<MODE>::issue(tDb, tDs, B.a2, B.b2, plane128, plane128, K2 / P::KSTEP, idesc2);
                tc::commit(&bar[1]);
            }
            mma2_pending = true;
        }
        if (failed) break;

        // ---- epilogue: last layer's D into the registers, then the partial slice ----
        if (mma2_pending && !drain_stage2()) { failed = true; break; }
        {
            const int y = y0 + trow;
            const size_t n3 = (size_t)nz * ny * nx;
            float* out = J.partial + (size_t)it.chunk * n3 + (size_t)z * ny * nx + (size_t)y * nx;
            if (y < ny) {
                const int xb = x0 + half * 64;
                if (xb + 64 <= nx && (nx & 3) == 0) {
#pragma unroll
                    for (int q = 0; q < 64; q += 4)
                        *reinterpret_cast<float4*>(out + xb + q) =
                            make_float4(dsum[q], dsum[q + 1], dsum[q + 2], dsum[q + 3]);
                } else {
#pragma unroll
                    for (int q = 0; q < 64; ++q)
                        if (xb + q < nx) out[xb + q] = dsum[q];
                }
            }
        }
        tc::fence_before_sync();
        __syncthreads();
    }

    if (failed) {
        if (tid == 0) atomicExch(err, 1);
        // drain what this CTA still has in flight (bounded), then release TMEM
        if (mma1_pending) (void)wait_bar(&bar[0], ph1);
        if (mma2_pending) (void)wait_bar(&bar[1], ph2);
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    if (warp == 0) tc::tmem_dealloc(tmem_base_s, kTmemCols);
}

template <int MODE>
size_t tc_smem_bytes(int K1, int N1) {
    using P = Prec<MODE>;
    const int narr = P::NPROD == 3 ? 2 : 1;
    return (size_t)narr * P::EB * (128u * K1 + (size_t)N1 * K1 + 2u * 128u * N1);
}

template <int MODE>
int launch_mode(JobDev* jobs, FwdItem* items, int total, int* counter, int* err, int K1, int N1,
                cudaStream_t s) {
    static thread_local int max_dyn = 0;
    if (max_dyn == 0) {
        int dev = 0, optin = 0;
        cudaFuncAttributes fa;
        if (cudaGetDevice(&dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) !=
                cudaSuccess ||
            cudaFuncGetAttributes(&fa, fwd_tc_kernel<MODE>) != cudaSuccess)
            return PBD_ERR_CUDA;
        const int avail = optin - (int)fa.sharedSizeBytes;
        if (avail <= 0 || cudaFuncSetAttribute(fwd_tc_kernel<MODE>,
                                               cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               avail) != cudaSuccess)
            return PBD_ERR_NO_SMEM;
        max_dyn = avail;
    }
    // At least 116 KiB so that one CTA (and its 512 TMEM columns) occupies an SM: a second
    // resident CTA would only wait in tcgen05.alloc for the first to finish.
    const size_t smem = std::max<size_t>(tc_smem_bytes<MODE>(K1, N1), 116u * 1024u);
    if (smem > (size_t)max_dyn) return PBD_ERR_NO_SMEM;
    const int grid = std::max(1, std::min(total, num_sms()));
    prof_mark(kProfFwd, 0, s);
    fwd_tc_kernel<MODE><<<grid, TNT, smem, s>>>(jobs, items, total, counter, err, K1, N1);
    PBD_LAUNCH_CHECK();
    prof_mark(kProfFwd, 1, s);
    return PBD_OK;
}

}  // namespace

int tc_operand_dims(int precision, int nsx, int nsy, int* K1, int* N1) {
    const int kstep = (precision == PBD_PREC_BF16X3 || precision == PBD_PREC_BF16) ? 16 : 8;
    *K1 = (nsx + kstep - 1) / kstep * kstep;
    *N1 = (nsy + 15) / 16 * 16;
    if (*K1 > 64 || *N1 > 64) return PBD_ERR_UNSUPPORTED;
    return PBD_OK;
}

int launch_forward_tc_main(int precision, JobDev* jobs, FwdItem* items, int total, int* counter,
                           int* err, int K1, int N1, cudaStream_t s) {
    switch (precision) {
        case PBD_PREC_TF32X3:
            return launch_mode<PBD_PREC_TF32X3>(jobs, items, total, counter, err, K1, N1, s);
        case PBD_PREC_TF32:
            return launch_mode<PBD_PREC_TF32>(jobs, items, total, counter, err, K1, N1, s);
        case PBD_PREC_BF16X3:
            return launch_mode<PBD_PREC_BF16X3>(jobs, items, total, counter, err, K1, N1, s);
        case PBD_PREC_BF16:
            return launch_mode<PBD_PREC_BF16>(jobs, items, total, counter, err, K1, N1, s);
        default:
            return PBD_ERR_BAD_VALUE;
    }
}

}  // namespace pbd
