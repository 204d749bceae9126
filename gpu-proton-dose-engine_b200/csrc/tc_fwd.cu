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
// TMEM, scaled, rounded and stored as stage 2's B operand; D stays in TMEM across the
// item's layers and is written once.  One thread issues the MMAs; completion is signalled
// through mbarriers by tcgen05.commit.  Every wait is bounded (2 s of %globaltimer): on
// expiry the CTA sets the workspace error word, drains, frees its TMEM and leaves, and the
// finalize pass turns the output into NaN.
//
// Precision modes (accumulation always FP32):
//   TF32X3  a b ~ ah bh + ah bl + al bh with ah = tf32(a), al = tf32(a - ah)  (~1e-7)
//   TF32    ah bh
//   BF16X3  the same split with bf16 hi / lo parts
//   BF16    ah bh in bf16
#include <algorithm>

#include "pbd_internal.cuh"
#include "tc_ptx.cuh"

namespace pbd {
namespace {

constexpr int TNT = 256;
constexpr uint32_t kTmemCols = 256;   // D: 128 columns, stage-1 accumulator: <= 64
constexpr uint64_t kWaitNs = 2000000000ull;

template <int MODE> struct Prec;
template <> struct Prec<PBD_PREC_TF32X3> {
    static constexpr int EB = 4, EPC = 4, KSTEP = 8, NPROD = 3;
    static constexpr uint32_t FMT = 2;
};
template <> struct Prec<PBD_PREC_TF32> {
    static constexpr int EB = 4, EPC = 4, KSTEP = 8, NPROD = 1;
    static constexpr uint32_t FMT = 2;
};
template <> struct Prec<PBD_PREC_BF16X3> {
    static constexpr int EB = 2, EPC = 8, KSTEP = 16, NPROD = 3;
    static constexpr uint32_t FMT = 1;
};
template <> struct Prec<PBD_PREC_BF16> {
    static constexpr int EB = 2, EPC = 8, KSTEP = 16, NPROD = 1;
    static constexpr uint32_t FMT = 1;
};

__device__ __forceinline__ float ex2_approx(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

__device__ __forceinline__ uint64_t now_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ bool wait_bar(uint64_t* bar, uint32_t parity) {
    if (tc::mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = now_ns();
    while (!tc::mbar_try_wait(bar, parity))
        if (now_ns() - t0 > kWaitNs) return false;
    return true;
}

__device__ __forceinline__ uint32_t bf16_bits(float v) {
    return (uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(v));
}

// Round one chunk (EPC values) to the operand type: hi part and, for split modes, lo part.
template <int MODE>
__device__ __forceinline__ void split_chunk(const float* v, uint4& hi, uint4& lo) {
    using P = Prec<MODE>;
    uint32_t h[4], l[4];
    if constexpr (P::EB == 4) {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            h[q] = tc::to_tf32(v[q]);
            l[q] = P::NPROD == 3 ? tc::to_tf32(v[q] - __uint_as_float(h[q])) : 0u;
        }
    } else {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const float a = v[2 * q], b = v[2 * q + 1];
            const uint32_t ha = bf16_bits(a), hb = bf16_bits(b);
            h[q] = ha | (hb << 16);
            if (P::NPROD == 3) {
                const float ra = a - __uint_as_float(ha << 16), rb = b - __uint_as_float(hb << 16);
                l[q] = bf16_bits(ra) | (bf16_bits(rb) << 16);
            } else {
                l[q] = 0u;
            }
        }
    }
    hi = make_uint4(h[0], h[1], h[2], h[3]);
    lo = make_uint4(l[0], l[1], l[2], l[3]);
}

struct Bufs {
    uint8_t *a1[2], *b1[2], *a2[2], *b2[2];
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
    const uint32_t tD = tmem_base_s, tD1 = tmem_base_s + 128u;
    const uint32_t lane_base = (uint32_t)(32 * (warp & 3)) << 16;
    const uint32_t idesc1 = tc::instr_desc(128, N1, P::FMT);
    const uint32_t idesc2 = tc::instr_desc(128, 128, P::FMT);
    const uint32_t plane128 = 128u * 16u, plane_n1 = (uint32_t)N1 * 16u;

    uint32_t ph1 = 0, ph2 = 0;
    bool mma1_pending = false, mma2_pending = false, failed = false;

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
        bool first = true;

        for (int l = it.lb; l < it.le && !failed; ++l) {
            const double c = J.idd[(size_t)l * nz + z];
            if (c == 0.0) continue;
            const double s = fmax(J.sigma[(size_t)l * nz + z], 1e-9);
            const double a2 = kLog2e / (2.0 * s * s);
            const float scale = (float)(c * kInv2Pi / (s * s));
            const float* wl = J.w + (size_t)l * nsy * nsx;

            // ---- stage-1 operands: A1 = Gx (128 x-rows, K1), B1 = W (N1 j-rows, K1) ----
            const int g1 = K1 / P::EPC;
            for (int e = tid; e < 128 * g1; e += TNT) {
                const int row = e & 127, g = e >> 7;
                const double xv = J.ox + (double)(x0 + row) * J.dx;
                float v[P::EPC];
#pragma unroll
                for (int q = 0; q < P::EPC; ++q) {
                    const int i = g * P::EPC + q;
                    const double d = xv - (J.sx0 + ((double)i - cx) * J.dsx);
                    v[q] = i < nsx ? ex2_approx((float)(-(d * d) * a2)) : 0.f;
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
                uint32_t acc = 0;
                for (int st = 0; st < K1 / P::KSTEP; ++st) {
#pragma unroll
                    for (int pr = 0; pr < P::NPROD; ++pr) {
                        const int ai = pr == 2 ? 1 : 0, bi = pr == 1 ? 1 : 0;
                        const uint64_t da = tc::smem_desc(
                            tc::smem_u32(B.a1[ai]) + (uint32_t)st * 2u * plane128, plane128, 128);
                        const uint64_t db = tc::smem_desc(
                            tc::smem_u32(B.b1[bi]) + (uint32_t)st * 2u * plane_n1, plane_n1, 128);
                        if (P::EB == 4) tc::mma_tf32(tD1, da, db, idesc1, acc);
                        else tc::mma_bf16(tD1, da, db, idesc1, acc);
                        acc = 1;
                    }
                }
                tc::commit(&bar[0]);
            }
            mma1_pending = true;

            // ---- stage-2 A operand: Gy (128 y-rows, K2); wait until MMA2(prev) read A2/B2 ----
            if (mma2_pending) {
                const bool ok = wait_bar(&bar[1], ph2);
                if (ok) { ph2 ^= 1; mma2_pending = false; }
                if (__syncthreads_or(!ok)) { failed = true; break; }
            }
            const int g2 = K2 / P::EPC;
            for (int e = tid; e < 128 * g2; e += TNT) {
                const int row = e & 127, g = e >> 7;
                const double yv = J.oy + (double)(y0 + row) * J.dy;
                float v[P::EPC];
#pragma unroll
                for (int q = 0; q < P::EPC; ++q) {
                    const int j = g * P::EPC + q;
                    const double d = yv - (J.sy0 + ((double)j - cy) * J.dsy);
                    v[q] = j < nsy ? ex2_approx((float)(-(d * d) * a2)) : 0.f;
                }
                uint4 hi, lo;
                split_chunk<MODE>(v, hi, lo);
                const uint32_t off = (uint32_t)g * plane128 + (uint32_t)row * 16u;
                *reinterpret_cast<uint4*>(B.a2[0] + off) = hi;
                if (NARR == 2) *reinterpret_cast<uint4*>(B.a2[1] + off) = lo;
            }

            // ---- U = s * stage-1 result -> B2 (128 x-rows, K2) ----
            {
                const bool ok = wait_bar(&bar[0], ph1);
                if (ok) { ph1 ^= 1; mma1_pending = false; }
                if (__syncthreads_or(!ok)) { failed = true; break; }
            }
            tc::fence_after_sync();
            {
                const int row = 32 * (warp & 3) + lane;
                const int half = warp >> 2, ncol = N1 / 2;
                for (int c0 = half * ncol; c0 < (half + 1) * ncol; c0 += 8) {
                    uint32_t r[8];
                    tc::tmem_ld8(tD1 + lane_base + (uint32_t)c0, r);
                    tc::tmem_wait_ld();
                    float v[8];
#pragma unroll
                    for (int q = 0; q < 8; ++q) v[q] = __uint_as_float(r[q]) * scale;
#pragma unroll
                    for (int part = 0; part < 8 / P::EPC; ++part) {
                        uint4 hi, lo;
                        split_chunk<MODE>(v + part * P::EPC, hi, lo);
                        const int g = (c0 + part * P::EPC) / P::EPC;
                        const uint32_t off = (uint32_t)g * plane128 + (uint32_t)row * 16u;
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
                uint32_t acc = first ? 0u : 1u;
                for (int st = 0; st < K2 / P::KSTEP; ++st) {
#pragma unroll
                    for (int pr = 0; pr < P::NPROD; ++pr) {
                        const int ai = pr == 2 ? 1 : 0, bi = pr == 1 ? 1 : 0;
                        const uint64_t da = tc::smem_desc(
                            tc::smem_u32(B.a2[ai]) + (uint32_t)st * 2u * plane128, plane128, 128);
                        const uint64_t db = tc::smem_desc(
                            tc::smem_u32(B.b2[bi]) + (uint32_t)st * 2u * plane128, plane128, 128);
                        if (P::EB == 4) tc::mma_tf32(tD, da, db, idesc2, acc);
                        else tc::mma_bf16(tD, da, db, idesc2, acc);
                        acc = 1;
                    }
                }
                tc::commit(&bar[1]);
            }
            mma2_pending = true;
            first = false;
        }
        if (failed) break;

        // ---- epilogue: D (lanes = y, columns = x) -> partial slice of this chunk ----
        if (mma2_pending) {
            const bool ok = wait_bar(&bar[1], ph2);
            if (ok) { ph2 ^= 1; mma2_pending = false; }
            if (__syncthreads_or(!ok)) { failed = true; break; }
        }
        tc::fence_after_sync();
        {
            const int yy = 32 * (warp & 3) + lane, half = warp >> 2;
            const int y = y0 + yy;
            const size_t n3 = (size_t)nz * ny * nx;
            float* out = J.partial + (size_t)it.chunk * n3 + (size_t)z * ny * nx + (size_t)y * nx;
            for (int c0 = half * 64; c0 < half * 64 + 64; c0 += 16) {
                uint32_t r[16];
                tc::tmem_ld16(tD + lane_base + (uint32_t)c0, r);
                tc::tmem_wait_ld();
                if (y < ny) {
                    const int xb = x0 + c0;
                    if (xb + 16 <= nx && (nx & 3) == 0) {
#pragma unroll
                        for (int q = 0; q < 16; q += 4)
                            *reinterpret_cast<float4*>(out + xb + q) =
                                make_float4(__uint_as_float(r[q]), __uint_as_float(r[q + 1]),
                                            __uint_as_float(r[q + 2]), __uint_as_float(r[q + 3]));
                    } else {
#pragma unroll
                        for (int q = 0; q < 16; ++q)
                            if (xb + q < nx) out[xb + q] = __uint_as_float(r[q]);
                    }
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
    // At least 116 KiB so that one CTA (and its 256 TMEM columns) occupies an SM: a second
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
