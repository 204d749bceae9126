// tc_common.cuh -- pieces shared by the tensor-core kernels: precision traits, operand
// rounding / splitting into the UMMA chunk layout, bounded mbarrier waits.
#pragma once

#include "pbd_internal.cuh"
#include "tc_ptx.cuh"

namespace pbd {
namespace tcc {

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

// Wait for phase `parity` of `bar` for at most `limit_ns` of %globaltimer; false when the
// limit ran out (the caller sets its error word and leaves).
__device__ __forceinline__ bool wait_bar(uint64_t* bar, uint32_t parity,
                                         uint64_t limit_ns = kWaitNs) {
    if (tc::mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = now_ns();
    while (!tc::mbar_try_wait(bar, parity))
        if (now_ns() - t0 > limit_ns) return false;
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

}  // namespace tcc
}  // namespace pbd
