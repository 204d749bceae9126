// adj_tc.cu -- adjoint of the separable dose on the tensor cores (tcgen05).
//
// Same mathematics as adj_simt.cu.  With G = dL/dD[z] and unnormalised Gaussians of
// width s = sigma_l(z), for every active (layer l, slice z):
//
//   stage 1   Y[m, x] = sum_y A[m, y] G[y, x]        A = [Gy | Gy']^T, m < 64: j, m >= 64: j'
//             M = 128 (m), N = 128 (x), K = 128 (y); A generated into TMEM, G^T in smem
//   stage 2   Q[m, n] = sum_x Y[m, x] B[n, x]        B = [Gx | Gx'], n < N1: i, n >= N1: i'
//             M = 128 (m), N = 2 N1 (n), K = 128 (x); Y split back into TMEM, B in smem
//
// P = Q[j, i] gives dL/dW_l += IDD P / (2 pi s^2) and dL/dIDD = <P, W> / (2 pi s^2);
// Q[j, i'] + Q[j', i] gives dL/dsigma = IDD <., W> / (2 pi s^2) (G' = dG/ds).  The
// Gaussian factors are regenerated per (layer, slice); nothing is stored.
//
// Work item = (slice z, chunk of <= C active layers): G^T for the slice is rounded and
// split into shared memory once per item.  dL/dW of a pair goes to its own (layer, slice)
// slot and the finalize kernel sums the slots of a layer in a fixed order (deterministic).
// One thread issues MMAs, tcgen05.commit signals mbarriers, every wait is bounded (2 s)
// and on expiry the CTA sets the error word, drains, frees TMEM and leaves.
// Grids of at most 128 x 128 voxels per slice; lattices up to 64 x 64 spots (48 in x
// for the TF32 modes, whose operands take twice the shared memory).
#include <algorithm>

#include "pbd_internal.cuh"
#include "tc_common.cuh"

namespace pbd {
namespace {
using namespace tcc;

constexpr int TNT = 256;
constexpr uint32_t kTmemCols = 512;   // A [0,256), Y [256,384), Q [384, 384 + 2 N1)

template <int MODE>
struct AdjOps {
    using P = Prec<MODE>;
    // TMEM columns per MMA k-step (8 tf32, or 16 bf16 packed two per column) and the
    // offset of the lo part of an A operand.
    static constexpr uint32_t kColsPerStep = 8;
    static constexpr uint32_t kLoOff = P::EB == 4 ? 128u : 64u;

    __device__ static void mma(uint32_t d, uint32_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
        if (P::EB == 4) tc::mma_tf32_ts(d, a, b, idesc, acc);
        else tc::mma_bf16_ts(d, a, b, idesc, acc);
    }
    // D = A (TMEM, K = 128) x B^T (smem, K-major, `rows` rows) with the 3 or 1 products.
    __device__ static void issue(uint32_t d, uint32_t a, uint8_t* const* b, uint32_t plane_b,
                                 uint32_t idesc) {
        uint32_t acc = 0;
        for (int st = 0; st < 128 / P::KSTEP; ++st) {
            const uint32_t ac = a + (uint32_t)st * kColsPerStep;
            const uint32_t ob = (uint32_t)st * 2u * plane_b;
            const uint64_t bh = tc::smem_desc(tc::smem_u32(b[0]) + ob, plane_b, 128);
            if (P::NPROD == 3) {
                const uint64_t bl = tc::smem_desc(tc::smem_u32(b[1]) + ob, plane_b, 128);
                mma(d, ac, bl, idesc, acc);          // small products first
                mma(d, ac + kLoOff, bh, idesc, 1u);
                acc = 1;
            }
            mma(d, ac, bh, idesc, acc);
            acc = 1;
        }
    }
};

// Round 16 (tf32) or 32 (bf16) values to hi / lo words for a TMEM store of 16 columns.
template <int MODE>
__device__ __forceinline__ void pack16(const float* v, uint32_t (&hi)[16], uint32_t (&lo)[16]) {
    using P = Prec<MODE>;
    if constexpr (P::EB == 4) {
#pragma unroll
        for (int q = 0; q < 16; ++q) {
            hi[q] = tc::to_tf32(v[q]);
            lo[q] = P::NPROD == 3 ? tc::to_tf32(v[q] - __uint_as_float(hi[q])) : 0u;
        }
    } else {
#pragma unroll
        for (int q = 0; q < 16; ++q) {
            const uint32_t ha = bf16_bits(v[2 * q]), hb = bf16_bits(v[2 * q + 1]);
            hi[q] = ha | (hb << 16);
            if (P::NPROD == 3) {
                const float ra = v[2 * q] - __uint_as_float(ha << 16);
                const float rb = v[2 * q + 1] - __uint_as_float(hb << 16);
                lo[q] = bf16_bits(ra) | (bf16_bits(rb) << 16);
            } else {
                lo[q] = 0u;
            }
        }
    }
}

__device__ __forceinline__ float block_sum256(float v, float* red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, ln = threadIdx.x & 31;
    __syncthreads();
    if (ln == 0) red[w] = v;
    __syncthreads();
    float s = 0.f;
    if (threadIdx.x < 32) {
        s = ln < TNT / 32 ? red[ln] : 0.f;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    }
    return s;   // valid in thread 0
}

template <int MODE>
__global__ void __launch_bounds__(TNT, 1)
adj_tc_kernel(const JobDev* __restrict__ jobs, const FwdItem* __restrict__ items, int total,
              int* counter, int* err, int N1) {
    using P = Prec<MODE>;
    using O = AdjOps<MODE>;
    constexpr int NARR = P::NPROD == 3 ? 2 : 1;
    constexpr int EPC = P::EPC;
    extern __shared__ __align__(1024) uint8_t smem[];
    __shared__ __align__(8) uint64_t bar[2];
    __shared__ uint32_t tmem_base_s;
    __shared__ int s_item;
    __shared__ float red[2][TNT / 32];

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int R2 = 2 * N1;
    const uint32_t gt_bytes = 128u * 128u * P::EB, b2_bytes = (uint32_t)R2 * 128u * P::EB;
    uint8_t* GT[2];
    uint8_t* B2[2];
    GT[0] = smem;
    GT[1] = smem + (NARR == 2 ? gt_bytes : 0);
    B2[0] = smem + NARR * gt_bytes;
    B2[1] = B2[0] + (NARR == 2 ? b2_bytes : 0);

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
    const uint32_t tA = tmem_base_s, tY = tmem_base_s + 256u, tQ = tmem_base_s + 384u;
    const uint32_t lane_base = (uint32_t)(32 * (warp & 3)) << 16;
    const uint32_t idesc1 = tc::instr_desc(128, 128, P::FMT);
    const uint32_t idesc2 = tc::instr_desc(128, R2, P::FMT);
    const uint32_t plane128 = 128u * 16u, planeR2 = (uint32_t)R2 * 16u;
    const int half = warp >> 2;
    const int m = 32 * (warp & 3) + lane;   // TMEM lane = row of A, Y, Q

    uint32_t ph1 = 0, ph2 = 0;
    bool pend1 = false, pend2 = false, failed = false;
    // the pair whose stage-2 result is still in TMEM
    int pl = -1;
    float pc = 0.f, pnrm = 0.f;

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
        const int z = it.z;
        const double cx = 0.5 * (double)(nsx - 1), cy = 0.5 * (double)(nsy - 1);

        // Q of the previous pair -> dL/dW slot, dL/dIDD, dL/dsigma
        auto drain = [&]() -> bool {
            const bool ok = wait_bar(&bar[1], ph2);
            if (ok) { ph2 ^= 1; pend2 = false; }
            if (__syncthreads_or(!ok)) return false;
            tc::fence_after_sync();
            const float* wl = J.w + (size_t)pl * nsy * nsx;
            float* slot = J.partial + ((size_t)pl * nz + z) * nsy * nsx;
            const int j = m & 63;
            const bool jrow = m < 64;
            float dcv = 0.f, dsv = 0.f;
            for (int c0 = 0; c0 < N1; c0 += 16) {
                uint32_t r[16];
                tc::tmem_ld16(tQ + lane_base + (uint32_t)(half * N1 + c0), r);
                tc::tmem_wait_ld();
                if (j < nsy && !(half == 1 && !jrow)) {
#pragma unroll
                    for (int q = 0; q < 16; ++q) {
                        const int i = c0 + q;
                        if (i < nsx) {
                            const float v = __uint_as_float(r[q]);
                            const float wv = wl[(size_t)j * nsx + i];
                            if (jrow && half == 0) {
                                slot[(size_t)j * nsx + i] = pc * pnrm * v;
                                dcv = fmaf(wv, v, dcv);
                            } else {
                                dsv = fmaf(wv, v, dsv);
                            }
                        }
                    }
                }
            }
            const float sdc = block_sum256(dcv, red[0]);
            const float sds = block_sum256(dsv, red[1]);
            if (tid == 0) {
                J.dc[(size_t)pl * nz + z] = pnrm * sdc;
                J.dsg[(size_t)pl * nz + z] = pc * pnrm * sds;
            }
            tc::fence_before_sync();
            __syncthreads();
            return true;
        };

        // ---- G^T of the slice: rows x, K = y (zero outside the grid) ----
        {
            const float* g = J.grad_dose + (size_t)z * ny * nx;
            for (int e = tid; e < 128 * (128 / EPC); e += TNT) {
                const int x = e & 127, gi = e >> 7;
                float v[EPC];
#pragma unroll
                for (int q = 0; q < EPC; ++q) {
                    const int y = gi * EPC + q;
                    v[q] = (y < ny && x < nx) ? g[(size_t)y * nx + x] : 0.f;
                }
                uint4 hi, lo;
                split_chunk<MODE>(v, hi, lo);
                const uint32_t off = (uint32_t)gi * plane128 + (uint32_t)x * 16u;
                *reinterpret_cast<uint4*>(GT[0] + off) = hi;
                if (NARR == 2) *reinterpret_cast<uint4*>(GT[1] + off) = lo;
            }
        }

        for (int l = it.lb; l < it.le && !failed; ++l) {
            const double c = J.idd[(size_t)l * nz + z];
            if (c == 0.0) continue;
            const double s = fmax(J.sigma[(size_t)l * nz + z], 1e-9);
            // d is formed in FP64 (voxel and spot coordinates of up to ~25 cm); d^2 and the
            // exponent in FP32 (relative rounding ~1e-7 of the exponent)
            const float a2 = (float)(kLog2e / (2.0 * s * s));
            const float inv_s3 = (float)(1.0 / (s * s * s)), inv_s = (float)(1.0 / s);

            if (pend2) {
                if (!drain()) { failed = true; break; }
            }
            // ---- A = [Gy | Gy']^T into TMEM: lane m, columns y ----
            {
                const int j = m & 63;
                const bool deriv = m >= 64;
                constexpr int VPS = P::EB == 4 ? 16 : 32;   // values per 16-column store
                const double ysj = J.sy0 + ((double)j - cy) * J.dsy;
                const float dyf = (float)J.dy;
                for (int y0 = half * 64; y0 < half * 64 + 64; y0 += VPS) {
                    // one FP64 difference per chunk, then FP32 steps of dy
                    const float base = (float)((J.oy + (double)y0 * J.dy) - ysj);
                    float v[VPS];
#pragma unroll
                    for (int q = 0; q < VPS; ++q) {
                        float val = 0.f;
                        if (j < nsy) {
                            const float df = fmaf((float)q, dyf, base), dd = df * df;
                            const float e = ex2_approx(-dd * a2);
                            val = deriv ? e * fmaf(dd, inv_s3, -inv_s) : e;
                        }
                        v[q] = val;
                    }
                    uint32_t hi[16], lo[16];
                    pack16<MODE>(v, hi, lo);
                    const uint32_t col = (uint32_t)(P::EB == 4 ? y0 : y0 / 2);
                    tc::tmem_st16(tA + lane_base + col, hi);
                    if (NARR == 2) tc::tmem_st16(tA + lane_base + O::kLoOff + col, lo);
                }
                tc::tmem_wait_st();
            }
            tc::fence_async_smem();   // G^T (first pair of the item) visible to the MMA
            tc::fence_before_sync();
            __syncthreads();
            if (tid == 0) {
                tc::fence_after_sync();
                O::issue(tY, tA, GT, plane128, idesc1);
                tc::commit(&bar[0]);
            }
            pend1 = true;

            // ---- B = [Gx | Gx'] in smem: rows n, K = x ----
            for (int e = tid; e < R2 * (128 / EPC); e += TNT) {
                const int n = e % R2, gi = e / R2;
                const int i = n < N1 ? n : n - N1;
                const bool deriv = n >= N1;
                const float base = (float)((J.ox + (double)(gi * EPC) * J.dx) -
                                           (J.sx0 + ((double)i - cx) * J.dsx));
                const float dxf = (float)J.dx;
                float v[EPC];
#pragma unroll
                for (int q = 0; q < EPC; ++q) {
                    float val = 0.f;
                    if (i < nsx) {
                        const float df = fmaf((float)q, dxf, base), dd = df * df;
                        const float g = ex2_approx(-dd * a2);
                        val = deriv ? g * fmaf(dd, inv_s3, -inv_s) : g;
                    }
                    v[q] = val;
                }
                uint4 hi, lo;
                split_chunk<MODE>(v, hi, lo);
                const uint32_t off = (uint32_t)gi * planeR2 + (uint32_t)n * 16u;
                *reinterpret_cast<uint4*>(B2[0] + off) = hi;
                if (NARR == 2) *reinterpret_cast<uint4*>(B2[1] + off) = lo;
            }

            // ---- Y (stage 1 result) -> split -> A region of TMEM ----
            {
                const bool ok = wait_bar(&bar[0], ph1);
                if (ok) { ph1 ^= 1; pend1 = false; }
                if (__syncthreads_or(!ok)) { failed = true; break; }
            }
            tc::fence_after_sync();
            {
                constexpr int VPS = P::EB == 4 ? 16 : 32;
                for (int x0 = half * 64; x0 < half * 64 + 64; x0 += VPS) {
                    float v[VPS];
                    {
                        uint32_t r[16];
                        tc::tmem_ld16(tY + lane_base + (uint32_t)x0, r);
                        tc::tmem_wait_ld();
#pragma unroll
                        for (int q = 0; q < 16; ++q) v[q] = __uint_as_float(r[q]);
                    }
                    if (VPS == 32) {
                        uint32_t r[16];
                        tc::tmem_ld16(tY + lane_base + (uint32_t)(x0 + 16), r);
                        tc::tmem_wait_ld();
#pragma unroll
                        for (int q = 0; q < 16; ++q) v[16 + (q & 15)] = __uint_as_float(r[q]);
                    }
                    uint32_t hi[16], lo[16];
                    pack16<MODE>(v, hi, lo);
                    const uint32_t col = (uint32_t)(P::EB == 4 ? x0 : x0 / 2);
                    tc::tmem_st16(tA + lane_base + col, hi);
                    if (NARR == 2) tc::tmem_st16(tA + lane_base + O::kLoOff + col, lo);
                }
                tc::tmem_wait_st();
            }
            tc::fence_async_smem();
            tc::fence_before_sync();
            __syncthreads();
            if (tid == 0) {
                tc::fence_after_sync();
                O::issue(tQ, tA, B2, planeR2, idesc2);
                tc::commit(&bar[1]);
            }
            pend2 = true;
            pl = l;
            pc = (float)c;
            pnrm = (float)(kInv2Pi / (s * s));
        }
        if (failed) break;
        if (pend2) {
            if (!drain()) { failed = true; break; }
        }
    }

    if (failed) {
        if (tid == 0) atomicExch(err, 1);
        if (pend1) (void)wait_bar(&bar[0], ph1);
        if (pend2) (void)wait_bar(&bar[1], ph2);
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    if (warp == 0) tc::tmem_dealloc(tmem_base_s, kTmemCols);
}

// dL/dW_l = sum over active slices of the (l, z) slots in a fixed order (deterministic);
// dL/dR_l in FP64; the loss total.  Grid (spot blocks of 128, layers, jobs): each block
// first compacts the layer's active slices into shared memory, then every thread sums its
// (j, i) entry over them with four independent accumulators (the loads of one slice are
// coalesced).
__global__ void adj_tc_finalize_kernel(const JobDev* __restrict__ jobs, int with_range,
                                       int finalize_loss, const int* __restrict__ err) {
    const JobDev& J = jobs[blockIdx.z];
    const int l = blockIdx.y;
    if (l >= J.nl) return;
    const int per = J.nsy * J.nsx;
    const bool bad = *err != 0 || (J.fwd_err != nullptr && *J.fwd_err != 0);
    const double* idd = J.idd + (size_t)l * J.nz;
    __shared__ int zl[1024];
    __shared__ int wcount[4];
    __shared__ int nact;
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    float a0 = 0.f, a1 = 0.f, a2 = 0.f, a3 = 0.f;
    for (int zc = 0; zc < J.nz; zc += 1024) {
        __syncthreads();
        if (threadIdx.x == 0) nact = 0;
        __syncthreads();
        // order-preserving compaction of the active slices, 128 at a time (4 warp ballots)
        for (int zb = zc; zb < min(J.nz, zc + 1024); zb += 128) {
            const int z = zb + threadIdx.x;
            const bool act = z < J.nz && z < zc + 1024 && idd[z] != 0.0;
            const unsigned bal = __ballot_sync(0xffffffffu, act);
            if (lane == 0) wcount[warp] = __popc(bal);
            __syncthreads();
            int off = nact;
            for (int w = 0; w < warp; ++w) off += wcount[w];
            if (act) zl[off + __popc(bal & ((1u << lane) - 1u))] = z;
            __syncthreads();
            if (threadIdx.x == 0) nact += wcount[0] + wcount[1] + wcount[2] + wcount[3];
            __syncthreads();
        }
        if (r < per) {
            const float* base = J.partial + (size_t)l * J.nz * per + r;
            int k = 0;
            for (; k + 4 <= nact; k += 4) {
                a0 += base[(size_t)zl[k] * per];
                a1 += base[(size_t)zl[k + 1] * per];
                a2 += base[(size_t)zl[k + 2] * per];
                a3 += base[(size_t)zl[k + 3] * per];
            }
            for (; k < nact; ++k) a0 += base[(size_t)zl[k] * per];
        }
    }
    if (r < per)
        J.grad_w[(size_t)l * per + r] = bad ? __int_as_float(0x7fc00000) : (a0 + a1) + (a2 + a3);
    if (with_range && blockIdx.x == 0) {
        __shared__ double redd[128];
        double acc = 0.0;
        for (int z = threadIdx.x; z < J.nz; z += blockDim.x) {
            const size_t o = (size_t)l * J.nz + z;
            if (idd[z] != 0.0)
                acc += (double)J.dc[o] * J.didd_dr[o] + (double)J.dsg[o] * J.dsig_dr[o];
        }
        redd[threadIdx.x] = acc;
        __syncthreads();
        for (int w = blockDim.x / 2; w > 0; w >>= 1) {
            if ((int)threadIdx.x < w) redd[threadIdx.x] += redd[threadIdx.x + w];
            __syncthreads();
        }
        if (threadIdx.x == 0) J.grad_range[l] = bad ? __int_as_float(0x7fc00000) : (float)redd[0];
    }
    if (finalize_loss && l == 0 && blockIdx.x == 0 && threadIdx.x == 0) {
        double s = 0.0;
        for (int b = 0; b < J.n_loss_part; ++b) s += J.loss_part[b];
        *J.loss = bad ? (double)__int_as_float(0x7fc00000) : s;
    }
}

template <int MODE>
size_t adj_smem_bytes(int N1) {
    using P = Prec<MODE>;
    const int narr = P::NPROD == 3 ? 2 : 1;
    return (size_t)narr * P::EB * (128u * 128u + 2u * (size_t)N1 * 128u);
}

template <int MODE>
int launch_mode(JobDev* jobs, FwdItem* items, int total, int* counter, int* err, int N1,
                cudaStream_t s) {
    static thread_local int max_dyn = 0;
    if (max_dyn == 0) {
        int dev = 0, optin = 0;
        cudaFuncAttributes fa;
        if (cudaGetDevice(&dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) !=
                cudaSuccess ||
            cudaFuncGetAttributes(&fa, adj_tc_kernel<MODE>) != cudaSuccess)
            return PBD_ERR_CUDA;
        const int avail = optin - (int)fa.sharedSizeBytes;
        if (avail <= 0 || cudaFuncSetAttribute(adj_tc_kernel<MODE>,
                                               cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               avail) != cudaSuccess)
            return PBD_ERR_NO_SMEM;
        max_dyn = avail;
    }
    // >= 116 KiB: one CTA, and its 512 TMEM columns, per SM
    const size_t smem = std::max<size_t>(adj_smem_bytes<MODE>(N1), 116u * 1024u);
    if (smem > (size_t)max_dyn) return PBD_ERR_NO_SMEM;
    const int grid = std::max(1, std::min(total, num_sms()));
    prof_mark(kProfAdj, 0, s);
    adj_tc_kernel<MODE><<<grid, TNT, smem, s>>>(jobs, items, total, counter, err, N1);
    PBD_LAUNCH_CHECK();
    prof_mark(kProfAdj, 1, s);
    return PBD_OK;
}

}  // namespace

int tc_adjoint_dims(int precision, const pbd_field* f, int* N1) {
    if (precision == PBD_PREC_FP32) return PBD_ERR_UNSUPPORTED;
    if (f->nx > kTile || f->ny > kTile || f->n_sy > 64) return PBD_ERR_UNSUPPORTED;
    *N1 = (f->n_sx + 15) / 16 * 16;
    const bool wide = precision == PBD_PREC_TF32X3 || precision == PBD_PREC_TF32;
    const int narr = (precision == PBD_PREC_TF32X3 || precision == PBD_PREC_BF16X3) ? 2 : 1;
    const size_t eb = wide ? 4 : 2;
    const size_t smem = (size_t)narr * eb * (128u * 128u + 2u * (size_t)(*N1) * 128u);
    if (*N1 > 64 || smem > 227u * 1024u - 2048u) return PBD_ERR_UNSUPPORTED;
    return PBD_OK;
}

int launch_adjoint_tc(int precision, JobDev* jobs_dev, const JobDev* jobs_host, int n_jobs,
                      FwdItem* items, int total_items, int* counter, int chunk, int with_range,
                      int finalize_loss, cudaStream_t s) {
    int N1 = 0;
    for (int j = 0; j < n_jobs; ++j) {
        pbd_field f{};
        f.nx = jobs_host[j].nx; f.ny = jobs_host[j].ny;
        f.n_sx = jobs_host[j].nsx; f.n_sy = jobs_host[j].nsy;
        int n1 = 0;
        PBD_TRY(tc_adjoint_dims(precision, &f, &n1));
        N1 = std::max(N1, n1);
    }
    PBD_TRY(cuda_rc(cudaMemsetAsync(counter, 0, 2 * sizeof(int), s)));
    PBD_TRY(launch_slice_schedule(jobs_dev, items, chunk, n_jobs, s));
    int rc = PBD_ERR_BAD_VALUE;
    switch (precision) {
        case PBD_PREC_TF32X3:
            rc = launch_mode<PBD_PREC_TF32X3>(jobs_dev, items, total_items, counter, counter + 1, N1, s);
            break;
        case PBD_PREC_TF32:
            rc = launch_mode<PBD_PREC_TF32>(jobs_dev, items, total_items, counter, counter + 1, N1, s);
            break;
        case PBD_PREC_BF16X3:
            rc = launch_mode<PBD_PREC_BF16X3>(jobs_dev, items, total_items, counter, counter + 1, N1, s);
            break;
        case PBD_PREC_BF16:
            rc = launch_mode<PBD_PREC_BF16>(jobs_dev, items, total_items, counter, counter + 1, N1, s);
            break;
        default:
            break;
    }
    PBD_TRY(rc);
    int max_l = 1, max_per = 1;
    for (int j = 0; j < n_jobs; ++j) {
        max_l = std::max(max_l, jobs_host[j].nl);
        max_per = std::max(max_per, jobs_host[j].nsy * jobs_host[j].nsx);
    }
    adj_tc_finalize_kernel<<<dim3((max_per + 127) / 128, max_l, n_jobs), 128, 0, s>>>(
        jobs_dev, with_range, finalize_loss, counter + 1);
    PBD_LAUNCH_CHECK();
    count_launch(3);
    return PBD_OK;
}

}  // namespace pbd
