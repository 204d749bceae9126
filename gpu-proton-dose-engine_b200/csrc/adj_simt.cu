// adj_simt.cu -- adjoint of the separable dose on the CUDA cores (FP32 FMA).
//
// With G_z = dL/dD[z] (ny x nx) and normalised Gaussians of width s = sigma_l(z):
//   P_l(z) = Gy^T G_z Gx                    (nsy x nsx)
//   dL/dW_l        = sum_z IDD_l(z) P_l(z)
//   dL/dIDD_l(z)   = <P_l(z), W_l>
//   dL/dsigma_l(z) = IDD_l(z) <Gy'^T G_z Gx + Gy^T G_z Gx', W_l>,  G' = dG/ds
// The reference has no adjoint; this is the transposed separable contraction of its
// forward (engines.py:191-197).  The Gaussian factors and their sigma-derivatives are
// regenerated per (layer, slice) in shared memory, never stored.
//
// Work item = (job, layer l, chunk of <= C active slices).  Per pair:
//   Y[m, x]  = sum_y A[y, m] G_z[y, x],  A = [Gy | Gy'] (m < 64: j, m >= 64: j')
//   P[j, i]  = sum_x Y[j, x] Gx[x, i]
//   Q[j, i]  = sum_x Y[j, x] Gx'[x, i] + Y[64+j, x] Gx[x, i]
// dL/dW accumulates in registers across the chunk and is written once per item; the
// finalize kernel sums the items of a layer in chunk order and forms dL/dR_l.
#include <algorithm>

#include "pbd_internal.cuh"

namespace pbd {
namespace {

constexpr int NT = 256;
constexpr int SA = kAdjMaxSpots;        // 64
constexpr int YS = kTile + 4;           // padded row of Y^T
constexpr size_t kAdjSmemBytes =
    (size_t)(kTile * kTile + kTile * 2 * SA + kTile * YS) * sizeof(float);   // 194 KiB

__device__ __forceinline__ float ex2_approx(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

constexpr int kActStage = 40 * 1024;

__global__ void adj_schedule_kernel(JobDev* jobs, AdjItem* items, int chunk) {
    const JobDev J = jobs[blockIdx.x];
    extern __shared__ unsigned char sact[];
    __shared__ int cnt[kMaxChunkCost + 1];
    __shared__ int cur[kMaxChunkCost + 1];
    __shared__ int total;
    for (int c = threadIdx.x; c <= kMaxChunkCost; c += blockDim.x) cnt[c] = 0;
    const bool staged = J.nl * J.nz <= kActStage;
    if (staged)
        for (int e = threadIdx.x; e < J.nl * J.nz; e += blockDim.x) sact[e] = J.idd[e] != 0.0;
    __syncthreads();
    auto active = [&](int l, int z) {
        return staged ? sact[l * J.nz + z] != 0 : J.idd[(size_t)l * J.nz + z] != 0.0;
    };
    for (int l = threadIdx.x; l < J.nl; l += blockDim.x) {
        int a = 0;
        for (int z = 0; z < J.nz; ++z) a += active(l, z);
        const int nch = (a + chunk - 1) / chunk;
        J.nchunks[l] = nch;
        for (int k = 0; k < nch; ++k) atomicAdd(&cnt[min(chunk, a - k * chunk)], 1);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        int pos = 0;
        for (int c = chunk; c >= 1; --c) { cur[c] = pos; pos += cnt[c]; }
        total = pos;
    }
    __syncthreads();
    for (int l = threadIdx.x; l < J.nl; l += blockDim.x) {
        int k = 0, in_chunk = 0, zb = 0, last = 0;
        for (int z = 0; z <= J.nz; ++z) {
            const bool act = z < J.nz && active(l, z);
            if (act) {
                if (in_chunk == 0) zb = z;
                ++in_chunk;
                last = z;
            }
            if ((act && in_chunk == chunk) || (z == J.nz && in_chunk > 0)) {
                const int p = atomicAdd(&cur[in_chunk], 1);
                AdjItem it;
                it.job = blockIdx.x; it.l = l; it.zb = zb; it.ze = last + 1; it.chunk = k;
                it.cost = in_chunk; it.pad0 = 0; it.pad1 = 0;
                items[J.item_base + p] = it;
                ++k;
                in_chunk = 0;
            }
        }
    }
    __syncthreads();
    for (int p = total + threadIdx.x; p < J.max_items; p += blockDim.x) {
        AdjItem it{};
        items[J.item_base + p] = it;
    }
}

__device__ __forceinline__ float block_sum(float v, float* red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, ln = threadIdx.x & 31;
    __syncthreads();
    if (ln == 0) red[w] = v;
    __syncthreads();
    float s = 0.f;
    if (threadIdx.x < 32) {
        s = ln < NT / 32 ? red[ln] : 0.f;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    }
    return s;   // valid in thread 0
}

__global__ void __launch_bounds__(NT, 1)
adj_simt_kernel(const JobDev* __restrict__ jobs, const AdjItem* __restrict__ items, int total,
                int* counter) {
    extern __shared__ float4 smem4[];
    float* Gs = reinterpret_cast<float*>(smem4);   // [128 y][128 x]
    float* AB = Gs + kTile * kTile;                 // [128 y][2*SA] then [128 x][2*SA]
    float* YT = AB + kTile * 2 * SA;                // [128 x][YS]
    __shared__ float red[2][NT / 32];
    __shared__ int s_item;
    const int tid = threadIdx.x, ty = tid >> 4, tx = tid & 15;

    for (;;) {
        if (tid == 0) s_item = atomicAdd(counter, 1);
        __syncthreads();
        const int it_idx = s_item;
        __syncthreads();
        if (it_idx >= total) break;
        const AdjItem it = items[it_idx];
        if (it.cost == 0) continue;
        const JobDev& J = jobs[it.job];
        const int nz = J.nz, nx = J.nx, ny = J.ny, nsx = J.nsx, nsy = J.nsy, l = it.l;
        const double cx = 0.5 * (double)(nsx - 1), cy = 0.5 * (double)(nsy - 1);
        const float* wl = J.w + (size_t)l * nsy * nsx;

        float wreg[4][4], dw[4][4];
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b) {
                const int j = ty * 4 + a, i = tx * 4 + b;
                wreg[a][b] = (j < nsy && i < nsx) ? wl[(size_t)j * nsx + i] : 0.f;
                dw[a][b] = 0.f;
            }

        for (int z = it.zb; z < it.ze; ++z) {
            const double c = J.idd[(size_t)l * nz + z];
            if (c == 0.0) continue;
            const double s = fmax(J.sigma[(size_t)l * nz + z], 1e-9);
            const double a2 = kLog2e / (2.0 * s * s);
            const double inv_s3 = 1.0 / (s * s * s), inv_s = 1.0 / s;
            float P[4][4], Q[4][4];
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int b = 0; b < 4; ++b) { P[a][b] = 0.f; Q[a][b] = 0.f; }

            for (int yt = 0; yt < J.nty; ++yt) {
                for (int xt = 0; xt < J.ntx; ++xt) {
                    const int y0 = yt * kTile, x0 = xt * kTile;
                    __syncthreads();
                    const float* gsrc = J.grad_dose + (size_t)z * ny * nx;
                    for (int e = tid; e < kTile * kTile; e += NT) {
                        const int yy = e >> 7, xx = e & (kTile - 1);
                        const int y = y0 + yy, x = x0 + xx;
                        Gs[e] = (y < ny && x < nx) ? gsrc[(size_t)y * nx + x] : 0.f;
                    }
                    for (int e = tid; e < kTile * 2 * SA; e += NT) {
                        const int yy = e / (2 * SA), m = e % (2 * SA);
                        const int j = m & (SA - 1);
                        float v = 0.f;
                        if (j < nsy) {
                            const double d = (J.oy + (double)(y0 + yy) * J.dy) -
                                             (J.sy0 + ((double)j - cy) * J.dsy);
                            const float g = ex2_approx((float)(-(d * d) * a2));
                            v = m < SA ? g : g * (float)(d * d * inv_s3 - inv_s);
                        }
                        AB[e] = v;
                    }
                    __syncthreads();
                    // Y[m, x] = sum_y A[y, m] G[y, x]; thread rows m = ty*8+a, cols x = tx+16b
                    float acc[8][8];
#pragma unroll
                    for (int a = 0; a < 8; ++a)
#pragma unroll
                        for (int b = 0; b < 8; ++b) acc[a][b] = 0.f;
                    for (int k = 0; k < kTile; ++k) {
                        const float4 q0 = *reinterpret_cast<const float4*>(&AB[k * 2 * SA + ty * 8]);
                        const float4 q1 =
                            *reinterpret_cast<const float4*>(&AB[k * 2 * SA + ty * 8 + 4]);
                        const float qa[8] = {q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, q1.z, q1.w};
                        float gb[8];
#pragma unroll
                        for (int b = 0; b < 8; ++b) gb[b] = Gs[k * kTile + tx + 16 * b];
#pragma unroll
                        for (int a = 0; a < 8; ++a)
#pragma unroll
                            for (int b = 0; b < 8; ++b) acc[a][b] = fmaf(qa[a], gb[b], acc[a][b]);
                    }
#pragma unroll
                    for (int b = 0; b < 8; ++b) {
                        float* row = YT + (tx + 16 * b) * YS + ty * 8;
                        *reinterpret_cast<float4*>(row) =
                            make_float4(acc[0][b], acc[1][b], acc[2][b], acc[3][b]);
                        *reinterpret_cast<float4*>(row + 4) =
                            make_float4(acc[4][b], acc[5][b], acc[6][b], acc[7][b]);
                    }
                    __syncthreads();
                    // B = [Gx | Gx'] over x rows
                    for (int e = tid; e < kTile * 2 * SA; e += NT) {
                        const int xx = e / (2 * SA), m = e % (2 * SA);
                        const int i = m & (SA - 1);
                        float v = 0.f;
                        if (i < nsx) {
                            const double d = (J.ox + (double)(x0 + xx) * J.dx) -
                                             (J.sx0 + ((double)i - cx) * J.dsx);
                            const float g = ex2_approx((float)(-(d * d) * a2));
                            v = m < SA ? g : g * (float)(d * d * inv_s3 - inv_s);
                        }
                        AB[e] = v;
                    }
                    __syncthreads();
                    // P[j,i] += sum_x Y[j,x] Gx[x,i];  Q[j,i] += Y[j,x] Gx'[x,i] + Y'[j,x] Gx[x,i]
                    for (int k = 0; k < kTile; ++k) {
                        const float4 y = *reinterpret_cast<const float4*>(&YT[k * YS + ty * 4]);
                        const float4 yd = *reinterpret_cast<const float4*>(&YT[k * YS + SA + ty * 4]);
                        const float4 g = *reinterpret_cast<const float4*>(&AB[k * 2 * SA + tx * 4]);
                        const float4 gd =
                            *reinterpret_cast<const float4*>(&AB[k * 2 * SA + SA + tx * 4]);
                        const float ya[4] = {y.x, y.y, y.z, y.w};
                        const float yda[4] = {yd.x, yd.y, yd.z, yd.w};
                        const float gb[4] = {g.x, g.y, g.z, g.w};
                        const float gdb[4] = {gd.x, gd.y, gd.z, gd.w};
#pragma unroll
                        for (int a = 0; a < 4; ++a)
#pragma unroll
                            for (int b = 0; b < 4; ++b) {
                                P[a][b] = fmaf(ya[a], gb[b], P[a][b]);
                                Q[a][b] = fmaf(ya[a], gdb[b], fmaf(yda[a], gb[b], Q[a][b]));
                            }
                    }
                }
            }
            // normalisation of both Gaussians: 1 / (2 pi s^2)
            const float nrm = (float)(kInv2Pi / (s * s));
            const float cf = (float)c;
            float pw = 0.f, qw = 0.f;
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int b = 0; b < 4; ++b) {
                    const float p = P[a][b] * nrm;
                    dw[a][b] = fmaf(cf, p, dw[a][b]);
                    pw = fmaf(p, wreg[a][b], pw);
                    qw = fmaf(Q[a][b] * nrm, wreg[a][b], qw);
                }
            const float dcv = block_sum(pw, red[0]);
            const float dsv = block_sum(qw, red[1]);
            if (tid == 0) {
                J.dc[(size_t)l * nz + z] = dcv;
                J.dsg[(size_t)l * nz + z] = cf * dsv;
            }
        }
        float* out = J.partial + ((size_t)l * J.max_chunks + it.chunk) * nsy * nsx;
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b) {
                const int j = ty * 4 + a, i = tx * 4 + b;
                if (j < nsy && i < nsx) out[(size_t)j * nsx + i] = dw[a][b];
            }
    }
}

// dL/dW = sum of the items of each layer (chunk order); dL/dR_l in FP64; final loss sum.
__global__ void adj_finalize_kernel(const JobDev* __restrict__ jobs, int with_range,
                                    int finalize_loss) {
    const JobDev& J = jobs[blockIdx.y];
    const int per_layer = J.nsy * J.nsx;
    const size_t n = (size_t)J.nl * per_layer;
    // a timed-out wait of a tensor-core forward leaves dL/dD invalid: poison the results
    const bool bad = J.fwd_err != nullptr && *J.fwd_err != 0;
    const float nan = __int_as_float(0x7fc00000);
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n;
         e += (size_t)gridDim.x * blockDim.x) {
        const int l = (int)(e / per_layer), r = (int)(e % per_layer);
        const int nch = J.nchunks[l];
        float s = bad ? nan : 0.f;
        for (int k = 0; k < nch; ++k)
            s += J.partial[((size_t)l * J.max_chunks + k) * per_layer + r];
        J.grad_w[e] = s;
    }
    if (blockIdx.x == 0) {
        if (with_range) {
            for (int l = threadIdx.x; l < J.nl; l += blockDim.x) {
                double acc = 0.0;
                for (int z = 0; z < J.nz; ++z) {
                    const size_t o = (size_t)l * J.nz + z;
                    if (J.idd[o] == 0.0) continue;
                    acc += (double)J.dc[o] * J.didd_dr[o] + (double)J.dsg[o] * J.dsig_dr[o];
                }
                J.grad_range[l] = bad ? nan : (float)acc;
            }
        }
        if (finalize_loss && threadIdx.x == 0) {
            double s = 0.0;
            for (int b = 0; b < J.n_loss_part; ++b) s += J.loss_part[b];
            *J.loss = bad ? (double)nan : s;
        }
    }
}

}  // namespace

int adj_chunk_depths(const pbd_field* f) {
    (void)f;
    return 4;
}

int adj_plan_sizes(const pbd_field* f, int chunk, size_t* partial_elems, int* items) {
    const int max_chunks = (f->nz + chunk - 1) / chunk;
    *partial_elems = (size_t)f->n_layers * max_chunks * f->n_sy * f->n_sx;
    *items = f->n_layers * max_chunks;
    return PBD_OK;
}

int launch_adjoint(JobDev* jobs_dev, const JobDev* jobs_host, int n_jobs, AdjItem* items,
                   int total_items, int* counter, int chunk, int with_range, int finalize_loss,
                   cudaStream_t s) {
    int set = 0;
    PBD_TRY(smem_optin((const void*)adj_simt_kernel, (int)kAdjSmemBytes, 0, &set));
    PBD_TRY(cuda_rc(cudaMemsetAsync(counter, 0, sizeof(int), s)));
    adj_schedule_kernel<<<n_jobs, 256, kActStage, s>>>(jobs_dev, items, chunk);
    PBD_LAUNCH_CHECK();
    const int grid = max(1, min(total_items, num_sms()));
    prof_mark(kProfAdj, 0, s);
    adj_simt_kernel<<<grid, NT, kAdjSmemBytes, s>>>(jobs_dev, items, total_items, counter);
    PBD_LAUNCH_CHECK();
    prof_mark(kProfAdj, 1, s);
    int blocks = 1;
    for (int j = 0; j < n_jobs; ++j) {
        const size_t n = (size_t)jobs_host[j].nl * jobs_host[j].nsy * jobs_host[j].nsx;
        blocks = max(blocks, (int)std::min<size_t>((n + 255) / 256, 1024));
    }
    adj_finalize_kernel<<<dim3(blocks, n_jobs), 256, 0, s>>>(jobs_dev, with_range, finalize_loss);
    PBD_LAUNCH_CHECK();
    count_launch(3);
    return PBD_OK;
}

}  // namespace pbd
