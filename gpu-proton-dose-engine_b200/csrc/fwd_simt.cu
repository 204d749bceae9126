// fwd_simt.cu -- forward dose on the CUDA cores (FP32 FMA), persistent and load-balanced.
//
// D[z,y,x] = sum_l IDD_l(z) sum_j Gy[y,j] sum_i W_l[j,i] Gx[x,i]   (engines.py:191-197)
//
// Work item = (job, depth slice z, 128x128 lateral tile, chunk of <= C active layers).
// For each active layer the CTA generates the Gaussian factors of that (layer, slice)
// in shared memory (never stored in HBM), contracts
//     U[j, x] = sum_i W'[j,i] Gx[x,i]      (W' = W * IDD / (2 pi sigma^2))
//     D[y, x] += sum_j Gy[y,j] U[j,x]
// with D held in registers across the chunk's layers, and writes the chunk's partial
// slice once.  The finalize kernel sums the (at most ceil(L/C)) partials of a slice in
// chunk order -- deterministic -- and fuses the masked quadratic loss and its gradient.
// Items are sorted by cost (longest first) by a device-side scheduler, and a
// persistent grid pulls them from an atomic counter: the deep slices that see few
// layers no longer bound the launch.
#include <algorithm>

#include "pbd_internal.cuh"

namespace pbd {
namespace {

constexpr int NT = 256;
constexpr int SC = kSpotChunk;                      // 64 spots per chunk
constexpr int kFwdSmemFloats = 3 * SC * kTile + SC * SC;
constexpr size_t kFwdSmemBytes = kFwdSmemFloats * sizeof(float);   // 112 KiB

__device__ __forceinline__ float ex2_approx(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// Scheduler: one CTA per job.  Items are written to the job's segment of the flat
// item array, bucket-sorted by cost (descending); unused slots get cost 0.
// Activity flags (IDD != 0) of a job staged in shared memory when they fit.
constexpr int kActStage = 40 * 1024;

__device__ __forceinline__ bool active(const JobDev& J, const unsigned char* sact, bool staged,
                                       int l, int z) {
    return staged ? sact[l * J.nz + z] != 0 : J.idd[(size_t)l * J.nz + z] != 0.0;
}

__device__ __forceinline__ bool stage_activity(const JobDev& J, unsigned char* sact) {
    const bool staged = J.nl * J.nz <= kActStage;
    if (staged)
        for (int e = threadIdx.x; e < J.nl * J.nz; e += blockDim.x) sact[e] = J.idd[e] != 0.0;
    __syncthreads();
    return staged;
}

__global__ void fwd_schedule_kernel(JobDev* jobs, FwdItem* items, int chunk) {
    const JobDev J = jobs[blockIdx.x];
    extern __shared__ unsigned char sact[];
    __shared__ int cnt[kMaxChunkCost + 1];
    __shared__ int cur[kMaxChunkCost + 1];
    __shared__ int total;
    const int ntiles = J.ntx * J.nty;
    for (int c = threadIdx.x; c <= kMaxChunkCost; c += blockDim.x) cnt[c] = 0;
    const bool staged = stage_activity(J, sact);
    for (int z = threadIdx.x; z < J.nz; z += blockDim.x) {
        int a = 0;
        for (int l = 0; l < J.nl; ++l) a += active(J, sact, staged, l, z);
        const int nch = (a + chunk - 1) / chunk;
        J.nchunks[z] = nch;
        for (int k = 0; k < nch; ++k) atomicAdd(&cnt[min(chunk, a - k * chunk)], ntiles);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        int pos = 0;
        for (int c = chunk; c >= 1; --c) { cur[c] = pos; pos += cnt[c]; }
        total = pos;
    }
    __syncthreads();
    for (int z = threadIdx.x; z < J.nz; z += blockDim.x) {
        int k = 0, in_chunk = 0, lb = 0, last = 0;
        for (int l = 0; l <= J.nl; ++l) {
            const bool act = l < J.nl && active(J, sact, staged, l, z);
            if (act) {
                if (in_chunk == 0) lb = l;
                ++in_chunk;
                last = l;
            }
            if ((act && in_chunk == chunk) || (l == J.nl && in_chunk > 0)) {
                for (int t = 0; t < ntiles; ++t) {
                    const int p = atomicAdd(&cur[in_chunk], 1);
                    FwdItem it;
                    it.job = blockIdx.x; it.z = z; it.ty = t / J.ntx; it.tx = t % J.ntx;
                    it.lb = lb; it.le = last + 1; it.chunk = k; it.cost = in_chunk;
                    items[J.item_base + p] = it;
                }
                ++k;
                in_chunk = 0;
            }
        }
    }
    __syncthreads();
    for (int p = total + threadIdx.x; p < J.max_items; p += blockDim.x) {
        FwdItem it{};
        items[J.item_base + p] = it;
    }
}

__device__ __forceinline__ int xcol(int tx, int b) { return tx * 4 + (b & 3) + ((b >> 2) << 6); }

__global__ void __launch_bounds__(NT, 2)
fwd_simt_kernel(const JobDev* __restrict__ jobs, const FwdItem* __restrict__ items, int total,
                int* counter) {
    extern __shared__ float4 smem4[];
    float* GxT = reinterpret_cast<float*>(smem4);   // [SC i][128 x]
    float* GyT = GxT + SC * kTile;                   // [SC j][128 y]
    float* U = GyT + SC * kTile;                     // [SC j][128 x]
    float* WT = U + SC * kTile;                      // [SC i][SC j]
    __shared__ int s_item;
    const int tid = threadIdx.x, ty = tid >> 4, tx = tid & 15;

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

        float dacc[8][8];
#pragma unroll
        for (int a = 0; a < 8; ++a)
#pragma unroll
            for (int b = 0; b < 8; ++b) dacc[a][b] = 0.f;

        for (int l = it.lb; l < it.le; ++l) {
            const double c = J.idd[(size_t)l * nz + z];
            if (c == 0.0) continue;
            const double s = fmax(J.sigma[(size_t)l * nz + z], 1e-9);
            const double a2 = kLog2e / (2.0 * s * s);
            const float nrm = (float)(c * kInv2Pi / (s * s));
            const float* wl = J.w + (size_t)l * nsy * nsx;

            for (int j0 = 0; j0 < nsy; j0 += SC) {
                const int nj = min(SC, nsy - j0);
                float uacc[4][8];
#pragma unroll
                for (int a = 0; a < 4; ++a)
#pragma unroll
                    for (int b = 0; b < 8; ++b) uacc[a][b] = 0.f;

                for (int i0 = 0; i0 < nsx; i0 += SC) {
                    const int ni = min(SC, nsx - i0);
                    __syncthreads();
                    for (int e = tid; e < ni * kTile; e += NT) {
                        const int ii = e >> 7, xx = e & (kTile - 1);
                        const double d = (J.ox + (double)(x0 + xx) * J.dx) -
                                         (J.sx0 + ((double)(i0 + ii) - cx) * J.dsx);
                        GxT[e] = ex2_approx((float)(-(d * d) * a2));
                    }
                    for (int e = tid; e < ni * SC; e += NT) {
                        const int ii = e / SC, jj = e % SC;
                        WT[e] = jj < nj ? nrm * wl[(size_t)(j0 + jj) * nsx + i0 + ii] : 0.f;
                    }
                    if (i0 == 0) {
                        for (int e = tid; e < nj * kTile; e += NT) {
                            const int jj = e >> 7, yy = e & (kTile - 1);
                            const double d = (J.oy + (double)(y0 + yy) * J.dy) -
                                             (J.sy0 + ((double)(j0 + jj) - cy) * J.dsy);
                            GyT[e] = ex2_approx((float)(-(d * d) * a2));
                        }
                    }
                    __syncthreads();
                    // stage 1: U[j, x] += sum_i W'[j,i] Gx[x,i]
                    for (int ii = 0; ii < ni; ++ii) {
                        const float4 wv = *reinterpret_cast<const float4*>(&WT[ii * SC + ty * 4]);
                        const float4 g0 = *reinterpret_cast<const float4*>(&GxT[ii * kTile + tx * 4]);
                        const float4 g1 =
                            *reinterpret_cast<const float4*>(&GxT[ii * kTile + 64 + tx * 4]);
                        const float wa[4] = {wv.x, wv.y, wv.z, wv.w};
                        const float gb[8] = {g0.x, g0.y, g0.z, g0.w, g1.x, g1.y, g1.z, g1.w};
#pragma unroll
                        for (int a = 0; a < 4; ++a)
#pragma unroll
                            for (int b = 0; b < 8; ++b) uacc[a][b] = fmaf(wa[a], gb[b], uacc[a][b]);
                    }
                }
                // U rows j = ty*4 + a
#pragma unroll
                for (int a = 0; a < 4; ++a) {
                    float* row = U + (ty * 4 + a) * kTile;
                    *reinterpret_cast<float4*>(&row[tx * 4]) =
                        make_float4(uacc[a][0], uacc[a][1], uacc[a][2], uacc[a][3]);
                    *reinterpret_cast<float4*>(&row[64 + tx * 4]) =
                        make_float4(uacc[a][4], uacc[a][5], uacc[a][6], uacc[a][7]);
                }
                __syncthreads();
                // stage 2: D[y, x] += sum_j Gy[y,j] U[j,x]
                for (int jj = 0; jj < nj; ++jj) {
                    const float4 q0 = *reinterpret_cast<const float4*>(&GyT[jj * kTile + ty * 8]);
                    const float4 q1 = *reinterpret_cast<const float4*>(&GyT[jj * kTile + ty * 8 + 4]);
                    const float4 u0 = *reinterpret_cast<const float4*>(&U[jj * kTile + tx * 4]);
                    const float4 u1 = *reinterpret_cast<const float4*>(&U[jj * kTile + 64 + tx * 4]);
                    const float ga[8] = {q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, q1.z, q1.w};
                    const float ub[8] = {u0.x, u0.y, u0.z, u0.w, u1.x, u1.y, u1.z, u1.w};
#pragma unroll
                    for (int a = 0; a < 8; ++a)
#pragma unroll
                        for (int b = 0; b < 8; ++b) dacc[a][b] = fmaf(ga[a], ub[b], dacc[a][b]);
                }
            }
        }
        // partial slice of this chunk
        const size_t n3 = (size_t)nz * ny * nx;
        float* out = J.partial + (size_t)it.chunk * n3 + (size_t)z * ny * nx;
#pragma unroll
        for (int a = 0; a < 8; ++a) {
            const int y = y0 + ty * 8 + a;
            if (y >= ny) continue;
#pragma unroll
            for (int b = 0; b < 8; ++b) {
                const int x = x0 + xcol(tx, b);
                if (x < nx) out[(size_t)y * nx + x] = dacc[a][b];
            }
        }
    }
}

// Sum of the chunk partials (chunk order), dose out, optional loss + dL/dD.
__global__ void fwd_finalize_kernel(const JobDev* __restrict__ jobs, int with_loss,
                                    const int* __restrict__ err) {
    const JobDev& J = jobs[blockIdx.y];
    const size_t plane = (size_t)J.nx * J.ny;
    const size_t n = plane * J.nz;
    const bool bad = *err != 0;   // a main-kernel wait timed out: make the result NaN
    double lsum = 0.0;
    for (size_t v = (size_t)blockIdx.x * blockDim.x + threadIdx.x; v < n;
         v += (size_t)gridDim.x * blockDim.x) {
        const int z = (int)(v / plane);
        const int nch = J.nchunks[z];
        float s = bad ? __int_as_float(0x7fc00000) : 0.f;
        for (int k = 0; k < nch; ++k) s += J.partial[(size_t)k * n + v];
        J.dose[v] = s;
        if (with_loss) {
            const float r = s - J.presc[v];
            const float m = J.mask[v];
            J.grad_dose[v] = 2.f * m * r;
            lsum += (double)m * (double)r * (double)r;
        }
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

}  // namespace

int launch_slice_schedule(JobDev* jobs_dev, FwdItem* items, int chunk, int n_jobs,
                          cudaStream_t s) {
    fwd_schedule_kernel<<<n_jobs, 256, kActStage, s>>>(jobs_dev, items, chunk);
    PBD_LAUNCH_CHECK();
    return PBD_OK;
}

int fwd_chunk_layers(const pbd_field* f, int precision) {
    // FP32: ~4 layers per item keeps items small next to the ~2 CTAs per SM.  Tensor cores:
    // the pipeline runs across unit boundaries, so larger units only save partial slices
    // (24 measured best, with 4-layer adjoint units, on the 128^3 / 41 x 41 x 40 field;
    // the autotuner refines it per geometry).
    // The split-FP16 forward: 20.  The largest unit bounds the balance (a slice with exactly C
    // active layers is one unit, claimed after the shallow slices), and 20 is just above the
    // clinical field's mean load of 18.4 steps per SM (measured 83.6 us against 90.2 at 24).
    (void)f;
    if (precision == PBD_PREC_FP16X3) return 20;
    return precision == PBD_PREC_FP32 ? 4 : 24;
}

int fwd_plan_sizes(const pbd_field* f, int chunk, size_t* partial_elems, int* items) {
    const int ntx = (f->nx + kTile - 1) / kTile, nty = (f->ny + kTile - 1) / kTile;
    const int max_chunks = (f->n_layers + chunk - 1) / chunk;
    *partial_elems = (size_t)max_chunks * f->nz * f->ny * f->nx;
    const long long it = (long long)f->nz * max_chunks * ntx * nty;
    if (it > (1LL << 30)) return PBD_ERR_UNSUPPORTED;
    *items = (int)it;
    return PBD_OK;
}

int launch_forward(JobDev* jobs_dev, const JobDev* jobs_host, int n_jobs, FwdItem* items,
                   int total_items, int* counter, size_t n_counter_ints, int* err, int chunk,
                   int with_loss, int precision, int poison, void* pack, size_t pack_bytes,
                   cudaStream_t s, const JobPair* inst, JobDev* inst_dst, int* inst_status) {
    const bool tc16 = precision == PBD_PREC_FP16X3 && jobs_host[0].layer_stride == 0;
    if (inst && !tc16) return PBD_ERR_UNSUPPORTED;   // only the split-FP16 pack installs views
    if (precision != PBD_PREC_FP32) {
        // the split-FP16 path clears its unit counter in its pack kernel (no memset node between
        // the job install and the dose kernels) and may install the job views there too
        if (tc16)
            return launch_forward_tc16(jobs_dev, jobs_host, n_jobs, counter, err, chunk,
                                       with_loss, poison, pack, pack_bytes, s, inst, inst_dst,
                                       inst_status);
        PBD_TRY(cuda_rc(cudaMemsetAsync(counter, 0, n_counter_ints * sizeof(int), s)));
        return launch_forward_tc(precision, jobs_dev, jobs_host, n_jobs, counter, err, chunk,
                                 with_loss, poison, s);
    }
    int set = 0;
    PBD_TRY(smem_optin((const void*)fwd_simt_kernel, (int)kFwdSmemBytes, 0, &set));
    PBD_TRY(cuda_rc(cudaMemsetAsync(counter, 0, sizeof(int), s)));
    fwd_schedule_kernel<<<n_jobs, 256, kActStage, s>>>(jobs_dev, items, chunk);
    PBD_LAUNCH_CHECK();
    {
        const int grid = max(1, min(total_items, 2 * num_sms()));
        prof_mark(kProfFwd, 0, s);
        fwd_simt_kernel<<<grid, NT, kFwdSmemBytes, s>>>(jobs_dev, items, total_items, counter);
        PBD_LAUNCH_CHECK();
        prof_mark(kProfFwd, 1, s);
    }
    int max_blocks = 1;
    for (int j = 0; j < n_jobs; ++j) {
        const size_t n = (size_t)jobs_host[j].nx * jobs_host[j].ny * jobs_host[j].nz;
        max_blocks = max(max_blocks, (int)std::min<size_t>((n + 255) / 256, 4096));
    }
    const int fin_blocks = with_loss ? kLossBlocks : max_blocks;
    fwd_finalize_kernel<<<dim3(fin_blocks, n_jobs), 256, 0, s>>>(jobs_dev, with_loss, err);
    PBD_LAUNCH_CHECK();
    count_launch(3);
    return PBD_OK;
}

}  // namespace pbd
