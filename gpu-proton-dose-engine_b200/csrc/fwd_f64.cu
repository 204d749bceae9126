// fwd_f64.cu -- forward dose in FP64 on the CUDA cores: the float64 form of the reference's
// engine on CUDA (engines.torch_separable with dtype=torch.float64, engines.py:223-224,
// 230-274), for callers that need the dose to ~1e-15 rather than ~1e-7.
//
//   D[z,y,x] = sum_l IDD_l(z) / (2 pi s^2) sum_j Gy[y,j] sum_i W_l[j,i] Gx[x,i]
//   Gx[x,i] = exp(-(x_v - xs_i)^2 / (2 s^2)),  s = max(sigma_l(z), 1e-9)
//
// One block per (64 x 64 lateral tile, depth slice), over every layer of the slice: the dose
// tile is summed in registers (layer order, then the spot chunks in order) and written once,
// so no scratch memory, no second pass and a deterministic result.  Per active layer and
// chunk of 32 spots the block generates Gx, Gy (exp in FP64, distances from FP64 differences)
// and W' = W IDD / (2 pi s^2) in shared memory, forms U[j, x] = sum_i W'[j,i] Gx[x,i] and
// adds D[y, x] += sum_j Gy[y,j] U[j,x].  256 threads: 2 x 4 U entries and 4 x 4 dose voxels
// each.
#include <math.h>

#include "pbd_internal.cuh"

namespace pbd {
namespace {

constexpr int kT = 64;        // tile edge (voxels)
constexpr int kSC = 32;       // spots per chunk
constexpr int kThreads = 256;
constexpr int kSmemDoubles = 3 * kSC * kT + kSC * kSC;
constexpr int kSmemBytes = kSmemDoubles * (int)sizeof(double);   // 56 KiB

__global__ void __launch_bounds__(kThreads) fwd_f64_kernel(pbd_field f, const double* __restrict__ w,
                                                           const double* __restrict__ idd,
                                                           const double* __restrict__ sigma,
                                                           double* __restrict__ dose) {
    extern __shared__ double sm[];
    double* GxT = sm;                  // [i][x]
    double* GyT = GxT + kSC * kT;      // [j][y]
    double* U = GyT + kSC * kT;        // [j][x]
    double* WT = U + kSC * kT;         // [i][j]
    const int tid = threadIdx.x, tr = tid >> 4, tc = tid & 15;
    const int x0 = blockIdx.x * kT, y0 = blockIdx.y * kT, z = blockIdx.z;
    const int nz = f.nz, nsx = f.n_sx, nsy = f.n_sy;
    const double cx = 0.5 * (double)(nsx - 1), cy = 0.5 * (double)(nsy - 1);

    double dacc[4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) dacc[a][b] = 0.0;

    for (int l = 0; l < f.n_layers; ++l) {
        const double c = idd[(size_t)l * nz + z];
        if (c == 0.0) continue;
        const double s = fmax(sigma[(size_t)l * nz + z], 1e-9);
        const double k2 = 1.0 / (2.0 * s * s);
        const double nrm = c * kInv2Pi / (s * s);
        const double* wl = w + (size_t)l * nsy * nsx;
        for (int j0 = 0; j0 < nsy; j0 += kSC) {
            const int nj = min(kSC, nsy - j0);
            double uacc[2][4];
#pragma unroll
            for (int a = 0; a < 2; ++a)
#pragma unroll
                for (int b = 0; b < 4; ++b) uacc[a][b] = 0.0;
            for (int i0 = 0; i0 < nsx; i0 += kSC) {
                const int ni = min(kSC, nsx - i0);
                __syncthreads();
                for (int e = tid; e < ni * kT; e += kThreads) {
                    const int ii = e / kT, xx = e % kT;
                    const double d = (f.ox + (double)(x0 + xx) * f.dx) -
                                     (f.x0 + ((double)(i0 + ii) - cx) * f.dx_spot);
                    GxT[e] = exp(-(d * d) * k2);
                }
                for (int e = tid; e < ni * kSC; e += kThreads) {
                    const int ii = e / kSC, jj = e % kSC;
                    WT[e] = jj < nj ? nrm * wl[(size_t)(j0 + jj) * nsx + i0 + ii] : 0.0;
                }
                if (i0 == 0) {
                    for (int e = tid; e < nj * kT; e += kThreads) {
                        const int jj = e / kT, yy = e % kT;
                        const double d = (f.oy + (double)(y0 + yy) * f.dy) -
                                         (f.y0 + ((double)(j0 + jj) - cy) * f.dy_spot);
                        GyT[e] = exp(-(d * d) * k2);
                    }
                }
                __syncthreads();
                // U[j, x] += sum_i W'[j,i] Gx[x,i]: rows j = 2 tr + a, columns x = 4 tc + b
                for (int ii = 0; ii < ni; ++ii) {
                    const double2 wv = *reinterpret_cast<const double2*>(&WT[ii * kSC + 2 * tr]);
                    const double4 g = *reinterpret_cast<const double4*>(&GxT[ii * kT + 4 * tc]);
                    const double wa[2] = {wv.x, wv.y};
                    const double gb[4] = {g.x, g.y, g.z, g.w};
#pragma unroll
                    for (int a = 0; a < 2; ++a)
#pragma unroll
                        for (int b = 0; b < 4; ++b) uacc[a][b] = fma(wa[a], gb[b], uacc[a][b]);
                }
            }
#pragma unroll
            for (int a = 0; a < 2; ++a)
                *reinterpret_cast<double4*>(&U[(2 * tr + a) * kT + 4 * tc]) =
                    make_double4(uacc[a][0], uacc[a][1], uacc[a][2], uacc[a][3]);
            __syncthreads();
            // D[y, x] += sum_j Gy[y,j] U[j,x]: rows y = 4 tr + a, columns x = 4 tc + b
            for (int jj = 0; jj < nj; ++jj) {
                const double4 q = *reinterpret_cast<const double4*>(&GyT[jj * kT + 4 * tr]);
                const double4 u = *reinterpret_cast<const double4*>(&U[jj * kT + 4 * tc]);
                const double ga[4] = {q.x, q.y, q.z, q.w};
                const double ub[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
                for (int a = 0; a < 4; ++a)
#pragma unroll
                    for (int b = 0; b < 4; ++b) dacc[a][b] = fma(ga[a], ub[b], dacc[a][b]);
            }
        }
    }
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        const int y = y0 + 4 * tr + a;
        if (y >= f.ny) continue;
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            const int x = x0 + 4 * tc + b;
            if (x < f.nx) dose[((size_t)z * f.ny + y) * f.nx + x] = dacc[a][b];
        }
    }
}

}  // namespace

int launch_forward_f64(const pbd_field* f, const double* w, const double* idd,
                       const double* sigma, double* dose, cudaStream_t s) {
    if (f->nz > 65535) return PBD_ERR_UNSUPPORTED;
    int set = 0;
    PBD_TRY(smem_optin((const void*)fwd_f64_kernel, kSmemBytes, 0, &set));
    const dim3 grid((f->nx + kT - 1) / kT, (f->ny + kT - 1) / kT, f->nz);
    prof_mark(kProfFwd, 0, s);
    fwd_f64_kernel<<<grid, kThreads, kSmemBytes, s>>>(*f, w, idd, sigma, dose);
    PBD_LAUNCH_CHECK();
    prof_mark(kProfFwd, 1, s);
    return PBD_OK;
}

}  // namespace pbd
