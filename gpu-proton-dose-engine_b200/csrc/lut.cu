// lut.cu -- FP64 depth-LUT builder on the device.
//
// Builds, for every energy layer, the integral depth dose IDD_l(z) (physics.py:328-387,
// normalize=False) and the lateral width sigma_l(z) (physics.py:221-286) at the dose
// grid's depths, plus their central differences in CSDA range for the range-shift
// gradient.  This file is compiled with -fmad=false: products and sums are rounded one
// at a time, in the order the reference's NumPy expressions evaluate them, so the
// tables agree with the reference to the last few ulps of the transcendental functions.
//
// Two steps are restated in a different but equivalent form:
//  * CSDA range table cumulative sum: one thread, sequential, as numpy.cumsum.
//  * Range-straggling convolution.  The reference multiplies the zero-padded rfft of
//    the binned dose (nfft = 16384 >= 2 n_fine) by exp(-2 (pi f sigma_R)^2).  By the
//    Poisson summation formula, irfft of that Gaussian spectrum is h * phi_sigma(k h)
//    summed over periods of nfft*h; all other periods and all frequencies past Nyquist
//    are below 1e-300 for any sigma_R >= 2 h, and the zero padding makes the circular
//    convolution linear.  The device therefore computes the linear convolution
//    smooth[n] = sum_m binned[m] * h * phi(|n-m| h) directly in FP64, truncated at
//    16 sigma_R (kernel weight < 1e-55).  The two agree to FFT round-off (~1e-16 of
//    the peak).
#include <math.h>
#include <stdio.h>

#include <algorithm>

#include "pbd_internal.cuh"
#include "tc_common.cuh"

namespace pbd {
namespace {

// physics.py:42-66
constexpr double kMp = 938.27208816;
constexpr double kMe = 0.51099895000;
constexpr double kKbb = 0.307075;
constexpr double kZA = 10.0 / 18.01528;
constexpr double kI = 75.0 * 1e-6;
constexpr double kRho = 1.0;
constexpr double kX0 = 36.08;
constexpr double kPowerP = 1.77;
constexpr double kHighland = 13.6;
constexpr double kElo = 0.5;
constexpr double kEhi = 400.0;
constexpr double kBohr = kKbb * kZA * kRho * kMe;   // physics.py:151
constexpr int kTableN = 3797;                        // 800 + 899 + 899 + 1199 points
constexpr int kBohrN = 4000;                         // physics.py:154

__device__ double g_etab[kTableN];
__device__ double g_rtab[kTableN];

// numpy.linspace(a, b, n)[k]: k*step + a, the last point set to b exactly.
__device__ __forceinline__ double lin(double a, double b, int n, int k) {
    if (k == n - 1) return b;
    double step = (b - a) / (double)(n - 1);
    return (double)k * step + a;
}

// Energy grid of the range table (physics.py:118-123): four linspace pieces with the
// shared end points 2, 20 and 60 MeV kept once.
__device__ double table_energy(int k) {
    if (k < 800) return lin(kElo, 2.0, 800, k);
    if (k < 1699) return lin(2.0, 20.0, 900, k - 799);
    if (k < 2598) return lin(20.0, 60.0, 900, k - 1698);
    return lin(60.0, kEhi, 1200, k - 2597);
}

// beta_gamma, physics.py:72-77
__device__ __forceinline__ void kinematics(double e, double& beta, double& gam, double& b2) {
    gam = 1.0 + e / kMp;
    b2 = 1.0 - 1.0 / (gam * gam);
    b2 = fmin(fmax(b2, 1e-14), 1.0);
    beta = sqrt(b2);
}

// bethe_bloch_water, physics.py:80-100
__device__ double stopping_power(double e) {
    double beta, gam, b2;
    kinematics(e, beta, gam, b2);
    const double me_mp = kMe / kMp;
    double g2 = gam * gam;
    double tmax = 2.0 * kMe * b2 * g2 / (1.0 + 2.0 * gam * me_mp + me_mp * me_mp);
    double arg = 2.0 * kMe * b2 * g2 * tmax / (kI * kI);
    arg = fmax(arg, 1.0 + 1e-12);
    return kKbb * kZA * kRho / b2 * (0.5 * log(arg) - b2);
}

// scattering_power(model="highland_local") at L = 1, physics.py:202-217
__device__ double highland_local(double e) {
    double beta, gam, b2;
    kinematics(e, beta, gam, b2);
    double pc = sqrt(fmax(gam * gam - 1.0, 0.0)) * kMp;
    double bpc = fmax(beta * pc, 1e-9);
    double q = kHighland / bpc;
    double base = q * q / kX0;
    const double lnl = 0.0;   // log(1)
    return base * (1.0 + 0.038 * lnl) * (1.076 + 0.038 * lnl);
}

// numpy.interp on a strictly increasing table.
__device__ double interp(double x, const double* xp, const double* fp, int n, double left,
                         double right) {
    if (x < xp[0]) return left;
    if (x > xp[n - 1]) return right;
    if (x == xp[n - 1]) return fp[n - 1];
    int lo = 0, hi = n - 1;
    while (hi - lo > 1) {
        int mid = (lo + hi) >> 1;
        if (xp[mid] <= x) lo = mid; else hi = mid;
    }
    if (xp[lo] == x) return fp[lo];
    double slope = (fp[lo + 1] - fp[lo]) / (xp[lo + 1] - xp[lo]);
    return slope * (x - xp[lo]) + fp[lo];
}

// numpy.interp where xp = linspace(a, b, n) is generated on the fly.
__device__ double interp_lin(double x, double a, double b, int n, const double* fp, double left,
                             double right) {
    if (x < a) return left;
    if (x > b) return right;
    if (x == b) return fp[n - 1];
    int lo = 0, hi = n - 1;
    while (hi - lo > 1) {
        int mid = (lo + hi) >> 1;
        if (lin(a, b, n, mid) <= x) lo = mid; else hi = mid;
    }
    double x0 = lin(a, b, n, lo);
    if (x0 == x) return fp[lo];
    double x1 = lin(a, b, n, lo + 1);
    double slope = (fp[lo + 1] - fp[lo]) / (x1 - x0);
    return slope * (x - x0) + fp[lo];
}

// numpy.linspace(a, b, n)[k] with its step (b - a) / (n - 1) passed in: the same value as lin().
__device__ __forceinline__ double lin_s(double a, double b, int n, int k, double step) {
    if (k == n - 1) return b;
    return (double)k * step + a;
}

// The interval of x on linspace(a, b, n) that interp_lin's binary search finds, for a <= x <= b:
// estimated from x * (1 / step) and corrected against the grid points themselves, whose values
// fk * step + a (fk = (double)lo kept in step with lo -- integers below 2^53, so fk +- 1 is
// exact) are those lin_s computes.  lo and its grid point x0 on return; x == b gives lo = n - 1,
// x0 = b.  step = (b - a) / (n - 1) and inv ~ 1 / step come from the caller.
__device__ __forceinline__ void locate_lin(double x, double a, double b, int n, double step,
                                           double inv, int& lo_out, double& x0_out) {
    if (x == b) {
        lo_out = n - 1;
        x0_out = b;
        return;
    }
    int lo = (int)((x - a) * inv);
    lo = lo < 0 ? 0 : (lo > n - 2 ? n - 2 : lo);
    double fk = (double)lo;
    double x0 = fk * step + a;
    while (lo > 0 && x0 > x) {
        --lo;
        fk -= 1.0;
        x0 = fk * step + a;
    }
    while (lo < n - 2) {
        const double x1 = lo + 1 == n - 1 ? b : (fk + 1.0) * step + a;
        if (!(x1 <= x)) break;
        ++lo;
        fk += 1.0;
        x0 = x1;
    }
    lo_out = lo;
    x0_out = x0;
}

__device__ __forceinline__ double csda(double e) {
    return interp(e, g_etab, g_rtab, kTableN, g_rtab[0], g_rtab[kTableN - 1]);
}
__device__ __forceinline__ double energy_at_range(double r) {
    double rc = fmin(fmax(r, 0.0), g_rtab[kTableN - 1]);
    return interp(rc, g_rtab, g_etab, kTableN, g_etab[0], g_etab[kTableN - 1]);
}

// _range_table, physics.py:111-127.  Trapezoid steps in parallel, cumulative sum in
// one thread in the order numpy.cumsum adds.
__global__ void range_table_kernel() {
    __shared__ double inv_s[kTableN];
    for (int k = threadIdx.x; k < kTableN; k += blockDim.x) {
        double e = table_energy(k);
        g_etab[k] = e;
        inv_s[k] = 1.0 / stopping_power(e);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double r = 0.0;
        g_rtab[0] = 0.0;
        double e_prev = g_etab[0];
        for (int k = 1; k < kTableN; ++k) {
            double e = g_etab[k];
            r = r + 0.5 * (inv_s[k] + inv_s[k - 1]) * (e - e_prev);
            g_rtab[k] = r;
            e_prev = e;
        }
    }
}

__global__ void csda_kernel(const double* in, double* out, int n, int inverse) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = inverse ? energy_at_range(in[i]) : csda(in[i]);
}

// Per (layer, variant) scalars.  Variant 0 is the nominal build, 1 and 2 are built at
// CSDA range +fd_step and -fd_step.
struct LayerScal {
    double e0, r0, sig_r, zmax, h;
    int conv_k;
    int pad_;
};

struct LutDims {
    int n_layers, nvar, nz, n_idd, n_fe;
    double fe_lo, fe_hi;      // Fermi-Eyges fine grid end points
    double fd_step;
};

// Setup of one (layer, variant): energy, range, sigma_R (physics.py:154-174, 310-322),
// the binned CSDA dose (physics.py:362-370), the Gaussian kernel table and the local
// scattering power on the Fermi-Eyges fine grid (physics.py:259-264).
__global__ void layer_setup_kernel(pbd_lut_spec spec, LutDims dm, const double* energies,
                                   const double* shift, LayerScal* scal, double* binned,
                                   double* ker, double* t_fe) {
    __shared__ double f_bohr[kBohrN];
    __shared__ double red[256];
    const int lv = blockIdx.x;
    const int l = lv / dm.nvar, v = lv % dm.nvar;
    const double off = v == 0 ? 0.0 : (v == 1 ? dm.fd_step : -dm.fd_step);
    const double s = (shift ? shift[l] : 0.0) + off;
    const double e_in = energies[l];
    const double e0 = (s == 0.0) ? e_in : energy_at_range(csda(e_in) + s);
    const double r0 = csda(e0);

    // range straggling
    double strag = 0.0;
    if (spec.straggling_model == 0) {
        double acc = 0.0;
        if (e0 > kElo) {
            for (int k = threadIdx.x; k < kBohrN; k += blockDim.x) {
                double e = lin(kElo, e0, kBohrN, k);
                double sp = stopping_power(e);
                double beta, gam, b2;
                kinematics(e, beta, gam, b2);
                f_bohr[k] = kBohr / (fmax(b2, 1e-12) * (sp * sp * sp));
            }
            __syncthreads();
            for (int k = threadIdx.x; k < kBohrN - 1; k += blockDim.x) {
                double de = lin(kElo, e0, kBohrN, k + 1) - lin(kElo, e0, kBohrN, k);
                acc += de * (f_bohr[k + 1] + f_bohr[k]) / 2.0;
            }
        }
        red[threadIdx.x] = acc;
        __syncthreads();
        for (int w = blockDim.x / 2; w > 0; w >>= 1) {
            if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
            __syncthreads();
        }
        strag = sqrt(red[0]);
    } else if (spec.straggling_model == 1) {
        strag = spec.strag_coef * pow(r0, spec.strag_exp);
    }
    const double espr = kPowerP * spec.energy_spread * r0;
    const double sig_r = hypot(strag, espr);
    const int n = dm.n_idd;
    const double zmax = r0 + 8.0 * sig_r + 0.2;
    const double h = lin(0.0, zmax, n, 1) - 0.0;
    int kk = 0;
    if (sig_r > 0.0) {
        double kf = ceil(16.0 * sig_r / h);
        kk = kf > (double)(n - 1) ? n - 1 : (int)kf;
    }
    if (threadIdx.x == 0) {
        LayerScal sc;
        sc.e0 = e0; sc.r0 = r0; sc.sig_r = sig_r; sc.zmax = zmax; sc.h = h; sc.conv_k = kk;
        sc.pad_ = 0;
        scal[lv] = sc;
    }
    double* bin = binned + (size_t)lv * n;
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        double zf = lin(0.0, zmax, n, k);
        double ea = lin(0.0, zmax, n + 1, k);
        double eb = lin(0.0, zmax, n + 1, k + 1);
        double ena = ea < r0 ? energy_at_range(fmax(r0 - ea, 0.0)) : 0.0;
        double enb = eb < r0 ? energy_at_range(fmax(r0 - eb, 0.0)) : 0.0;
        double fl = exp(-zf / spec.atten_len);
        bin[k] = fl * (ena - enb) / h;
    }
    if (sig_r > 0.0) {
        double* kr = ker + (size_t)lv * n;
        const double c = kInvSqrt2Pi / sig_r;
        for (int k = threadIdx.x; k <= kk; k += blockDim.x) {
            double t = (double)k * h;
            kr[k] = h * (c * exp(-(t * t) / (2.0 * sig_r * sig_r)));
        }
    }
    double* tf = t_fe + (size_t)lv * dm.n_fe;
    for (int i = threadIdx.x; i < dm.n_fe; i += blockDim.x) {
        double zf = lin(dm.fe_lo, dm.fe_hi, dm.n_fe, i);
        double t = 0.0;
        if (zf < r0) {
            double el = energy_at_range(fmax(r0 - zf, 0.0));
            t = highland_local(fmax(el, 1e-3));
        }
        tf[i] = t;
    }
}

// Range-straggling convolution (see the file comment): smooth[i] = sum_m bin[m] kr[|i - m|]
// over |i - m| <= K, bins outside [0, n) being zero, each output summed in ascending m with
// FMA.  A thread owns kConvB consecutive outputs i0 .. i0 + B - 1 and walks the steps
// s = m - i0 + K = 0 .. 2K + B - 1: at each step one bin (shared by its B outputs) and one
// kernel value kr[|K - s|] (the same for every thread of the block) are read from shared
// memory, and the kernel value is kept in a ring of B registers whose slot is the step
// modulo B -- output b needs the value loaded b steps earlier -- so the unrolled body needs
// no register moves.  Steps run in chunks of kConvChunk whose bins and kernel values are
// staged in shared memory; B is odd so that the threads' strided bin reads do not collide
// in the banks.
constexpr int kConvB = 9;
constexpr int kConvThreads = 128;
constexpr int kConvSeg = kConvB * kConvThreads;          // outputs per block
constexpr int kConvChunk = 112 * kConvB;                 // steps per staged chunk
constexpr int kConvSmem = (kConvSeg + kConvChunk + kConvChunk) * (int)sizeof(double);

__global__ void __launch_bounds__(kConvThreads)
conv_kernel(LutDims dm, const LayerScal* scal, const double* binned, const double* ker,
            double* smooth) {
    extern __shared__ double csm[];
    double* sbin = csm;                                   // kConvSeg + kConvChunk bins
    double* skw = csm + kConvSeg + kConvChunk;            // kConvChunk kernel values
    const int lv = blockIdx.x;
    const int n = dm.n_idd;
    const int s0 = blockIdx.y * kConvSeg;
    const double* bin = binned + (size_t)lv * n;
    double* out = smooth + (size_t)lv * n;
    const LayerScal sc = scal[lv];
    if (sc.sig_r <= 0.0) {
        for (int i = s0 + threadIdx.x; i < min(n, s0 + kConvSeg); i += kConvThreads)
            out[i] = bin[i];
        return;
    }
    const double* kr = ker + (size_t)lv * n;
    const int K = sc.conv_k;
    const int n_steps = 2 * K + kConvB;
    const int i0 = s0 + threadIdx.x * kConvB;             // this thread's first output
    double acc[kConvB], ring[kConvB];
#pragma unroll
    for (int b = 0; b < kConvB; ++b) { acc[b] = 0.0; ring[b] = 0.0; }
    for (int c0 = 0; c0 < n_steps; c0 += kConvChunk) {
        // bins m = s0 - K + c0 + j, j < kConvSeg + kConvChunk; kernel kr[|K - c0 - j|], j < chunk
        __syncthreads();
        for (int j = threadIdx.x; j < kConvSeg + kConvChunk; j += kConvThreads) {
            const int m = s0 - K + c0 + j;
            sbin[j] = (m >= 0 && m < n) ? bin[m] : 0.0;
        }
        for (int j = threadIdx.x; j < kConvChunk; j += kConvThreads) {
            const int t = K - c0 - j;
            const int a = t < 0 ? -t : t;
            skw[j] = a <= K ? kr[a] : 0.0;
        }
        __syncthreads();
        const double* sb = sbin + threadIdx.x * kConvB;   // bin of step c0 + j is sb[j]
        for (int j = 0; j < kConvChunk; j += kConvB) {
#pragma unroll
            for (int q = 0; q < kConvB; ++q) {
                ring[q] = skw[j + q];                     // kr[|K - s|], s = c0 + j + q
                const double bv = sb[j + q];
#pragma unroll
                for (int b = 0; b < kConvB; ++b)
                    acc[b] = __fma_rn(bv, ring[(q - b + kConvB) % kConvB], acc[b]);
            }
        }
    }
#pragma unroll
    for (int b = 0; b < kConvB; ++b)
        if (i0 + b < n) out[i0 + b] = acc[b];
}

// Fermi-Eyges direct scattering integral B(zf_i) = sum_{j<i} (zf_i - zf_j)^2 T_j h_j,
// physics.py:266-270, with h = numpy.gradient(zf).
__device__ __forceinline__ double fe_h(const LutDims& dm, int j) {
    const int n = dm.n_fe;
    if (j == 0) return lin(dm.fe_lo, dm.fe_hi, n, 1) - lin(dm.fe_lo, dm.fe_hi, n, 0);
    if (j == n - 1) return lin(dm.fe_lo, dm.fe_hi, n, n - 1) - lin(dm.fe_lo, dm.fe_hi, n, n - 2);
    return (lin(dm.fe_lo, dm.fe_hi, n, j + 1) - lin(dm.fe_lo, dm.fe_hi, n, j - 1)) / 2.0;
}

__global__ void fe_grid_kernel(LutDims dm, double* zf, double* hf) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < dm.n_fe; i += gridDim.x * blockDim.x) {
        zf[i] = lin(dm.fe_lo, dm.fe_hi, dm.n_fe, i);
        hf[i] = fe_h(dm, i);
    }
}

__global__ void fe_b_kernel(LutDims dm, const double* zf, const double* hf, const double* t_fe,
                            double* b_fe) {
    const int lv = blockIdx.x;
    const int i = blockIdx.y * blockDim.x + threadIdx.x;
    if (i >= dm.n_fe) return;
    const double* tf = t_fe + (size_t)lv * dm.n_fe;
    const double zi = zf[i];
    double acc = 0.0;
    for (int j = 0; j < i; ++j) {
        double d = zi - zf[j];
        acc += d * d * tf[j] * hf[j];
    }
    b_fe[(size_t)lv * dm.n_fe + i] = acc;
}

// Tables at the requested depths, all variants of one layer per block; the variants
// combine into the range derivatives.
__global__ void lut_output_kernel(pbd_lut_spec spec, LutDims dm, const LayerScal* scal,
                                  const double* smooth, const double* zf_fe, const double* b_fe,
                                  double single_depth, double* idd, double* sigma,
                                  double* didd, double* dsig) {
    const int l = blockIdx.x;
    for (int k = threadIdx.x; k < dm.nz; k += blockDim.x) {
        double d = spec.depth_scale * (spec.z0 + (double)k * spec.dz);
        double dz_eval = (dm.nz == 1 && !spec.anchor_surface) ? single_depth : d;
        double out_i[3], out_s[3];
        for (int v = 0; v < dm.nvar; ++v) {
            const int lv = l * dm.nvar + v;
            const LayerScal sc = scal[lv];
            out_i[v] = interp_lin(d, 0.0, sc.zmax, dm.n_idd, smooth + (size_t)lv * dm.n_idd, 0.0,
                                  0.0);
            double b = 0.0;
            if (!(spec.anchor_surface && d <= 0.0))
                b = interp(dz_eval, zf_fe, b_fe + (size_t)lv * dm.n_fe, dm.n_fe,
                           b_fe[(size_t)lv * dm.n_fe], b_fe[(size_t)lv * dm.n_fe + dm.n_fe - 1]);
            double zp = dz_eval / spec.depth_scale;
            double var = spec.sigma_x0 * spec.sigma_x0
                       + 2.0 * spec.rho0 * spec.sigma_x0 * spec.sigma_theta0 * zp
                       + spec.sigma_theta0 * spec.sigma_theta0 * (zp * zp)
                       + b / (spec.depth_scale * spec.depth_scale);
            out_s[v] = sqrt(fmax(var, 0.0));
        }
        const size_t o = (size_t)l * dm.nz + k;
        idd[o] = out_i[0];
        sigma[o] = out_s[0];
        if (dm.nvar == 3) {
            if (didd) didd[o] = (out_i[1] - out_i[2]) / (2.0 * dm.fd_step);
            if (dsig) dsig[o] = (out_s[1] - out_s[2]) / (2.0 * dm.fd_step);
        }
    }
}

// Heterogeneous media: dose = sum_l IDD_l(WED) * lateral_l per voxel, IDD_l the layer's
// smoothed depth curve evaluated at the voxel's water-equivalent depth with the same
// interpolation as the tables (lut_output_kernel).  Accumulated in FP64, in layer order.
constexpr int kWedLayers = 256;   // layers whose curve scalars are staged in shared memory

// The combine streams each layer's lateral values of a 1024-voxel tile into a ring of
// shared-memory stages with 1-D bulk copies (cp.async.bulk, completion on an mbarrier), so the
// bytes in flight do not depend on the registers the FP64 interpolation needs.  Layers that
// no voxel of the tile reaches (tile's smallest WED above zmax, or largest below 0) are
// neither copied nor evaluated.  Waits are bounded (2 s); a block whose wait runs out sets
// the error word, waits (bounded) for its own copies in flight and leaves, and the poison pass
// turns the dose into NaN.
constexpr int kCmbThreads = 256;
constexpr int kCmbPer = 4;                              // voxels per thread
constexpr int kCmbTile = kCmbThreads * kCmbPer;         // voxels per tile (4 KB of one layer)
constexpr int kCmbStages = 6;

__device__ __forceinline__ void bulk_load_s(void* dst, const void* src, uint32_t bytes,
                                            uint64_t* bar) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(tc::smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
    asm volatile(
        "cp.async.bulk.shared::cta.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            tc::smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(tc::smem_u32(bar))
        : "memory");
}

// 48 registers, no spills: 5 blocks per SM (64 registers without the bound: 4)
__global__ void __launch_bounds__(kCmbThreads, 5) wed_combine_kernel(
    LutDims dm, const LayerScal* scal, const double2* pts, const float* lateral, size_t lstride,
    const double* wed, size_t nvox, int n_layers, float* dose, int* err) {
    __shared__ __align__(128) float lat[kCmbStages][kCmbTile];
    __shared__ __align__(8) uint64_t full[kCmbStages];
    __shared__ double zmax[kWedLayers], stp[kWedLayers], istp[kWedLayers];
    __shared__ double rmin[kCmbThreads / 32], rmax[kCmbThreads / 32];
    __shared__ int rnan[kCmbThreads / 32];
    __shared__ int abort_s;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int l = tid; l < n_layers && l < kWedLayers; l += kCmbThreads) {
        zmax[l] = scal[l].zmax;
        stp[l] = (scal[l].zmax - 0.0) / (double)(dm.n_idd - 1);
        istp[l] = 1.0 / stp[l];
    }
    if (tid == 0) {
        for (int q = 0; q < kCmbStages; ++q) tc::mbar_init(&full[q], 1);
        tc::fence_mbar_init();
        abort_s = 0;
    }
    __syncthreads();
    const int n = dm.n_idd;
    const double inf = __longlong_as_double(0x7FF0000000000000ll);
    const size_t n_tiles = (nvox + kCmbTile - 1) / kCmbTile;
    uint32_t it = 0;       // copies consumed: stage it % kCmbStages, parity (it / kCmbStages) & 1
    uint32_t issued = 0;   // copies issued (thread 0)
    int next_l = 0;        // next layer thread 0 considers (thread 0)
    for (size_t t = blockIdx.x; t < n_tiles; t += gridDim.x) {
        const size_t v0 = t * kCmbTile;
        const int cnt = (int)((nvox - v0) < (size_t)kCmbTile ? (nvox - v0) : (size_t)kCmbTile);
        double d[kCmbPer], acc[kCmbPer];
        double mn = inf, mx = -inf;
        int has_nan = 0;
#pragma unroll
        for (int j = 0; j < kCmbPer; ++j) {
            const int i = tid + j * kCmbThreads;
            acc[j] = 0.0;
            d[j] = 0.0;
            if (i < cnt) {
                d[j] = __ldcs(wed + v0 + i);
                if (d[j] != d[j]) {
                    has_nan = 1;
                } else {
                    mn = fmin(mn, d[j]);
                    mx = fmax(mx, d[j]);
                }
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            mn = fmin(mn, __shfl_xor_sync(0xffffffffu, mn, o));
            mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
            has_nan |= __shfl_xor_sync(0xffffffffu, has_nan, o);
        }
        if (lane == 0) {
            rmin[warp] = mn;
            rmax[warp] = mx;
            rnan[warp] = has_nan;
        }
        __syncthreads();
        double tmin = inf, tmax = -inf;
        bool tnan = false;
#pragma unroll
        for (int q = 0; q < kCmbThreads / 32; ++q) {
            tmin = fmin(tmin, rmin[q]);
            tmax = fmax(tmax, rmax[q]);
            tnan = tnan || rnan[q] != 0;
        }
        // the same answer in every thread: layer l is copied and evaluated for this tile
        auto active = [&](int l) -> bool {
            const double zm = l < kWedLayers ? zmax[l] : scal[l].zmax;
            return tnan || (tmin <= zm && tmax >= 0.0);
        };
        const uint32_t bytes = (uint32_t)((cnt + 3) / 4) * 16u;
        auto refill = [&]() {
            while (issued - it < (uint32_t)kCmbStages && next_l < n_layers) {
                if (active(next_l)) {
                    const uint32_t q = issued % kCmbStages;
                    bulk_load_s(lat[q], lateral + (size_t)next_l * lstride + v0, bytes, &full[q]);
                    ++issued;
                }
                ++next_l;
            }
        };
        if (tid == 0) {
            next_l = 0;
            refill();
        }
        for (int l = 0; l < n_layers; ++l) {
            if (!active(l)) continue;
            const uint32_t q = it % kCmbStages;
            if (!tcc::wait_bar(&full[q], (it / kCmbStages) & 1u)) {
                abort_s = 1;
                atomicExch(err, 1);
            } else {
                const double zm = l < kWedLayers ? zmax[l] : scal[l].zmax;
                const double st = l < kWedLayers ? stp[l] : (zm - 0.0) / (double)(n - 1);
                const double is = l < kWedLayers ? istp[l] : 1.0 / st;
                const double2* lp = pts + (size_t)l * n;
                // A voxel counts only where its WED lies inside the curve (or is NaN): outside
                // [0, zmax] the curve's fill values are 0 and nothing is added, and a (layer,
                // slice) the activity table marked inactive has every WED above zmax, so the
                // unwritten part of a lateral map is copied at most, never used.
                int lo[kCmbPer];
                double x0[kCmbPer];
#pragma unroll
                for (int j = 0; j < kCmbPer; ++j) {
                    lo[j] = 0;
                    x0[j] = 0.0;
                    if (tid + j * kCmbThreads < cnt && !(d[j] < 0.0 || d[j] > zm))
                        locate_lin(d[j], 0.0, zm, n, st, is, lo[j], x0[j]);
                }
#pragma unroll
                for (int j = 0; j < kCmbPer; ++j) {
                    const int i = tid + j * kCmbThreads;
                    if (i >= cnt || d[j] < 0.0 || d[j] > zm) continue;
                    const double2 pt = __ldg(lp + lo[j]);
                    // interp_lin's value: fp[lo] on a grid point, else slope * (x - x0) + fp[lo]
                    // with the slope np.interp rounds; the sum in layer order
                    const double idd = x0[j] == d[j] ? pt.x : pt.y * (d[j] - x0[j]) + pt.x;
                    if (idd == 0.0) continue;
                    acc[j] += idd * (double)lat[q][i];
                }
            }
            __syncthreads();   // stage q is free again; abort_s is visible to every thread
            ++it;
            if (abort_s) break;
            if (tid == 0) refill();
        }
        if (abort_s) {
            // the copies still in flight (the one whose wait ran out included) land before
            // the block's shared memory is released
            if (tid == 0)
                for (uint32_t c = it - 1; c != issued; ++c)
                    (void)tcc::wait_bar(&full[c % kCmbStages], (c / kCmbStages) & 1u);
            return;
        }
#pragma unroll
        for (int j = 0; j < kCmbPer; ++j) {
            const int i = tid + j * kCmbThreads;
            if (i < cnt) __stcs(dose + v0 + i, (float)acc[j]);
        }
        __syncthreads();   // the next tile's reduction reuses rmin / rmax / rnan
    }
}

// After a combine (or the lateral maps' forward, err2) whose wait ran out: the whole dose is
// invalid, NaN.
__global__ void wed_poison_kernel(float* dose, size_t nvox, const int* err, const int* err2) {
    if (*err == 0 && (err2 == nullptr || *err2 == 0)) return;
    for (size_t v = (size_t)blockIdx.x * blockDim.x + threadIdx.x; v < nvox;
         v += (size_t)gridDim.x * blockDim.x)
        dose[v] = __int_as_float(0x7fc00000);
}

// The heterogeneous dose's dL/dD seen by layer l: maps[l * lstride + v] = IDD_l(WED[v]) *
// grad[v] (FP64 product, rounded once to FP32), 0 outside the curve.  The adjoint of layer l
// with this map and depth dose 1 on its active slices is dL/dW_l.  Every (layer, voxel) entry
// is written.
__global__ void __launch_bounds__(256) wed_grad_maps_kernel(LutDims dm, const LayerScal* scal,
                                                            const double2* pts, const float* grad,
                                                            const double* wed, size_t nvox,
                                                            int n_layers, size_t lstride,
                                                            float* maps) {
    __shared__ double zmax[kWedLayers], stp[kWedLayers], istp[kWedLayers];
    for (int l = threadIdx.x; l < n_layers && l < kWedLayers; l += blockDim.x) {
        zmax[l] = scal[l].zmax;
        stp[l] = (scal[l].zmax - 0.0) / (double)(dm.n_idd - 1);
        istp[l] = 1.0 / stp[l];
    }
    __syncthreads();
    const int n = dm.n_idd;
    for (size_t v = (size_t)blockIdx.x * blockDim.x + threadIdx.x; v < nvox;
         v += (size_t)gridDim.x * blockDim.x) {
        const double d = wed[v];
        const double g = (double)grad[v];
        for (int l = 0; l < n_layers; ++l) {
            const double zm = l < kWedLayers ? zmax[l] : scal[l].zmax;
            float out = 0.0f;
            if (!(d < 0.0 || d > zm)) {
                const double st = l < kWedLayers ? stp[l] : (zm - 0.0) / (double)(n - 1);
                const double is = l < kWedLayers ? istp[l] : 1.0 / st;
                int lo = 0;
                double x0 = 0.0;
                locate_lin(d, 0.0, zm, n, st, is, lo, x0);
                const double2 pt = __ldg(pts + (size_t)l * n + lo);
                const double idd = x0 == d ? pt.x : pt.y * (d - x0) + pt.x;
                out = (float)(idd * g);
            }
            maps[(size_t)l * lstride + v] = out;
        }
    }
}

// Depth dose of a layer's curve at depth d (the curve's interval search and np.interp
// semantics, as in wed_grad_maps_kernel): 0 outside [0, zmax].
__device__ __forceinline__ double curve_at(const LayerScal& sc, const double2* pts, int n, double d) {
    const double zm = sc.zmax;
    if (d < 0.0 || d > zm) return 0.0;
    const double st = (zm - 0.0) / (double)(n - 1), is = 1.0 / st;
    int lo = 0;
    double x0 = 0.0;
    locate_lin(d, 0.0, zm, n, st, is, lo, x0);
    const double2 pt = __ldg(pts + lo);
    return x0 == d ? pt.x : pt.y * (d - x0) + pt.x;
}

// maps (L, lstride): dL/dD times the range derivative of each layer's depth dose at the WED,
// (IDD+_l(WED) - IDD-_l(WED)) / (2 h), from the curves at range shifts +h and -h (FP64 difference,
// one FP32 rounding of the product).
__global__ void __launch_bounds__(256) wed_grad_maps_dr_kernel(
    LutDims dm, const LayerScal* scp, const double2* ptp, const LayerScal* scm,
    const double2* ptm, const float* grad, const double* wed, size_t nvox, int n_layers,
    size_t lstride, double inv2h, float* maps) {
    const int n = dm.n_idd;
    for (size_t v = (size_t)blockIdx.x * blockDim.x + threadIdx.x; v < nvox;
         v += (size_t)gridDim.x * blockDim.x) {
        const double d = wed[v];
        const double g = (double)grad[v];
        for (int l = 0; l < n_layers; ++l) {
            const double dp = curve_at(scp[l], ptp + (size_t)l * n, n, d);
            const double dmn = curve_at(scm[l], ptm + (size_t)l * n, n, d);
            maps[(size_t)l * lstride + v] = (float)((dp - dmn) * inv2h * g);
        }
    }
}

// Curve points of the smoothed depth curves: {fp[k], slope_k} with slope_k = (fp[k+1] - fp[k])
// / (x[k+1] - x[k]) on the grid linspace(0, zmax, n) -- the operands and the single rounding
// of np.interp's slope (and of interp_lin) -- and 0 at the last point.  Value and slope share a
// 16-byte load in the combine, which needs no division per voxel.
__global__ void wed_slope_kernel(LutDims dm, const LayerScal* scal, const double* smooth,
                                 double2* pts) {
    const int l = blockIdx.x;
    const int n = dm.n_idd;
    const double zm = scal[l].zmax;
    const double st = (zm - 0.0) / (double)(n - 1);
    const double* fp = smooth + (size_t)l * n;
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        double s = 0.0;
        if (k < n - 1) {
            const double x0 = lin_s(0.0, zm, n, k, st), x1 = lin_s(0.0, zm, n, k + 1, st);
            s = (fp[k + 1] - fp[k]) / (x1 - x0);
        }
        pts[(size_t)l * n + k] = make_double2(fp[k], s);
    }
}

// Per (layer, slice) activity of the heterogeneous dose: 1 when some voxel of the slice has a
// WED inside the layer's depth curve (<= zmax), else 0 (the layer adds nothing there).  One
// block per slice: the slice's smallest WED, then one entry per layer.
constexpr int kActThreads = 1024;

__global__ void __launch_bounds__(kActThreads) wed_activity_kernel(const LayerScal* scal,
                                                                   const LayerScal* scal2,
                                                                   const double* wed,
                                                                   size_t nslice, int nz,
                                                                   int n_layers, double* act) {
    __shared__ double red[kActThreads / 32];
    const int z = blockIdx.x;
    const double* p = wed + (size_t)z * nslice;
    const double inf = __longlong_as_double(0x7FF0000000000000ll);
    // eight independent loads in flight per thread; fmin is exact in any order (NaN ignored)
    double m[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) m[q] = inf;
    size_t v = threadIdx.x;
    for (; v + 7 * (size_t)kActThreads < nslice; v += 8 * (size_t)kActThreads) {
#pragma unroll
        for (int q = 0; q < 8; ++q) m[q] = fmin(m[q], __ldcs(p + v + (size_t)q * kActThreads));
    }
    for (; v < nslice; v += kActThreads) m[0] = fmin(m[0], __ldcs(p + v));
    double t = fmin(fmin(fmin(m[0], m[1]), fmin(m[2], m[3])), fmin(fmin(m[4], m[5]), fmin(m[6], m[7])));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t = fmin(t, __shfl_xor_sync(0xffffffffu, t, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = t;
    __syncthreads();
    if (threadIdx.x < 32) {
        t = red[threadIdx.x];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) t = fmin(t, __shfl_xor_sync(0xffffffffu, t, o));
        if (threadIdx.x == 0) red[0] = t;
    }
    __syncthreads();
    const double smin = red[0];
    // with a second curve set: active where either set's curve reaches
    for (int l = threadIdx.x; l < n_layers; l += kActThreads) {
        const double zm = scal2 ? fmax(scal[l].zmax, scal2[l].zmax) : scal[l].zmax;
        act[(size_t)l * nz + z] = smin <= zm ? 1.0 : 0.0;
    }
}

// Water-equivalent depth at the voxel centres z_k = oz + k dz along +z (the beam axis):
// the sum of rho * path length from depth 0 (physics.py:421-423 per voxel path), voxel i
// filling [z_i - dz/2, z_i + dz/2] with rho_i, water above the first voxel, path lengths
// clipped at depth 0.  One thread per (y, x) column, FP64, in depth order.
constexpr int kRayThreads = 64;   // 64-thread blocks: a 128 x 128 field still fills every SM
constexpr int kRayBatch = 16;     // depths whose rho one thread loads before the running sum

__global__ void __launch_bounds__(kRayThreads) wed_raytrace_kernel(int nz, size_t ncol, double oz,
                                                                   double dz, const float* rho,
                                                                   double* wed) {
    for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < ncol;
         c += (size_t)gridDim.x * blockDim.x) {
        const double top0 = oz - 0.5 * dz;
        double acc = top0 > 0.0 ? top0 : 0.0;          // water above the first voxel
        for (int k0 = 0; k0 < nz; k0 += kRayBatch) {
            float r[kRayBatch];
#pragma unroll
            for (int q = 0; q < kRayBatch; ++q)
                r[q] = k0 + q < nz ? __ldcs(rho + (size_t)(k0 + q) * ncol + c) : 0.0f;
#pragma unroll
            for (int q = 0; q < kRayBatch; ++q) {
                const int k = k0 + q;
                if (k >= nz) break;
                const double zc = oz + (double)k * dz;
                const double lo = fmax(zc - 0.5 * dz, 0.0), mid = fmax(zc, 0.0);
                const double hi = fmax(zc + 0.5 * dz, 0.0);
                const double rr = (double)r[q];
                __stcs(wed + (size_t)k * ncol + c, acc + rr * (mid - lo));
                acc += rr * (hi - lo);
            }
        }
    }
}

// Depth list of the Fermi-Eyges integral (host): its first and last points and size.
struct FeList {
    int n_list;
    double lo, hi, single_depth;
    int n_fine;
};

FeList fe_list(const pbd_lut_spec* s) {
    FeList fl{};
    const int nz = s->nz;
    auto depth = [&](int k) { return s->depth_scale * (s->z0 + (double)k * s->dz); };
    fl.single_depth = 0.0;
    if (!s->anchor_surface) {
        if (nz == 1) {  // physics.py:249-253
            double z1 = depth(0);
            fl.single_depth = z1 > 0 ? z1 : 1e-6;
            fl.lo = 0.0; fl.hi = fl.single_depth; fl.n_list = 2;
        } else {
            fl.lo = depth(0); fl.hi = depth(nz - 1); fl.n_list = nz;
        }
    } else {
        int pos = 0;
        for (int k = 0; k < nz; ++k) pos += depth(k) > 0.0;
        fl.lo = 0.0;
        fl.hi = pos > 0 ? depth(nz - 1) : 1e-6;
        fl.n_list = pos + 1;
    }
    double span = fl.hi - fl.lo;   // physics.py:256-258
    int need = span > 0 ? (int)ceil(span / fmax(s->fe_max_step, 1e-6)) + 1 : 2;
    int a = (fl.n_list - 1) * s->fe_n_sub + 1;
    int nf = a > need ? a : need;
    fl.n_fine = nf > 2 ? nf : 2;
    return fl;
}

int validate_spec(const pbd_lut_spec* s, int n_layers) {
    if (!s) return PBD_ERR_NULL_ARG;
    if (n_layers <= 0 || s->nz <= 0 || s->idd_n_fine < 3 || s->fe_n_sub < 1) return PBD_ERR_BAD_DIM;
    if (!(s->dz > 0.0) || !(s->depth_scale > 0.0) || !(s->atten_len > 0.0) ||
        !(s->fe_max_step > 0.0) || !(s->fd_step >= 0.0) || !(s->sigma_x0 >= 0.0) ||
        !(s->energy_spread >= 0.0))
        return PBD_ERR_BAD_VALUE;
    if (s->straggling_model < 0 || s->straggling_model > 2) return PBD_ERR_BAD_VALUE;
    if (s->idd_n_fine > (1 << 20)) return PBD_ERR_UNSUPPORTED;
    FeList fl = fe_list(s);
    if (fl.n_fine > (1 << 16)) return PBD_ERR_UNSUPPORTED;
    return PBD_OK;
}

// The range table is a constant of the physics: the first call on a device builds it and
// waits for it (once per process and device), so that later calls on any stream find it
// ready.  Inside a stream capture the build is recorded into the graph instead and the
// device is not marked.
bool g_range_built[64];

int ensure_range_table(cudaStream_t st) {
    int dev = 0;
    PBD_TRY(cuda_rc(cudaGetDevice(&dev)));
    if (dev >= 0 && dev < 64 && g_range_built[dev]) return PBD_OK;
    range_table_kernel<<<1, 1024, 0, st>>>();
    PBD_LAUNCH_CHECK();
    count_launch(1);
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    PBD_TRY(cuda_rc(cudaStreamIsCapturing(st, &cs)));
    if (cs == cudaStreamCaptureStatusNone && dev >= 0 && dev < 64) {
        PBD_TRY(cuda_rc(cudaStreamSynchronize(st)));
        g_range_built[dev] = true;
    }
    return PBD_OK;
}

struct LutWs {
    LayerScal* scal;
    double *binned, *ker, *smooth, *t_fe, *b_fe, *zf_fe, *hf_fe;
};

size_t carve_lut(Carve& c, LutWs& w, int n_layers, int nvar, int n_idd, int n_fe) {
    const size_t lv = (size_t)n_layers * nvar;
    w.scal = c.take<LayerScal>(lv);
    w.binned = c.take<double>(lv * n_idd);
    w.ker = c.take<double>(lv * n_idd);
    w.smooth = c.take<double>(lv * n_idd);
    w.t_fe = c.take<double>(lv * n_fe);
    w.b_fe = c.take<double>(lv * n_fe);
    w.zf_fe = c.take<double>(n_fe);
    w.hf_fe = c.take<double>(n_fe);
    return c.used;
}

}  // namespace

int lut_workspace_bytes(const pbd_lut_spec* s, int n_layers, size_t* bytes) {
    PBD_TRY(validate_spec(s, n_layers));
    if (!bytes) return PBD_ERR_NULL_ARG;
    FeList fl = fe_list(s);
    Carve c(nullptr);
    LutWs w;
    *bytes = carve_lut(c, w, n_layers, s->fd_step > 0 ? 3 : 1, s->idd_n_fine, fl.n_fine) + 256;
    return PBD_OK;
}

int lut_build(const pbd_lut_spec* s, int n_layers, const double* energies, const double* shift,
              double* idd, double* sigma, double* didd, double* dsig, void* ws, size_t ws_bytes,
              cudaStream_t st) {
    PBD_TRY(validate_spec(s, n_layers));
    if (!energies || !idd || !sigma) return PBD_ERR_NULL_ARG;
    if (s->fd_step > 0 && (!didd || !dsig)) return PBD_ERR_NULL_ARG;
    size_t need = 0;
    PBD_TRY(lut_workspace_bytes(s, n_layers, &need));
    if (!ws || ws_bytes < need) return PBD_ERR_WORKSPACE;
    FeList fl = fe_list(s);
    LutDims dm;
    dm.n_layers = n_layers;
    dm.nvar = s->fd_step > 0 ? 3 : 1;
    dm.nz = s->nz;
    dm.n_idd = s->idd_n_fine;
    dm.n_fe = fl.n_fine;
    dm.fe_lo = fl.lo;
    dm.fe_hi = fl.hi;
    dm.fd_step = s->fd_step;
    Carve c(ws);
    LutWs w;
    carve_lut(c, w, n_layers, dm.nvar, dm.n_idd, dm.n_fe);
    const int lvn = n_layers * dm.nvar;

    PBD_TRY(ensure_range_table(st));
    fe_grid_kernel<<<(dm.n_fe + 255) / 256, 256, 0, st>>>(dm, w.zf_fe, w.hf_fe);
    PBD_LAUNCH_CHECK();
    layer_setup_kernel<<<lvn, 256, 0, st>>>(*s, dm, energies, shift, w.scal, w.binned, w.ker,
                                            w.t_fe);
    PBD_LAUNCH_CHECK();
    conv_kernel<<<dim3(lvn, (dm.n_idd + kConvSeg - 1) / kConvSeg), kConvThreads, kConvSmem, st>>>(
        dm, w.scal, w.binned, w.ker, w.smooth);
    PBD_LAUNCH_CHECK();
    fe_b_kernel<<<dim3(lvn, (dm.n_fe + 127) / 128), 128, 0, st>>>(dm, w.zf_fe, w.hf_fe, w.t_fe,
                                                                  w.b_fe);
    PBD_LAUNCH_CHECK();
    lut_output_kernel<<<n_layers, 128, 0, st>>>(*s, dm, w.scal, w.smooth, w.zf_fe, w.b_fe,
                                                 fl.single_depth, idd, sigma, didd, dsig);
    PBD_LAUNCH_CHECK();
    count_launch(5);
    return PBD_OK;
}

// The depth-curve blob of the heterogeneous dose: the table builder's nominal-variant
// workspace followed by the curve points {value, slope} (n_layers, n_idd).
static size_t carve_curves(Carve& c, LutWs& w, double2*& pts, int n_layers, int n_idd, int n_fe) {
    carve_lut(c, w, n_layers, 1, n_idd, n_fe);
    pts = c.take<double2>((size_t)n_layers * n_idd);
    return c.used;
}

int lut_curve_workspace(const pbd_lut_spec* s, int n_layers, size_t* bytes) {
    PBD_TRY(validate_spec(s, n_layers));
    if (!bytes) return PBD_ERR_NULL_ARG;
    FeList fl = fe_list(s);
    Carve c(nullptr);
    LutWs w;
    double2* pts = nullptr;
    *bytes = carve_curves(c, w, pts, n_layers, s->idd_n_fine, fl.n_fine) + 256;
    return PBD_OK;
}

static int wed_dims(const pbd_lut_spec* s, int n_layers, const void* ws, size_t ws_bytes,
                    LutDims& dm, LutWs& w, double2*& pts) {
    size_t need = 0;
    PBD_TRY(lut_curve_workspace(s, n_layers, &need));
    if (!ws || ws_bytes < need) return PBD_ERR_WORKSPACE;
    FeList fl = fe_list(s);
    dm.n_layers = n_layers;
    dm.nvar = 1;
    dm.nz = s->nz;
    dm.n_idd = s->idd_n_fine;
    dm.n_fe = fl.n_fine;
    dm.fe_lo = fl.lo;
    dm.fe_hi = fl.hi;
    dm.fd_step = 0.0;
    Carve c(const_cast<void*>(ws));
    carve_curves(c, w, pts, n_layers, dm.n_idd, dm.n_fe);
    return PBD_OK;
}

int lut_wed_curves(const pbd_lut_spec* s, int n_layers, const double* energies,
                   const double* shift, void* curves, size_t curves_bytes, cudaStream_t st) {
    PBD_TRY(validate_spec(s, n_layers));
    if (!energies) return PBD_ERR_NULL_ARG;
    LutDims dm;
    LutWs w;
    double2* pts = nullptr;
    PBD_TRY(wed_dims(s, n_layers, curves, curves_bytes, dm, w, pts));
    PBD_TRY(ensure_range_table(st));
    layer_setup_kernel<<<n_layers, 256, 0, st>>>(*s, dm, energies, shift, w.scal, w.binned, w.ker,
                                                 w.t_fe);
    PBD_LAUNCH_CHECK();
    conv_kernel<<<dim3(n_layers, (dm.n_idd + kConvSeg - 1) / kConvSeg), kConvThreads, kConvSmem, st>>>(
        dm, w.scal, w.binned, w.ker, w.smooth);
    PBD_LAUNCH_CHECK();
    wed_slope_kernel<<<n_layers, 256, 0, st>>>(dm, w.scal, w.smooth, pts);
    PBD_LAUNCH_CHECK();
    count_launch(3);
    return PBD_OK;
}

int lut_wed_activity(const pbd_lut_spec* s, int n_layers, const void* curves, size_t curves_bytes,
                     const double* wed, int nz, size_t nslice, double* act, cudaStream_t st,
                     const void* curves2, size_t curves2_bytes) {
    PBD_TRY(validate_spec(s, n_layers));
    if (!wed || !act) return PBD_ERR_NULL_ARG;
    LutDims dm;
    LutWs w;
    double2* pts = nullptr;
    PBD_TRY(wed_dims(s, n_layers, curves, curves_bytes, dm, w, pts));
    const LayerScal* scal2 = nullptr;
    if (curves2) {
        LutDims dm2;
        LutWs w2;
        double2* pts2 = nullptr;
        PBD_TRY(wed_dims(s, n_layers, curves2, curves2_bytes, dm2, w2, pts2));
        scal2 = w2.scal;
    }
    wed_activity_kernel<<<nz, kActThreads, 0, st>>>(w.scal, scal2, wed, nslice, nz, n_layers, act);
    PBD_LAUNCH_CHECK();
    count_launch(1);
    return PBD_OK;
}

int lut_wed_combine(const pbd_lut_spec* s, int n_layers, const float* lateral, size_t lstride,
                    const double* wed, size_t nvox, float* dose, int* err, const int* err2,
                    const void* curves, size_t curves_bytes, cudaStream_t st) {
    PBD_TRY(validate_spec(s, n_layers));
    if (!lateral || !wed || !dose || !err) return PBD_ERR_NULL_ARG;
    // 1-D bulk copies: 16-byte aligned rows, the tile's copy rounded up to 16 bytes inside
    // the row
    if ((reinterpret_cast<size_t>(lateral) & 15) || (lstride & 3) || lstride < ((nvox + 3) & ~(size_t)3))
        return PBD_ERR_BAD_VALUE;
    LutDims dm;
    LutWs w;
    double2* pts = nullptr;
    PBD_TRY(wed_dims(s, n_layers, curves, curves_bytes, dm, w, pts));
    static int per_sm = 0;
    if (per_sm == 0) {
        int b = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, wed_combine_kernel, kCmbThreads, 0) !=
                cudaSuccess || b < 1)
            b = 1;
        per_sm = b;
    }
    const size_t n_tiles = (nvox + kCmbTile - 1) / kCmbTile;
    const int blocks = (int)std::min<size_t>(n_tiles, (size_t)num_sms() * per_sm);
    wed_combine_kernel<<<std::max(blocks, 1), kCmbThreads, 0, st>>>(dm, w.scal, pts, lateral,
                                                                    lstride, wed, nvox, n_layers,
                                                                    dose, err);
    PBD_LAUNCH_CHECK();
    const int pb = (int)std::min<size_t>((nvox + 255) / 256, (size_t)num_sms() * 4);
    wed_poison_kernel<<<std::max(pb, 1), 256, 0, st>>>(dose, nvox, err, err2);
    PBD_LAUNCH_CHECK();
    count_launch(2);
    return PBD_OK;
}

int lut_wed_grad_maps(const pbd_lut_spec* s, int n_layers, const void* curves,
                      size_t curves_bytes, const float* grad, const double* wed, size_t nvox,
                      size_t lstride, float* maps, cudaStream_t st) {
    PBD_TRY(validate_spec(s, n_layers));
    if (!grad || !wed || !maps) return PBD_ERR_NULL_ARG;
    if (lstride < nvox) return PBD_ERR_BAD_VALUE;
    LutDims dm;
    LutWs w;
    double2* pts = nullptr;
    PBD_TRY(wed_dims(s, n_layers, curves, curves_bytes, dm, w, pts));
    const int blocks = (int)std::min<size_t>((nvox + 255) / 256, (size_t)num_sms() * 8);
    wed_grad_maps_kernel<<<std::max(blocks, 1), 256, 0, st>>>(dm, w.scal, pts, grad, wed, nvox,
                                                              n_layers, lstride, maps);
    PBD_LAUNCH_CHECK();
    count_launch(1);
    return PBD_OK;
}

int lut_wed_grad_maps_dr(const pbd_lut_spec* s, int n_layers, const void* curves_p,
                         size_t curves_p_bytes, const void* curves_m, size_t curves_m_bytes,
                         double h, const float* grad, const double* wed, size_t nvox,
                         size_t lstride, float* maps, cudaStream_t st) {
    PBD_TRY(validate_spec(s, n_layers));
    if (!grad || !wed || !maps || !curves_p || !curves_m) return PBD_ERR_NULL_ARG;
    if (lstride < nvox) return PBD_ERR_BAD_VALUE;
    if (!(h > 0.0) || !isfinite(h)) return PBD_ERR_BAD_VALUE;
    LutDims dp, dmm;
    LutWs wp, wm;
    double2* pp = nullptr;
    double2* pm = nullptr;
    PBD_TRY(wed_dims(s, n_layers, curves_p, curves_p_bytes, dp, wp, pp));
    PBD_TRY(wed_dims(s, n_layers, curves_m, curves_m_bytes, dmm, wm, pm));
    const int blocks = (int)std::min<size_t>((nvox + 255) / 256, (size_t)num_sms() * 8);
    wed_grad_maps_dr_kernel<<<std::max(blocks, 1), 256, 0, st>>>(dp, wp.scal, pp, wm.scal, pm, grad,
                                                                 wed, nvox, n_layers, lstride,
                                                                 0.5 / h, maps);
    PBD_LAUNCH_CHECK();
    count_launch(1);
    return PBD_OK;
}

int lut_wed_raytrace(int nz, int ny, int nx, double oz, double dz, const float* rho, double* wed,
                     cudaStream_t st) {
    if (!rho || !wed) return PBD_ERR_NULL_ARG;
    if (nz <= 0 || ny <= 0 || nx <= 0) return PBD_ERR_BAD_DIM;
    if (!isfinite(oz) || !(dz > 0.0) || !isfinite(dz)) return PBD_ERR_BAD_VALUE;
    const size_t ncol = (size_t)ny * nx;
    const int blocks = (int)std::min<size_t>((ncol + kRayThreads - 1) / kRayThreads,
                                             (size_t)num_sms() * 32);
    wed_raytrace_kernel<<<std::max(blocks, 1), kRayThreads, 0, st>>>(nz, ncol, oz, dz, rho, wed);
    PBD_LAUNCH_CHECK();
    count_launch(1);
    return PBD_OK;
}

int lut_csda(const double* e, double* r, int n, int inverse, cudaStream_t st) {
    if (!e || !r) return PBD_ERR_NULL_ARG;
    if (n < 0) return PBD_ERR_BAD_DIM;
    PBD_TRY(ensure_range_table(st));
    if (n == 0) return PBD_OK;
    csda_kernel<<<(n + 255) / 256, 256, 0, st>>>(e, r, n, inverse);
    PBD_LAUNCH_CHECK();
    count_launch(1);
    return PBD_OK;
}

}  // namespace pbd
