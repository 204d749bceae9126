// optim.cu -- on-device steps of a plan-optimisation loop: a projected Adam update of a
// parameter vector (spot weights, per-layer range shifts) and the combination of the
// scenario gradients of a robust objective.  No counterpart in the reference, which
// computes dose only; these are the callers that consume the adjoint.
//
// Both kernels keep all of their state on the device (moments, step count, loss history),
// so a whole iteration -- tables, loss gradient, combination, update -- can be captured
// into one CUDA graph and replayed without host work.
//
// Arithmetic: Adam as in Kingma & Ba, "Adam: A Method for Stochastic Optimization"
// (ICLR 2015), Algorithm 1, in FP32 with every product and sum rounded separately
// (__fmul_rn / __fadd_rn: no contraction into FMA), IEEE division and square root, and
// the bias corrections 1 - beta^t formed in FP64 and rounded once to FP32; the result is
// then projected onto the box [lo, hi].  The same sequence of FP32 roundings in NumPy
// reproduces it bit for bit.
#include "pbd_internal.cuh"

namespace pbd {
namespace {

constexpr int kOptThreads = 256;
constexpr int kOptPer = 4;          // elements per thread
constexpr int kCombThreads = 256;

__global__ void __launch_bounds__(kOptThreads)
adam_kernel(pbd_adam_params p, int n, float* __restrict__ x, float* __restrict__ m,
            float* __restrict__ v, const float* __restrict__ g, int* __restrict__ state,
            double* __restrict__ x64, const double* __restrict__ loss, double* __restrict__ hist,
            int hist_len) {
    // state[0]: completed steps; state[1]: blocks of this launch that have finished
    const int t = __ldcg(state) + 1;
    const float b1 = p.beta1, b2 = p.beta2;
    const float bc1 = (float)(1.0 - pow((double)b1, (double)t));
    const float bc2 = (float)(1.0 - pow((double)b2, (double)t));
    const float omb1 = __fsub_rn(1.0f, b1), omb2 = __fsub_rn(1.0f, b2);
    const int base = blockIdx.x * (kOptThreads * kOptPer) + threadIdx.x;
#pragma unroll
    for (int k = 0; k < kOptPer; ++k) {
        const int i = base + k * kOptThreads;
        if (i >= n) break;
        const float gi = __fmul_rn(g[i], p.grad_scale);
        const float mi = __fadd_rn(__fmul_rn(b1, m[i]), __fmul_rn(omb1, gi));
        const float vi = __fadd_rn(__fmul_rn(b2, v[i]), __fmul_rn(omb2, __fmul_rn(gi, gi)));
        const float mh = __fdiv_rn(mi, bc1);
        const float vh = __fdiv_rn(vi, bc2);
        const float upd = __fdiv_rn(mh, __fadd_rn(__fsqrt_rn(vh), p.eps));
        float xi = __fsub_rn(x[i], __fmul_rn(p.lr, upd));
        xi = xi < p.lo ? p.lo : (xi > p.hi ? p.hi : xi);   // a NaN stays NaN
        m[i] = mi;
        v[i] = vi;
        x[i] = xi;
        if (x64) x64[i] = (double)xi;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0 && hist && loss && t <= hist_len) hist[t - 1] = *loss;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const int done = atomicAdd(state + 1, 1);
        if (done == (int)gridDim.x - 1) {     // last block: every block has read state[0]
            state[0] = t;
            state[1] = 0;
            __threadfence();
        }
    }
}

// Robust objective over S scenarios of one field.  Every block finds the selected
// scenario itself from the S losses (S <= PBD_MAX_JOBS), in index order.
__global__ void __launch_bounds__(kCombThreads)
combine_kernel(int mode, int n_scen, int n, const float* __restrict__ grads,
               const double* __restrict__ losses, float* __restrict__ out,
               double* __restrict__ out_loss) {
    int sel = 0;
    if (mode == PBD_OBJ_MAX) {
        double best = losses[0];
        for (int s = 1; s < n_scen; ++s) {
            const double ls = losses[s];
            if (ls > best) { best = ls; sel = s; }   // first index wins ties
        }
    }
    const int i = blockIdx.x * kCombThreads + threadIdx.x;
    if (i < n) {
        if (mode == PBD_OBJ_MAX) {
            out[i] = grads[(size_t)sel * n + i];
        } else {
            float acc = 0.f;
            for (int s = 0; s < n_scen; ++s) acc = __fadd_rn(acc, grads[(size_t)s * n + i]);
            out[i] = __fdiv_rn(acc, (float)n_scen);
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0 && out_loss) {
        if (mode == PBD_OBJ_MAX) {
            *out_loss = losses[sel];
        } else {
            double acc = 0.0;
            for (int s = 0; s < n_scen; ++s) acc += losses[s];
            *out_loss = acc / n_scen;
        }
    }
}

bool finite(float a) { return a == a && a - a == 0.f; }

}  // namespace
}  // namespace pbd

using namespace pbd;

int pbd_adam_step(const pbd_adam_params* p, int n, float* x, float* m, float* v, const float* grad,
                  int* state, double* x64, const double* loss, double* loss_hist, int hist_len,
                  void* stream) {
    if (!p || !state) return PBD_ERR_NULL_ARG;
    if (n < 0 || hist_len < 0) return PBD_ERR_BAD_DIM;
    if (n > 0 && (!x || !m || !v || !grad)) return PBD_ERR_NULL_ARG;
    if (hist_len > 0 && (!loss_hist || !loss)) return PBD_ERR_NULL_ARG;
    if (!finite(p->lr) || !(p->lr >= 0.f) || !(p->beta1 >= 0.f && p->beta1 < 1.f) ||
        !(p->beta2 >= 0.f && p->beta2 < 1.f) || !finite(p->eps) || !(p->eps > 0.f) ||
        !finite(p->grad_scale) || p->lo != p->lo || p->hi != p->hi || p->lo > p->hi)
        return PBD_ERR_BAD_VALUE;
    if (n == 0) return PBD_OK;
    const int blocks = (n + kOptThreads * kOptPer - 1) / (kOptThreads * kOptPer);
    adam_kernel<<<blocks, kOptThreads, 0, (cudaStream_t)stream>>>(
        *p, n, x, m, v, grad, state, x64, loss, hist_len > 0 ? loss_hist : nullptr, hist_len);
    PBD_LAUNCH_CHECK();
    count_launch(1);
    return PBD_OK;
}

int pbd_scenario_combine(int mode, int n_scen, int n, const float* grads, const double* losses,
                         float* out_grad, double* out_loss, void* stream) {
    if (!losses) return PBD_ERR_NULL_ARG;
    if (mode != PBD_OBJ_MEAN && mode != PBD_OBJ_MAX) return PBD_ERR_BAD_VALUE;
    if (n_scen < 1 || n_scen > PBD_MAX_JOBS || n < 0) return PBD_ERR_BAD_DIM;
    if (n > 0 && (!grads || !out_grad)) return PBD_ERR_NULL_ARG;
    if (n == 0 && !out_loss) return PBD_OK;
    const int blocks = n > 0 ? (n + kCombThreads - 1) / kCombThreads : 1;
    combine_kernel<<<blocks, kCombThreads, 0, (cudaStream_t)stream>>>(mode, n_scen, n, grads,
                                                                      losses, out_grad, out_loss);
    PBD_LAUNCH_CHECK();
    count_launch(1);
    return PBD_OK;
}
