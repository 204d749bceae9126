/*
 * pbdose_b200.h -- C ABI of the B200 (sm_100a) separable proton pencil-beam dose engine.
 *
 * Dose model (per-energy-layer exact separable pencil beam, water):
 *
 *   D[z,y,x] = sum_l IDD_l(z) * sum_{j,i} Gy_l(z)[y,j] * W_l[j,i] * Gx_l(z)[x,i]
 *   Gx_l(z)[x,i] = exp(-(x_v - xs_i)^2 / (2 s^2)) / (sqrt(2 pi) s),  s = sigma_l(z)
 *
 * Conventions (the same as the reference's Python engine, engines.py:208-283):
 *   - dose is (nz, ny, nx), x innermost; voxel centres x_v = ox + k*dx (model.py:7-9, 48-52);
 *   - weights are (L, nsy, nsx) float32; spot centres xs_i = x0 + (i - (nsx-1)/2)*dx_spot
 *     (model.py:106-113);
 *   - depth tables idd, sigma are (L, nz) float64, row l = energy layer, column k = voxel
 *     slice k (model.py:137-151).
 *
 * Every entry point validates its arguments first, returns 0 (PBD_OK) or a negative
 * PBD_ERR_* code readable with pbd_strerror(), never exits the process and never throws
 * across the ABI (the reference's ABI rules, pencil_beam.cu:647-730).  All array pointers
 * are DEVICE pointers unless stated otherwise.  Work is enqueued on `stream` (a
 * cudaStream_t passed as void*; NULL = legacy default stream) and is asynchronous: the
 * caller synchronises.  The caller owns all memory; scratch comes from the caller's
 * `workspace`, sized by the matching *_workspace() query; a workspace needs no particular
 * alignment (the library starts each of its sub-arrays on a 256-byte address boundary inside
 * it, and the queries include the slack for that).
 */
#ifndef PBDOSE_B200_H
#define PBDOSE_B200_H

#include <stddef.h>

#if defined(__GNUC__)
#define PBD_API __attribute__((visibility("default")))
#else
#define PBD_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* Error codes; pencil_beam.cu:647-653.  The values the reference defines keep their meaning
 * (-3, its z-grid mismatch, cannot occur here: tables are built at the grid's depths);
 * new codes start at -7. */
#define PBD_OK                0
#define PBD_ERR_NULL_ARG     -1
#define PBD_ERR_BAD_DIM      -2
#define PBD_ERR_BAD_VALUE   -10   /* non-finite or out-of-range value (spacing, step, mode) */
#define PBD_ERR_CUDA         -4
#define PBD_ERR_UNSUPPORTED  -5
#define PBD_ERR_NO_SMEM      -6
#define PBD_ERR_WORKSPACE    -7   /* workspace missing or smaller than the query result */
#define PBD_ERR_TIMEOUT      -8   /* a bounded device-side wait ran out; results invalid */
#define PBD_ERR_TOO_MANY     -9   /* more jobs than PBD_MAX_JOBS in one launch */

/* Arithmetic used for the two Gaussian contractions.  All accumulate in FP32. */
#define PBD_PREC_FP32    0   /* FP32 FMA on the CUDA cores */
#define PBD_PREC_TF32X3  1   /* tcgen05 TF32, hi/lo split, three products */
#define PBD_PREC_TF32    2   /* tcgen05 TF32, one product */
#define PBD_PREC_BF16X3  3   /* tcgen05 BF16, hi/lo split, three products */
#define PBD_PREC_BF16    4   /* tcgen05 BF16, one product */
#define PBD_PREC_FP16X3  5   /* tcgen05 FP16, hi/lo split, three products; operands scaled by
                                powers of two into FP16's range */

#define PBD_MAX_JOBS 128     /* jobs (fields x scenarios) per batched launch */

/* One field: dose grid (DoseGrid, model.py:27-38) + spot lattice (SpotLattice,
 * model.py:85-100).  Host memory, read during the call only. */
typedef struct pbd_field {
    int nx, ny, nz;
    double dx, dy, dz;
    double ox, oy, oz;
    int n_sx, n_sy, n_layers;
    double dx_spot, dy_spot;
    double x0, y0;
} pbd_field;

/* Parameters of the depth-LUT builder (physics.py:221-387 with the defaults of
 * IDDModel, physics.py:292-308, and fermi_eyges_moments).  The tables are built at the
 * water-equivalent depths d_k = depth_scale * (z0 + k*dz), k < nz.  depth_scale = 1 and
 * z0 = the grid's oz give exactly the reference's tables; other values model a
 * depth shift (z0 = oz - shift) or a stopping-power scaling (depth_scale = s, in which
 * case B is divided by s^2 to return to physical lateral units). */
typedef struct pbd_lut_spec {
    int nz;
    double z0, dz, depth_scale;
    int anchor_surface;                    /* 0: scattering integral starts at the first depth
                                              (reference semantics); 1: starts at depth 0 and
                                              depths <= 0 get sigma_x0 and IDD 0 */
    double sigma_x0, sigma_theta0, rho0;   /* initial beam phase space, cm / rad */
    int fe_n_sub;                          /* fine-grid subdivision (4) */
    double fe_max_step;                    /* fine-grid max step, cm (0.02) */
    int straggling_model;                  /* 0 bohr, 1 icru49, 2 none */
    double strag_coef, strag_exp;          /* icru49: coef * R0^exp */
    double energy_spread;                  /* relative 1-sigma (0.0033) */
    double atten_len;                      /* nuclear attenuation length, cm (150) */
    int idd_n_fine;                        /* CSDA binning points (6000) */
    double fd_step;                        /* range step of the derivative tables, cm; 0 = none */
} pbd_lut_spec;

/* One job of a batched launch: a field, its device arrays and its outputs. */
typedef struct pbd_job {
    pbd_field field;
    const float *w;          /* (L, nsy, nsx) */
    const double *idd;       /* (L, nz) */
    const double *sigma;     /* (L, nz) */
    float *dose;             /* (nz, ny, nx) out */
} pbd_job;

/* ---- utilities --------------------------------------------------------------- */
/* Replaces pb_strerror, pencil_beam.cu:687-699. Never NULL. */
PBD_API const char *pbd_strerror(int code);
/* ABI version, major*10000 + minor*100 + patch. */
PBD_API int pbd_version(void);
/* Validates a field descriptor; replaces pb_problem_validate, pencil_beam.cu:717-730. */
PBD_API int pbd_field_validate(const pbd_field *f);
/* Work-item granularity of the calling host thread's subsequent calls (0 = built-in
 * default): energy layers per forward item, depth slices per adjoint item.  The setting is
 * per host thread (calls from other threads keep their own), and the workspace queries use
 * it too, so set it before sizing.  No counterpart in the reference (it plays the role of
 * engines.torch_separable's layer_chunk knob). */
PBD_API int pbd_set_schedule(int fwd_layers_per_item, int adj_depths_per_item);
/* Measurement utilities (no counterpart in the reference).  Between begin and end, the
 * calling thread's forward and adjoint calls record CUDA events around their main dose
 * kernel; end() waits for them and returns the summed kernel time (ms) and the number
 * of launches of each.  Not for use inside stream capture. */
PBD_API int pbd_profile_begin(void);
PBD_API int pbd_profile_end(double *fwd_ms, int *n_fwd, double *adj_ms, int *n_adj);
/* Number of kernels this library has launched from the calling thread so far. */
PBD_API int pbd_launch_count(long long *n);

/* Status of the last call that used `workspace` (no counterpart in the reference, whose
 * kernels never wait on one another).  The kernels' waits on each other are bounded (2 s);
 * a wait that runs out makes the call's results NaN and sets a status word at the start of
 * its workspace.  This reads those words on `stream`, waits for the stream, and stores
 * PBD_OK or PBD_ERR_TIMEOUT in *status.  Valid after pbd_forward, pbd_adjoint, pbd_loss_grad,
 * pbd_forward_batch, pbd_loss_grad_batch, pbd_forward_wed(_curves) and pbd_adjoint_wed(_range); not
 * for use inside stream capture. */
PBD_API int pbd_workspace_status(const void *workspace, size_t workspace_bytes, int *status,
                                 void *stream);
/* Test hook of the timeout path (no counterpart in the reference).  For the calling thread's
 * later calls: wait_limit_ns bounds every device wait of the tensor-core forward and adjoint
 * (0 = the default 2 s), and hold_schedulers = 1 makes their scheduler warps publish no work,
 * so that every other warp's first wait runs out after wait_limit_ns (which must then be
 * non-zero) -- no tensor-core instruction is issued, the kernels end, the outputs are NaN and
 * pbd_workspace_status reports PBD_ERR_TIMEOUT.  pbd_test_hook(0, 0) restores the defaults. */
PBD_API int pbd_test_hook(unsigned long long wait_limit_ns, int hold_schedulers);

/* ---- depth-LUT builder (FP64, on the device) -------------------------------------
 * Replaces the per-layer host loop of model.py:225-233 (physics.idd_pristine with
 * normalize=False and physics.fermi_eyges_moments(...)["sigma_x"]).
 * energies: (L) MeV; range_shift: (L) cm or NULL (layer l is built at the CSDA range
 * R0_l + range_shift_l); outputs idd, sigma (L, nz); didd_dr, dsigma_dr (L, nz) central
 * differences in range with step spec->fd_step (may be NULL when fd_step == 0). */
PBD_API int pbd_lut_workspace(const pbd_lut_spec *spec, int n_layers, size_t *bytes);
PBD_API int pbd_build_luts(const pbd_lut_spec *spec, int n_layers, const double *energies,
                   const double *range_shift, double *idd, double *sigma,
                   double *didd_dr, double *dsigma_dr,
                   void *workspace, size_t workspace_bytes, void *stream);
/* CSDA range table lookups (physics.py:130-139), elementwise on device arrays. */
PBD_API int pbd_csda_range(const double *energy, double *range_cm, int n, void *stream);
PBD_API int pbd_energy_from_range(const double *range_cm, double *energy, int n, void *stream);

/* ---- forward dose -----------------------------------------------------------------
 * Replaces engines.torch_separable(per_layer=True), engines.py:208-283, and the
 * reference ABI's pb_dose_forward_separable, pencil_beam.cu:799-851. */
PBD_API int pbd_forward_workspace(const pbd_field *f, int precision, size_t *bytes);
PBD_API int pbd_forward(const pbd_field *f, const float *w, const double *idd, const double *sigma,
                float *dose, int precision, void *workspace, size_t workspace_bytes,
                void *stream);

/* ---- forward dose in FP64 ----------------------------------------------------------
 * Replaces engines.torch_separable(..., dtype=torch.float64) on CUDA, engines.py:223-224 and
 * 230-274 (operands and both batched matmuls in float64).  The dose of pbd_forward with the
 * weights, Gaussians, products and sums in float64 on the CUDA cores: w (L, nsy, nsx) and
 * dose (nz, ny, nx) are float64.  No workspace: one block per (64 x 64 voxel tile, slice) sums
 * every layer in layer order and writes its voxels once. */
PBD_API int pbd_forward_f64(const pbd_field *f, const double *w, const double *idd,
                            const double *sigma, double *dose, void *stream);

/* ---- forward dose without any device allocation ----------------------------------
 * No counterpart in the reference.  For callers that cannot allocate device memory: a
 * real-time adaptive-therapy loop that reserves its memory once at start-up and must not
 * block or fail on an allocation mid-treatment, or a host that owns the GPU through its
 * own memory pool.  Same inputs and output as pbd_forward, but no workspace argument:
 * the scratch is a fixed 1 MiB array inside the library (held by every GPU that loads
 * it, until exit).  Limits: n_layers <= 64 and nz * ceil(nx/128) * ceil(ny/128) work
 * items must fit the 1 MiB (about 32,000 items); otherwise PBD_ERR_UNSUPPORTED or
 * PBD_ERR_WORKSPACE.  The first call on a device resolves the array's device address,
 * so make it before any stream capture.  Calls share the array: two calls that overlap
 * on the GPU race, so order them (same stream) or do not overlap them.  The resolved address
 * belongs to the device's primary context: after cudaDeviceReset(), or from a context the
 * caller created through the driver API, this entry point must not be used on that device. */
PBD_API int pbd_forward_noalloc(const pbd_field *f, const float *w, const double *idd,
                                const double *sigma, float *dose, int precision, void *stream);

/* ---- adjoint (no counterpart in the reference, which has no gradient) --------------
 * Given grad_dose = dL/dD (nz, ny, nx), writes grad_w = dL/dW (L, nsy, nsx) and
 * grad_range = dL/d(range shift) (L), the latter through didd_dr and dsigma_dr
 * (either may be NULL together with grad_range == NULL to skip it). */
PBD_API int pbd_adjoint_workspace(const pbd_field *f, int precision, size_t *bytes);
PBD_API int pbd_adjoint(const pbd_field *f, const float *w, const double *idd, const double *sigma,
                const double *didd_dr, const double *dsigma_dr, const float *grad_dose,
                float *grad_w, float *grad_range, int precision,
                void *workspace, size_t workspace_bytes, void *stream);

/* ---- fused plan-loss gradient evaluation --------------------------------------------
 * L = sum_v mask_v (D_v - presc_v)^2.  Writes dose, grad_dose = 2 mask (D - presc),
 * loss (device float64 scalar), grad_w and grad_range, in one call. */
PBD_API int pbd_loss_grad_workspace(const pbd_field *f, int precision, size_t *bytes);
PBD_API int pbd_loss_grad(const pbd_field *f, const float *w, const double *idd, const double *sigma,
                  const double *didd_dr, const double *dsigma_dr,
                  const float *mask, const float *presc,
                  float *dose, float *grad_dose, double *loss, float *grad_w, float *grad_range,
                  int precision, void *workspace, size_t workspace_bytes, void *stream);

/* ---- batched forward: several fields / scenarios in one persistent launch ----------
 * jobs: HOST array of n_jobs <= PBD_MAX_JOBS descriptors (copied into the launch's
 * parameters; may be freed on return). */
PBD_API int pbd_forward_batch_workspace(const pbd_job *jobs, int n_jobs, int precision, size_t *bytes);
PBD_API int pbd_forward_batch(const pbd_job *jobs, int n_jobs, int precision,
                      void *workspace, size_t workspace_bytes, void *stream);

/* ---- batched loss gradient: several fields / scenarios in one forward and one adjoint ----
 * No counterpart in the reference.  Each job has its own field, tables, loss arrays and
 * outputs, with the meaning they have in pbd_loss_grad; all jobs' forwards (with the fused
 * loss) run in one persistent launch and all adjoints in another.  Tensor-core precisions
 * only (PBD_ERR_UNSUPPORTED for PBD_PREC_FP32); grad_range (with didd_dr, dsigma_dr) on every
 * job or on none.  jobs: HOST array of n_jobs <= PBD_MAX_JOBS descriptors. */
typedef struct pbd_grad_job {
    pbd_field field;
    const float *w;
    const double *idd, *sigma, *didd_dr, *dsigma_dr;
    const float *mask, *presc;
    float *dose, *grad_dose;
    double *loss;
    float *grad_w, *grad_range;
} pbd_grad_job;
PBD_API int pbd_loss_grad_batch_workspace(const pbd_grad_job *jobs, int n_jobs, int precision,
                                          size_t *bytes);
PBD_API int pbd_loss_grad_batch(const pbd_grad_job *jobs, int n_jobs, int precision,
                                void *workspace, size_t workspace_bytes, void *stream);

/* ---- heterogeneous media: water-equivalent depth (WED) -----------------------------
 * The reference has a stub, physics.wed_from_density_path (physics.py:421-423: WED = sum of
 * rho * L), and lists heterogeneous media as not implemented.
 * pbd_wed_raytrace: WED at every voxel centre z_k = oz + k dz along the beam axis (+z),
 * through the relative stopping-power map rho (nz, ny, nx, float32): the sum of rho * path
 * length from depth 0, voxel k filling [z_k - dz/2, z_k + dz/2], water above the first voxel,
 * lengths clipped at depth 0; wed (nz, ny, nx) float64.  rho = 1 gives WED = max(z, 0).
 * pbd_forward_wed: the dose with every layer's depth dose evaluated at the voxel's WED
 * instead of its depth -- the same curve and interpolation as the depth tables --
 *   D[z,y,x] = sum_l IDD_l(WED[z,y,x]) * sum_{j,i} Gy_l(z)[y,j] W_l[j,i] Gx_l(z)[x,i]
 * with the lateral widths sigma (L, nz) of water at the geometric depth (the tables of
 * pbd_build_luts).  spec / energies / range_shift: as for pbd_build_luts.  The per-layer
 * lateral maps come from one launch of the tensor-core forward that writes every layer's map
 * (PBD_PREC_FP32: single-layer jobs of the batched forward).
 * pbd_build_wed_curves: the per-layer smoothed depth curves and their interval slopes, built
 * once into an opaque device blob of pbd_wed_curves_workspace bytes; pbd_forward_wed_curves
 * computes the dose from such a blob (built with the same spec and n_layers) without
 * rebuilding it; pbd_forward_wed builds the curves inside its workspace on every call.  Both
 * forwards take a workspace of pbd_forward_wed_workspace bytes. */
PBD_API int pbd_wed_raytrace(int nz, int ny, int nx, double oz, double dz, const float *rho,
                             double *wed, void *stream);
PBD_API int pbd_forward_wed_workspace(const pbd_field *f, const pbd_lut_spec *spec, int precision,
                                      size_t *bytes);
PBD_API int pbd_forward_wed(const pbd_field *f, const pbd_lut_spec *spec, const double *energies,
                            const double *range_shift, const float *w, const double *sigma,
                            const double *wed, float *dose, int precision, void *workspace,
                            size_t workspace_bytes, void *stream);
PBD_API int pbd_wed_curves_workspace(const pbd_lut_spec *spec, int n_layers, size_t *bytes);
PBD_API int pbd_build_wed_curves(const pbd_lut_spec *spec, int n_layers, const double *energies,
                                 const double *range_shift, void *curves, size_t curves_bytes,
                                 void *stream);
PBD_API int pbd_forward_wed_curves(const pbd_field *f, const pbd_lut_spec *spec,
                                   const void *curves, size_t curves_bytes, const float *w,
                                   const double *sigma, const double *wed, float *dose,
                                   int precision, void *workspace, size_t workspace_bytes,
                                   void *stream);

/* dL/dW of the heterogeneous dose for a given dL/dD (grad_dose, (nz, ny, nx) float32):
 * grad_w (L, nsy, nsx) float32, sum over voxels of grad_dose * IDD_l(WED) * dLateral_l/dW_l --
 * the adjoint of pbd_forward_wed_curves (same field, spec, curve blob, w, sigma, wed).  No
 * counterpart in the reference.  Per layer: dL/dD times the layer's depth dose at the WED,
 * then the layer's adjoint (the kernels of pbd_adjoint; on the tensor cores one launch over
 * every layer). */
PBD_API int pbd_adjoint_wed_workspace(const pbd_field *f, const pbd_lut_spec *spec, int precision,
                                      size_t *bytes);
PBD_API int pbd_adjoint_wed(const pbd_field *f, const pbd_lut_spec *spec, const void *curves,
                            size_t curves_bytes, const float *w, const double *sigma,
                            const double *wed, const float *grad_dose, float *grad_w,
                            int precision, void *workspace, size_t workspace_bytes, void *stream);

/* dL/dW and dL/d(range shift) of the heterogeneous dose for a given dL/dD: grad_w as
 * pbd_adjoint_wed, grad_range (L) float32.  No counterpart in the reference (its only
 * heterogeneous code is the WED stub, physics.py:421-423).  A range shift moves each layer's
 * depth curve and its water widths: dL/dR_l = sum_v g IDD'_l(WED) Lat_l + sum_z dL/dsigma_lz
 * dsigma_lz/dR, with IDD'_l the central difference (curves_p - curves_m) / (2 h) of the layer's
 * curves built by pbd_build_wed_curves at range shifts +h and -h (same spec, energies and
 * blob size as `curves`), and dsigma_dr (L, nz) float64 the widths' range derivative
 * (pbd_build_luts with fd_step = h).  Both terms come from one adjoint launch on the tensor
 * cores (FP32: one SIMT adjoint per layer and term). */
PBD_API int pbd_adjoint_wed_range_workspace(const pbd_field *f, const pbd_lut_spec *spec,
                                            int precision, size_t *bytes);
PBD_API int pbd_adjoint_wed_range(const pbd_field *f, const pbd_lut_spec *spec,
                                  const void *curves, size_t curves_bytes, const void *curves_p,
                                  const void *curves_m, double h, const float *w,
                                  const double *sigma, const double *dsigma_dr, const double *wed,
                                  const float *grad_dose, float *grad_w, float *grad_range,
                                  int precision, void *workspace, size_t workspace_bytes,
                                  void *stream);

/* ---- plan-optimisation steps (no counterpart in the reference) ---------------------
 * Device-resident state, so that an optimisation iteration (tables, loss gradient,
 * combination, update) can be captured into one CUDA graph and replayed. */

/* Projected Adam (Kingma & Ba 2015, Algorithm 1) in FP32:
 *   g' = grad_scale * g;  m = b1 m + (1-b1) g';  v = b2 v + (1-b2) g'^2;
 *   x = clamp(x - lr * (m / (1-b1^t)) / (sqrt(v / (1-b2^t)) + eps), lo, hi)
 * with t = state[0] + 1.  state: device int[2], zero before the first step; state[0] counts
 * completed steps (the call increments it), state[1] is scratch and stays 0 between calls.
 * n == 0 enqueues nothing (x, m, v, grad may then be NULL; the count does not advance).
 * x64 (may be NULL) receives a float64 copy of x (e.g. the range shifts the LUT builder
 * reads).  If hist_len > 0, the value at `loss` (a device float64 scalar, the loss of the
 * gradient being applied) is stored at loss_hist[t-1] for t <= hist_len. */
typedef struct pbd_adam_params {
    float lr, beta1, beta2, eps;
    float lo, hi;          /* projection box; -inf / +inf for none */
    float grad_scale;      /* multiplies the gradient before the update */
} pbd_adam_params;
PBD_API int pbd_adam_step(const pbd_adam_params *p, int n, float *x, float *m, float *v,
                          const float *grad, int *state, double *x64, const double *loss,
                          double *loss_hist, int hist_len, void *stream);

/* Robust objective over n_scen scenarios of one field: grads is (n_scen, n), losses
 * (n_scen) float64.  PBD_OBJ_MEAN: out_grad = (sum_s grads[s]) / n_scen in scenario order,
 * out_loss = mean loss.  PBD_OBJ_MAX (min-max): the scenario with the largest loss (the
 * first on ties) gives out_grad and out_loss.  out_loss may be NULL. */
#define PBD_OBJ_MEAN 0
#define PBD_OBJ_MAX  1
PBD_API int pbd_scenario_combine(int mode, int n_scen, int n, const float *grads,
                                 const double *losses, float *out_grad, double *out_loss,
                                 void *stream);

/* ---- gamma index (replaces gamma.py:41-60 dta_offsets, 81-160 gamma_index and 213-261
 * gamma_index_torch) -------------------------------------------------------------------------
 *   gamma(r)^2 = min over integer voxel offsets o, |o| <= DTA (at most max_vox voxels per axis),
 *                of (|o|/DTA)^2 + ((E[r+o] - R[r]) / dose_crit(r))^2,   E = 0 outside the grid
 *   dose_crit = pct/100 * ref_max (global) or pct/100 * max(R[r], 1e-12) (local)
 *   mask = R >= threshold_pct/100 * ref_max, or R > 0 when that mask is empty
 *   ref_max = max(R), or ref_dose when use_ref_dose.
 * Computed in float64 with the reference's order of operations: the gamma map, mask, counts,
 * maximum and the NumPy-'linear' 95th / 99th percentiles equal the reference's float64
 * results; the mean is a fixed-order sum.  reference / evaluation: (nz, ny, nx) device arrays
 * of `dtype`; gamma_map (float64) and mask_map (0/1 bytes) may be NULL; `stats` is a DEVICE
 * pointer, written at the end of the call (status = PBD_ERR_BAD_VALUE when ref_max <= 0 or no
 * voxel is evaluated, as gamma.py:112-113 raises). */
#define PBD_GAMMA_GLOBAL 0
#define PBD_GAMMA_LOCAL  1
#define PBD_DTYPE_F32 0
#define PBD_DTYPE_F64 1
typedef struct pbd_gamma_spec {
    double dz, dy, dx;          /* voxel spacing, cm */
    double dose_crit_pct;       /* 3.0 = 3 % */
    double dta_mm;
    double threshold_pct;       /* low-dose threshold, % of ref_max */
    int normalization;          /* PBD_GAMMA_GLOBAL or PBD_GAMMA_LOCAL */
    int use_ref_dose;           /* 1: ref_max = ref_dose */
    double ref_dose;
    int max_vox;                /* search radius cap per axis, 0..6 (the reference uses 6) */
} pbd_gamma_spec;
typedef struct pbd_gamma_stats {
    double pass_rate, gamma_mean, gamma_max, gamma_p95, gamma_p99, ref_max;
    long long n_eval, n_pass;
    int n_dta_offsets;
    int mask_fallback;          /* 1: the statistics used R > 0 */
    int status;
    int reserved;
} pbd_gamma_stats;
/* Host only: the search offsets of a spec (count, radii z/y/x, and the weights (|o|/DTA)^2
 * as a 7x7x7 table over (|a|, |b|, |c|), -1 outside the ball); radii / weights may be NULL. */
PBD_API int pbd_gamma_offsets(const pbd_gamma_spec *spec, int *n_offsets, int *radii,
                              double *weights);
PBD_API int pbd_gamma_workspace(int nz, int ny, int nx, size_t *bytes);
PBD_API int pbd_gamma_index(const pbd_gamma_spec *spec, int nz, int ny, int nx,
                            const void *reference, const void *evaluation, int dtype,
                            double *gamma_map, unsigned char *mask_map, pbd_gamma_stats *stats,
                            void *workspace, size_t workspace_bytes, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* PBDOSE_B200_H */
