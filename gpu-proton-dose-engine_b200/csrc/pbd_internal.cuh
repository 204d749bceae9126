// Internal declarations shared by the CUDA translation units of libpbdose_b200.so.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "../../include/pbdose_b200.h"

namespace pbd {

constexpr double kInvSqrt2Pi = 0.39894228040143267794;   // 1/sqrt(2 pi)
constexpr double kInv2Pi = 0.15915494309189533577;       // 1/(2 pi)
constexpr double kLog2e = 1.44269504088896340736;

// ---------------------------------------------------------------------------
// Device-side view of one job (field x scenario).  Written into the workspace by
// the scheduling kernels from the launch parameters, read by the compute kernels.
// ---------------------------------------------------------------------------
struct JobDev {
    int nx, ny, nz, nsx, nsy, nl;
    int ntx, nty;                 // lateral tiles of 128 x 128 voxels
    int max_chunks;               // forward: layer chunks per depth slice; adjoint: z chunks per layer
    int item_base, max_items;     // slice of the flat item array owned by this job
    int n_loss_part;              // loss partial sums written by the forward (summed in order)
    double ox, oy, dx, dy;        // voxel centres x = ox + k dx
    double sx0, sy0, dsx, dsy;    // spot centres xs = sx0 + (i - (nsx-1)/2) dsx
    const float* w;               // (nl, nsy, nsx)
    const double* idd;            // (nl, nz)
    const double* sigma;          // (nl, nz)
    const double* didd_dr;        // (nl, nz) or null
    const double* dsig_dr;        // (nl, nz) or null
    float* dose;                  // (nz, ny, nx)
    float* partial;               // forward: (max_chunks, nz, ny, nx); adjoint: (nl, max_chunks, nsy, nsx)
    int* nchunks;                 // forward: (nz); adjoint: (nl)
    int* arrive;                  // tensor-core forward: chunks of each (slice, tile) written so far
    const int* fwd_err;           // adjoint view: the forward's error word (poisons the results)
    const float* mask;            // loss
    const float* presc;
    float* grad_dose;             // (nz, ny, nx): written by the loss, read by the adjoint
    double* loss_part;            // per-block partial sums of the loss
    double* loss;                 // device scalar
    float* grad_w;                // (nl, nsy, nsx)
    float* grad_range;            // (nl)
    float* dc;                    // (nl, nz) dL/dIDD
    float* dsg;                   // (nl, nz) dL/dsigma
    size_t layer_stride;          // tensor-core forward: > 0 writes each layer's own dose
                                  // (its lateral map times idd) to dose + l * layer_stride
                                  // instead of the sum over layers; 0 = the dose
    int direct;                   // forward: partial == dose (one work item per slice writes
                                  // the dose itself)
};

// A call's job views, installed into the device array by the call's first kernel (which also
// clears the status header and `zero`).
struct JobPair {
    JobDev j[2];
    int n;
    int nzero;           // ints of `zero` to clear (<= 32), e.g. the adjoint's counter block
    int* zero;
};

struct FwdItem { int job, z, ty, tx, lb, le, chunk, cost; };
struct AdjItem { int job, l, zb, ze, chunk, cost, pad0, pad1; };

constexpr int kTile = 128;          // lateral tile edge (voxels)
constexpr int kSpotChunk = 64;      // spots per lattice chunk in the FP32 forward
constexpr int kAdjMaxSpots = 64;    // adjoint lattice limit per axis
constexpr int kMaxChunkCost = 64;   // largest layers-per-item / z-per-item
constexpr int kLossBlocks = 296;    // fixed grid of the loss reduction (deterministic order)
constexpr int kLossBlocks16 = 592;  // the same for the split-FP16 forward's finalize (4 per SM:
                                    // one wave at its 64 registers per thread)
constexpr int kTcAdjChunk = 4;      // host unit size of the single-job tensor-core adjoint: it
                                    // sizes the grid (min(units, SMs)); with no explicit schedule
                                    // the CTAs then use ceil(active pairs / grid) + 1 layers
constexpr int kTcFwdWarps = 8;      // math warps of the tensor-core forward: each owns 32 rows x
                                    // 64 columns of a tile, its own arrival counter and loss partial

// ---------------------------------------------------------------------------
// small helpers
// ---------------------------------------------------------------------------
inline size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

inline int cuda_rc(cudaError_t e) { return e == cudaSuccess ? PBD_OK : PBD_ERR_CUDA; }

#define PBD_TRY(expr)                         \
    do {                                      \
        int pbd_rc_ = (expr);                 \
        if (pbd_rc_ != PBD_OK) return pbd_rc_; \
    } while (0)

#define PBD_LAUNCH_CHECK()                                       \
    do {                                                         \
        cudaError_t pbd_e_ = cudaGetLastError();                 \
        if (pbd_e_ != cudaSuccess) return PBD_ERR_CUDA;          \
    } while (0)

// Launch `kernel` as a programmatic dependent of the previous kernel on `s`: its CTAs may
// start (and run their prologue) while the previous kernel's last CTAs finish; the kernel
// itself executes griddepcontrol.wait before touching that kernel's results.
template <class... KArgs, class... Args>
int launch_dependent(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem,
                     cudaStream_t s, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cuda_rc(cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...));
}

// Bump allocator over the caller's workspace.  With base == nullptr it only sizes.
// Sub-arrays of a caller's workspace, each starting on a 256-byte ADDRESS boundary (the base
// need not be aligned).  Sized with base = nullptr, which assumes an aligned base: every
// workspace query adds 256 bytes of slack for the first alignment step of an unaligned one.
struct Carve {
    char* base;
    size_t used;
    explicit Carve(void* b) : base(static_cast<char*>(b)), used(0) {}
    template <class T>
    T* take(size_t count) {
        const size_t b = reinterpret_cast<size_t>(base);
        used = align_up(b + used, 256) - b;
        T* p = base ? reinterpret_cast<T*>(base + used) : nullptr;
        used += count * sizeof(T);
        return p;
    }
};

// Host-side planning of one job (shared by the forward and adjoint paths).
struct JobPlan {
    JobDev dev;
    size_t partial_elems;
    size_t nchunk_elems;
    int items;
};

int fill_job(const pbd_field* f, JobDev* j);

// Loss partial sums the forward of `precision` writes for one field (summed in index order by
// the adjoint's reduce): per (slice, tile, math warp) for the tensor-core forward that forms the
// loss in its output, per finalize block (kLossBlocks) for the paths with a finalize pass.
int loss_partials(const pbd_field* f, int precision);

// Status header: the first sub-array of every workspace whose kernels run bounded waits
// (kStatusInts ints at the workspace's first 256-byte boundary).  Word kStatFwd is the
// forward's error word, kStatAdj the adjoint's, kStatCmb the heterogeneous combine's; the
// call's first kernel (or memset) clears the header, a wait that runs out sets its word, and
// pbd_workspace_status() reads them back.
constexpr int kStatusInts = 16;
enum StatusWord { kStatFwd = 0, kStatAdj = 1, kStatCmb = 2 };

// Dynamic shared memory opt-in of kernel `fn` on the CURRENT device, done once per (device,
// kernel) and cached: bytes >= 0 sets that size; bytes < 0 sets the device's opt-in maximum
// minus the kernel's static shared memory.  *set_bytes receives the value in force.  With
// min_regs > 0 a kernel compiled with fewer registers per thread is refused
// (PBD_ERR_UNSUPPORTED): a setmaxnreg split needs the launch allotment it was written for.
int smem_optin(const void* fn, int bytes, int min_regs, int* set_bytes);

// Bounded device waits: the limit in ns (2 s unless the calling thread set a test limit) and
// whether the calling thread asked the tensor-core schedulers to publish no work (a test of
// the timeout path: every consumer wait then runs out).  Both from pbd_test_hook().
unsigned long long wait_limit_ns();
int test_hold();

// Profiling hooks (api.cu): event pairs around the dominant kernels while enabled on
// the calling thread, and a per-thread count of kernels this library launched.
enum ProfKernel { kProfFwd = 0, kProfAdj = 1 };
void prof_mark(int which, int end, cudaStream_t s);
void count_launch(int n = 1);
int host_validate_field(const pbd_field* f);
int num_sms();

// forward (FP32 SIMT) -- fwd_simt.cu
int fwd_chunk_layers(const pbd_field* f, int precision);
int fwd_plan_sizes(const pbd_field* f, int chunk, size_t* partial_elems, int* items);
// counter[0] = item counter; `err` = the error word (set by a timed-out device wait, read by
// the finalize / poison passes; the caller clears it).  FP32 path: schedule + persistent
// kernel + finalize.  Tensor-core precisions go to launch_forward_tc after clearing
// `n_counter_ints` ints from `counter` (the counters and the jobs' arrival arrays, laid out
// contiguously by the caller).
int launch_forward(JobDev* jobs_dev, const JobDev* jobs_host, int n_jobs, FwdItem* items,
                   int total_items, int* counter, size_t n_counter_ints, int* err, int chunk,
                   int with_loss, int precision, int poison, void* pack, size_t pack_bytes,
                   cudaStream_t s, const JobPair* inst = nullptr,
                   JobDev* inst_dst = nullptr, int* inst_status = nullptr);

// (slice, tile, layer-chunk) work items sorted longest-first, one CTA per job.
int launch_slice_schedule(JobDev* jobs_dev, FwdItem* items, int chunk, int n_jobs, cudaStream_t s);

// adjoint (tcgen05) -- adj_tc.cu.  Units (slice, chunk of `chunk` active layers) are
// pulled z-major; `partial` holds one (layer, slice) slot plane of nsy * nsx floats and the
// warps' dot-product partials of every pair (tc_adjoint_slot_elems); counter[0] = unit
// counter, counter[1] unused; `err` = the error word (cleared by the caller).
int tc_adjoint_dims(int precision, const pbd_field* f, int* N1);
// The calling thread's explicit adjoint item size (pbd_set_schedule), 0 when none is set.
int schedule_adj_override();
size_t tc_adjoint_slot_elems(const pbd_field* f);
// Ints of the adjoint's counter block (the unit counter and one unused word, for any number of
// jobs and layers).
size_t tc_adjoint_counter_ints(int n_jobs, int max_layers);
// counters_zeroed: the caller cleared the counter block earlier on the stream (so that no
// memset sits between the forward and this launch, which runs as its programmatic dependent).
int launch_adjoint_tc(int precision, JobDev* jobs_dev, const JobDev* jobs_host, int n_jobs,
                      int* counter, int* err, int chunk, int with_range, int finalize_loss,
                      int counters_zeroed, cudaStream_t s);

// forward (tcgen05) -- tc_fwd.cu.  Work units (slice, layer chunk, tile) are enumerated
// z-major; counter[0] = unit counter; every job's `arrive` array (nz * tiles ints, only read
// when a slice spans several chunks) must be zero at launch; `err` = the error word.
// `poison`: a follow-up kernel turns every job's dose into NaN if a device wait ran out.
int tc_operand_dims(int precision, int nsx, int nsy, int* K1, int* N1);
int tc_forward_units(const JobDev* jobs_host, int n_jobs, int chunk, int* cmax, int* tmax,
                     int* n_units);
int launch_forward_tc(int precision, JobDev* jobs_dev, const JobDev* jobs_host, int n_jobs,
                      int* counter, int* err, int chunk, int with_loss, int poison,
                      cudaStream_t s);

// forward in FP64 on the CUDA cores -- fwd_f64.cu.  One block per (slice, 64 x 64 tile)
// over all layers, writing the dose directly (no scratch).
int launch_forward_f64(const pbd_field* f, const double* w, const double* idd,
                       const double* sigma, double* dose, cudaStream_t s);

// forward (tcgen05, split FP16) -- tc_fwd16.cu.  Same units, counters and outputs as
// launch_forward_tc; `pack` (tc16_pack_bytes) receives the packed spot maps of every job.
size_t tc16_pack_bytes(int n_jobs, int max_layers, int nsx, int nsy);
int launch_forward_tc16(JobDev* jobs_dev, const JobDev* jobs_host, int n_jobs, int* counter,
                        int* err, int chunk, int with_loss, int poison, void* pack,
                        size_t pack_bytes, cudaStream_t s, const JobPair* inst = nullptr,
                        JobDev* inst_dst = nullptr, int* inst_status = nullptr);

// adjoint (FP32 SIMT) -- adj_simt.cu
int adj_chunk_depths(const pbd_field* f);
int adj_plan_sizes(const pbd_field* f, int chunk, size_t* partial_elems, int* items);
int launch_adjoint(JobDev* jobs_dev, const JobDev* jobs_host, int n_jobs, AdjItem* items,
                   int total_items, int* counter, int chunk, int with_range, int finalize_loss,
                   cudaStream_t s);

// LUT builder -- lut.cu
int lut_workspace_bytes(const pbd_lut_spec* s, int n_layers, size_t* bytes);
int lut_build(const pbd_lut_spec* s, int n_layers, const double* energies, const double* shift,
              double* idd, double* sigma, double* didd, double* dsig, void* ws, size_t ws_bytes,
              cudaStream_t st);
int lut_csda(const double* e, double* r, int n, int inverse, cudaStream_t st);
// Heterogeneous media (lut.cu): size of the depth-curve blob; curves builds the per-layer
// smoothed depth curves and their interval slopes into it; activity fills the (layer, slice)
// table act (L, nz) from a WED map; combine forms dose = sum_l IDD_l(WED) * lateral_l with
// layer l's lateral map at lateral + l * lstride (16-byte aligned, lstride a multiple of 4
// floats, >= nvox rounded up to 4), its error word err (set when a bounded wait ran out) and
// optionally the lateral maps' forward error word err2 (either one makes the dose NaN); the
// WED ray trace along +z.
int lut_curve_workspace(const pbd_lut_spec* s, int n_layers, size_t* bytes);
int lut_wed_curves(const pbd_lut_spec* s, int n_layers, const double* energies,
                   const double* shift, void* curves, size_t curves_bytes, cudaStream_t st);
// act (L, nz): 1 where some voxel of the slice lies within the layer's curve (of either set,
// when a second curve set is given)
int lut_wed_activity(const pbd_lut_spec* s, int n_layers, const void* curves, size_t curves_bytes,
                     const double* wed, int nz, size_t nslice, double* act, cudaStream_t st,
                     const void* curves2 = nullptr, size_t curves2_bytes = 0);
int lut_wed_combine(const pbd_lut_spec* s, int n_layers, const float* lateral, size_t lstride,
                    const double* wed, size_t nvox, float* dose, int* err, const int* err2,
                    const void* curves, size_t curves_bytes, cudaStream_t st);
// maps (L, lstride): dL/dD times each layer's depth dose at the WED (the heterogeneous
// adjoint's per-layer input).
int lut_wed_grad_maps(const pbd_lut_spec* s, int n_layers, const void* curves,
                      size_t curves_bytes, const float* grad, const double* wed, size_t nvox,
                      size_t lstride, float* maps, cudaStream_t st);
// maps (L, lstride): dL/dD times (IDD+_l(WED) - IDD-_l(WED)) / (2 h), the curves built at range
// shifts +h and -h (the heterogeneous range gradient's per-layer input).
int lut_wed_grad_maps_dr(const pbd_lut_spec* s, int n_layers, const void* curves_p,
                         size_t curves_p_bytes, const void* curves_m, size_t curves_m_bytes,
                         double h, const float* grad, const double* wed, size_t nvox,
                         size_t lstride, float* maps, cudaStream_t st);
int lut_wed_raytrace(int nz, int ny, int nx, double oz, double dz, const float* rho, double* wed,
                     cudaStream_t st);

}  // namespace pbd
