// api.cu -- extern "C" entry points of libpbdose_b200.so (declared in include/pbdose_b200.h).
//
// Rules of the boundary (the reference ABI's, pencil_beam.cu:647-730): validate first,
// return PBD_OK or a negative code, never exit, never throw across the boundary.  Work
// goes onto the caller's stream; no host<->device copies and no allocation happen here:
// per-call device state (job descriptors, schedules, partial sums) lives in the
// caller's workspace and is written by kernels from launch parameters, so every call
// can be captured into a CUDA graph.
#include <algorithm>
#include <math.h>
#include <string.h>

#include <mutex>
#include <vector>

#include "pbd_internal.cuh"

namespace pbd {

namespace {
thread_local int g_fwd_chunk = 0;   // 0 = default
thread_local int g_adj_chunk = 0;

// Installs the call's job views and clears its status header (may be null) and p.zero.
__global__ void install_jobs_kernel(JobPair p, JobDev* dst, int* status) {
    if ((int)threadIdx.x < p.n) dst[threadIdx.x] = p.j[threadIdx.x];
    if (status && (int)threadIdx.x < kStatusInts) status[threadIdx.x] = 0;
    if (p.zero && (int)threadIdx.x < p.nzero) p.zero[threadIdx.x] = 0;
}

struct JobLite {
    int nx, ny, nz, nsx, nsy, nl;
    int item_base, max_items, max_chunks, direct;   // direct: items write the output slice
    double ox, oy, dx, dy, sx0, sy0, dsx, dsy;
    const float* w;
    const double* idd;
    const double* sigma;
    float* dose;
    size_t partial_off, nchunk_off, arrive_off;
};

struct JobTable {
    int n;
    JobLite j[PBD_MAX_JOBS];
};
static_assert(sizeof(JobTable) < 32000, "kernel parameter limit");

__global__ void install_table_kernel(JobTable t, JobDev* dst, float* partial_base, int* nchunk_base,
                                     int* arrive_base, int* status) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < kStatusInts) status[k] = 0;
    if (k >= t.n) return;
    const JobLite& a = t.j[k];
    JobDev J;
    memset(&J, 0, sizeof(J));
    J.nx = a.nx; J.ny = a.ny; J.nz = a.nz; J.nsx = a.nsx; J.nsy = a.nsy; J.nl = a.nl;
    J.ntx = (a.nx + kTile - 1) / kTile;
    J.nty = (a.ny + kTile - 1) / kTile;
    J.max_chunks = a.max_chunks; J.item_base = a.item_base; J.max_items = a.max_items;
    J.ox = a.ox; J.oy = a.oy; J.dx = a.dx; J.dy = a.dy;
    J.sx0 = a.sx0; J.sy0 = a.sy0; J.dsx = a.dsx; J.dsy = a.dsy;
    J.w = a.w; J.idd = a.idd; J.sigma = a.sigma; J.dose = a.dose;
    J.partial = a.direct ? a.dose : partial_base + a.partial_off;
    J.direct = a.direct;
    J.nchunks = nchunk_base + a.nchunk_off;
    J.arrive = arrive_base + a.arrive_off;
    dst[k] = J;
}

// Batched loss gradient: per-job descriptors installed in groups of kGradInstall (kernel
// parameter size) into the forward and adjoint views.
struct GradLite {
    int nx, ny, nz, nsx, nsy, nl;
    int max_chunks_f, max_chunks_a, direct, n_loss_part;
    double ox, oy, dx, dy, sx0, sy0, dsx, dsy;
    const float* w;
    const double *idd, *sigma, *didd, *dsig;
    const float *mask, *presc;
    float *dose, *grad_dose;
    double* loss;
    float *grad_w, *grad_range;
    size_t fpart_off, arrive_off, loss_off, slot_off, dcs_off;
};
constexpr int kGradInstall = 64;
struct GradTable {
    int n, base;
    GradLite j[kGradInstall];
};
static_assert(sizeof(GradTable) < 32000, "kernel parameter limit");

struct GradBufs {
    JobDev *fwd, *adj;
    float* fpart;
    int* farr;
    double* lpart;
    float *apart, *dcs, *dsgs;
    const int* fwd_err;
    int* status;         // cleared by the first group's launch
};

__global__ void install_grad_kernel(GradTable t, GradBufs b) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (t.base == 0 && k < kStatusInts) b.status[k] = 0;
    if (k >= t.n) return;
    const GradLite& a = t.j[k];
    JobDev J;
    memset(&J, 0, sizeof(J));
    J.nx = a.nx; J.ny = a.ny; J.nz = a.nz; J.nsx = a.nsx; J.nsy = a.nsy; J.nl = a.nl;
    J.ntx = (a.nx + kTile - 1) / kTile;
    J.nty = (a.ny + kTile - 1) / kTile;
    J.ox = a.ox; J.oy = a.oy; J.dx = a.dx; J.dy = a.dy;
    J.sx0 = a.sx0; J.sy0 = a.sy0; J.dsx = a.dsx; J.dsy = a.dsy;
    J.w = a.w; J.idd = a.idd; J.sigma = a.sigma; J.didd_dr = a.didd; J.dsig_dr = a.dsig;
    J.dose = a.dose; J.mask = a.mask; J.presc = a.presc; J.grad_dose = a.grad_dose;
    J.loss = a.loss; J.grad_w = a.grad_w; J.grad_range = a.grad_range;
    J.n_loss_part = a.n_loss_part;
    J.loss_part = b.lpart + a.loss_off;
    JobDev F = J, A = J;
    F.max_chunks = a.max_chunks_f;
    F.partial = a.direct ? a.dose : b.fpart + a.fpart_off;
    F.direct = a.direct;
    F.arrive = b.farr + a.arrive_off;
    A.max_chunks = a.max_chunks_a;
    A.partial = b.apart + a.slot_off;
    A.dc = b.dcs + a.dcs_off;
    A.dsg = b.dsgs + a.dcs_off;
    A.fwd_err = b.fwd_err;
    b.fwd[t.base + k] = F;
    b.adj[t.base + k] = A;
}

int g_sms[64] = {0};
std::mutex g_sms_mu;

// smem_optin's cache: one entry per (device, kernel).
struct OptIn {
    int dev;
    const void* fn;
    int bytes;   // value set, or a negative error code
};
std::vector<OptIn> g_optin;
std::mutex g_optin_mu;

// pbd_test_hook's settings (calling thread)
thread_local unsigned long long g_wait_ns = 0;   // 0 = the default 2 s
thread_local int g_hold = 0;

struct ProfState {
    bool on = false;
    std::vector<cudaEvent_t> ev[2];   // alternating begin/end per kernel kind
    size_t used[2] = {0, 0};
    long long launches = 0;
};
thread_local ProfState g_prof;

int choose_fwd_chunk(const pbd_field* f, int precision) {
    int c = g_fwd_chunk > 0 ? g_fwd_chunk : fwd_chunk_layers(f, precision);
    return c < 1 ? 1 : (c > kMaxChunkCost ? kMaxChunkCost : c);
}
int choose_adj_chunk(const pbd_field* f) {
    int c = g_adj_chunk > 0 ? g_adj_chunk : adj_chunk_depths(f);
    return c < 1 ? 1 : (c > kMaxChunkCost ? kMaxChunkCost : c);
}

bool finite_pos(double v) { return isfinite(v) && v > 0.0; }

int check_precision(int p) {
    if (p >= PBD_PREC_FP32 && p <= PBD_PREC_FP16X3) return PBD_OK;
    return PBD_ERR_BAD_VALUE;
}

int check_field_precision(const pbd_field* f, int p) {
    PBD_TRY(check_precision(p));
    if (p == PBD_PREC_FP32) return PBD_OK;
    int k1 = 0, n1 = 0;
    return tc_operand_dims(p, f->n_sx, f->n_sy, &k1, &n1);
}

int adjoint_supported(const pbd_field* f) {
    if (f->n_sx > kAdjMaxSpots || f->n_sy > kAdjMaxSpots) return PBD_ERR_UNSUPPORTED;
    return PBD_OK;
}

// Workspace of the single-job paths.
struct Ws {
    int* status;         // status header: [kStatFwd], [kStatAdj] error words
    JobDev* jobs;        // [0] forward view, [1] adjoint view
    int* counters;       // [0] forward items, [2] adjoint items (FP32); then the forward's
                         // arrival counters
    int* farr;           // tensor-core forward: per (slice, tile) arrival counters
    size_t n_fcount;     // ints the forward clears at launch (counters + arrivals)
    int n_loss_part;
    FwdItem* fitems;
    int* fnch;
    float* fpart;
    double* loss_part;
    void* aitems;        // AdjItem (FP32 path) or FwdItem (tensor-core path), 32 B each
    int adj_tc;          // 1: tensor-core adjoint, (layer, slice) dL/dW slots
    int* anch;
    void* pack;          // split-FP16 forward: packed spot maps
    size_t pack_bytes;
    int* acnt;           // tensor-core adjoint: its counter block (unit counter)
    float* apart;
    float* dc;
    float* dsg;
    int f_items, a_items, f_chunk, a_chunk;
};

int carve_ws(const pbd_field* f, bool fwd, bool adj, bool loss, int precision, void* base, Ws& w,
             size_t* used) {
    Carve c(base);
    w.status = c.take<int>(kStatusInts);
    w.jobs = c.take<JobDev>(2);
    const int tiles = ((f->nx + kTile - 1) / kTile) * ((f->ny + kTile - 1) / kTile);
    const size_t narr = fwd ? (size_t)f->nz * tiles * kTcFwdWarps : 0;
    w.counters = c.take<int>(8 + narr);
    w.farr = w.counters ? w.counters + 8 : nullptr;
    w.n_fcount = 8 + narr;
    w.n_loss_part = loss_partials(f, precision);
    w.f_chunk = choose_fwd_chunk(f, precision);
    w.a_chunk = choose_adj_chunk(f);
    w.fitems = nullptr; w.fnch = nullptr; w.fpart = nullptr; w.loss_part = nullptr;
    w.aitems = nullptr; w.anch = nullptr; w.apart = nullptr; w.dc = nullptr; w.dsg = nullptr;
    w.acnt = nullptr;
    w.f_items = w.a_items = 0;
    w.pack = nullptr;
    w.pack_bytes = 0;
    if (fwd) {
        size_t pe = 0;
        PBD_TRY(fwd_plan_sizes(f, w.f_chunk, &pe, &w.f_items));
        w.fitems = c.take<FwdItem>(w.f_items);
        w.fnch = c.take<int>(f->nz);
        w.fpart = c.take<float>(pe);
        if (precision == PBD_PREC_FP16X3) {
            w.pack_bytes = tc16_pack_bytes(1, f->n_layers, f->n_sx, f->n_sy);
            w.pack = c.take<char>(w.pack_bytes);
        }
    }
    if (loss) w.loss_part = c.take<double>(w.n_loss_part);
    w.adj_tc = 0;
    if (adj) {
        size_t pe = 0;
        int n1 = 0;
        if (tc_adjoint_dims(precision, f, &n1) == PBD_OK) {
            // tensor-core adjoint: (slice, layer-chunk) units, one slot and the warps' dot
            // products per active (layer, slice)
            w.adj_tc = 1;
            w.a_chunk = g_adj_chunk > 0 ? w.a_chunk : kTcAdjChunk;
            pe = tc_adjoint_slot_elems(f);
            w.acnt = c.take<int>(tc_adjoint_counter_ints(1, f->n_layers));
        } else {
            PBD_TRY(adj_plan_sizes(f, w.a_chunk, &pe, &w.a_items));
            w.aitems = c.take<AdjItem>(w.a_items);
            w.anch = c.take<int>(f->n_layers);
        }
        w.apart = c.take<float>(pe);
        w.dc = c.take<float>((size_t)f->n_layers * f->nz);
        w.dsg = c.take<float>((size_t)f->n_layers * f->nz);
    }
    *used = c.used + 256;
    return PBD_OK;
}

}  // namespace

int smem_optin(const void* fn, int bytes, int min_regs, int* set_bytes) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return PBD_ERR_CUDA;
    std::lock_guard<std::mutex> g(g_optin_mu);
    for (const OptIn& o : g_optin)
        if (o.dev == dev && o.fn == fn) {
            if (o.bytes < 0) return o.bytes;
            *set_bytes = o.bytes;
            return PBD_OK;
        }
    int optin = 0;
    cudaFuncAttributes fa;
    if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) !=
            cudaSuccess ||
        cudaFuncGetAttributes(&fa, fn) != cudaSuccess)
        return PBD_ERR_CUDA;
    int rc = PBD_OK;
    const int want = bytes >= 0 ? bytes : optin - (int)fa.sharedSizeBytes;
    if (min_regs > 0 && fa.numRegs < min_regs) {
        rc = PBD_ERR_UNSUPPORTED;
    } else if (want <= 0 || want + (int)fa.sharedSizeBytes > optin ||
               cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, want) !=
                   cudaSuccess) {
        rc = PBD_ERR_NO_SMEM;
    }
    g_optin.push_back({dev, fn, rc == PBD_OK ? want : rc});
    if (rc == PBD_OK) *set_bytes = want;
    return rc;
}

unsigned long long wait_limit_ns() { return g_wait_ns ? g_wait_ns : 2000000000ull; }
int test_hold() { return g_hold; }

int schedule_adj_override() { return g_adj_chunk; }

int num_sms() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
    std::lock_guard<std::mutex> g(g_sms_mu);
    if (g_sms[dev] == 0) {
        int v = 0;
        if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0)
            v = 148;
        g_sms[dev] = v;
    }
    return g_sms[dev];
}

void prof_mark(int which, int end, cudaStream_t s) {
    if (!g_prof.on) return;
    std::vector<cudaEvent_t>& v = g_prof.ev[which];
    size_t& u = g_prof.used[which];
    if ((end == 0) != (u % 2 == 0)) return;   // keep begin/end paired
    if (u == v.size()) {
        cudaEvent_t e;
        if (cudaEventCreate(&e) != cudaSuccess) return;
        v.push_back(e);
    }
    cudaEventRecord(v[u], s);
    ++u;
}

void count_launch(int n) { g_prof.launches += n; }

int host_validate_field(const pbd_field* f) {
    if (!f) return PBD_ERR_NULL_ARG;
    if (f->nx <= 0 || f->ny <= 0 || f->nz <= 0 || f->n_sx <= 0 || f->n_sy <= 0 || f->n_layers <= 0)
        return PBD_ERR_BAD_DIM;
    if (f->n_sx > 4096 || f->n_sy > 4096 || f->n_layers > 4096) return PBD_ERR_UNSUPPORTED;
    if ((double)f->nx * f->ny * f->nz > 2147483647.0) return PBD_ERR_UNSUPPORTED;
    if (!finite_pos(f->dx) || !finite_pos(f->dy) || !finite_pos(f->dz) ||
        !finite_pos(f->dx_spot) || !finite_pos(f->dy_spot))
        return PBD_ERR_BAD_VALUE;
    if (!isfinite(f->ox) || !isfinite(f->oy) || !isfinite(f->oz) || !isfinite(f->x0) ||
        !isfinite(f->y0))
        return PBD_ERR_BAD_VALUE;
    return PBD_OK;
}

int loss_partials(const pbd_field* f, int precision) {
    const int tiles = ((f->nx + kTile - 1) / kTile) * ((f->ny + kTile - 1) / kTile);
    if (precision == PBD_PREC_FP32) return kLossBlocks;
    if (precision == PBD_PREC_FP16X3) return kLossBlocks16;
    return f->nz * tiles * kTcFwdWarps;
}

int fill_job(const pbd_field* f, JobDev* J) {
    memset(J, 0, sizeof(*J));
    J->nx = f->nx; J->ny = f->ny; J->nz = f->nz;
    J->nsx = f->n_sx; J->nsy = f->n_sy; J->nl = f->n_layers;
    J->ntx = (f->nx + kTile - 1) / kTile;
    J->nty = (f->ny + kTile - 1) / kTile;
    J->ox = f->ox; J->oy = f->oy; J->dx = f->dx; J->dy = f->dy;
    J->sx0 = f->x0; J->sy0 = f->y0; J->dsx = f->dx_spot; J->dsy = f->dy_spot;
    return PBD_OK;
}

// ---- heterogeneous media helpers ------------------------------------------------------
// Jobs of one forward launch of the per-layer lateral maps: one single-layer job per layer,
// depth dose 1 where the layer reaches the slice at all (`act`, (L, nz)), else 0.
// Row stride (floats) of the per-layer lateral maps: the voxel count rounded up to 64 floats,
// so every row starts on a 256-byte boundary for the combine's bulk copies.
static size_t wed_lateral_stride(const pbd_field* f) {
    return align_up((size_t)f->nz * f->ny * f->nx, 64);
}

static void wed_jobs(const pbd_field* f, int l0, int n, const float* w, const double* sigma,
                     const double* act, float* lateral, pbd_job* jobs) {
    const size_t lstride = wed_lateral_stride(f);
    for (int q = 0; q < n; ++q) {
        const int l = l0 + q;
        pbd_job& j = jobs[q];
        j.field = *f;
        j.field.n_layers = 1;
        j.w = w ? w + (size_t)l * f->n_sy * f->n_sx : nullptr;
        j.idd = act ? act + (size_t)l * f->nz : nullptr;
        j.sigma = sigma ? sigma + (size_t)l * f->nz : nullptr;
        j.dose = lateral ? lateral + (size_t)l * lstride : nullptr;
    }
}

struct WedCarve {
    int* status;         // status header: forward, combine error words
    double* act;
    float* lateral;      // (L, wed_lateral_stride) per-layer lateral maps
    void* curves;
    size_t curves_bytes;
    void* batch;         // the lateral maps' forward: batch (FP32) or single-job workspace
    size_t batch_bytes;
};

static int carve_wed(const pbd_field* f, const pbd_lut_spec* spec, int precision, void* base,
                     WedCarve& w, size_t* used) {
    const int L = f->n_layers;
    pbd_job jobs[PBD_MAX_JOBS];
    const int nb = L < PBD_MAX_JOBS ? L : PBD_MAX_JOBS;
    wed_jobs(f, 0, nb, nullptr, nullptr, nullptr, nullptr, jobs);
    size_t bb = 0, cb = 0;
    if (precision == PBD_PREC_FP32) {
        PBD_TRY(pbd_forward_batch_workspace(jobs, nb, precision, &bb));
    } else {
        Ws fw;
        PBD_TRY(carve_ws(f, true, false, false, precision, nullptr, fw, &bb));
    }
    PBD_TRY(lut_curve_workspace(spec, L, &cb));
    Carve c(base);
    w.status = c.take<int>(kStatusInts);
    w.act = c.take<double>((size_t)L * f->nz);
    w.lateral = c.take<float>((size_t)L * wed_lateral_stride(f));
    w.curves = c.take<char>(cb);
    w.curves_bytes = cb;
    w.batch = c.take<char>(bb);
    w.batch_bytes = bb;
    *used = c.used + 256;
    return PBD_OK;
}

}  // namespace pbd

using namespace pbd;

extern "C" {

const char* pbd_strerror(int code) {
    switch (code) {
        case PBD_OK: return "ok";
        case PBD_ERR_NULL_ARG: return "null argument";
        case PBD_ERR_BAD_DIM: return "invalid dimension";
        case PBD_ERR_BAD_VALUE: return "invalid value (non-finite or non-positive spacing, step or sigma)";
        case PBD_ERR_CUDA: return "CUDA runtime error";
        case PBD_ERR_UNSUPPORTED: return "unsupported configuration";
        case PBD_ERR_NO_SMEM: return "insufficient shared memory per block";
        case PBD_ERR_WORKSPACE: return "workspace missing or too small";
        case PBD_ERR_TIMEOUT: return "bounded device wait ran out";
        case PBD_ERR_TOO_MANY: return "too many jobs for one launch";
        default: return "unknown error";
    }
}

int pbd_version(void) { return 100; }

int pbd_field_validate(const pbd_field* f) { return host_validate_field(f); }

int pbd_set_schedule(int fwd_layers_per_item, int adj_depths_per_item) {
    if (fwd_layers_per_item < 0 || fwd_layers_per_item > kMaxChunkCost ||
        adj_depths_per_item < 0 || adj_depths_per_item > kMaxChunkCost)
        return PBD_ERR_BAD_VALUE;
    g_fwd_chunk = fwd_layers_per_item;
    g_adj_chunk = adj_depths_per_item;
    return PBD_OK;
}

int pbd_profile_begin(void) {
    g_prof.on = true;
    g_prof.used[0] = g_prof.used[1] = 0;
    return PBD_OK;
}

int pbd_profile_end(double* fwd_ms, int* n_fwd, double* adj_ms, int* n_adj) {
    double* ms[2] = {fwd_ms, adj_ms};
    int* cnt[2] = {n_fwd, n_adj};
    int rc = PBD_OK;
    for (int k = 0; k < 2; ++k) {
        double tot = 0.0;
        int n = 0;
        for (size_t i = 0; i + 1 < g_prof.used[k]; i += 2) {
            float t = 0.f;
            if (cudaEventSynchronize(g_prof.ev[k][i + 1]) != cudaSuccess ||
                cudaEventElapsedTime(&t, g_prof.ev[k][i], g_prof.ev[k][i + 1]) != cudaSuccess) {
                rc = PBD_ERR_CUDA;
                break;
            }
            tot += t;
            ++n;
        }
        if (ms[k]) *ms[k] = tot;
        if (cnt[k]) *cnt[k] = n;
    }
    g_prof.on = false;
    g_prof.used[0] = g_prof.used[1] = 0;
    return rc;
}

int pbd_launch_count(long long* n) {
    if (!n) return PBD_ERR_NULL_ARG;
    *n = g_prof.launches;
    return PBD_OK;
}

int pbd_test_hook(unsigned long long wait_limit_ns, int hold_schedulers) {
    if (hold_schedulers != 0 && hold_schedulers != 1) return PBD_ERR_BAD_VALUE;
    if (hold_schedulers && wait_limit_ns == 0) return PBD_ERR_BAD_VALUE;   // keep 2 s holds out
    g_wait_ns = wait_limit_ns;
    g_hold = hold_schedulers;
    return PBD_OK;
}

int pbd_workspace_status(const void* workspace, size_t workspace_bytes, int* status,
                         void* stream) {
    if (!workspace || !status) return PBD_ERR_NULL_ARG;
    Carve c(const_cast<void*>(workspace));
    const int* hdr = c.take<int>(kStatusInts);
    if (c.used > workspace_bytes) return PBD_ERR_WORKSPACE;
    int h[kStatusInts];
    cudaStream_t s = (cudaStream_t)stream;
    if (cudaMemcpyAsync(h, hdr, sizeof(h), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return PBD_ERR_CUDA;
    int st = PBD_OK;
    for (int k = 0; k < kStatusInts; ++k)
        if (h[k] != 0) st = PBD_ERR_TIMEOUT;
    *status = st;
    return PBD_OK;
}

int pbd_forward_f64(const pbd_field* f, const double* w, const double* idd, const double* sigma,
                    double* dose, void* stream) {
    PBD_TRY(host_validate_field(f));
    if (!w || !idd || !sigma || !dose) return PBD_ERR_NULL_ARG;
    PBD_TRY(launch_forward_f64(f, w, idd, sigma, dose, (cudaStream_t)stream));
    count_launch(1);
    return PBD_OK;
}

int pbd_lut_workspace(const pbd_lut_spec* spec, int n_layers, size_t* bytes) {
    return lut_workspace_bytes(spec, n_layers, bytes);
}

int pbd_build_luts(const pbd_lut_spec* spec, int n_layers, const double* energies,
                   const double* range_shift, double* idd, double* sigma, double* didd_dr,
                   double* dsigma_dr, void* workspace, size_t workspace_bytes, void* stream) {
    return lut_build(spec, n_layers, energies, range_shift, idd, sigma, didd_dr, dsigma_dr,
                     workspace, workspace_bytes, (cudaStream_t)stream);
}

int pbd_csda_range(const double* energy, double* range_cm, int n, void* stream) {
    return lut_csda(energy, range_cm, n, 0, (cudaStream_t)stream);
}

int pbd_energy_from_range(const double* range_cm, double* energy, int n, void* stream) {
    return lut_csda(range_cm, energy, n, 1, (cudaStream_t)stream);
}

int pbd_forward_workspace(const pbd_field* f, int precision, size_t* bytes) {
    PBD_TRY(host_validate_field(f));
    PBD_TRY(check_field_precision(f, precision));
    if (!bytes) return PBD_ERR_NULL_ARG;
    Ws w;
    return carve_ws(f, true, false, false, precision, nullptr, w, bytes);
}

int pbd_forward(const pbd_field* f, const float* w, const double* idd, const double* sigma,
                float* dose, int precision, void* workspace, size_t workspace_bytes, void* stream) {
    PBD_TRY(host_validate_field(f));
    PBD_TRY(check_field_precision(f, precision));
    if (!w || !idd || !sigma || !dose) return PBD_ERR_NULL_ARG;
    size_t need = 0;
    Ws ws;
    PBD_TRY(carve_ws(f, true, false, false, precision, nullptr, ws, &need));
    if (!workspace || workspace_bytes < need) return PBD_ERR_WORKSPACE;
    PBD_TRY(carve_ws(f, true, false, false, precision, workspace, ws, &need));
    cudaStream_t s = (cudaStream_t)stream;
    JobPair p;
    memset(&p, 0, sizeof(p));
    p.n = 1;
    JobDev& J = p.j[0];
    fill_job(f, &J);
    J.w = w; J.idd = idd; J.sigma = sigma; J.dose = dose;
    J.max_chunks = (f->n_layers + ws.f_chunk - 1) / ws.f_chunk;
    J.item_base = 0; J.max_items = ws.f_items;
    J.partial = ws.fpart; J.nchunks = ws.fnch; J.arrive = ws.farr;
    // split FP16: the pack kernel installs the views (one launch fewer before the dose kernel)
    const bool merged = precision == PBD_PREC_FP16X3;
    if (!merged) {
        install_jobs_kernel<<<1, 32, 0, s>>>(p, ws.jobs, ws.status);
        PBD_LAUNCH_CHECK();
        count_launch(1);
    }
    return launch_forward(ws.jobs, &J, 1, ws.fitems, ws.f_items, ws.counters, ws.n_fcount,
                          ws.status + kStatFwd, ws.f_chunk, 0, precision, 1, ws.pack,
                          ws.pack_bytes, s, merged ? &p : nullptr, ws.jobs, ws.status);
}

// err: the adjoint's error word (the workspace's own status word unless a caller passes its
// own, as the heterogeneous adjoint does for its per-layer calls)
static int run_adjoint(const Ws& ws, int precision, const JobDev* A, int with_range,
                       int finalize_loss, int counters_zeroed, int* err, cudaStream_t s) {
    if (ws.adj_tc)
        return launch_adjoint_tc(precision, ws.jobs + 1, A, 1, ws.acnt, err, ws.a_chunk,
                                 with_range, finalize_loss, counters_zeroed, s);
    return launch_adjoint(ws.jobs + 1, A, 1, static_cast<AdjItem*>(ws.aitems), ws.a_items,
                          ws.counters + 2, ws.a_chunk, with_range, finalize_loss, s);
}

int pbd_adjoint_workspace(const pbd_field* f, int precision, size_t* bytes) {
    PBD_TRY(host_validate_field(f));
    PBD_TRY(check_field_precision(f, precision));
    PBD_TRY(adjoint_supported(f));
    if (!bytes) return PBD_ERR_NULL_ARG;
    Ws w;
    return carve_ws(f, false, true, false, precision, nullptr, w, bytes);
}

static void fill_adj_view(const pbd_field* f, const Ws& ws, JobDev& A) {
    A.max_chunks = ws.adj_tc ? (f->n_layers + ws.a_chunk - 1) / ws.a_chunk
                             : (f->nz + ws.a_chunk - 1) / ws.a_chunk;
    A.item_base = 0;
    A.max_items = ws.a_items;
    A.partial = ws.apart;
    A.nchunks = ws.anch;
    A.dc = ws.dc;
    A.dsg = ws.dsg;
}

// One adjoint call; `err` (may be null: the workspace's own status word) receives a timed-out
// wait.
static int adjoint_one(const pbd_field* f, const float* w, const double* idd, const double* sigma,
                       const double* didd_dr, const double* dsigma_dr, const float* grad_dose,
                       float* grad_w, float* grad_range, int precision, void* workspace,
                       size_t workspace_bytes, int* err, cudaStream_t s) {
    PBD_TRY(host_validate_field(f));
    PBD_TRY(check_field_precision(f, precision));
    PBD_TRY(adjoint_supported(f));
    if (!w || !idd || !sigma || !grad_dose || !grad_w) return PBD_ERR_NULL_ARG;
    const int with_range = grad_range != nullptr;
    if (with_range && (!didd_dr || !dsigma_dr)) return PBD_ERR_NULL_ARG;
    size_t need = 0;
    Ws ws;
    PBD_TRY(carve_ws(f, false, true, false, precision, nullptr, ws, &need));
    if (!workspace || workspace_bytes < need) return PBD_ERR_WORKSPACE;
    PBD_TRY(carve_ws(f, false, true, false, precision, workspace, ws, &need));
    JobPair p;
    memset(&p, 0, sizeof(p));
    p.n = 2;
    JobDev& A = p.j[1];
    fill_job(f, &A);
    A.w = w; A.idd = idd; A.sigma = sigma; A.didd_dr = didd_dr; A.dsig_dr = dsigma_dr;
    A.grad_dose = const_cast<float*>(grad_dose);
    A.grad_w = grad_w; A.grad_range = grad_range;
    fill_adj_view(f, ws, A);
    p.j[0] = A;
    install_jobs_kernel<<<1, 32, 0, s>>>(p, ws.jobs, ws.status);
    PBD_LAUNCH_CHECK();
    count_launch(1);
    return run_adjoint(ws, precision, &A, with_range, 0, 0, err ? err : ws.status + kStatAdj, s);
}

int pbd_adjoint(const pbd_field* f, const float* w, const double* idd, const double* sigma,
                const double* didd_dr, const double* dsigma_dr, const float* grad_dose,
                float* grad_w, float* grad_range, int precision, void* workspace,
                size_t workspace_bytes, void* stream) {
    return adjoint_one(f, w, idd, sigma, didd_dr, dsigma_dr, grad_dose, grad_w, grad_range,
                       precision, workspace, workspace_bytes, nullptr, (cudaStream_t)stream);
}

int pbd_loss_grad_workspace(const pbd_field* f, int precision, size_t* bytes) {
    PBD_TRY(host_validate_field(f));
    PBD_TRY(check_field_precision(f, precision));
    PBD_TRY(adjoint_supported(f));
    if (!bytes) return PBD_ERR_NULL_ARG;
    Ws w;
    return carve_ws(f, true, true, true, precision, nullptr, w, bytes);
}

int pbd_loss_grad(const pbd_field* f, const float* w, const double* idd, const double* sigma,
                  const double* didd_dr, const double* dsigma_dr, const float* mask,
                  const float* presc, float* dose, float* grad_dose, double* loss, float* grad_w,
                  float* grad_range, int precision, void* workspace, size_t workspace_bytes,
                  void* stream) {
    PBD_TRY(host_validate_field(f));
    PBD_TRY(check_field_precision(f, precision));
    PBD_TRY(adjoint_supported(f));
    if (!w || !idd || !sigma || !mask || !presc || !dose || !grad_dose || !loss || !grad_w)
        return PBD_ERR_NULL_ARG;
    const int with_range = grad_range != nullptr;
    if (with_range && (!didd_dr || !dsigma_dr)) return PBD_ERR_NULL_ARG;
    size_t need = 0;
    Ws ws;
    PBD_TRY(carve_ws(f, true, true, true, precision, nullptr, ws, &need));
    if (!workspace || workspace_bytes < need) return PBD_ERR_WORKSPACE;
    PBD_TRY(carve_ws(f, true, true, true, precision, workspace, ws, &need));
    cudaStream_t s = (cudaStream_t)stream;
    JobPair p;
    memset(&p, 0, sizeof(p));
    p.n = 2;
    JobDev& F = p.j[0];
    fill_job(f, &F);
    F.w = w; F.idd = idd; F.sigma = sigma; F.didd_dr = didd_dr; F.dsig_dr = dsigma_dr;
    F.dose = dose; F.mask = mask; F.presc = presc; F.grad_dose = grad_dose;
    F.loss_part = ws.loss_part; F.loss = loss; F.grad_w = grad_w; F.grad_range = grad_range;
    F.n_loss_part = ws.n_loss_part;
    JobDev A = F;
    F.max_chunks = (f->n_layers + ws.f_chunk - 1) / ws.f_chunk;
    F.item_base = 0; F.max_items = ws.f_items;
    F.partial = ws.fpart; F.nchunks = ws.fnch; F.arrive = ws.farr;
    fill_adj_view(f, ws, A);
    A.fwd_err = ws.status + kStatFwd;
    p.j[1] = A;
    // the adjoint's counters are cleared by the install, before the forward, so that forward
    // -> adjoint -> reduce run back to back (programmatic dependent launches)
    if (ws.adj_tc) {
        const size_t nc = tc_adjoint_counter_ints(1, f->n_layers);
        if (nc > 32) return PBD_ERR_UNSUPPORTED;
        p.zero = ws.acnt;
        p.nzero = (int)nc;
    }
    // split FP16: the pack kernel installs the views (one launch fewer before the dose kernel)
    const bool merged = precision == PBD_PREC_FP16X3;
    if (!merged) {
        install_jobs_kernel<<<1, 32, 0, s>>>(p, ws.jobs, ws.status);
        PBD_LAUNCH_CHECK();
        count_launch(1);
    }
    PBD_TRY(launch_forward(ws.jobs, &F, 1, ws.fitems, ws.f_items, ws.counters, ws.n_fcount,
                           ws.status + kStatFwd, ws.f_chunk, 1, precision, 0, ws.pack,
                           ws.pack_bytes, s, merged ? &p : nullptr, ws.jobs, ws.status));
    return run_adjoint(ws, precision, &A, with_range, 1, ws.adj_tc, ws.status + kStatAdj, s);
}

// ---- batched loss gradient ------------------------------------------------------------
// layers per tensor-core adjoint unit of a batch: many jobs balance the grid by themselves,
// so larger units only amortise the per-unit set-up (the 100-job loss gradient: 14.31 ms at
// 8, 14.06 at 20, 13.98 at 40)
constexpr int kBatchAdjChunk = 40;

struct GradPlan {
    int chunk, direct, with_range, max_l;
    int fprec;           // the forward's precision (split FP16 needs direct mode here)
    size_t arr, fpart, lpart, apart, dcs, pack;
};

static int plan_grad_batch(const pbd_grad_job* jobs, int n_jobs, int precision, GradPlan* gp) {
    if (!jobs) return PBD_ERR_NULL_ARG;
    if (n_jobs <= 0) return PBD_ERR_BAD_DIM;
    if (n_jobs > PBD_MAX_JOBS) return PBD_ERR_TOO_MANY;
    PBD_TRY(check_precision(precision));
    if (precision == PBD_PREC_FP32) return PBD_ERR_UNSUPPORTED;
    int max_l = 0, chunk = kMaxChunkCost, max_sx = 1, max_sy = 1;
    gp->with_range = jobs[0].grad_range != nullptr;
    for (int k = 0; k < n_jobs; ++k) {
        const pbd_field* f = &jobs[k].field;
        PBD_TRY(host_validate_field(f));
        PBD_TRY(check_field_precision(f, precision));
        PBD_TRY(adjoint_supported(f));
        int n1 = 0;
        PBD_TRY(tc_adjoint_dims(precision, f, &n1));
        if ((jobs[k].grad_range != nullptr) != (gp->with_range != 0)) return PBD_ERR_BAD_VALUE;
        max_l = max_l > f->n_layers ? max_l : f->n_layers;
        max_sx = max_sx > f->n_sx ? max_sx : f->n_sx;
        max_sy = max_sy > f->n_sy ? max_sy : f->n_sy;
        const int ch = choose_fwd_chunk(f, precision);
        chunk = ch < chunk ? ch : chunk;
    }
    gp->max_l = max_l;
    gp->direct = (max_l <= kMaxChunkCost && g_fwd_chunk == 0) ? 1 : 0;
    // the split-FP16 forward's partial slices need per-slice chunk counts, which this path
    // keeps only in direct mode; otherwise its forward runs split TF32 (same accuracy class)
    gp->fprec = (precision == PBD_PREC_FP16X3 && !gp->direct) ? PBD_PREC_TF32X3 : precision;
    gp->pack = gp->fprec == PBD_PREC_FP16X3 ? tc16_pack_bytes(n_jobs, max_l, max_sx, max_sy) : 0;
    gp->chunk = gp->direct ? max_l : chunk;
    gp->arr = gp->fpart = gp->lpart = gp->apart = gp->dcs = 0;
    for (int k = 0; k < n_jobs; ++k) {
        const pbd_field& f = jobs[k].field;
        const size_t tiles = (size_t)((f.nx + kTile - 1) / kTile) * ((f.ny + kTile - 1) / kTile);
        size_t pe = 0;
        int it = 0;
        PBD_TRY(fwd_plan_sizes(&f, gp->chunk, &pe, &it));
        gp->arr += (size_t)f.nz * tiles * kTcFwdWarps;
        gp->fpart += gp->direct ? 0 : pe;
        gp->lpart += (size_t)loss_partials(&f, gp->fprec);
        gp->apart += tc_adjoint_slot_elems(&f);
        gp->dcs += (size_t)f.n_layers * f.nz;
    }
    return PBD_OK;
}

struct GradCarve {
    int* status;
    void* pack;
    JobDev *fwd, *adj;
    int *fcnt, *acnt;
    float* fpart;
    double* lpart;
    float *apart, *dcs, *dsgs;
};

static size_t carve_grad(void* base, int n_jobs, const GradPlan& gp, GradCarve& g) {
    Carve c(base);
    g.status = c.take<int>(kStatusInts);
    g.fwd = c.take<JobDev>(n_jobs);
    g.adj = c.take<JobDev>(n_jobs);
    g.fcnt = c.take<int>(2 + gp.arr);
    g.acnt = c.take<int>(tc_adjoint_counter_ints(n_jobs, gp.max_l));
    g.fpart = c.take<float>(gp.fpart);
    g.lpart = c.take<double>(gp.lpart);
    g.apart = c.take<float>(gp.apart);
    g.dcs = c.take<float>(gp.dcs);
    g.dsgs = c.take<float>(gp.dcs);
    g.pack = c.take<char>(gp.pack);
    return c.used + 256;
}

// Planning of a batched launch (host).  When every job has at most kMaxChunkCost layers,
// one work item covers all layers of a (job, slice, tile) and writes the output slice
// directly ("direct" mode: no partial sums, no partial buffer; the many jobs keep the
// grid balanced).  Otherwise items hold `chunk` layers and partial slices are summed.
struct BatchPlan {
    int chunk, direct, items;
    size_t nch, part, arr, pack;
};

static int plan_batch(const pbd_job* jobs, int n_jobs, int precision, BatchPlan* bp) {
    if (!jobs) return PBD_ERR_NULL_ARG;
    if (n_jobs <= 0) return PBD_ERR_BAD_DIM;
    if (n_jobs > PBD_MAX_JOBS) return PBD_ERR_TOO_MANY;
    PBD_TRY(check_precision(precision));
    int max_l = 0, chunk = kMaxChunkCost, max_sx = 1, max_sy = 1;
    for (int k = 0; k < n_jobs; ++k) {
        PBD_TRY(host_validate_field(&jobs[k].field));
        PBD_TRY(check_field_precision(&jobs[k].field, precision));
        max_l = max_l > jobs[k].field.n_layers ? max_l : jobs[k].field.n_layers;
        max_sx = max_sx > jobs[k].field.n_sx ? max_sx : jobs[k].field.n_sx;
        max_sy = max_sy > jobs[k].field.n_sy ? max_sy : jobs[k].field.n_sy;
        const int ch = choose_fwd_chunk(&jobs[k].field, precision);
        chunk = ch < chunk ? ch : chunk;
    }
    bp->direct = (max_l <= kMaxChunkCost && g_fwd_chunk == 0) ? 1 : 0;
    bp->chunk = bp->direct ? max_l : chunk;
    size_t items = 0;
    bp->nch = 0;
    bp->part = 0;
    bp->arr = 0;
    for (int k = 0; k < n_jobs; ++k) {
        size_t pe = 0;
        int it = 0;
        PBD_TRY(fwd_plan_sizes(&jobs[k].field, bp->chunk, &pe, &it));
        items += it;
        bp->nch += jobs[k].field.nz;
        const pbd_field& f = jobs[k].field;
        bp->arr += (size_t)f.nz * ((f.nx + kTile - 1) / kTile) * ((f.ny + kTile - 1) / kTile) *
                   kTcFwdWarps;
        bp->part += bp->direct ? 0 : pe;
    }
    if (items > (size_t)1 << 30) return PBD_ERR_UNSUPPORTED;
    bp->items = (int)items;
    bp->pack = precision == PBD_PREC_FP16X3 ? tc16_pack_bytes(n_jobs, max_l, max_sx, max_sy) : 0;
    return PBD_OK;
}

int pbd_forward_batch_workspace(const pbd_job* jobs, int n_jobs, int precision, size_t* bytes) {
    if (!bytes) return PBD_ERR_NULL_ARG;
    BatchPlan bp;
    PBD_TRY(plan_batch(jobs, n_jobs, precision, &bp));
    Carve c(nullptr);
    c.take<int>(kStatusInts);
    c.take<JobDev>(n_jobs);
    c.take<int>(2 + bp.arr);
    c.take<FwdItem>(bp.items);
    c.take<int>(bp.nch);
    c.take<float>(bp.part);
    c.take<char>(bp.pack);
    *bytes = c.used + 256;
    return PBD_OK;
}

int pbd_forward_batch(const pbd_job* jobs, int n_jobs, int precision, void* workspace,
                      size_t workspace_bytes, void* stream) {
    BatchPlan bp;
    PBD_TRY(plan_batch(jobs, n_jobs, precision, &bp));
    size_t need = 0;
    PBD_TRY(pbd_forward_batch_workspace(jobs, n_jobs, precision, &need));
    if (!workspace || workspace_bytes < need) return PBD_ERR_WORKSPACE;
    for (int k = 0; k < n_jobs; ++k)
        if (!jobs[k].w || !jobs[k].idd || !jobs[k].sigma || !jobs[k].dose) return PBD_ERR_NULL_ARG;
    static JobTable t;                 // large; filled under the lock below
    static std::mutex mu;
    std::lock_guard<std::mutex> g(mu);
    memset(&t, 0, sizeof(t));
    t.n = n_jobs;
    int item_base = 0;
    size_t nch_off = 0, part_off = 0, arr_off = 0;
    JobDev host_view[PBD_MAX_JOBS];
    for (int k = 0; k < n_jobs; ++k) {
        const pbd_field* f = &jobs[k].field;
        size_t pe = 0;
        int it = 0;
        PBD_TRY(fwd_plan_sizes(f, bp.chunk, &pe, &it));
        JobLite& a = t.j[k];
        a.nx = f->nx; a.ny = f->ny; a.nz = f->nz; a.nsx = f->n_sx; a.nsy = f->n_sy;
        a.nl = f->n_layers;
        a.item_base = item_base; a.max_items = it;
        a.max_chunks = bp.direct ? 1 : (f->n_layers + bp.chunk - 1) / bp.chunk;
        a.direct = bp.direct;
        a.ox = f->ox; a.oy = f->oy; a.dx = f->dx; a.dy = f->dy;
        a.sx0 = f->x0; a.sy0 = f->y0; a.dsx = f->dx_spot; a.dsy = f->dy_spot;
        a.w = jobs[k].w; a.idd = jobs[k].idd; a.sigma = jobs[k].sigma; a.dose = jobs[k].dose;
        a.partial_off = part_off; a.nchunk_off = nch_off; a.arrive_off = arr_off;
        fill_job(f, &host_view[k]);
        host_view[k].direct = bp.direct;
        item_base += it;
        nch_off += f->nz;
        arr_off += (size_t)f->nz * ((f->nx + kTile - 1) / kTile) * ((f->ny + kTile - 1) / kTile) *
                   kTcFwdWarps;
        part_off += bp.direct ? 0 : pe;
    }
    Carve c(workspace);
    int* status = c.take<int>(kStatusInts);
    JobDev* jd = c.take<JobDev>(n_jobs);
    int* counter = c.take<int>(2 + arr_off);
    FwdItem* items = c.take<FwdItem>(item_base);
    int* nchb = c.take<int>(nch_off);
    float* partb = c.take<float>(part_off);
    void* packb = c.take<char>(bp.pack);
    cudaStream_t s = (cudaStream_t)stream;
    install_table_kernel<<<(n_jobs + 31) / 32, 32, 0, s>>>(t, jd, partb, nchb, counter + 2,
                                                             status);
    PBD_LAUNCH_CHECK();
    count_launch(1);
    return launch_forward(jd, host_view, n_jobs, items, item_base, counter, 2 + arr_off,
                          status + kStatFwd, bp.chunk, 0, precision, 1, packb, bp.pack, s);
}

// ---- heterogeneous media ------------------------------------------------------------
int pbd_wed_raytrace(int nz, int ny, int nx, double oz, double dz, const float* rho, double* wed,
                     void* stream) {
    return lut_wed_raytrace(nz, ny, nx, oz, dz, rho, wed, (cudaStream_t)stream);
}

int pbd_forward_wed_workspace(const pbd_field* f, const pbd_lut_spec* spec, int precision,
                              size_t* bytes) {
    PBD_TRY(host_validate_field(f));
    PBD_TRY(check_field_precision(f, precision));
    if (!spec || !bytes) return PBD_ERR_NULL_ARG;
    WedCarve w;
    return carve_wed(f, spec, precision, nullptr, w, bytes);
}

int pbd_wed_curves_workspace(const pbd_lut_spec* spec, int n_layers, size_t* bytes) {
    if (!spec || !bytes) return PBD_ERR_NULL_ARG;
    return lut_curve_workspace(spec, n_layers, bytes);
}

int pbd_build_wed_curves(const pbd_lut_spec* spec, int n_layers, const double* energies,
                         const double* range_shift, void* curves, size_t curves_bytes,
                         void* stream) {
    if (!spec || !energies || !curves) return PBD_ERR_NULL_ARG;
    return lut_wed_curves(spec, n_layers, energies, range_shift, curves, curves_bytes,
                          (cudaStream_t)stream);
}

// Tensor-core precisions: every layer's lateral map (depth dose = the activity table) from
// one launch of the forward in its per-layer-maps mode, so that a unit's layers share its
// distance tables.  err: the forward's error word (the caller's status header).
static int forward_layer_maps(const pbd_field* f, const float* w, const double* act,
                              const double* sigma, float* lateral, size_t lstride, int precision,
                              void* base, size_t bytes, cudaStream_t s, int* err) {
    size_t need = 0;
    Ws ws;
    PBD_TRY(carve_ws(f, true, false, false, precision, nullptr, ws, &need));
    if (!base || bytes < need) return PBD_ERR_WORKSPACE;
    PBD_TRY(carve_ws(f, true, false, false, precision, base, ws, &need));
    JobPair p;
    memset(&p, 0, sizeof(p));
    p.n = 1;
    JobDev& J = p.j[0];
    fill_job(f, &J);
    J.w = w; J.idd = act; J.sigma = sigma; J.dose = lateral;
    J.layer_stride = lstride;
    J.max_chunks = (f->n_layers + ws.f_chunk - 1) / ws.f_chunk;
    J.item_base = 0; J.max_items = ws.f_items;
    J.partial = ws.fpart; J.nchunks = ws.fnch; J.arrive = ws.farr;
    install_jobs_kernel<<<1, 32, 0, s>>>(p, ws.jobs, nullptr);
    PBD_LAUNCH_CHECK();
    count_launch(1);
    // no poison pass here: the combine's poison pass reads this error word too
    return launch_forward(ws.jobs, &J, 1, ws.fitems, ws.f_items, ws.counters, ws.n_fcount, err,
                          ws.f_chunk, 0, precision, 0, nullptr, 0, s);
}

// Activity table, the per-layer lateral maps, then the combine.
static int forward_wed_body(const pbd_field* f, const pbd_lut_spec* spec, const void* curves,
                            size_t curves_bytes, const float* w, const double* sigma,
                            const double* wed, float* dose, int precision, const WedCarve& wc,
                            void* stream) {
    cudaStream_t s = (cudaStream_t)stream;
    const size_t nslice = (size_t)f->ny * f->nx;
    const size_t lstride = wed_lateral_stride(f);
    PBD_TRY(lut_wed_activity(spec, f->n_layers, curves, curves_bytes, wed, f->nz, nslice, wc.act,
                             s));
    PBD_TRY(cuda_rc(cudaMemsetAsync(wc.status, 0, kStatusInts * sizeof(int), s)));
    const int* fwd_err = nullptr;
    if (precision != PBD_PREC_FP32) {
        PBD_TRY(forward_layer_maps(f, w, wc.act, sigma, wc.lateral, lstride, precision, wc.batch,
                                   wc.batch_bytes, s, wc.status + kStatFwd));
        fwd_err = wc.status + kStatFwd;
    } else {
        // FP32: one single-layer job per layer through the batched forward (its own poison)
        pbd_job jobs[PBD_MAX_JOBS];
        for (int l0 = 0; l0 < f->n_layers; l0 += PBD_MAX_JOBS) {
            const int n = f->n_layers - l0 < PBD_MAX_JOBS ? f->n_layers - l0 : PBD_MAX_JOBS;
            wed_jobs(f, l0, n, w, sigma, wc.act, wc.lateral, jobs);
            PBD_TRY(pbd_forward_batch(jobs, n, precision, wc.batch, wc.batch_bytes, stream));
        }
    }
    return lut_wed_combine(spec, f->n_layers, wc.lateral, lstride, wed, (size_t)f->nz * nslice,
                           dose, wc.status + kStatCmb, fwd_err, curves, curves_bytes, s);
}

static int wed_setup(const pbd_field* f, const pbd_lut_spec* spec, int precision, void* workspace,
                     size_t workspace_bytes, WedCarve& wc) {
    PBD_TRY(host_validate_field(f));
    PBD_TRY(check_field_precision(f, precision));
    size_t need = 0;
    PBD_TRY(carve_wed(f, spec, precision, nullptr, wc, &need));
    if (!workspace || workspace_bytes < need) return PBD_ERR_WORKSPACE;
    return carve_wed(f, spec, precision, workspace, wc, &need);
}

int pbd_forward_wed(const pbd_field* f, const pbd_lut_spec* spec, const double* energies,
                    const double* range_shift, const float* w, const double* sigma,
                    const double* wed, float* dose, int precision, void* workspace,
                    size_t workspace_bytes, void* stream) {
    if (!f || !spec || !energies || !w || !sigma || !wed || !dose) return PBD_ERR_NULL_ARG;
    WedCarve wc;
    PBD_TRY(wed_setup(f, spec, precision, workspace, workspace_bytes, wc));
    PBD_TRY(lut_wed_curves(spec, f->n_layers, energies, range_shift, wc.curves, wc.curves_bytes,
                           (cudaStream_t)stream));
    return forward_wed_body(f, spec, wc.curves, wc.curves_bytes, w, sigma, wed, dose, precision,
                            wc, stream);
}

int pbd_forward_wed_curves(const pbd_field* f, const pbd_lut_spec* spec, const void* curves,
                           size_t curves_bytes, const float* w, const double* sigma,
                           const double* wed, float* dose, int precision, void* workspace,
                           size_t workspace_bytes, void* stream) {
    if (!f || !spec || !curves || !w || !sigma || !wed || !dose) return PBD_ERR_NULL_ARG;
    WedCarve wc;
    PBD_TRY(wed_setup(f, spec, precision, workspace, workspace_bytes, wc));
    return forward_wed_body(f, spec, curves, curves_bytes, w, sigma, wed, dose, precision, wc,
                            stream);
}

// ---- heterogeneous media: dL/dW and dL/dR -------------------------------------------
// D = sum_l IDD_l(WED) Lat_l, Lat_l = Gy_l W_l Gx_l^T with water's widths at the geometric depth.
//  * dL/dW_l = A_l^T (g IDD_l(WED)): the adjoint of layer l's map g IDD_l(WED) with depth dose 1
//    on its active slices.
//  * dL/dR_l = sum_v g dIDD_l/dR(WED) Lat_l + sum_z dL/dsigma_lz dsigma_lz/dR.  The first term is
//    <A_l^T (g dIDD_l/dR(WED)), W_l> = sum_z <P_lz, W_l> of a second job set whose maps use the
//    curves' central difference at range shifts +-h; the second is the first set's per-pair
//    dL/dsigma dotted with dsigma/dR.
// Tensor-core precisions: one adjoint launch over every job (set s, layer l), the batched
// adjoint's machinery with single-layer jobs.  FP32: one SIMT adjoint per (set, layer).
struct WedAdjCarve {
    int sets;            // 1: dL/dW; 2: dL/dW and dL/dR
    int* status;         // status header: the adjoint's error word
    double* act;         // (sets, L, nz) activity tables
    float* maps;         // (sets, L, wed_lateral_stride) the jobs' dL/dD maps
    double* zeros;       // FP32 with dL/dR: (L, nz) zero table
    float* gw2;          // set 1's dL/dW (unused), (L, nsy, nsx)
    float* r1;           // set 1's part of dL/dR, (L)
    void* adj;           // FP32: one single-layer adjoint's workspace, reused job after job
    size_t adj_bytes;
    JobDev *fwd, *jobs;  // tensor cores: the install kernel's (unused) forward views, the jobs
    float *apart, *dcs, *dsgs;
    int* acnt;           // the adjoint's unit counter block
    size_t slot_elems;   // slots of one single-layer job
};

static int carve_wed_adj(const pbd_field* f, int precision, int sets, void* base, WedAdjCarve& w,
                         size_t* used) {
    pbd_field f1 = *f;
    f1.n_layers = 1;
    const size_t L = (size_t)f->n_layers, per = (size_t)f->n_sy * f->n_sx;
    const size_t nj = (size_t)sets * L;
    Carve c(base);
    w.sets = sets;
    w.status = c.take<int>(kStatusInts);
    w.act = c.take<double>(nj * f->nz);
    w.maps = c.take<float>(nj * wed_lateral_stride(f));
    w.zeros = nullptr; w.gw2 = nullptr; w.r1 = nullptr;
    if (sets == 2) {
        w.gw2 = c.take<float>(L * per);
        w.r1 = c.take<float>(L);
        if (precision == PBD_PREC_FP32) w.zeros = c.take<double>(L * f->nz);
    }
    w.adj = nullptr; w.adj_bytes = 0;
    w.fwd = w.jobs = nullptr; w.apart = w.dcs = w.dsgs = nullptr; w.acnt = nullptr;
    w.slot_elems = 0;
    if (precision == PBD_PREC_FP32) {
        size_t ab = 0;
        PBD_TRY(pbd_adjoint_workspace(&f1, precision, &ab));
        w.adj = c.take<char>(ab);
        w.adj_bytes = ab;
    } else {
        int n1 = 0;
        PBD_TRY(tc_adjoint_dims(precision, &f1, &n1));
        w.slot_elems = tc_adjoint_slot_elems(&f1);
        w.fwd = c.take<JobDev>(nj);
        w.jobs = c.take<JobDev>(nj);
        w.apart = c.take<float>(nj * w.slot_elems);
        w.dcs = c.take<float>(nj * f->nz);
        w.dsgs = c.take<float>(nj * f->nz);
        w.acnt = c.take<int>(tc_adjoint_counter_ints((int)nj, 1));
    }
    *used = c.used + 256;
    return PBD_OK;
}

__global__ void wed_range_combine_kernel(float* grad_range, const float* r1, int n) {
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l < n) grad_range[l] += r1[l];
}

// The adjoints of the carve's job sets (maps and activity tables already written).
static int wed_adjoint_jobs(const pbd_field* f, const WedAdjCarve& wc, const float* w,
                            const double* sigma, const double* dsigma_dr, float* grad_w,
                            float* grad_range, int precision, cudaStream_t s) {
    pbd_field f1 = *f;
    f1.n_layers = 1;
    const int L = f->n_layers;
    const size_t per = (size_t)f->n_sy * f->n_sx, lstride = wed_lateral_stride(f);
    const size_t nzL = (size_t)L * f->nz;
    const bool rng = wc.sets == 2;
    if (precision == PBD_PREC_FP32) {
        PBD_TRY(cuda_rc(cudaMemsetAsync(wc.status, 0, kStatusInts * sizeof(int), s)));
        if (rng) PBD_TRY(cuda_rc(cudaMemsetAsync(wc.zeros, 0, nzL * sizeof(double), s)));
        for (int st = 0; st < wc.sets; ++st)
            for (int l = 0; l < L; ++l) {
                const size_t lz = (size_t)l * f->nz;
                const double* act = wc.act + (size_t)st * nzL + lz;
                const double* didd = !rng ? nullptr : (st == 0 ? wc.zeros + lz : act);
                const double* dsig = !rng ? nullptr : (st == 0 ? dsigma_dr + lz : wc.zeros + lz);
                float* gw = (st == 0 ? grad_w : wc.gw2) + (size_t)l * per;
                float* gr = !rng ? nullptr : (st == 0 ? grad_range : wc.r1) + l;
                PBD_TRY(adjoint_one(&f1, w + (size_t)l * per, act, sigma + lz, didd, dsig,
                                    wc.maps + ((size_t)st * L + l) * lstride, gw, gr, precision,
                                    wc.adj, wc.adj_bytes, wc.status + kStatAdj, s));
            }
    } else {
        // the jobs installed kGradInstall at a time (the first group also clears the status
        // header), then one adjoint launch and one reduce launch over them
        const int nj = wc.sets * L;
        std::vector<JobDev> views((size_t)nj);
        GradBufs b{};
        b.fwd = wc.fwd; b.adj = wc.jobs; b.fpart = nullptr; b.farr = nullptr; b.lpart = nullptr;
        b.apart = wc.apart; b.dcs = wc.dcs; b.dsgs = wc.dsgs; b.fwd_err = nullptr;
        b.status = wc.status;
        JobDev base{};
        fill_job(&f1, &base);
        for (int g0 = 0; g0 < nj; g0 += kGradInstall) {
            GradTable t;
            memset(&t, 0, sizeof(t));
            t.base = g0;
            t.n = std::min(kGradInstall, nj - g0);
            for (int k = 0; k < t.n; ++k) {
                const int jb = g0 + k, st = jb / L, l = jb % L;
                const size_t lz = (size_t)l * f->nz;
                GradLite& a = t.j[k];
                a.nx = base.nx; a.ny = base.ny; a.nz = base.nz;
                a.nsx = base.nsx; a.nsy = base.nsy; a.nl = 1;
                a.max_chunks_f = 1; a.max_chunks_a = 1; a.direct = 0; a.n_loss_part = 0;
                a.ox = base.ox; a.oy = base.oy; a.dx = base.dx; a.dy = base.dy;
                a.sx0 = base.sx0; a.sy0 = base.sy0; a.dsx = base.dsx; a.dsy = base.dsy;
                a.w = w + (size_t)l * per;
                a.idd = wc.act + (size_t)st * nzL + lz;
                a.sigma = sigma + lz;
                // set 0: the sigma term of dL/dR; set 1: sum_z <P, W> (the activity is 1 on
                // every slice that the reduce reads)
                a.didd = rng && st == 1 ? a.idd : nullptr;
                a.dsig = rng && st == 0 ? dsigma_dr + lz : nullptr;
                a.grad_dose = wc.maps + (size_t)jb * lstride;
                a.grad_w = (st == 0 ? grad_w : wc.gw2) + (size_t)l * per;
                a.grad_range = !rng ? nullptr : (st == 0 ? grad_range : wc.r1) + l;
                a.slot_off = (size_t)jb * wc.slot_elems;
                a.dcs_off = (size_t)jb * f->nz;
                JobDev& v = views[(size_t)jb];
                v = base;
                v.nl = 1; v.max_chunks = 1;
                v.w = a.w; v.idd = a.idd; v.sigma = a.sigma; v.grad_dose = a.grad_dose;
                v.didd_dr = a.didd; v.dsig_dr = a.dsig;
                v.grad_w = a.grad_w; v.grad_range = a.grad_range;
                v.partial = wc.apart + a.slot_off;
                v.dc = wc.dcs + a.dcs_off; v.dsg = wc.dsgs + a.dcs_off;
            }
            install_grad_kernel<<<(std::max(t.n, kStatusInts) + 63) / 64, 64, 0, s>>>(t, b);
            PBD_LAUNCH_CHECK();
            count_launch(1);
        }
        PBD_TRY(launch_adjoint_tc(precision, wc.jobs, views.data(), nj, wc.acnt,
                                  wc.status + kStatAdj, 1, rng ? 1 : 0, 0, 0, s));
    }
    if (rng) {
        wed_range_combine_kernel<<<(L + 127) / 128, 128, 0, s>>>(grad_range, wc.r1, L);
        PBD_LAUNCH_CHECK();
        count_launch(1);
    }
    return PBD_OK;
}

int pbd_adjoint_wed_workspace(const pbd_field* f, const pbd_lut_spec* spec, int precision,
                              size_t* bytes) {
    PBD_TRY(host_validate_field(f));
    PBD_TRY(check_field_precision(f, precision));
    PBD_TRY(adjoint_supported(f));
    if (!spec || !bytes) return PBD_ERR_NULL_ARG;
    WedAdjCarve w;
    return carve_wed_adj(f, precision, 1, nullptr, w, bytes);
}

int pbd_adjoint_wed(const pbd_field* f, const pbd_lut_spec* spec, const void* curves,
                    size_t curves_bytes, const float* w, const double* sigma, const double* wed,
                    const float* grad_dose, float* grad_w, int precision, void* workspace,
                    size_t workspace_bytes, void* stream) {
    if (!f || !spec || !curves || !w || !sigma || !wed || !grad_dose || !grad_w)
        return PBD_ERR_NULL_ARG;
    PBD_TRY(host_validate_field(f));
    PBD_TRY(check_field_precision(f, precision));
    PBD_TRY(adjoint_supported(f));
    WedAdjCarve wc;
    size_t need = 0;
    PBD_TRY(carve_wed_adj(f, precision, 1, nullptr, wc, &need));
    if (!workspace || workspace_bytes < need) return PBD_ERR_WORKSPACE;
    PBD_TRY(carve_wed_adj(f, precision, 1, workspace, wc, &need));
    cudaStream_t s = (cudaStream_t)stream;
    const size_t nslice = (size_t)f->ny * f->nx, nvox = (size_t)f->nz * nslice;
    PBD_TRY(lut_wed_activity(spec, f->n_layers, curves, curves_bytes, wed, f->nz, nslice, wc.act,
                             s));
    PBD_TRY(lut_wed_grad_maps(spec, f->n_layers, curves, curves_bytes, grad_dose, wed, nvox,
                              wed_lateral_stride(f), wc.maps, s));
    return wed_adjoint_jobs(f, wc, w, sigma, nullptr, grad_w, nullptr, precision, s);
}

int pbd_adjoint_wed_range_workspace(const pbd_field* f, const pbd_lut_spec* spec, int precision,
                                    size_t* bytes) {
    PBD_TRY(host_validate_field(f));
    PBD_TRY(check_field_precision(f, precision));
    PBD_TRY(adjoint_supported(f));
    if (!spec || !bytes) return PBD_ERR_NULL_ARG;
    WedAdjCarve w;
    return carve_wed_adj(f, precision, 2, nullptr, w, bytes);
}

int pbd_adjoint_wed_range(const pbd_field* f, const pbd_lut_spec* spec, const void* curves,
                          size_t curves_bytes, const void* curves_p, const void* curves_m,
                          double h, const float* w, const double* sigma, const double* dsigma_dr,
                          const double* wed, const float* grad_dose, float* grad_w,
                          float* grad_range, int precision, void* workspace,
                          size_t workspace_bytes, void* stream) {
    if (!f || !spec || !curves || !curves_p || !curves_m || !w || !sigma || !dsigma_dr || !wed ||
        !grad_dose || !grad_w || !grad_range)
        return PBD_ERR_NULL_ARG;
    if (!(h > 0.0) || !isfinite(h)) return PBD_ERR_BAD_VALUE;
    PBD_TRY(host_validate_field(f));
    PBD_TRY(check_field_precision(f, precision));
    PBD_TRY(adjoint_supported(f));
    WedAdjCarve wc;
    size_t need = 0;
    PBD_TRY(carve_wed_adj(f, precision, 2, nullptr, wc, &need));
    if (!workspace || workspace_bytes < need) return PBD_ERR_WORKSPACE;
    PBD_TRY(carve_wed_adj(f, precision, 2, workspace, wc, &need));
    cudaStream_t s = (cudaStream_t)stream;
    const int L = f->n_layers;
    const size_t nslice = (size_t)f->ny * f->nx, nvox = (size_t)f->nz * nslice;
    const size_t lstride = wed_lateral_stride(f);
    // set 0: g IDD_l(WED) on the nominal curves' active slices; set 1: g dIDD_l/dR(WED) on the
    // slices that either shifted curve reaches
    PBD_TRY(lut_wed_activity(spec, L, curves, curves_bytes, wed, f->nz, nslice, wc.act, s));
    PBD_TRY(lut_wed_grad_maps(spec, L, curves, curves_bytes, grad_dose, wed, nvox, lstride,
                              wc.maps, s));
    PBD_TRY(lut_wed_activity(spec, L, curves_p, curves_bytes, wed, f->nz, nslice,
                             wc.act + (size_t)L * f->nz, s, curves_m, curves_bytes));
    PBD_TRY(lut_wed_grad_maps_dr(spec, L, curves_p, curves_bytes, curves_m, curves_bytes, h,
                                 grad_dose, wed, nvox, lstride, wc.maps + (size_t)L * lstride, s));
    return wed_adjoint_jobs(f, wc, w, sigma, dsigma_dr, grad_w, grad_range, precision, s);
}

int pbd_loss_grad_batch_workspace(const pbd_grad_job* jobs, int n_jobs, int precision,
                                  size_t* bytes) {
    if (!bytes) return PBD_ERR_NULL_ARG;
    GradPlan gp;
    PBD_TRY(plan_grad_batch(jobs, n_jobs, precision, &gp));
    GradCarve g;
    *bytes = carve_grad(nullptr, n_jobs, gp, g);
    return PBD_OK;
}

int pbd_loss_grad_batch(const pbd_grad_job* jobs, int n_jobs, int precision, void* workspace,
                        size_t workspace_bytes, void* stream) {
    GradPlan gp;
    PBD_TRY(plan_grad_batch(jobs, n_jobs, precision, &gp));
    for (int k = 0; k < n_jobs; ++k) {
        const pbd_grad_job& j = jobs[k];
        if (!j.w || !j.idd || !j.sigma || !j.mask || !j.presc || !j.dose || !j.grad_dose ||
            !j.loss || !j.grad_w)
            return PBD_ERR_NULL_ARG;
        if (gp.with_range && (!j.didd_dr || !j.dsigma_dr)) return PBD_ERR_NULL_ARG;
    }
    GradCarve g;
    const size_t need = carve_grad(nullptr, n_jobs, gp, g);
    if (!workspace || workspace_bytes < need) return PBD_ERR_WORKSPACE;
    carve_grad(workspace, n_jobs, gp, g);
    cudaStream_t s = (cudaStream_t)stream;
    GradBufs b{g.fwd, g.adj, g.fpart, g.fcnt + 2, g.lpart, g.apart, g.dcs, g.dsgs,
               g.status + kStatFwd, g.status};
    PBD_TRY(cuda_rc(cudaMemsetAsync(g.acnt, 0,
                                    tc_adjoint_counter_ints(n_jobs, gp.max_l) * sizeof(int), s)));
    const int a_chunk = g_adj_chunk > 0 ? g_adj_chunk : kBatchAdjChunk;
    JobDev fview[PBD_MAX_JOBS], aview[PBD_MAX_JOBS];
    size_t arr = 0, fpart = 0, lpart = 0, apart = 0, dcs = 0;
    GradTable t;
    for (int base = 0; base < n_jobs; base += kGradInstall) {
        memset(&t, 0, sizeof(t));
        t.base = base;
        t.n = n_jobs - base < kGradInstall ? n_jobs - base : kGradInstall;
        for (int q = 0; q < t.n; ++q) {
            const int k = base + q;
            const pbd_grad_job& j = jobs[k];
            const pbd_field* f = &j.field;
            const size_t tiles =
                (size_t)((f->nx + kTile - 1) / kTile) * ((f->ny + kTile - 1) / kTile);
            size_t pe = 0;
            int it = 0;
            PBD_TRY(fwd_plan_sizes(f, gp.chunk, &pe, &it));
            GradLite& a = t.j[q];
            a.nx = f->nx; a.ny = f->ny; a.nz = f->nz; a.nsx = f->n_sx; a.nsy = f->n_sy;
            a.nl = f->n_layers;
            a.max_chunks_f = gp.direct ? 1 : (f->n_layers + gp.chunk - 1) / gp.chunk;
            a.max_chunks_a = (f->n_layers + a_chunk - 1) / a_chunk;
            a.direct = gp.direct;
            a.n_loss_part = loss_partials(f, gp.fprec);
            a.ox = f->ox; a.oy = f->oy; a.dx = f->dx; a.dy = f->dy;
            a.sx0 = f->x0; a.sy0 = f->y0; a.dsx = f->dx_spot; a.dsy = f->dy_spot;
            a.w = j.w; a.idd = j.idd; a.sigma = j.sigma; a.didd = j.didd_dr; a.dsig = j.dsigma_dr;
            a.mask = j.mask; a.presc = j.presc; a.dose = j.dose; a.grad_dose = j.grad_dose;
            a.loss = j.loss; a.grad_w = j.grad_w; a.grad_range = j.grad_range;
            a.fpart_off = fpart; a.arrive_off = arr; a.loss_off = lpart; a.slot_off = apart;
            a.dcs_off = dcs;
            fill_job(f, &fview[k]);
            fview[k].max_chunks = a.max_chunks_f;
            fview[k].direct = a.direct;
            aview[k] = fview[k];
            aview[k].max_chunks = a.max_chunks_a;
            aview[k].grad_dose = j.grad_dose;   // the adjoint checks its alignment
            arr += (size_t)f->nz * tiles * kTcFwdWarps;
            fpart += gp.direct ? 0 : pe;
            lpart += (size_t)a.n_loss_part;
            apart += tc_adjoint_slot_elems(f);
            dcs += (size_t)f->n_layers * f->nz;
        }
        install_grad_kernel<<<(t.n + 63) / 64, 64, 0, s>>>(t, b);
        PBD_LAUNCH_CHECK();
        count_launch(1);
    }
    PBD_TRY(launch_forward(g.fwd, fview, n_jobs, nullptr, 0, g.fcnt, 2 + gp.arr,
                           g.status + kStatFwd, gp.chunk, 1, gp.fprec, 0, g.pack, gp.pack, s));
    return launch_adjoint_tc(precision, g.adj, aview, n_jobs, g.acnt, g.status + kStatAdj, a_chunk,
                             gp.with_range, 1, 1, s);
}

}  // extern "C"
