// noalloc.cu -- forward dose for callers that cannot allocate device memory.
//
// The regular entry points take their scratch from a workspace the caller allocates.  Some
// callers cannot do that: a real-time adaptive-therapy loop that reserves all device memory
// once at start-up and must not risk a blocking or failing allocation while the patient is
// on the table, or a host application that owns the GPU through its own memory pool and
// forbids any other allocator.  pbd_forward_noalloc serves them: the caller passes only
// inputs and the output, and the little scratch the forward needs (the job descriptor,
// the work-item counter and error word, the work-item list and the per-slice chunk
// counts) lives in the fixed array below.
//
// The array is a file-scope __device__ object: every GPU that loads this library holds
// its 1 MiB until the process exits.  On the host its name is only a stand-in for the
// device object, never a usable address, so the entry point resolves the device address
// with cudaGetSymbolAddress once per device (on that device's first call, with the device
// current) and passes that address to the kernels.  Because the first call on a device
// does this set-up, it should come before any stream capture on that device.
//
// All calls on a device share the array and it keeps the last call's contents: the
// counter and error word are cleared on every call and the work list is rewritten, but two
// calls that overlap on the GPU (different streams, no ordering between them) race on the
// array and must not be issued.
//
// The cached address belongs to the device's primary context, the one the CUDA runtime
// uses.  It stays valid until that context is destroyed: a caller that runs
// cudaDeviceReset() after its first call on a device, or drives the device through a
// context of its own (the driver API), must not use this entry point on that device.
#include <mutex>

#include "pbd_internal.cuh"

namespace pbd {
namespace {

constexpr size_t kNoAllocScratchBytes = (size_t)1 << 20;   // 1 MiB

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_noalloc_mu;
void* g_noalloc_addr[64] = {nullptr};

// Device address of the scratch array on the current device (resolved once per device).
int noalloc_scratch(void** out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return PBD_ERR_CUDA;
    if (dev < 0 || dev >= 64) return PBD_ERR_UNSUPPORTED;
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (g_noalloc_addr[dev] == nullptr) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || p == nullptr)
            return PBD_ERR_CUDA;
        g_noalloc_addr[dev] = p;
    }
    *out = g_noalloc_addr[dev];
    return PBD_OK;
}

// Installs the job view and clears the error word (counters[1]).
__global__ void noalloc_install_kernel(JobDev J, JobDev* dst, int* err) {
    if (threadIdx.x == 0) {
        *dst = J;
        *err = 0;
    }
}

}  // namespace
}  // namespace pbd

using namespace pbd;

extern "C" int pbd_forward_noalloc(const pbd_field* f, const float* w, const double* idd,
                                   const double* sigma, float* dose, int precision,
                                   void* stream) {
    PBD_TRY(host_validate_field(f));
    if (precision < PBD_PREC_FP32 || precision > PBD_PREC_FP16X3) return PBD_ERR_BAD_VALUE;
    if (precision == PBD_PREC_FP16X3) return PBD_ERR_UNSUPPORTED;   // its spot maps need scratch
    if (precision != PBD_PREC_FP32) {
        int k1 = 0, n1 = 0;
        PBD_TRY(tc_operand_dims(precision, f->n_sx, f->n_sy, &k1, &n1));
    }
    if (!w || !idd || !sigma || !dose) return PBD_ERR_NULL_ARG;
    // One work item per (slice, tile) holding all of the slice's active layers, so each
    // item writes its slice of `dose` directly and no partial sums need scratch.
    if (f->n_layers > kMaxChunkCost) return PBD_ERR_UNSUPPORTED;
    const int chunk = f->n_layers;
    size_t partial_elems = 0;
    int items = 0;
    PBD_TRY(fwd_plan_sizes(f, chunk, &partial_elems, &items));
    Carve sizing(nullptr);
    sizing.take<JobDev>(1);
    sizing.take<int>(2);
    sizing.take<FwdItem>(items);
    sizing.take<int>(f->nz);
    if (sizing.used > kNoAllocScratchBytes) return PBD_ERR_WORKSPACE;   // beyond the fixed 1 MiB

    void* base = nullptr;
    PBD_TRY(noalloc_scratch(&base));
    Carve c(base);
    JobDev* jd = c.take<JobDev>(1);
    int* counters = c.take<int>(2);
    FwdItem* it = c.take<FwdItem>(items);
    int* nch = c.take<int>(f->nz);

    JobDev J;
    fill_job(f, &J);
    J.w = w; J.idd = idd; J.sigma = sigma; J.dose = dose;
    J.max_chunks = 1;
    J.item_base = 0;
    J.max_items = items;
    J.partial = dose;     // chunk 0 of every slice is the output itself
    J.direct = 1;
    J.nchunks = nch;
    cudaStream_t s = (cudaStream_t)stream;
    noalloc_install_kernel<<<1, 32, 0, s>>>(J, jd, counters + 1);
    PBD_LAUNCH_CHECK();
    count_launch(1);
    return launch_forward(jd, &J, 1, it, items, counters, 2, counters + 1, chunk, 0, precision, 1,
                          nullptr, 0, s);
}
