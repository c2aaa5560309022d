// Allocation-free variant of the few-column FP64 T contraction.
//
// Some callers cannot allocate device memory while they call into the solver:
// a host code whose device memory is owned by another runtime or framework
// (the buffers it hands over come from that allocator), a code running inside
// a memory-budgeted or preallocated serving loop, or one that must not
// introduce allocation calls (which synchronise the device) into a timed
// inner loop.  plx_contract_noalloc computes S = T X for a few columns on
// buffers the caller already owns and allocates nothing itself: its only
// scratch space is the file-scope device array below.
//
// The scratch array holds the split-K partial sums of the contraction; every
// element the reduction reads is written by the same call first, so nothing
// has to start at zero.  All calls on a device share the one array and it
// keeps the last call's contents: two calls whose kernels overlap on the GPU
// (different streams, host threads or processes sharing a context) race on it.
// The kernels run on the context's own stream, which is not ordered after the
// caller's streams: the caller finishes writing X on the device before the
// call.  The call waits for its kernels, so S is complete when it returns.
#include <mutex>

#include "plx_internal.h"
#include "skinny.cuh"

namespace {

// Maximum scratch: 2^21 doubles (16 MiB), held by every GPU that loads the
// library until the process exits.
constexpr size_t kNoAllocScratchDoubles = size_t(1) << 21;
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocScratchDoubles];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
double *g_scratch_ptr[kMaxDevices] = {};

// The device address of the scratch array on the current device.  In host
// code `g_noalloc_scratch` is only a host-side stand-in for the symbol; the
// address a kernel can use comes from cudaGetSymbolAddress, taken once per
// device with that device current.
double *scratch_for_device(int dev) {
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (dev < 0 || dev >= kMaxDevices) throw plx::Error(PLX_ERR_ARG, "device ordinal out of range");
    if (!g_scratch_ptr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess)
            throw plx::Error(PLX_ERR_CUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
        g_scratch_ptr[dev] = static_cast<double *>(p);
    }
    return g_scratch_ptr[dev];
}

template <int R>
void launch_partial(dim3 grid, cudaStream_t st, int n, int kchunk, const double *X, const double *T, double *part) {
    plx::skinny_partial<R><<<grid, plx::kSkinnyCols, 0, st>>>(n, kchunk, X, T, part);
}

}  // namespace

extern "C" plx_status plx_contract_noalloc(plx_geom *g, int32_t count, const double *d_X, double *d_S) {
    if (!g || !d_X || !d_S) return PLX_ERR_ARG;
    plx_ctx *ctx = g->ctx;
    try {
        PLX_CHECK_CUDA(cudaSetDevice(ctx->device));
        if (!g->has_T) throw plx::Error(PLX_ERR_ARG, "geometry was created without the dense T matrix");
        if (count < 1 || count > 16)
            throw plx::Error(PLX_ERR_ARG, "plx_contract_noalloc takes 1 to 16 columns, got " + std::to_string(count));
        const int n = g->n_var;
        int ks, kchunk;
        plx::skinny_split(n, ks, kchunk);
        const size_t need = (size_t)ks * count * n;
        if (need > kNoAllocScratchDoubles)
            throw plx::Error(PLX_ERR_ARG, "plx_contract_noalloc: " + std::to_string(count) + " columns of order " +
                                              std::to_string(n) + " need " + std::to_string(need) +
                                              " scratch doubles, above the fixed maximum of " +
                                              std::to_string(kNoAllocScratchDoubles));
        double *part = scratch_for_device(ctx->device);
        cudaStream_t st = ctx->stream;
        dim3 grid(plx::n_blocks(n, plx::kSkinnyCols), ks);
        switch (count) {
#define PLX_NA(RR) \
    case RR: launch_partial<RR>(grid, st, n, kchunk, d_X, g->d_T.p, part); break;
            PLX_NA(1) PLX_NA(2) PLX_NA(3) PLX_NA(4) PLX_NA(5) PLX_NA(6) PLX_NA(7) PLX_NA(8)
            PLX_NA(9) PLX_NA(10) PLX_NA(11) PLX_NA(12) PLX_NA(13) PLX_NA(14) PLX_NA(15) PLX_NA(16)
#undef PLX_NA
        }
        plx::skinny_reduce<<<plx::n_blocks((int64_t)count * n, 256), 256, 0, st>>>(n, count, ks, part, d_S);
        ctx->launches += 2;
        PLX_CHECK_CUDA(cudaGetLastError());
        PLX_CHECK_CUDA(cudaStreamSynchronize(st));
        return PLX_OK;
    } catch (const plx::Error &e) {
        ctx->last_error = e.msg;
        return e.code;
    } catch (const std::exception &e) {
        // a failed lock or message allocation must not leave the C ABI as an exception
        try {
            ctx->last_error = e.what();
        } catch (...) {
        }
        return PLX_ERR_ARG;
    }
}
