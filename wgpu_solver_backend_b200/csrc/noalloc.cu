// wsb_dot_tree256_noalloc: the reference-arithmetic dot product (the pass
// structure of encode_dot_scalar_into) with its scratch in a file-scope
// device array instead of memory the caller or the library allocates.
//
// Some callers cannot call cudaMalloc at the point where they need a dot
// product: a host loop that runs under a memory budget which the rest of
// its process has already spent, code that must not pay the device-wide
// synchronisation that cudaMalloc/cudaFree can cause, or a caller whose only
// device memory is the buffers it was handed. For them this entry point
// touches no allocator: inputs and output are the caller's, and the
// partial sums between passes go to g_dot_scratch below, which every GPU
// that loads this library keeps (about 257 KiB) until the process exits.
#include <mutex>

#include "kernels_ref.cuh"

namespace wsb {
namespace {

constexpr uint32_t kMaxN = WSB_NOALLOC_DOT_MAX_N;
// Partials of the first pass, then of the second, as ref_dot lays them out.
constexpr size_t kScratchFloats = (kMaxN + 255u) / 256u + ((kMaxN + 255u) / 256u + 255u) / 256u + 2u;

static __device__ __align__(256) float g_dot_scratch[kScratchFloats];

// Device address of g_dot_scratch per device. In host code the symbol is
// only a stand-in; cudaGetSymbolAddress with the device current gives the
// address a kernel can use. It is looked up once per device and kept for the
// life of the process, which assumes the device's primary context (and with
// it this module's copy of the array) is never reset while the library is in
// use: after a cudaDeviceReset the kept address would be stale.
std::mutex g_mu;
float *g_addr[64] = {};

int scratch_for(Context *ctx, float **out) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (ctx->device < 0 || ctx->device >= 64) return fail(ctx, WSB_ERR_UNSUPPORTED, "device ordinal %d", ctx->device);
    if (!g_addr[ctx->device]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_dot_scratch);
        if (e != cudaSuccess)
            return fail(ctx, WSB_ERR_CUDA, "cudaGetSymbolAddress(scratch) failed: %s", cudaGetErrorString(e));
        g_addr[ctx->device] = static_cast<float *>(p);
    }
    *out = g_addr[ctx->device];
    return WSB_OK;
}

}  // namespace
}  // namespace wsb

using namespace wsb;

// The first call on a device looks up the scratch address (set-up); make
// that first call before any stream capture. Calls that overlap on the GPU
// (other streams, other host threads on the same device) share the scratch
// and race; order them on one stream. Nothing needs clearing between calls:
// every pass writes the partials it later reads.
extern "C" int wsb_dot_tree256_noalloc(wsb_context *ctx_in, const float *d_a, const float *d_b, uint32_t n,
                                       float *d_out) {
    Context *ctx = reinterpret_cast<Context *>(ctx_in);
    if (!ctx) return fail(nullptr, WSB_ERR_BAD_INPUT, "context is null");
    if (n > kMaxN)
        return fail(ctx, WSB_ERR_BAD_INPUT, "wsb_dot_tree256_noalloc: n = %u exceeds the static scratch limit %u", n,
                    kMaxN);
    if (!d_out || (n && (!d_a || !d_b))) return fail(ctx, WSB_ERR_BAD_INPUT, "wsb_dot_tree256_noalloc: null pointer");
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e != cudaSuccess) return fail(ctx, WSB_ERR_CUDA, "cudaSetDevice: %s", cudaGetErrorString(e));
    float *scratch = nullptr;
    int rc = scratch_for(ctx, &scratch);
    if (rc) return rc;
    e = ref_dot(ctx->stream, n, d_a, d_b, scratch, d_out);
    if (e != cudaSuccess) return fail(ctx, WSB_ERR_CUDA, "wsb_dot_tree256_noalloc launch: %s", cudaGetErrorString(e));
    return WSB_OK;
}
