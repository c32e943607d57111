// extern "C" entry points of include/wsb.h: context, buffers, the reference
// executors, the reference-arithmetic solve, matrices, plain and batched
// solves.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <memory>

#include "engine.h"
#include "kernels_ref.cuh"

namespace wsb {

static thread_local std::string g_thread_error;

void set_thread_error(const std::string &msg) { g_thread_error = msg; }
const char *thread_error() { return g_thread_error.c_str(); }

int fail(Context *ctx, int status, const char *f, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, f);
    vsnprintf(buf, sizeof buf, f, ap);
    va_end(ap);
    g_thread_error = buf;
    if (ctx) {
        std::lock_guard<std::mutex> lk(ctx->mu);
        ctx->last_error = buf;
    }
    return status;
}

cudaMemPool_t &thread_alloc_pool() {
    static thread_local cudaMemPool_t pool = nullptr;
    return pool;
}

int dev_alloc(Context *ctx, void **p, size_t bytes, bool zero, cudaStream_t stream) {
    *p = nullptr;
    if (bytes == 0) bytes = 16;
    cudaMemPool_t pool = thread_alloc_pool();
    cudaError_t e = pool ? cudaMallocFromPoolAsync(p, bytes, pool, stream) : cudaMalloc(p, bytes);
    if (e != cudaSuccess) {
        *p = nullptr;
        return fail(ctx, e == cudaErrorMemoryAllocation ? WSB_ERR_OUT_OF_MEMORY : WSB_ERR_CUDA,
                    "cudaMalloc(%zu) failed: %s", bytes, cudaGetErrorString(e));
    }
    if (zero) {
        e = cudaMemsetAsync(*p, 0, bytes, stream);
        if (e != cudaSuccess) return fail(ctx, WSB_ERR_CUDA, "cudaMemsetAsync failed: %s", cudaGetErrorString(e));
    }
    return WSB_OK;
}

void dev_free(void *p) {
    if (p) cudaFree(p);
}

static inline unsigned grid_for(uint64_t n, unsigned block) { return (unsigned)std::max<uint64_t>(1, (n + block - 1) / block); }

// Converged / breakdown / max-iteration messages of compute.rs:473-494.
static int solve_status_message(Context *ctx, int status, int breakdown, uint64_t max_iter) {
    if (status == WSB_ERR_BREAKDOWN)
        return fail(ctx, status, breakdown == 2 ? "PCG(BlockJacobiGpu): rz_old is zero (breakdown)"
                                                : "PCG(BlockJacobiGpu): dot(p,Ap) is zero (breakdown)");
    if (status == WSB_ERR_NOT_CONVERGED)
        return fail(ctx, status, "PCG(BlockJacobiGpu): did not converge in %llu iterations",
                    (unsigned long long)max_iter);
    return status;
}

// ---------------------------------------------------------------------------
// Reference-arithmetic solve: the reference's passes one by one
// (compute.rs:226-489) with the scalars and stop test kept on the device.
// The iteration body runs inside a CUDA graph while loop.
// ---------------------------------------------------------------------------
static int solve_reference(Context *ctx, const MatA &A, const Precond &M, const float *b, float *x, bool dev,
                           uint64_t max_iter, float rel_tol, float abs_tol, bool always_x, SolveOutcome *out,
                           double *hist_host, uint64_t hist_cap, uint64_t *hist_len, double *device_ms) {
    if (A.layout != LAYOUT_CSR)
        return fail(ctx, WSB_ERR_UNSUPPORTED,
                    "reference arithmetic runs on the CSR layout; create the matrix with WSB_LAYOUT_CSR");
    cudaStream_t st = ctx->stream;
    const uint32_t n = A.n;
    hist_cap = std::min<uint64_t>(hist_cap, std::max<uint64_t>(max_iter, 1));
    const size_t vb = ((size_t)n + kPadElems) * sizeof(float);
    const size_t scratch_f = ref_dot_scratch_floats(n);
    const size_t total = 6 * vb + 64 * sizeof(float) + scratch_f * sizeof(float) + 256 + 64 +
                         (hist_cap + 1) * sizeof(double);
    static_assert(sizeof(RefState) <= 256, "RefState fits its slot");
    void *mem = nullptr;
    int rc = dev_alloc(ctx, &mem, total, true, st);  // zero: wgpu buffers start zeroed
    if (rc) return rc;
    std::unique_ptr<void, void (*)(void *)> guard(mem, dev_free);
    char *p = static_cast<char *>(mem);
    RefState *dst = reinterpret_cast<RefState *>(p);
    p += 256;
    float *s = reinterpret_cast<float *>(p);
    p += 64 * sizeof(float);
    float *db = reinterpret_cast<float *>(p), *dx = db + vb / 4, *dr = dx + vb / 4, *dp = dr + vb / 4, *dz = dp + vb / 4,
          *dap = dz + vb / 4;
    float *scratch = dap + vb / 4;
    double *dhist = reinterpret_cast<double *>(scratch + scratch_f + (scratch_f & 1));
    const cudaMemcpyKind kind = dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    if (n) {
        WSB_CUDA_TRY(ctx, cudaMemcpyAsync(db, b, sizeof(float) * n, kind, st));
        WSB_CUDA_TRY(ctx, cudaMemcpyAsync(dx, x, sizeof(float) * n, kind, st));
    }
    RefState hs;
    std::memset(&hs, 0, sizeof hs);
    hs.rel_tol = rel_tol;
    hs.abs_tol = abs_tol;
    hs.max_iter = (uint32_t)std::min<uint64_t>(max_iter, 0xffffffffu);
    WSB_CUDA_TRY(ctx, cudaMemcpyAsync(dst, &hs, sizeof hs, cudaMemcpyHostToDevice, st));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, st);
    const unsigned gb = grid_for(n, 256), gblk = grid_for(M.nb, 128);
    // 1) ||b||^2 (compute.rs:228-250), 2) init (compute.rs:283-331).
    WSB_CUDA_TRY(ctx, ref_dot(st, n, db, db, scratch, s + 0));
    k_ref_after_bnorm<<<1, 32, 0, st>>>(dst, s);
    if (n) WSB_CUDA_TRY(ctx, cudaMemcpyAsync(dr, db, sizeof(float) * n, cudaMemcpyDeviceToDevice, st));
    k_ref_spmv<<<gb, 256, 0, st>>>(n, A.row_ptr, A.col, A.val, dx, dap);
    k_ref_axpy<<<gb, 256, 0, st>>>(n, -1.0f, dap, dr);
    k_ref_block_jacobi<<<gblk, 128, 0, st>>>(n, M.nb, M.lu, M.bs, dr, dz);
    if (n) WSB_CUDA_TRY(ctx, cudaMemcpyAsync(dp, dz, sizeof(float) * n, cudaMemcpyDeviceToDevice, st));
    WSB_CUDA_TRY(ctx, ref_dot(st, n, dr, dz, scratch, s + 3));
    k_ref_after_init<<<1, 32, 0, st>>>(dst, s);
    WSB_CUDA_TRY(ctx, cudaGetLastError());
    // 3) the loop (compute.rs:336-489) as a graph: gate + while(body).
    cudaGraph_t g = nullptr;
    cudaGraphExec_t ge = nullptr;
    WSB_CUDA_TRY(ctx, cudaGraphCreate(&g, 0));
    std::unique_ptr<CUgraph_st, cudaError_t (*)(cudaGraph_t)> gguard(g, cudaGraphDestroy);
    cudaGraphConditionalHandle h;
    WSB_CUDA_TRY(ctx, cudaGraphConditionalHandleCreate(&h, g, 0, 0));
    cudaKernelNodeParams kp = {};
    const RefState *cst = dst;
    void *gate_args[] = {(void *)&cst, &h};
    kp.func = (void *)k_ref_gate;
    kp.gridDim = dim3(1);
    kp.blockDim = dim3(32);
    kp.kernelParams = gate_args;
    cudaGraphNode_t gate, wn;
    WSB_CUDA_TRY(ctx, cudaGraphAddKernelNode(&gate, g, nullptr, 0, &kp));
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    WSB_CUDA_TRY(ctx, cudaGraphAddNode(&wn, g, &gate, 1, &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    cudaStream_t cs;
    WSB_CUDA_TRY(ctx, cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    cudaError_t ce = cudaStreamBeginCaptureToGraph(cs, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed);
    if (ce == cudaSuccess) {
        k_ref_spmv<<<gb, 256, 0, cs>>>(n, A.row_ptr, A.col, A.val, dp, dap);            // A
        ref_dot(cs, n, dp, dap, scratch, s + 0);                                        // B
        k_ref_write_rz_old<<<1, 32, 0, cs>>>(dst, s);                                    // C
        k_ref_update_scalars<<<1, 32, 0, cs>>>(s, 0, 2, 3, 4, 5, 6);                     // D
        k_ref_axpy_s<<<gb, 256, 0, cs>>>(n, dp, dx, s, 4);                               // E
        k_ref_axpy_s<<<gb, 256, 0, cs>>>(n, dap, dr, s, 5);
        ref_dot(cs, n, dr, dr, scratch, s + 1);                                         // F
        k_ref_block_jacobi<<<gblk, 128, 0, cs>>>(n, M.nb, M.lu, M.bs, dr, dz);         // G
        ref_dot(cs, n, dr, dz, scratch, s + 2);                                         // H
        k_ref_update_scalars<<<1, 32, 0, cs>>>(s, 0, 2, 3, 4, 5, 6);                     // I
        k_ref_scale_s<<<gb, 256, 0, cs>>>(n, dp, s, 6);                                  // J
        k_ref_axpy<<<gb, 256, 0, cs>>>(n, 1.0f, dz, dp);
        k_ref_check<<<1, 32, 0, cs>>>(dst, s, hist_cap ? dhist : nullptr, hist_cap, h);  // readback + checks
        ce = cudaStreamEndCapture(cs, &body);
    }
    cudaStreamDestroy(cs);
    if (ce != cudaSuccess) return fail(ctx, WSB_ERR_CUDA, "capturing the reference loop failed: %s", cudaGetErrorString(ce));
    WSB_CUDA_TRY(ctx, cudaGraphInstantiate(&ge, g, 0));
    std::unique_ptr<CUgraphExec_st, cudaError_t (*)(cudaGraphExec_t)> eguard(ge, cudaGraphExecDestroy);
    WSB_CUDA_TRY(ctx, cudaGraphLaunch(ge, st));
    cudaEventRecord(e1, st);
    WSB_CUDA_TRY(ctx, cudaMemcpyAsync(&hs, dst, sizeof hs, cudaMemcpyDeviceToHost, st));
    WSB_CUDA_TRY(ctx, cudaStreamSynchronize(st));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (device_ms) *device_ms = ms;
    out->iterations = hs.iter;
    out->bb = hs.b_norm2;
    out->rr = hs.last_rr;
    out->relres = hs.b_norm2 > 0 ? std::sqrt((double)hs.last_rr / hs.b_norm2) : 0.0;
    out->breakdown = (int)hs.breakdown;
    out->status = hs.status == ST_CONVERGED ? WSB_OK : hs.status == ST_BREAKDOWN ? WSB_ERR_BREAKDOWN : WSB_ERR_NOT_CONVERGED;
    if (hs.status == ST_RUNNING) out->status = WSB_ERR_CUDA;
    // b.b == 0 returns Ok(0) with x untouched (compute.rs:252-254).
    const bool x_changed = !(hs.status == ST_CONVERGED && hs.iter == 0);
    if (n && x_changed && (out->status == WSB_OK || always_x))
        WSB_CUDA_TRY(ctx, cudaMemcpyAsync(x, dx, sizeof(float) * n, dev ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, st));
    const uint64_t hl = std::min<uint64_t>(hs.iter, hist_cap);
    if (hist_host && hl) WSB_CUDA_TRY(ctx, cudaMemcpyAsync(hist_host, dhist, sizeof(double) * hl, cudaMemcpyDeviceToHost, st));
    if (hist_len) *hist_len = hist_host ? hl : 0;
    WSB_CUDA_TRY(ctx, cudaStreamSynchronize(st));
    return WSB_OK;
}

}  // namespace wsb

using namespace wsb;

struct wsb_context : Context {};
struct wsb_buffer : Buffer {};

struct wsb_spmv_executor {
    Context *ctx = nullptr;
    MatA A;
    std::unique_ptr<Engine> eng;
    const Precond *eng_M = nullptr;
    uint32_t slot = 0;
    SolveCfg slot_cfg;
};
struct wsb_dot_scalar_executor {
    Context *ctx = nullptr;
    uint64_t n_max = 0;
    uint32_t len = 0;
    wsb_buffer *scalars = nullptr;
    float *scratch = nullptr;
};
struct wsb_block_jacobi_executor {
    Context *ctx = nullptr;
    Precond M;
};
struct wsb_matrix {
    Context *ctx = nullptr;
    MatA A;
    Precond M;
    std::unique_ptr<Engine> eng;
    uint32_t slot = 0;
    SolveCfg slot_cfg;
    // wsb_matrix_spmv_device: the plain SpMV kernel's one-system descriptor
    // and error word (device), allocated on the first call and owned by the
    // matrix; a pinned host copy of the error word refreshed after every
    // launch, and the event that marks that copy.
    SysDesc *spmv_dd = nullptr;
    StepParams *spmv_sp = nullptr;
    uint32_t *spmv_err_h = nullptr;
    cudaEvent_t spmv_err_ev = nullptr;
    bool spmv_err_pending = false;
    ~wsb_matrix() {
        dev_free(spmv_dd);
        dev_free(spmv_sp);
        if (spmv_err_h) cudaFreeHost(spmv_err_h);
        if (spmv_err_ev) cudaEventDestroy(spmv_err_ev);
    }
};

#define CHECK_CTX(c)                                                              \
    do {                                                                          \
        if (!(c)) return fail(nullptr, WSB_ERR_BAD_INPUT, "context is null");     \
        cudaError_t _se = cudaSetDevice((c)->device);                             \
        if (_se != cudaSuccess) return fail((c), WSB_ERR_CUDA, "cudaSetDevice: %s", cudaGetErrorString(_se)); \
    } while (0)

// ---------------------------------------------------------------------------
// Context
// ---------------------------------------------------------------------------
extern "C" int wsb_context_create(int device, wsb_context **out) {
    if (!out) return fail(nullptr, WSB_ERR_BAD_INPUT, "out is null");
    *out = nullptr;
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0)
        return fail(nullptr, WSB_ERR_NO_DEVICE, "no suitable GPU adapter found (%s)",
                    e != cudaSuccess ? cudaGetErrorString(e) : "no CUDA device");
    if (device < 0 || device >= count)
        return fail(nullptr, WSB_ERR_NO_DEVICE, "device %d out of range (%d devices)", device, count);
    auto *c = new wsb_context();
    c->device = device;
    if ((e = cudaSetDevice(device)) != cudaSuccess || (e = cudaGetDeviceProperties(&c->prop, device)) != cudaSuccess) {
        delete c;
        return fail(nullptr, WSB_ERR_CUDA, "request device failed: %s", cudaGetErrorString(e));
    }
    if (c->prop.major < 10) {
        const int maj = c->prop.major, min = c->prop.minor;
        delete c;
        return fail(nullptr, WSB_ERR_UNSUPPORTED, "device compute capability %d.%d; this build targets sm_100a",
                    maj, min);
    }
    c->sm_count = c->prop.multiProcessorCount;
    if ((e = cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking)) != cudaSuccess) {
        delete c;
        return fail(nullptr, WSB_ERR_CUDA, "stream creation failed: %s", cudaGetErrorString(e));
    }
    c->stream = c->own_stream;
    *out = c;
    return WSB_OK;
}

extern "C" void wsb_context_destroy(wsb_context *ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
    delete ctx;
}

extern "C" const char *wsb_last_error(const wsb_context *ctx) {
    if (ctx) return ctx->last_error.c_str();
    return thread_error();
}

extern "C" int wsb_context_describe(const wsb_context *ctx, char *buf, size_t cap) {
    if (!ctx || !buf || !cap) return fail(nullptr, WSB_ERR_BAD_INPUT, "bad arguments");
    // Same shape as GpuContext::describe (context.rs:111-120).
    snprintf(buf, cap, "%s (DiscreteGpu, backend=Cuda, vendor=0x10de, device=0x%04x) sm_%d%d, %d SMs, %.1f GiB",
             ctx->prop.name, ctx->prop.pciDeviceID, ctx->prop.major, ctx->prop.minor, ctx->sm_count,
             ctx->prop.totalGlobalMem / 1073741824.0);
    return WSB_OK;
}

extern "C" int wsb_context_adapter_info(const wsb_context *ctx, wsb_adapter_info *out) {
    if (!ctx || !out) return fail(nullptr, WSB_ERR_BAD_INPUT, "bad arguments");
    std::memset(out, 0, sizeof *out);
    snprintf(out->name, sizeof out->name, "%s", ctx->prop.name);
    snprintf(out->backend, sizeof out->backend, "Cuda");
    snprintf(out->device_type, sizeof out->device_type, "DiscreteGpu");
    out->vendor = 0x10de;
    out->device = 0;
    out->sm_count = (uint32_t)ctx->sm_count;
    out->cc_major = ctx->prop.major;
    out->cc_minor = ctx->prop.minor;
    out->total_mem_bytes = ctx->prop.totalGlobalMem;
    return WSB_OK;
}

extern "C" int wsb_context_set_stream(wsb_context *ctx, void *stream) {
    CHECK_CTX(ctx);
    ctx->stream = stream ? static_cast<cudaStream_t>(stream) : ctx->own_stream;
    return WSB_OK;
}

extern "C" int wsb_context_set_wait_limit(wsb_context *ctx, uint64_t cycles) {
    CHECK_CTX(ctx);
    ctx->wait_cycles = cycles;
    return WSB_OK;
}

extern "C" int wsb_context_synchronize(wsb_context *ctx) {
    CHECK_CTX(ctx);
    WSB_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    return WSB_OK;
}

// ---------------------------------------------------------------------------
// Buffers
// ---------------------------------------------------------------------------
extern "C" int wsb_buffer_create(wsb_context *ctx, const void *data, size_t bytes, wsb_buffer **out) {
    CHECK_CTX(ctx);
    if (!out) return fail(ctx, WSB_ERR_BAD_INPUT, "out is null");
    auto *b = new wsb_buffer();
    b->ctx = ctx;
    b->bytes = bytes;
    int rc = dev_alloc(ctx, &b->ptr, bytes + 64, true, ctx->stream);
    if (rc) {
        delete b;
        return rc;
    }
    cudaError_t e = cudaSuccess;
    if (data && bytes) e = cudaMemcpyAsync(b->ptr, data, bytes, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) {
        dev_free(b->ptr);
        delete b;
        return fail(ctx, WSB_ERR_CUDA, "buffer upload failed: %s", cudaGetErrorString(e));
    }
    *out = b;
    return WSB_OK;
}

extern "C" int wsb_buffer_write(wsb_context *ctx, wsb_buffer *buf, size_t offset, const void *src, size_t bytes) {
    CHECK_CTX(ctx);
    if (!buf || (bytes && !src) || offset + bytes > buf->bytes)
        return fail(ctx, WSB_ERR_BAD_INPUT, "buffer write out of range");
    if (bytes) {
        WSB_CUDA_TRY(ctx, cudaMemcpyAsync(static_cast<char *>(buf->ptr) + offset, src, bytes, cudaMemcpyHostToDevice, ctx->stream));
        WSB_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    }
    return WSB_OK;
}

extern "C" int wsb_buffer_read(wsb_context *ctx, const wsb_buffer *buf, size_t offset, void *dst, size_t bytes) {
    CHECK_CTX(ctx);
    if (!buf || (bytes && !dst) || offset + bytes > buf->bytes)
        return fail(ctx, WSB_ERR_BAD_INPUT, "buffer read out of range");
    if (bytes) WSB_CUDA_TRY(ctx, cudaMemcpyAsync(dst, static_cast<const char *>(buf->ptr) + offset, bytes, cudaMemcpyDeviceToHost, ctx->stream));
    WSB_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    return WSB_OK;
}

extern "C" size_t wsb_buffer_size(const wsb_buffer *buf) { return buf ? buf->bytes : 0; }
extern "C" void *wsb_buffer_device_ptr(const wsb_buffer *buf) { return buf ? buf->ptr : nullptr; }
extern "C" void wsb_buffer_destroy(wsb_buffer *buf) {
    if (!buf) return;
    dev_free(buf->ptr);
    delete buf;
}

static bool holds(const wsb_buffer *b, uint64_t floats) { return b && b->bytes >= floats * 4; }

// ---------------------------------------------------------------------------
// Executors
// ---------------------------------------------------------------------------
extern "C" int wsb_spmv_executor_create(wsb_context *ctx, uint32_t n_rows, const uint32_t *row_ptr,
                                        const uint32_t *col_idx, const float *values, uint64_t nnz,
                                        wsb_spmv_executor **out) {
    CHECK_CTX(ctx);
    if (!out || !row_ptr) return fail(ctx, WSB_ERR_BAD_INPUT, "bad arguments");
    std::string err;
    const uint32_t bs_dummy[1] = {0};
    (void)bs_dummy;
    if (row_ptr[0] != 0 || row_ptr[n_rows] != nnz) return fail(ctx, WSB_ERR_BAD_INPUT, "CSR row_ptr must start with 0 and end with nnz");
    for (uint32_t i = 0; i < n_rows; ++i)
        if (row_ptr[i + 1] < row_ptr[i]) return fail(ctx, WSB_ERR_BAD_INPUT, "CSR row_ptr must be non-decreasing");
    for (uint64_t k = 0; k < nnz; ++k)
        if (col_idx[k] >= n_rows)
            return fail(ctx, WSB_ERR_BAD_INPUT, "CSR col_idx contains out-of-range column %u for n_cols=%u", col_idx[k], n_rows);
    auto *ex = new wsb_spmv_executor();
    ex->ctx = ctx;
    int rc = upload_matA(ctx, n_rows, row_ptr, col_idx, values, nnz, nullptr, 0, WSB_LAYOUT_CSR, ctx->stream, &ex->A);
    if (rc) {
        delete ex;
        return rc;
    }
    *out = ex;
    return WSB_OK;
}

extern "C" int wsb_spmv_executor_spmv(wsb_spmv_executor *ex, const wsb_buffer *x, wsb_buffer *y) {
    if (!ex) return fail(nullptr, WSB_ERR_BAD_INPUT, "executor is null");
    Context *ctx = ex->ctx;
    CHECK_CTX(ctx);
    if (!holds(x, ex->A.n) || !holds(y, ex->A.n)) return fail(ctx, WSB_ERR_BAD_INPUT, "x/y buffers must hold n_rows floats");
    k_ref_spmv<<<grid_for(ex->A.n, 256), 256, 0, ctx->stream>>>(ex->A.n, ex->A.row_ptr, ex->A.col, ex->A.val,
                                                                 (const float *)x->ptr, (float *)y->ptr);
    WSB_CUDA_TRY(ctx, cudaGetLastError());
    return WSB_OK;
}

extern "C" void wsb_spmv_executor_destroy(wsb_spmv_executor *ex) {
    if (!ex) return;
    cudaSetDevice(ex->ctx->device);
    ex->eng.reset();
    delete ex;
}

extern "C" int wsb_dot_scalar_executor_create(wsb_context *ctx, uint64_t n_max, uint32_t len, wsb_dot_scalar_executor **out) {
    CHECK_CTX(ctx);
    if (!out) return fail(ctx, WSB_ERR_BAD_INPUT, "out is null");
    auto *ex = new wsb_dot_scalar_executor();
    ex->ctx = ctx;
    ex->n_max = n_max;
    ex->len = len;
    int rc = wsb_buffer_create(ctx, nullptr, std::max<size_t>(len, 1) * sizeof(float), &ex->scalars);
    if (!rc) {
        void *p = nullptr;
        rc = dev_alloc(ctx, &p, ref_dot_scratch_floats(n_max) * sizeof(float), true, ctx->stream);
        ex->scratch = static_cast<float *>(p);
    }
    if (rc) {
        wsb_buffer_destroy(ex->scalars);
        delete ex;
        return rc;
    }
    ex->scalars->bytes = (size_t)len * sizeof(float);
    *out = ex;
    return WSB_OK;
}

extern "C" int wsb_dot_scalar_executor_dot_into(wsb_dot_scalar_executor *ex, const wsb_buffer *a, const wsb_buffer *b,
                                                uint32_t n, uint32_t out_index) {
    if (!ex) return fail(nullptr, WSB_ERR_BAD_INPUT, "executor is null");
    Context *ctx = ex->ctx;
    CHECK_CTX(ctx);
    if (out_index >= ex->len) return fail(ctx, WSB_ERR_BAD_INPUT, "DotScalarExecutor: out_index out of range");
    if (n > ex->n_max) return fail(ctx, WSB_ERR_BAD_INPUT, "DotScalarExecutor: n %u exceeds n_max %llu", n, (unsigned long long)ex->n_max);
    if (!holds(a, n) || !holds(b, n)) return fail(ctx, WSB_ERR_BAD_INPUT, "a/b buffers must hold n floats");
    WSB_CUDA_TRY(ctx, ref_dot(ctx->stream, n, (const float *)a->ptr, (const float *)b->ptr, ex->scratch,
                              (float *)ex->scalars->ptr + out_index));
    return WSB_OK;
}

extern "C" wsb_buffer *wsb_dot_scalar_executor_scalar_results(wsb_dot_scalar_executor *ex) { return ex ? ex->scalars : nullptr; }

extern "C" int wsb_dot_scalar_executor_readback(wsb_dot_scalar_executor *ex, float *out, uint32_t len) {
    if (!ex) return fail(nullptr, WSB_ERR_BAD_INPUT, "executor is null");
    return wsb_buffer_read(static_cast<wsb_context *>(ex->ctx), ex->scalars, 0, out, (size_t)std::min(len, ex->len) * 4);
}

extern "C" void wsb_dot_scalar_executor_destroy(wsb_dot_scalar_executor *ex) {
    if (!ex) return;
    wsb_buffer_destroy(ex->scalars);
    dev_free(ex->scratch);
    delete ex;
}

extern "C" int wsb_vec_axpy_inplace(wsb_context *ctx, const wsb_buffer *x, wsb_buffer *y, uint32_t n, float alpha) {
    CHECK_CTX(ctx);
    if (!holds(x, n) || !holds(y, n)) return fail(ctx, WSB_ERR_BAD_INPUT, "x/y buffers must hold n floats");
    if (n) k_ref_axpy<<<grid_for(n, 256), 256, 0, ctx->stream>>>(n, alpha, (const float *)x->ptr, (float *)y->ptr);
    WSB_CUDA_TRY(ctx, cudaGetLastError());
    return WSB_OK;
}

extern "C" int wsb_vec_axpy_inplace_from_scalar_results(wsb_context *ctx, const wsb_buffer *x, wsb_buffer *y, uint32_t n,
                                                        const wsb_buffer *s, uint32_t k) {
    CHECK_CTX(ctx);
    if (!holds(x, n) || !holds(y, n) || !holds(s, (uint64_t)k + 1))
        return fail(ctx, WSB_ERR_BAD_INPUT, "buffer too small for n or scalar index");
    if (n) k_ref_axpy_s<<<grid_for(n, 256), 256, 0, ctx->stream>>>(n, (const float *)x->ptr, (float *)y->ptr, (const float *)s->ptr, k);
    WSB_CUDA_TRY(ctx, cudaGetLastError());
    return WSB_OK;
}

extern "C" int wsb_vec_scale_inplace_from_scalar_results(wsb_context *ctx, wsb_buffer *x, uint32_t n, const wsb_buffer *s,
                                                         uint32_t k) {
    CHECK_CTX(ctx);
    if (!holds(x, n) || !holds(s, (uint64_t)k + 1)) return fail(ctx, WSB_ERR_BAD_INPUT, "buffer too small for n or scalar index");
    if (n) k_ref_scale_s<<<grid_for(n, 256), 256, 0, ctx->stream>>>(n, (float *)x->ptr, (const float *)s->ptr, k);
    WSB_CUDA_TRY(ctx, cudaGetLastError());
    return WSB_OK;
}

extern "C" int wsb_block_jacobi_executor_create(wsb_context *ctx, uint32_t n, const float *lu, uint64_t lu_len,
                                                const uint32_t *bs, uint64_t bs_len, wsb_block_jacobi_executor **out) {
    CHECK_CTX(ctx);
    if (!out || !bs || bs_len < 1) return fail(ctx, WSB_ERR_BAD_INPUT, "block_starts must not be empty");
    if (bs[0] != 0 || bs[bs_len - 1] != n) return fail(ctx, WSB_ERR_BAD_INPUT, "block_starts must start with 0 and end with n (%u)", n);
    for (uint64_t i = 0; i + 1 < bs_len; ++i)
        if (bs[i + 1] <= bs[i]) return fail(ctx, WSB_ERR_BAD_INPUT, "block_starts must be strictly increasing");
    if (lu_len < (bs_len - 1) * 36) return fail(ctx, WSB_ERR_BAD_INPUT, "lu_blocks must hold 36 floats per block");
    auto *ex = new wsb_block_jacobi_executor();
    ex->ctx = ctx;
    int rc = upload_precond(ctx, n, lu, bs, bs_len, ctx->stream, &ex->M);
    if (rc) {
        delete ex;
        return rc;
    }
    *out = ex;
    return WSB_OK;
}

extern "C" int wsb_block_jacobi_executor_apply(wsb_block_jacobi_executor *ex, const wsb_buffer *r, wsb_buffer *z) {
    if (!ex) return fail(nullptr, WSB_ERR_BAD_INPUT, "executor is null");
    Context *ctx = ex->ctx;
    CHECK_CTX(ctx);
    if (!holds(r, ex->M.n) || !holds(z, ex->M.n)) return fail(ctx, WSB_ERR_BAD_INPUT, "r/z buffers must hold n floats");
    if (ex->M.nb)
        k_ref_block_jacobi<<<grid_for(ex->M.nb, 128), 128, 0, ctx->stream>>>(ex->M.n, ex->M.nb, ex->M.lu, ex->M.bs,
                                                                             (const float *)r->ptr, (float *)z->ptr);
    WSB_CUDA_TRY(ctx, cudaGetLastError());
    return WSB_OK;
}

extern "C" void wsb_block_jacobi_executor_destroy(wsb_block_jacobi_executor *ex) {
    if (!ex) return;
    cudaSetDevice(ex->ctx->device);
    delete ex;
}

extern "C" int wsb_pcg_update_scalars(wsb_context *ctx, wsb_buffer *s, uint32_t p_ap, uint32_t rz_new, uint32_t rz_old,
                                      uint32_t alpha, uint32_t minus_alpha, uint32_t beta) {
    CHECK_CTX(ctx);
    const uint32_t mx = std::max({p_ap, rz_new, rz_old, alpha, minus_alpha, beta});
    if (!holds(s, (uint64_t)mx + 1)) return fail(ctx, WSB_ERR_BAD_INPUT, "scalar index out of range");
    k_ref_update_scalars<<<1, 32, 0, ctx->stream>>>((float *)s->ptr, p_ap, rz_new, rz_old, alpha, minus_alpha, beta);
    WSB_CUDA_TRY(ctx, cudaGetLastError());
    return WSB_OK;
}

// ---------------------------------------------------------------------------
// Host LU
// ---------------------------------------------------------------------------
extern "C" int wsb_lu_factor_inplace_6(float *mat, uint64_t mat_len, uint32_t n) {
    if (!mat || mat_len < 36) return fail(nullptr, WSB_ERR_BAD_INPUT, "lu_factor_inplace_6: mat must have len >= 36");
    if (n > 6) return fail(nullptr, WSB_ERR_BAD_INPUT, "lu_factor_inplace_6: n must be <= 6, got %u", n);
    uint32_t k = 0;
    if (lu_factor_inplace_6(mat, n, &k) != WSB_OK) return fail(nullptr, WSB_ERR_ZERO_PIVOT, "LU zero pivot at k = %u", k);
    return WSB_OK;
}

extern "C" int wsb_build_lu_blocks_from_csr_block_starts_6(uint32_t n, const uint32_t *row_ptr, uint64_t row_ptr_len,
                                                           const uint32_t *col, uint64_t col_len, const float *val,
                                                           uint64_t val_len, const uint32_t *bs, uint64_t bs_len,
                                                           float *out) {
    if (!row_ptr || (bs_len && !bs) || (bs_len >= 2 && !out)) return fail(nullptr, WSB_ERR_BAD_INPUT, "null argument");
    std::string err;
    int rc = build_lu_blocks_6(n, row_ptr, row_ptr_len, col, col_len, val, val_len, bs, bs_len, out, &err);
    if (rc) return fail(nullptr, rc, "%s", err.c_str());
    return WSB_OK;
}

// ---------------------------------------------------------------------------
// Solves through an engine slot cached on an executor or matrix.
// ---------------------------------------------------------------------------
void wsb_solve_opts_default(wsb_solve_opts *o);

static SolveCfg make_cfg(uint64_t max_iter, float rel, float abs_tol, const wsb_solve_opts *o) {
    SolveCfg c;
    c.max_iter = max_iter;
    c.rel_tol = rel;
    c.abs_tol = abs_tol;
    if (o) {
        c.precision = o->precision;
        if (o->target_relres > 0) c.target_relres = o->target_relres;
        if (o->inner_rel_tol > 0) c.inner_rel_tol = o->inner_rel_tol;
        if (o->max_refine > 0) c.max_refine = o->max_refine;
        c.hist_cap = o->history_out ? o->history_capacity : 0;
        c.algorithm = o->algorithm;
    }
    return c;
}

static bool same_layout(const SolveCfg &a, const SolveCfg &b) {
    return (a.precision == WSB_PREC_MIXED_F64_IR) == (b.precision == WSB_PREC_MIXED_F64_IR) &&
           a.algorithm == b.algorithm &&
           std::min<uint64_t>(a.hist_cap, std::max<uint64_t>(a.max_iter, 1)) ==
               std::min<uint64_t>(b.hist_cap, std::max<uint64_t>(b.max_iter, 1));
}

static int engine_solve(Context *ctx, std::unique_ptr<Engine> *eng, uint32_t *slot, SolveCfg *slot_cfg, const MatA &A,
                        const Precond &M, const float *b, float *x, bool dev, const SolveCfg &cfg,
                        const wsb_solve_opts *o, wsb_solve_result *res) {
    const auto t0 = std::chrono::steady_clock::now();
    int rc;
    if (!*eng || (*eng)->stream() != ctx->stream) {
        eng->reset(new Engine(ctx, ctx->stream));
        if ((rc = (*eng)->add(&A, &M, cfg, slot))) {
            eng->reset();
            return rc;
        }
        *slot_cfg = cfg;
    } else if (!same_layout(*slot_cfg, cfg)) {
        (*eng)->remove(*slot);
        if ((rc = (*eng)->add(&A, &M, cfg, slot))) return rc;
        *slot_cfg = cfg;
    } else {
        (*eng)->reset_slot(*slot, cfg);
        *slot_cfg = cfg;
    }
    Engine &E = **eng;
    const uint64_t launches0 = E.launches();
    if ((rc = E.set_rhs(*slot, b, x, dev))) return rc;
    if ((rc = E.run())) return rc;
    SolveOutcome out;
    uint64_t hl = 0;
    const bool always_x = o && o->always_write_x;
    if ((rc = E.fetch(*slot, x, dev, always_x, &out, o ? o->history_out : nullptr, o ? o->history_capacity : 0, &hl,
                      o ? o->x64_out : nullptr)))
        return rc;
    if (res) {
        std::memset(res, 0, sizeof *res);
        res->status = out.status;
        res->breakdown_kind = out.breakdown;
        res->iterations = out.iterations;
        res->refine_sweeps = out.sweeps;
        res->b_norm2 = out.bb;
        res->final_r_norm2 = out.rr;
        res->final_relres = out.relres;
        res->device_ms = E.last_device_ms();
        res->total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        res->history_len = hl;
        res->kernel_launches = E.launches() - launches0;
    }
    return solve_status_message(ctx, out.status, out.breakdown, cfg.max_iter);
}

static int fill_ref_result(Context *ctx, const SolveOutcome &out, double ms, double t_ms, uint64_t hl, uint64_t max_iter,
                           wsb_solve_result *res) {
    if (res) {
        std::memset(res, 0, sizeof *res);
        res->status = out.status;
        res->breakdown_kind = out.breakdown;
        res->iterations = out.iterations;
        res->b_norm2 = out.bb;
        res->final_r_norm2 = out.rr;
        res->final_relres = out.relres;
        res->device_ms = ms;
        res->total_ms = t_ms;
        res->history_len = hl;
    }
    return solve_status_message(ctx, out.status, out.breakdown, max_iter);
}

extern "C" int wsb_pcg_block_jacobi_csr(wsb_context *ctx, uint64_t n, const float *b, uint64_t b_len, float *x,
                                        uint64_t x_len, uint64_t max_iter, float rel_tol, float abs_tol,
                                        wsb_spmv_executor *spmv, wsb_block_jacobi_executor *bj,
                                        const wsb_solve_opts *opts, uint64_t *iterations, wsb_solve_result *result) {
    CHECK_CTX(ctx);
    if (b_len != n || x_len != n)
        return fail(ctx, WSB_ERR_BAD_INPUT, "PCG(BlockJacobiGpu): dimension mismatch: n=%llu, b len %llu, x len %llu",
                    (unsigned long long)n, (unsigned long long)b_len, (unsigned long long)x_len);
    if (!spmv || !bj) return fail(ctx, WSB_ERR_BAD_INPUT, "executors must not be null");
    if (spmv->A.n != n || bj->M.n != n)
        return fail(ctx, WSB_ERR_BAD_INPUT, "PCG(BlockJacobiGpu): executor sizes (%u, %u) differ from n=%llu", spmv->A.n,
                    bj->M.n, (unsigned long long)n);
    if (n && (!b || !x)) return fail(ctx, WSB_ERR_BAD_INPUT, "b and x must not be null");
    const SolveCfg cfg = make_cfg(max_iter, rel_tol, abs_tol, opts);
    int rc;
    if (cfg.precision == WSB_PREC_REFERENCE_F32) {
        const auto t0 = std::chrono::steady_clock::now();
        SolveOutcome out;
        double ms = 0;
        uint64_t hl = 0;
        rc = solve_reference(ctx, spmv->A, bj->M, b, x, false, max_iter, rel_tol, abs_tol, opts && opts->always_write_x,
                             &out, opts ? opts->history_out : nullptr, opts ? opts->history_capacity : 0, &hl, &ms);
        if (rc) return rc;
        const double t_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        if (iterations && out.status == WSB_OK) *iterations = out.iterations;
        return fill_ref_result(ctx, out, ms, t_ms, hl, max_iter, result);
    }
    if (spmv->eng && spmv->eng_M != &bj->M) spmv->eng.reset();
    spmv->eng_M = &bj->M;
    wsb_solve_result local;
    rc = engine_solve(ctx, &spmv->eng, &spmv->slot, &spmv->slot_cfg, spmv->A, bj->M, b, x, false, cfg, opts,
                      result ? result : &local);
    if (iterations && rc == WSB_OK) *iterations = (result ? result : &local)->iterations;
    return rc;
}

// ---------------------------------------------------------------------------
// Matrices
// ---------------------------------------------------------------------------
extern "C" void wsb_solve_opts_default(wsb_solve_opts *o) {
    if (!o) return;
    std::memset(o, 0, sizeof *o);
    o->struct_size = sizeof *o;
    o->precision = WSB_PREC_F32_F64DOT;
    o->target_relres = 1e-10;
    o->inner_rel_tol = 1e-4f;
    o->max_refine = 50;
}

extern "C" int wsb_matrix_create(wsb_context *ctx, uint32_t n, const uint32_t *row_ptr, const uint32_t *col,
                                 const float *val, uint64_t nnz, const uint32_t *bs, uint64_t bs_len, int32_t layout,
                                 wsb_matrix **out) {
    CHECK_CTX(ctx);
    if (!out) return fail(ctx, WSB_ERR_BAD_INPUT, "out is null");
    *out = nullptr;
    if (nnz > 0xfffff000ull) return fail(ctx, WSB_ERR_BAD_INPUT, "nnz %llu exceeds the u32 index range", (unsigned long long)nnz);
    if (!row_ptr || (nnz && (!col || !val))) return fail(ctx, WSB_ERR_BAD_INPUT, "null CSR array");
    auto *m = new wsb_matrix();
    m->ctx = ctx;
    int rc = prepare_system_device(ctx, n, row_ptr, col, val, nnz, bs, bs_len, layout, ctx->stream, &m->A, &m->M);
    if (rc) {
        delete m;
        return rc;
    }
    *out = m;
    return WSB_OK;
}

extern "C" int wsb_matrix_info_get(const wsb_matrix *m, wsb_matrix_info *out) {
    if (!m || !out) return fail(nullptr, WSB_ERR_BAD_INPUT, "bad arguments");
    std::memset(out, 0, sizeof *out);
    out->n = m->A.n;
    out->nnz = m->A.nnz;
    out->num_blocks = m->M.nb;
    out->layout = m->A.layout == LAYOUT_BSR6 ? WSB_LAYOUT_BSR6 : WSB_LAYOUT_CSR;
    out->device_bytes = m->A.bytes + m->M.bytes;
    out->spmv_bytes = spmv_algorithmic_bytes(m->A);
    out->iteration_bytes = iteration_algorithmic_bytes(m->A, m->M);
    return WSB_OK;
}

extern "C" int wsb_matrix_autotune(wsb_context *ctx, wsb_matrix *m, uint32_t iterations, wsb_tune_result *out) {
    CHECK_CTX(ctx);
    if (!m) return fail(ctx, WSB_ERR_BAD_INPUT, "matrix is null");
    m->eng.reset();  // its systems point at the tiles being replaced
    return autotune_matrix(ctx, &m->A, &m->M, iterations, out);
}

extern "C" void wsb_autotune_clear(void) { tile_caps_clear(); }

extern "C" int wsb_matrix_read_lu(wsb_context *ctx, const wsb_matrix *m, float *out, uint64_t out_len) {
    CHECK_CTX(ctx);
    if (!m || (!out && m->M.nb)) return fail(ctx, WSB_ERR_BAD_INPUT, "bad arguments");
    const uint64_t need = 36ull * m->M.nb;
    if (out_len < need) return fail(ctx, WSB_ERR_BAD_INPUT, "out_len %llu < %llu", (unsigned long long)out_len,
                                    (unsigned long long)need);
    if (need) {
        WSB_CUDA_TRY(ctx, cudaMemcpyAsync(out, m->M.lu, sizeof(float) * need, cudaMemcpyDeviceToHost, ctx->stream));
        WSB_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    }
    return WSB_OK;
}

extern "C" void wsb_matrix_destroy(wsb_matrix *m) {
    if (!m) return;
    cudaSetDevice(m->ctx->device);
    m->eng.reset();
    delete m;
}

static int matrix_solve(wsb_context *ctx, wsb_matrix *m, const float *b, float *x, bool dev, uint64_t max_iter, float rel,
                        float abs_tol, const wsb_solve_opts *o, wsb_solve_result *res) {
    CHECK_CTX(ctx);
    if (!m) return fail(ctx, WSB_ERR_BAD_INPUT, "matrix is null");
    if (m->A.n && (!b || !x)) return fail(ctx, WSB_ERR_BAD_INPUT, "b and x must not be null");
    const SolveCfg cfg = make_cfg(max_iter, rel, abs_tol, o);
    if (cfg.precision < WSB_PREC_F32_F64DOT || cfg.precision > WSB_PREC_MIXED_F64_IR)
        return fail(ctx, WSB_ERR_BAD_INPUT, "unknown precision %d", cfg.precision);
    if (cfg.precision == WSB_PREC_REFERENCE_F32 && cfg.algorithm != WSB_ALG_CLASSIC)
        return fail(ctx, WSB_ERR_BAD_INPUT, "reference arithmetic runs the reference's classic recurrence only");
    if (cfg.precision == WSB_PREC_REFERENCE_F32) {
        const auto t0 = std::chrono::steady_clock::now();
        SolveOutcome out;
        double ms = 0;
        uint64_t hl = 0;
        int rc = solve_reference(ctx, m->A, m->M, b, x, dev, max_iter, rel, abs_tol, o && o->always_write_x, &out,
                                 o ? o->history_out : nullptr, o ? o->history_capacity : 0, &hl, &ms);
        if (rc) return rc;
        const double t_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        return fill_ref_result(ctx, out, ms, t_ms, hl, max_iter, res);
    }
    wsb_solve_result local;
    return engine_solve(ctx, &m->eng, &m->slot, &m->slot_cfg, m->A, m->M, b, x, dev, cfg, o, res ? res : &local);
}

extern "C" int wsb_solve(wsb_context *ctx, wsb_matrix *m, const float *b, float *x, uint64_t max_iter, float rel,
                         float abs_tol, const wsb_solve_opts *o, wsb_solve_result *res) {
    return matrix_solve(ctx, m, b, x, false, max_iter, rel, abs_tol, o, res);
}

extern "C" int wsb_solve_device(wsb_context *ctx, wsb_matrix *m, const float *d_b, float *d_x, uint64_t max_iter, float rel,
                                float abs_tol, const wsb_solve_opts *o, wsb_solve_result *res) {
    return matrix_solve(ctx, m, d_b, d_x, true, max_iter, rel, abs_tol, o, res);
}

// The error word of the plain SpMV kernel is sticky: launches OR their codes
// into it and only a reported error clears it, so a code survives later
// launches until a call reads it.
static int spmv_error_status(wsb_matrix *m, uint32_t code) {
    m->spmv_err_pending = false;
    *m->spmv_err_h = 0;
    cudaMemsetAsync(&m->spmv_sp->error, 0, sizeof(uint32_t), m->ctx->stream);
    return fail(m->ctx, (code & kErrWaitMask) ? WSB_ERR_TIMEOUT : WSB_ERR_CUDA,
                "an earlier wsb_matrix_spmv_device launch on this matrix failed (kernel code %u)", code);
}

extern "C" int wsb_matrix_spmv_device(wsb_context *ctx, wsb_matrix *m, const float *d_x, float *d_y) {
    CHECK_CTX(ctx);
    if (!m || !d_x || !d_y) return fail(ctx, WSB_ERR_BAD_INPUT, "bad arguments");
    if (m->ctx->device != ctx->device)
        return fail(ctx, WSB_ERR_BAD_INPUT, "the matrix lives on device %d, the context on device %d", m->ctx->device,
                    ctx->device);
    if (!m->spmv_dd) {
        void *dd = nullptr, *sp = nullptr;
        WSB_CUDA_TRY(ctx, cudaMalloc(&dd, sizeof(SysDesc)));
        m->spmv_dd = static_cast<SysDesc *>(dd);
        WSB_CUDA_TRY(ctx, cudaMalloc(&sp, sizeof(StepParams)));
        m->spmv_sp = static_cast<StepParams *>(sp);
        WSB_CUDA_TRY(ctx, cudaMemsetAsync(m->spmv_sp, 0, sizeof(StepParams), ctx->stream));
        WSB_CUDA_TRY(ctx, cudaHostAlloc((void **)&m->spmv_err_h, sizeof(uint32_t), cudaHostAllocDefault));
        *m->spmv_err_h = 0;
        WSB_CUDA_TRY(ctx, cudaEventCreateWithFlags(&m->spmv_err_ev, cudaEventDisableTiming));
        WSB_CUDA_TRY(ctx, cudaFuncSetAttribute(k_spmv_plain, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               (int)kSpmvSmem));
    }
    // A finished read-back of the error word with a code in it: report it.
    if (m->spmv_err_pending && cudaEventQuery(m->spmv_err_ev) == cudaSuccess) {
        m->spmv_err_pending = false;
        if (*m->spmv_err_h) return spmv_error_status(m, *m->spmv_err_h);
    }
    // The one-system descriptor (rewritten every call: the tiles may have
    // been rebuilt by the autotuner since the last one).
    SysDesc d;
    std::memset(&d, 0, sizeof d);
    d.n = m->A.n;
    d.layout = m->A.layout;
    d.row_ptr = m->A.row_ptr;
    d.col = m->A.col;
    d.val = m->A.val;
    d.brow_ptr = m->A.brow_ptr;
    d.bcol = m->A.bcol;
    d.bval = m->A.bval;
    d.stiles = m->A.stiles;
    d.n_stiles = m->A.n_stiles;
    WSB_CUDA_TRY(ctx, cudaMemcpyAsync(m->spmv_dd, &d, sizeof d, cudaMemcpyHostToDevice, ctx->stream));
    int occ = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_spmv_plain, kSpmvThreads, kSpmvSmem);
    const uint32_t g = std::max<uint32_t>(1, std::min<uint32_t>(m->A.n_stiles, (uint32_t)(std::max(occ, 1) * ctx->sm_count)));
    k_spmv_plain<<<g, kSpmvThreads, kSpmvSmem, ctx->stream>>>(m->spmv_dd, m->spmv_sp, d_x, d_y);
    WSB_CUDA_TRY(ctx, cudaGetLastError());
    WSB_CUDA_TRY(ctx, cudaMemcpyAsync(m->spmv_err_h, &m->spmv_sp->error, sizeof(uint32_t), cudaMemcpyDeviceToHost,
                                      ctx->stream));
    WSB_CUDA_TRY(ctx, cudaEventRecord(m->spmv_err_ev, ctx->stream));
    m->spmv_err_pending = true;
    return WSB_OK;
}

extern "C" int wsb_matrix_spmv_check(wsb_context *ctx, wsb_matrix *m) {
    CHECK_CTX(ctx);
    if (!m) return fail(ctx, WSB_ERR_BAD_INPUT, "matrix is null");
    if (!m->spmv_err_pending) return WSB_OK;
    WSB_CUDA_TRY(ctx, cudaEventSynchronize(m->spmv_err_ev));
    m->spmv_err_pending = false;
    if (*m->spmv_err_h) return spmv_error_status(m, *m->spmv_err_h);
    return WSB_OK;
}

extern "C" int wsb_matrix_kernel_times(wsb_context *ctx, wsb_matrix *m, const float *d_b, uint32_t iterations,
                                       double *ms) {
    CHECK_CTX(ctx);
    if (!m || !d_b || !ms || iterations == 0) return fail(ctx, WSB_ERR_BAD_INPUT, "bad arguments");
    Engine E(ctx, ctx->stream);
    SolveCfg cfg;
    cfg.max_iter = iterations + 1;
    uint32_t slot;
    int rc = E.add(&m->A, &m->M, cfg, &slot);
    if (rc) return rc;
    float *d_x0 = nullptr;
    const size_t xbytes = sizeof(float) * std::max<uint32_t>(m->A.n, 1);
    WSB_CUDA_TRY(ctx, cudaMallocAsync((void **)&d_x0, xbytes, ctx->stream));
    const cudaError_t me = cudaMemsetAsync(d_x0, 0, xbytes, ctx->stream);
    if (me != cudaSuccess) {
        cudaFreeAsync(d_x0, ctx->stream);
        return fail(ctx, WSB_ERR_CUDA, "kernel times: cudaMemsetAsync failed: %s", cudaGetErrorString(me));
    }
    rc = E.set_rhs(slot, d_b, d_x0, true);
    if (!rc) rc = E.profile_kernels(slot, iterations, ms);
    cudaFreeAsync(d_x0, ctx->stream);
    return rc;
}

// ---------------------------------------------------------------------------
// Batch
// ---------------------------------------------------------------------------
struct wsb_batch {
    Context *ctx = nullptr;
    std::unique_ptr<Engine> eng;
    struct Item {
        wsb_matrix *m;
        uint32_t slot;
        SolveCfg cfg;
        bool always_x;
        double *hist;
        uint64_t hist_cap;
        double *x64_out;
    };
    std::vector<Item> items;
    double device_ms = 0.0;
    bool solved = false;
};

extern "C" int wsb_batch_create(wsb_context *ctx, wsb_batch **out) {
    CHECK_CTX(ctx);
    if (!out) return fail(ctx, WSB_ERR_BAD_INPUT, "out is null");
    auto *bt = new wsb_batch();
    bt->ctx = ctx;
    bt->eng.reset(new Engine(ctx, ctx->stream));
    *out = bt;
    return WSB_OK;
}

extern "C" int wsb_batch_add(wsb_batch *bt, wsb_matrix *m, const float *b, const float *x0, uint64_t max_iter, float rel,
                             float abs_tol, const wsb_solve_opts *o, uint32_t *id) {
    if (!bt) return fail(nullptr, WSB_ERR_BAD_INPUT, "batch is null");
    Context *ctx = bt->ctx;
    CHECK_CTX(ctx);
    if (!m || (m->A.n && (!b || !x0))) return fail(ctx, WSB_ERR_BAD_INPUT, "bad arguments");
    SolveCfg cfg = make_cfg(max_iter, rel, abs_tol, o);
    if (cfg.precision != WSB_PREC_F32_F64DOT && cfg.precision != WSB_PREC_MIXED_F64_IR)
        return fail(ctx, WSB_ERR_UNSUPPORTED, "batched solves use FP64 reductions (F32_F64DOT or MIXED_F64_IR)");
    uint32_t slot;
    int rc = bt->eng->add(&m->A, &m->M, cfg, &slot);
    if (rc) return rc;
    if ((rc = bt->eng->set_rhs(slot, b, x0, false))) return rc;
    bt->items.push_back({m, slot, cfg, o && o->always_write_x, o ? o->history_out : nullptr,
                         o ? o->history_capacity : 0, o ? o->x64_out : nullptr});
    if (id) *id = (uint32_t)bt->items.size() - 1;
    return WSB_OK;
}

extern "C" int wsb_batch_solve(wsb_batch *bt) {
    if (!bt) return fail(nullptr, WSB_ERR_BAD_INPUT, "batch is null");
    Context *ctx = bt->ctx;
    CHECK_CTX(ctx);
    // Steps of 64 iterations: finished systems leave the work lists between steps.
    bool left = true;
    double ms = 0.0;
    while (left) {
        int rc = bt->eng->step(64, &left);
        if (rc) return rc;
        ms += bt->eng->last_device_ms();
    }
    bt->device_ms = ms;
    bt->solved = true;
    return WSB_OK;
}

extern "C" int wsb_batch_result(wsb_batch *bt, uint32_t id, float *x, wsb_solve_result *res) {
    if (!bt || id >= bt->items.size()) return fail(nullptr, WSB_ERR_BAD_INPUT, "bad batch id");
    Context *ctx = bt->ctx;
    CHECK_CTX(ctx);
    auto &it = bt->items[id];
    SolveOutcome out;
    uint64_t hl = 0;
    int rc = bt->eng->fetch(it.slot, x, false, it.always_x, &out, it.hist, it.hist_cap, &hl, it.x64_out);
    if (rc) return rc;
    if (res) {
        std::memset(res, 0, sizeof *res);
        res->status = out.status;
        res->breakdown_kind = out.breakdown;
        res->iterations = out.iterations;
        res->refine_sweeps = out.sweeps;
        res->b_norm2 = out.bb;
        res->final_r_norm2 = out.rr;
        res->final_relres = out.relres;
        res->device_ms = bt->device_ms;
        res->history_len = hl;
        res->kernel_launches = bt->eng->launches();
    }
    return solve_status_message(ctx, out.status, out.breakdown, it.cfg.max_iter);
}

extern "C" void wsb_batch_destroy(wsb_batch *bt) {
    if (!bt) return;
    cudaSetDevice(bt->ctx->device);
    bt->eng.reset();
    delete bt;
}
