// Multi-system PCG engine: device-resident systems iterated together by the
// fused kernels inside one CUDA graph whose while loop runs on the device.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <queue>
#include <vector>

#include "engine.h"

namespace wsb {

static inline size_t a256(size_t x) { return (x + 255) & ~size_t(255); }

// Launch with programmatic stream serialisation: the kernel may begin while
// the previous kernel in the stream drains; it waits for that kernel's
// completion itself (griddepcontrol.wait) before touching its results.
template <typename... Params, typename... Args>
static cudaError_t launch_pdl(void (*kernel)(Params...), uint32_t grid, uint32_t block, size_t smem,
                              cudaStream_t st, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, args...);
}

static void release(void *p, bool pooled, cudaStream_t st) {
    if (!p) return;
    if (pooled) cudaFreeAsync(p, st);
    else dev_free(p);
}

MatA::~MatA() {
    for (void *p : {(void *)row_ptr, (void *)col, (void *)val, (void *)brow_ptr, (void *)bcol, (void *)bval,
                    (void *)stiles})
        release(p, pooled, free_stream);
}

Precond::~Precond() {
    for (void *p : {(void *)lu, (void *)bs, (void *)utiles}) release(p, pooled, free_stream);
}

template <class T>
static int upload(Context *ctx, T **dst, const T *src, size_t count, size_t pad, cudaStream_t st, uint64_t *bytes) {
    void *p = nullptr;
    const size_t nbytes = (count + pad) * sizeof(T);
    int rc = dev_alloc(ctx, &p, nbytes, pad > 0, st);
    if (rc) return rc;
    *dst = static_cast<T *>(p);
    if (count) WSB_CUDA_TRY(ctx, cudaMemcpyAsync(p, src, count * sizeof(T), cudaMemcpyHostToDevice, st));
    *bytes += nbytes;
    return WSB_OK;
}

int upload_matA(Context *ctx, uint32_t n, const uint32_t *row_ptr, const uint32_t *col, const float *val,
                uint64_t nnz, const uint32_t *bs, uint64_t bs_len, int layout_req, cudaStream_t st, MatA *out) {
    out->ctx = ctx;
    out->n = n;
    out->nnz = nnz;
    bool bsr = false;
    if (layout_req != WSB_LAYOUT_CSR && bs) bsr = bsr6_convertible(n, row_ptr, col, bs, bs_len);
    if (layout_req == WSB_LAYOUT_BSR6 && !bsr)
        return fail(ctx, WSB_ERR_BAD_INPUT,
                    "BSR6 layout needs blocks of exactly 6 rows whose rows store complete 6x6 blocks with "
                    "strictly increasing columns");
    int rc;
    if (bsr) {
        std::vector<uint32_t> brow_ptr, bcol;
        std::vector<float> bval;
        out->nbsr = csr_to_bsr6(n, row_ptr, col, val, &brow_ptr, &bcol, &bval);
        out->layout = LAYOUT_BSR6;
        if ((rc = upload(ctx, &out->brow_ptr, brow_ptr.data(), brow_ptr.size(), 8, st, &out->bytes))) return rc;
        if ((rc = upload(ctx, &out->bcol, bcol.data(), bcol.size(), kPadElems, st, &out->bytes))) return rc;
        if ((rc = upload(ctx, &out->bval, bval.data(), bval.size(), 16, st, &out->bytes))) return rc;
        const TileCaps caps = tile_caps_for(LAYOUT_BSR6, n, nnz);
        std::vector<SpmvTile> tiles;
        build_spmv_tiles_bsr(n / 6, brow_ptr.data(), &tiles, caps.spmv_rows / 6, caps.spmv_cap);
        out->h_rows = brow_ptr;
        out->tile_rows = caps.spmv_rows;
        out->tile_cap = caps.spmv_cap;
        out->n_stiles = (uint32_t)tiles.size();
        if ((rc = upload(ctx, &out->stiles, tiles.data(), tiles.size(), 1, st, &out->bytes))) return rc;
        WSB_CUDA_TRY(ctx, cudaStreamSynchronize(st));
        return WSB_OK;
    }
    out->layout = LAYOUT_CSR;
    if ((rc = upload(ctx, &out->row_ptr, row_ptr, (size_t)n + 1, 8, st, &out->bytes))) return rc;
    if ((rc = upload(ctx, &out->col, col, nnz, kPadElems, st, &out->bytes))) return rc;
    if ((rc = upload(ctx, &out->val, val, nnz, kPadElems, st, &out->bytes))) return rc;
    const TileCaps caps = tile_caps_for(LAYOUT_CSR, n, nnz);
    std::vector<SpmvTile> tiles;
    build_spmv_tiles_csr(n, row_ptr, &tiles, caps.spmv_rows, caps.spmv_cap);
    out->h_rows.assign(row_ptr, row_ptr + (size_t)n + 1);
    out->tile_rows = caps.spmv_rows;
    out->tile_cap = caps.spmv_cap;
    out->n_stiles = (uint32_t)tiles.size();
    if ((rc = upload(ctx, &out->stiles, tiles.data(), tiles.size(), 1, st, &out->bytes))) return rc;
    WSB_CUDA_TRY(ctx, cudaStreamSynchronize(st));
    return WSB_OK;
}

int upload_precond(Context *ctx, uint32_t n, const float *lu, const uint32_t *bs, uint64_t bs_len, cudaStream_t st,
                   Precond *out) {
    out->ctx = ctx;
    out->n = n;
    out->nb = bs_len >= 1 ? (uint32_t)(bs_len - 1) : 0;
    int rc;
    if ((rc = upload(ctx, &out->lu, lu, (size_t)out->nb * 36, 4, st, &out->bytes))) return rc;
    if ((rc = upload(ctx, &out->bs, bs, (size_t)bs_len, 8, st, &out->bytes))) return rc;
    std::vector<UpdTile> tiles;
    build_upd_tiles(n, bs, out->nb, &tiles, kUpdTileRows, kUpdBlocks);
    out->h_bs.assign(bs, bs + bs_len);
    out->tile_rows = kUpdTileRows;
    out->tile_blocks = kUpdBlocks;
    out->n_utiles = (uint32_t)tiles.size();
    if ((rc = upload(ctx, &out->utiles, tiles.data(), tiles.size(), 1, st, &out->bytes))) return rc;
    WSB_CUDA_TRY(ctx, cudaStreamSynchronize(st));
    return WSB_OK;
}

// Algorithmic bytes of one SpMV: matrix storage + row pointers + x read once +
// y written once.
uint64_t spmv_algorithmic_bytes(const MatA &A) {
    if (A.layout == LAYOUT_BSR6) return 148ull * A.nbsr + 4ull * (A.n / 6 + 1) + 8ull * A.n;
    return 8ull * A.nnz + 4ull * ((uint64_t)A.n + 1) + 8ull * A.n;
}

// One fused iteration: SpMV (reads p, writes Ap) + update (reads x, p, r, Ap,
// LU (24 B/row); writes x, r, z) + p update (reads z, p; writes p).
uint64_t iteration_algorithmic_bytes(const MatA &A, const Precond &M) {
    return spmv_algorithmic_bytes(A) + 28ull * A.n + 144ull * M.nb + 12ull * A.n;
}

// ---------------------------------------------------------------------------
// Engine
// ---------------------------------------------------------------------------
struct Engine::Slot {
    const MatA *A = nullptr;
    const Precond *M = nullptr;
    SolveCfg cfg;
    void *mem = nullptr;
    size_t mem_bytes = 0;
    float *b = nullptr, *x = nullptr, *r = nullptr, *z = nullptr, *p = nullptr, *ap = nullptr, *b_orig = nullptr;
    float *s = nullptr;  // single reduction: s = A p
    double *x64 = nullptr, *part_a = nullptr, *hist = nullptr;
    double2 *part_b = nullptr;
    uint32_t sgroups = 0, ugroups = 0;  // reduction groups of the SpMV and update tiles
    uint64_t hist_cap = 0;
    enum Phase { IDLE, NEED_INIT, RUNNING, NEED_REFINE, DONE } phase = IDLE;
    bool mixed = false;
    bool stalled = false;
    uint64_t iters_total = 0;
    SolveOutcome out;
};

enum { AUX_REFINE = 0, AUX_RESID = 1, AUX_X32 = 2 };

Engine::Engine(Context *ctx, cudaStream_t stream) : ctx_(ctx), stream_(stream) {
    cudaEventCreate(&ev0_);
    cudaEventCreate(&ev1_);
    cudaFuncSetAttribute(k_spmv_loop, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSpmvSmem);
    cudaFuncSetAttribute(k_spmv_init, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSpmvSmem);
    cudaFuncSetAttribute(k_spmv_plain, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSpmvSmem);
    cudaFuncSetAttribute(k_update, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kUpdSmem);
    cudaFuncSetAttribute(k_update_sr, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kUpdSmemSr);
    cudaFuncSetAttribute(k_init, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kUpdSmem);
    int occ_a = 0, occ_b = 0, occ_c = 0, occ_s = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_a, k_spmv_loop, kSpmvThreads, kSpmvSmem);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_b, k_update, kUpdThreads, kUpdSmem);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_c, k_pupdate, kThreads, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_s, k_update_sr, kUpdThreads, kUpdSmemSr);
    max_grid_sr_ = std::max(1, occ_s) * std::max(1, ctx->sm_count);
    max_grid_a_ = std::max(1, occ_a) * std::max(1, ctx->sm_count);
    max_grid_b_ = std::max(1, occ_b) * std::max(1, ctx->sm_count);
    max_grid_c_ = std::max(1, occ_c) * std::max(1, ctx->sm_count);
    const char *loop_env = getenv("WSB_LOOP");
    use_graph_ = !(loop_env && std::strcmp(loop_env, "launch") == 0);
    cudaMallocHost(&h_sp_, sizeof(StepParams));
    cudaMallocHost(&h_sp_rb_, sizeof(StepParams));
    std::memset(h_sp_, 0, sizeof(StepParams));
    std::memset(h_sp_rb_, 0, sizeof(StepParams));
    cudaMalloc(&d_sp_, sizeof(StepParams));
    cudaMemsetAsync(d_sp_, 0, sizeof(StepParams), stream_);
}

Engine::~Engine() {
    cudaStreamSynchronize(stream_);
    if (exec_) cudaGraphExecDestroy(exec_);
    if (graph_) cudaGraphDestroy(graph_);
    for (auto &s : slots_)
        if (s && s->mem) cudaFree(s->mem);
    cudaFree(d_sys_);
    cudaFree(d_state_);
    cudaFree(d_sp_);
    cudaFree(d_work_);
    cudaFreeHost(h_sys_);
    cudaFreeHost(h_state_);
    cudaFreeHost(h_sp_);
    cudaFreeHost(h_sp_rb_);
    cudaFreeHost(h_work_);
    cudaEventDestroy(ev0_);
    cudaEventDestroy(ev1_);
}

int Engine::ensure_capacity(uint32_t need) {
    if (need <= cap_) return WSB_OK;
    uint32_t nc = std::max<uint32_t>(need, std::max<uint32_t>(8, cap_ * 2));
    WSB_CUDA_TRY(ctx_, cudaStreamSynchronize(stream_));
    SysDesc *ds = nullptr, *hs = nullptr;
    SysState *dst = nullptr, *hst = nullptr;
    WSB_CUDA_TRY(ctx_, cudaMalloc(&ds, sizeof(SysDesc) * nc));
    WSB_CUDA_TRY(ctx_, cudaMalloc(&dst, sizeof(SysState) * nc));
    WSB_CUDA_TRY(ctx_, cudaMallocHost(&hs, sizeof(SysDesc) * nc));
    WSB_CUDA_TRY(ctx_, cudaMallocHost(&hst, sizeof(SysState) * nc));
    std::memset(hs, 0, sizeof(SysDesc) * nc);
    std::memset(hst, 0, sizeof(SysState) * nc);
    WSB_CUDA_TRY(ctx_, cudaMemsetAsync(ds, 0, sizeof(SysDesc) * nc, stream_));
    WSB_CUDA_TRY(ctx_, cudaMemsetAsync(dst, 0, sizeof(SysState) * nc, stream_));
    if (cap_) {
        std::memcpy(hs, h_sys_, sizeof(SysDesc) * cap_);
        WSB_CUDA_TRY(ctx_, cudaMemcpyAsync(dst, d_state_, sizeof(SysState) * cap_, cudaMemcpyDeviceToDevice, stream_));
        std::memcpy(hst, h_state_, sizeof(SysState) * cap_);
    }
    // Re-point every slot's state pointer at the new state array.
    for (uint32_t i = 0; i < cap_; ++i) hs[i].st = dst + i;
    if (cap_) WSB_CUDA_TRY(ctx_, cudaMemcpyAsync(ds, hs, sizeof(SysDesc) * cap_, cudaMemcpyHostToDevice, stream_));
    WSB_CUDA_TRY(ctx_, cudaStreamSynchronize(stream_));
    cudaFree(d_sys_);
    cudaFree(d_state_);
    cudaFreeHost(h_sys_);
    cudaFreeHost(h_state_);
    d_sys_ = ds;
    d_state_ = dst;
    h_sys_ = hs;
    h_state_ = hst;
    cap_ = nc;
    // The captured graph holds d_sys_ as a kernel argument.
    if (exec_) cudaGraphExecDestroy(exec_);
    if (graph_) cudaGraphDestroy(graph_);
    exec_ = nullptr;
    graph_ = nullptr;
    graph_grid_a_ = graph_grid_b_ = graph_grid_c_ = 0;
    return WSB_OK;
}

int Engine::push_desc(uint32_t s) {
    WSB_CUDA_TRY(ctx_, cudaMemcpyAsync(d_sys_ + s, h_sys_ + s, sizeof(SysDesc), cudaMemcpyHostToDevice, stream_));
    return WSB_OK;
}

int Engine::push_state(uint32_t s) {
    WSB_CUDA_TRY(ctx_, cudaMemcpyAsync(d_state_ + s, h_state_ + s, sizeof(SysState), cudaMemcpyHostToDevice, stream_));
    return WSB_OK;
}

int Engine::add(const MatA *A, const Precond *M, const SolveCfg &cfg, uint32_t *slot_out) {
    if (A->n != M->n) return fail(ctx_, WSB_ERR_BAD_INPUT, "matrix and preconditioner sizes differ (%u vs %u)", A->n, M->n);
    if (cfg.algorithm != WSB_ALG_CLASSIC && cfg.algorithm != WSB_ALG_SINGLE_REDUCTION)
        return fail(ctx_, WSB_ERR_BAD_INPUT, "unknown algorithm %d", cfg.algorithm);
    // One recurrence per engine (its captured loop body is that recurrence's
    // kernels); an engine with no system left takes the next one's.
    bool empty = true;
    for (auto &sl : slots_)
        if (sl) empty = false;
    if (empty && algo_ != (uint32_t)cfg.algorithm) {
        algo_ = (uint32_t)cfg.algorithm;
        if (exec_) cudaGraphExecDestroy(exec_);
        if (graph_) cudaGraphDestroy(graph_);
        exec_ = nullptr;
        graph_ = nullptr;
        graph_grid_a_ = graph_grid_b_ = graph_grid_c_ = 0;
    }
    if (algo_ != (uint32_t)cfg.algorithm)
        return fail(ctx_, WSB_ERR_UNSUPPORTED,
                    "systems iterated together use one recurrence: this batch or server already runs algorithm %u",
                    algo_);
    // The lists may still name stopped systems (their tiles skipped); a
    // slot they name must not take a new system before they are re-laid out.
    if (retired_tiles_) work_dirty_ = true;
    uint32_t s = (uint32_t)slots_.size();
    for (uint32_t i = 0; i < slots_.size(); ++i)
        if (!slots_[i]) {
            s = i;
            break;
        }
    int rc = ensure_capacity(s + 1);
    if (rc) return rc;
    auto sl = std::make_unique<Slot>();
    sl->A = A;
    sl->M = M;
    sl->cfg = cfg;
    sl->mixed = cfg.precision == WSB_PREC_MIXED_F64_IR;
    const size_t n = A->n, vf = a256((n + kPadElems) * sizeof(float));
    const uint64_t max_hist = cfg.max_iter > 0 ? cfg.max_iter : 1;
    sl->hist_cap = std::min<uint64_t>(cfg.hist_cap, max_hist);
    size_t off[12], tot = 0;
    auto take = [&](int k, size_t bytes) {
        off[k] = tot;
        tot += a256(bytes);
    };
    take(0, vf);  // b (inner right-hand side)
    take(1, vf);  // x
    take(2, vf);  // r
    take(3, vf);  // z
    take(4, vf);  // p
    take(5, vf);  // ap
    take(6, sl->mixed ? vf : 0);                                       // b_orig
    take(7, sl->mixed ? a256((n + kPadElems) * sizeof(double)) : 0);  // x64
    take(8, sizeof(double) * (A->n_stiles + 1));
    take(9, sizeof(double2) * (M->n_utiles + 1));
    take(10, sizeof(double) * (sl->hist_cap + 1));
    take(11, cfg.algorithm == WSB_ALG_SINGLE_REDUCTION ? vf : 0);  // s
    void *mem = nullptr;
    cudaError_t e = cudaMallocAsync(&mem, tot, stream_);
    if (e != cudaSuccess)
        return fail(ctx_, e == cudaErrorMemoryAllocation ? WSB_ERR_OUT_OF_MEMORY : WSB_ERR_CUDA,
                    "device allocation of %zu bytes for a system failed: %s", tot, cudaGetErrorString(e));
    WSB_CUDA_TRY(ctx_, cudaMemsetAsync(mem, 0, tot, stream_));
    char *base = static_cast<char *>(mem);
    sl->mem = mem;
    sl->mem_bytes = tot;
    sl->b = (float *)(base + off[0]);
    sl->x = (float *)(base + off[1]);
    sl->r = (float *)(base + off[2]);
    sl->z = (float *)(base + off[3]);
    sl->p = (float *)(base + off[4]);
    sl->ap = (float *)(base + off[5]);
    sl->b_orig = sl->mixed ? (float *)(base + off[6]) : nullptr;
    sl->x64 = sl->mixed ? (double *)(base + off[7]) : nullptr;
    sl->part_a = (double *)(base + off[8]);
    sl->part_b = (double2 *)(base + off[9]);
    sl->hist = sl->hist_cap ? (double *)(base + off[10]) : nullptr;
    sl->s = cfg.algorithm == WSB_ALG_SINGLE_REDUCTION ? (float *)(base + off[11]) : nullptr;

    SysDesc &d = h_sys_[s];
    std::memset(&d, 0, sizeof d);
    d.n = A->n;
    d.nb = M->nb;
    d.layout = A->layout;
    d.hist_cap = (uint32_t)std::min<uint64_t>(sl->hist_cap, 0xffffffffu);
    d.row_ptr = A->row_ptr;
    d.col = A->col;
    d.val = A->val;
    d.brow_ptr = A->brow_ptr;
    d.bcol = A->bcol;
    d.bval = A->bval;
    d.lu = M->lu;
    d.bstart = M->bs;
    d.b = sl->b;
    d.x = sl->x;
    d.r = sl->r;
    d.z = sl->z;
    d.p = sl->p;
    d.ap = sl->ap;
    d.b_orig = sl->b_orig;
    d.x64 = sl->x64;
    d.stiles = A->stiles;
    d.utiles = M->utiles;
    d.n_stiles = A->n_stiles;
    d.n_utiles = M->n_utiles;
    d.part_a = sl->part_a;
    d.part_b = sl->part_b;
    // As many reduction groups as the kernel has resident CTAs (or one per
    // tile): the last CTA of a reduction then sums at most one partial per
    // CTA instead of one per tile. The groups depend only on the tile count
    // and the device, so a system's sums are the same alone and batched.
    sl->sgroups = std::min<uint32_t>(A->n_stiles, (uint32_t)max_grid_a_);
    sl->ugroups = std::min<uint32_t>(M->n_utiles, (uint32_t)update_grid_max());
    d.n_sgroups = sl->sgroups;
    d.n_ugroups = sl->ugroups;
    d.st = d_state_ + s;
    d.history = sl->hist;
    d.algo = (uint32_t)cfg.algorithm;
    d.s = sl->s;
    std::memset(h_state_ + s, 0, sizeof(SysState));
    if ((rc = push_desc(s))) return rc;
    if ((rc = push_state(s))) return rc;
    if (s == slots_.size())
        slots_.push_back(std::move(sl));
    else
        slots_[s] = std::move(sl);
    *slot_out = s;
    return WSB_OK;
}

int Engine::reset_slot(uint32_t s, const SolveCfg &cfg) {
    Slot &sl = *slots_[s];
    sl.cfg = cfg;
    sl.phase = Slot::IDLE;
    sl.iters_total = 0;
    sl.stalled = false;
    sl.out = SolveOutcome();
    return WSB_OK;
}

int Engine::set_rhs(uint32_t s, const float *b, const float *x0, bool dev) {
    Slot &sl = *slots_[s];
    const size_t nb = sizeof(float) * sl.A->n;
    const cudaMemcpyKind kind = dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    if (nb) {
        WSB_CUDA_TRY(ctx_, cudaMemcpyAsync(sl.mixed ? sl.b_orig : sl.b, b, nb, kind, stream_));
        WSB_CUDA_TRY(ctx_, cudaMemcpyAsync(sl.x, x0, nb, kind, stream_));
        if (sl.mixed) WSB_CUDA_TRY(ctx_, cudaMemsetAsync(sl.x64, 0, sizeof(double) * sl.A->n, stream_));
    }
    sl.phase = sl.mixed ? Slot::NEED_REFINE : Slot::NEED_INIT;
    sl.iters_total = 0;
    sl.stalled = false;
    sl.out = SolveOutcome();
    // Restore the history window (mixed solves move it per sweep).
    h_sys_[s].history = sl.hist;
    h_sys_[s].hist_cap = (uint32_t)std::min<uint64_t>(sl.hist_cap, 0xffffffffu);
    return push_desc(s);
}

bool Engine::done(uint32_t s) const { return slots_[s] && slots_[s]->phase == Slot::DONE; }
uint64_t Engine::slot_bytes(uint32_t s) const { return slots_[s] ? slots_[s]->mem_bytes : 0; }
uint32_t Engine::active_count() const {
    uint32_t c = 0;
    for (auto &s : slots_)
        if (s && (s->phase == Slot::RUNNING || s->phase == Slot::NEED_INIT || s->phase == Slot::NEED_REFINE)) ++c;
    return c;
}

void Engine::remove(uint32_t s) {
    if (s >= slots_.size() || !slots_[s]) return;
    if (slots_[s]->phase == Slot::RUNNING) work_dirty_ = true;
    cudaFreeAsync(slots_[s]->mem, stream_);
    slots_[s].reset();
    std::memset(h_sys_ + s, 0, sizeof(SysDesc));
}

// Work-list storage: six lists (loop a/b/c, init a/b, aux b) of work_cap_
// items each, in one device array with a pinned host mirror. The host only
// rewrites a region before the copy that feeds the next kernel reading it, so
// a copy still pending from earlier in the same step carries either the same
// content or content that a later copy replaces before any kernel reads it.
namespace {

struct GroupSrc {
    uint32_t sys, tiles, groups;
};

// The tiles of some systems laid out in columns for the column walk of the
// loop kernels (StepParams). A system of T tiles in G reduction groups has
// group g = tiles g, g + G, g + 2G, ... (strided: CTAs that walk one group
// each then sweep the system together, as a grid-stride loop would, which
// keeps the DRAM streams and the reuse of x in the L2 of neighbouring tiles;
// contiguous groups of T/G tiles measured slower). The groups of the
// systems, in order, go round-robin to the columns (a system's groups differ
// in size by at most one tile, so the columns stay balanced); a column lists
// its groups' tiles in increasing order (the kernels derive a tile's group
// and its place in it from the tile index), and positions past the end of a
// column are marked kNoSys.
// The layout is rebuilt whenever the active set changes, so it is two
// linear passes with no sorting: layout_size gives the columns (at most
// max_cols) and the longest column, layout_fill writes w x len items.
struct ColLayout {
    uint32_t w = 0, len = 0;
};

ColLayout layout_size(const std::vector<GroupSrc> &src, uint32_t max_cols, std::vector<uint32_t> *col_len) {
    uint64_t groups = 0;
    for (const GroupSrc &q : src) groups += q.groups;
    ColLayout l;
    l.w = (uint32_t)std::min<uint64_t>(groups, std::max<uint32_t>(max_cols, 1u));
    if (l.w == 0) return l;
    col_len->assign(l.w, 0u);
    uint32_t *len = col_len->data(), c = 0;
    for (const GroupSrc &q : src) {
        const uint32_t base = q.tiles / q.groups, rem = q.tiles % q.groups;  // group g has base + (g < rem) tiles
        for (uint32_t g = 0; g < q.groups; ++g) {
            len[c] += base + (g < rem ? 1u : 0u);
            if (++c == l.w) c = 0;
        }
    }
    for (uint32_t i = 0; i < l.w; ++i) l.len = std::max(l.len, len[i]);
    return l;
}

void layout_fill(const std::vector<GroupSrc> &src, const ColLayout &l, std::vector<uint32_t> *cur, WorkItem *dst) {
    if (l.w == 0) return;
    cur->assign(l.w, 0u);
    uint32_t *cj = cur->data(), c = 0;
    const size_t w = l.w;
    for (const GroupSrc &q : src) {
        const uint32_t base = q.tiles / q.groups, rem = q.tiles % q.groups;
        for (uint32_t g = 0; g < q.groups; ++g) {
            const uint32_t sz = base + (g < rem ? 1u : 0u);
            uint32_t j = cj[c];
            WorkItem *o = dst + c + w * j;
            for (uint32_t t = 0; t < sz; ++t, ++j, o += w) *o = WorkItem{q.sys, g + t * q.groups};
            cj[c] = j;
            if (++c == l.w) c = 0;
        }
    }
    for (uint32_t cc = 0; cc < l.w; ++cc)
        for (uint32_t j = cj[cc]; j < l.len; ++j) dst[cc + w * j] = WorkItem{kNoSys, 0u};
}

}  // namespace

// Grows the list storage to at least `per` items per list, keeping every
// list's contents (host and device).
int Engine::ensure_work_cap(size_t per) {
    if (per <= work_cap_) return WSB_OK;
    WSB_CUDA_TRY(ctx_, cudaStreamSynchronize(stream_));
    const size_t nc = std::max(per, work_cap_ * 2);
    WorkItem *d = nullptr, *h = nullptr;
    WSB_CUDA_TRY(ctx_, cudaMalloc(&d, sizeof(WorkItem) * nc * kLists));
    const cudaError_t he = cudaMallocHost(&h, sizeof(WorkItem) * nc * kLists);
    if (he != cudaSuccess) {
        cudaFree(d);
        return fail(ctx_, WSB_ERR_OUT_OF_MEMORY, "pinned work-list allocation failed: %s", cudaGetErrorString(he));
    }
    if (work_cap_) {
        for (int l = 0; l < kLists; ++l) {
            std::memcpy(h + l * nc, h_work_ + l * work_cap_, sizeof(WorkItem) * work_cap_);
            const cudaError_t ce = cudaMemcpy(d + l * nc, d_work_ + l * work_cap_, sizeof(WorkItem) * work_cap_,
                                              cudaMemcpyDeviceToDevice);
            if (ce != cudaSuccess) {
                cudaFree(d);
                cudaFreeHost(h);
                return fail(ctx_, WSB_ERR_CUDA, "work-list copy failed: %s", cudaGetErrorString(ce));
            }
        }
    }
    cudaFree(d_work_);
    cudaFreeHost(h_work_);
    d_work_ = d;
    h_work_ = h;
    work_cap_ = nc;
    return WSB_OK;
}

int Engine::rebuild_work() {
    std::vector<GroupSrc> ga, gb;
    size_t per = 1;
    for (uint32_t s = 0; s < slots_.size(); ++s) {
        const Slot *sl = slots_[s].get();
        if (!sl) continue;
        per += std::max<size_t>(std::max(sl->A->n_stiles, sl->M->n_utiles), chunks_of(sl->A->n));
        if (sl->phase != Slot::RUNNING) continue;
        ga.push_back({s, sl->A->n_stiles, sl->sgroups});
        gb.push_back({s, sl->M->n_utiles, sl->ugroups});
    }
    const ColLayout la = layout_size(ga, (uint32_t)max_grid_a_, &layout_tmp_);
    const ColLayout lb = layout_size(gb, (uint32_t)update_grid_max(), &layout_tmp_);
    const uint32_t na = la.w * la.len, nb = lb.w * lb.len;
    int rc = ensure_work_cap(std::max<size_t>(per, std::max(na, nb) + 1));
    if (rc) return rc;
    uint32_t nch = 0;
    WorkItem *wa = h_work_ + L_A * work_cap_, *wb = h_work_ + L_B * work_cap_, *wc = h_work_ + L_C * work_cap_;
    layout_fill(ga, la, &layout_tmp_, wa);
    layout_fill(gb, lb, &layout_tmp_, wb);
    w_work_a_ = la.w;
    w_work_b_ = lb.w;
    for (uint32_t s = 0; s < slots_.size(); ++s) {
        const Slot *sl = slots_[s].get();
        if (!sl || sl->phase != Slot::RUNNING) continue;
        for (uint32_t t = 0; t < chunks_of(sl->A->n); ++t) wc[nch++] = {s, t};
    }
    n_work_a_ = na;
    n_work_b_ = nb;
    n_work_c_ = nch;
    listed_tiles_ = 0;
    for (const GroupSrc &q : ga) listed_tiles_ += q.tiles;
    for (const GroupSrc &q : gb) listed_tiles_ += q.tiles;
    retired_tiles_ = 0;
    if (na) WSB_CUDA_TRY(ctx_, cudaMemcpyAsync(d_work_ + L_A * work_cap_, wa, sizeof(WorkItem) * na, cudaMemcpyHostToDevice, stream_));
    if (nb) WSB_CUDA_TRY(ctx_, cudaMemcpyAsync(d_work_ + L_B * work_cap_, wb, sizeof(WorkItem) * nb, cudaMemcpyHostToDevice, stream_));
    if (nch) WSB_CUDA_TRY(ctx_, cudaMemcpyAsync(d_work_ + L_C * work_cap_, wc, sizeof(WorkItem) * nch, cudaMemcpyHostToDevice, stream_));
    work_dirty_ = false;
    return WSB_OK;
}

void Engine::fill_list_ptrs() {
    h_sp_->num_sys = cap_;
    h_sp_->work_a = d_work_ + L_A * work_cap_;
    h_sp_->work_b = d_work_ + L_B * work_cap_;
    h_sp_->work_c = d_work_ + L_C * work_cap_;
    h_sp_->init_a = d_work_ + L_IA * work_cap_;
    h_sp_->init_b = d_work_ + L_IB * work_cap_;
    h_sp_->aux_b = d_work_ + L_X * work_cap_;
}

int Engine::capture_loop(uint32_t ga, uint32_t gb, uint32_t gc) {
    if (exec_) cudaGraphExecDestroy(exec_);
    if (graph_) cudaGraphDestroy(graph_);
    exec_ = nullptr;
    graph_ = nullptr;
    WSB_CUDA_TRY(ctx_, cudaGraphCreate(&graph_, 0));
    cudaGraphConditionalHandle h;
    WSB_CUDA_TRY(ctx_, cudaGraphConditionalHandleCreate(&h, graph_, 0, 0));
    cudaKernelNodeParams kp = {};
    StepParams *sp = d_sp_;
    void *gate_args[] = {&sp, &h};
    kp.func = (void *)k_loop_gate;
    kp.gridDim = dim3(1);
    kp.blockDim = dim3(32);
    kp.kernelParams = gate_args;
    cudaGraphNode_t gate;
    WSB_CUDA_TRY(ctx_, cudaGraphAddKernelNode(&gate, graph_, nullptr, 0, &kp));
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t wn;
    WSB_CUDA_TRY(ctx_, cudaGraphAddNode(&wn, graph_, &gate, 1, &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    cudaStream_t cs;
    WSB_CUDA_TRY(ctx_, cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    cudaError_t e = cudaStreamBeginCaptureToGraph(cs, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed);
    if (e == cudaSuccess) {
        const SysDesc *dsys = d_sys_;
        StepParams *dsp = d_sp_;
        cudaError_t le = launch_pdl(k_spmv_loop, ga, kSpmvThreads, kSpmvSmem, cs, dsys, dsp);
        if (algo_ == WSB_ALG_SINGLE_REDUCTION) {
            // Two kernels per iteration: the update kernel also forms the new
            // direction and ends the loop body.
            if (le == cudaSuccess) le = launch_pdl(k_update_sr, gb, kUpdThreads, kUpdSmemSr, cs, dsys, dsp, h);
        } else {
            if (le == cudaSuccess) le = launch_pdl(k_update, gb, kUpdThreads, kUpdSmem, cs, dsys, dsp);
            if (le == cudaSuccess) le = launch_pdl(k_pupdate, gc, kThreads, (size_t)0, cs, dsys, dsp, h);
        }
        e = cudaStreamEndCapture(cs, &body);
        if (e == cudaSuccess && le != cudaSuccess) e = le;
    }
    cudaStreamDestroy(cs);
    if (e != cudaSuccess) return fail(ctx_, WSB_ERR_CUDA, "capturing the PCG loop body failed: %s", cudaGetErrorString(e));
    WSB_CUDA_TRY(ctx_, cudaGraphInstantiate(&exec_, graph_, 0));
    graph_grid_a_ = ga;
    graph_grid_b_ = gb;
    graph_grid_c_ = gc;
    return WSB_OK;
}

int Engine::launch_init(const std::vector<uint32_t> &ids) {
    std::vector<GroupSrc> ga, gb;
    for (uint32_t s : ids) {
        const Slot &sl = *slots_[s];
        ga.push_back({s, sl.A->n_stiles, sl.sgroups});
        gb.push_back({s, sl.M->n_utiles, sl.ugroups});
    }
    const ColLayout la = layout_size(ga, (uint32_t)max_grid_a_, &layout_tmp_);
    const ColLayout lb = layout_size(gb, (uint32_t)max_grid_b_, &layout_tmp_);
    const uint32_t na = la.w * la.len, nb = lb.w * lb.len;
    int rc = ensure_work_cap(std::max(na, nb) + 1);
    if (rc) return rc;
    WorkItem *ia = h_work_ + L_IA * work_cap_, *ib = h_work_ + L_IB * work_cap_;
    layout_fill(ga, la, &layout_tmp_, ia);
    layout_fill(gb, lb, &layout_tmp_, ib);
    h_sp_->w_init_a = la.w;
    h_sp_->w_init_b = lb.w;
    if (na) WSB_CUDA_TRY(ctx_, cudaMemcpyAsync(d_work_ + L_IA * work_cap_, ia, sizeof(WorkItem) * na, cudaMemcpyHostToDevice, stream_));
    if (nb) WSB_CUDA_TRY(ctx_, cudaMemcpyAsync(d_work_ + L_IB * work_cap_, ib, sizeof(WorkItem) * nb, cudaMemcpyHostToDevice, stream_));
    h_sp_->n_init_a = na;
    h_sp_->n_init_b = nb;
    return WSB_OK;
}

int Engine::launch_aux(const std::vector<uint32_t> &ids, int which) {
    if (ids.empty()) return WSB_OK;
    size_t need = 1;
    for (uint32_t s : ids) need += slots_[s]->M->n_utiles;
    int rc = ensure_work_cap(need);  // the loop lists stay as they are
    if (rc) return rc;
    WorkItem *xb = h_work_ + L_X * work_cap_;
    uint32_t nb = 0;
    for (uint32_t s : ids) {
        const Slot &sl = *slots_[s];
        for (uint32_t t = 0; t < sl.M->n_utiles; ++t) xb[nb++] = {s, t};
    }
    WSB_CUDA_TRY(ctx_, cudaMemcpyAsync(d_work_ + L_X * work_cap_, xb, sizeof(WorkItem) * nb, cudaMemcpyHostToDevice, stream_));
    fill_list_ptrs();
    h_sp_->n_aux_b = nb;
    WSB_CUDA_TRY(ctx_, cudaMemcpyAsync(d_sp_, h_sp_, sizeof(StepParams), cudaMemcpyHostToDevice, stream_));
    const uint32_t g = std::min<uint32_t>(nb, (uint32_t)max_grid_b_);
    if (which == AUX_REFINE) k_refine<<<g, kThreads, 0, stream_>>>(d_sys_, d_sp_);
    else if (which == AUX_RESID) k_resid64<<<g, kThreads, 0, stream_>>>(d_sys_, d_sp_);
    else k_x64_to_x32<<<g, kThreads, 0, stream_>>>(d_sys_, d_sp_);
    WSB_CUDA_TRY(ctx_, cudaGetLastError());
    launches_ += 1;
    return WSB_OK;
}

int Engine::read_states(const std::vector<uint32_t> &ids) {
    (void)ids;
    WSB_CUDA_TRY(ctx_, cudaMemcpyAsync(h_state_, d_state_, sizeof(SysState) * cap_, cudaMemcpyDeviceToHost, stream_));
    WSB_CUDA_TRY(ctx_, cudaStreamSynchronize(stream_));
    return WSB_OK;
}

static int map_status(uint32_t st) {
    switch (st) {
        case ST_CONVERGED: return WSB_OK;
        case ST_BREAKDOWN: return WSB_ERR_BREAKDOWN;
        case ST_MAXITER: return WSB_ERR_NOT_CONVERGED;
        default: return WSB_ERR_CUDA;
    }
}

int Engine::finish_slot(uint32_t s, int status) {
    Slot &sl = *slots_[s];
    sl.phase = Slot::DONE;
    sl.out.status = status;
    sl.out.iterations = sl.iters_total;
    return WSB_OK;
}

int Engine::step(uint32_t loop_limit, bool *any_left) {
    int rc;
    // The lists change only when the active set does (work_dirty_); the
    // layout is not free (a linear pass over every tile of every active
    // system), so it is not redone every step.
    if ((work_dirty_ || work_cap_ == 0) && (rc = rebuild_work())) return rc;
    const bool timing = true;
    if (timing) cudaEventRecord(ev0_, stream_);
    // 1) Mixed precision: refinement sweeps (x64 += d; r64 = b - A x64).
    std::vector<uint32_t> refine;
    for (uint32_t s = 0; s < slots_.size(); ++s)
        if (slots_[s] && slots_[s]->phase == Slot::NEED_REFINE) refine.push_back(s);
    if (!refine.empty()) {
        if ((rc = launch_aux(refine, AUX_REFINE))) return rc;
        if ((rc = launch_aux(refine, AUX_RESID))) return rc;
        if ((rc = read_states(refine))) return rc;
        std::vector<uint32_t> finalize;
        for (uint32_t s : refine) {
            Slot &sl = *slots_[s];
            const SysState &st = h_state_[s];
            const double relres = st.bb64 > 0.0 ? std::sqrt(st.rr64 / st.bb64) : 0.0;
            sl.out.relres = relres;
            sl.out.bb = st.bb64;
            int fin = -1;
            if (st.bb64 == 0.0 || relres <= sl.cfg.target_relres) fin = WSB_OK;
            else if (sl.stalled) fin = sl.out.breakdown ? WSB_ERR_BREAKDOWN : WSB_ERR_NOT_CONVERGED;
            else if (sl.out.sweeps >= sl.cfg.max_refine || sl.iters_total >= sl.cfg.max_iter) fin = WSB_ERR_NOT_CONVERGED;
            if (fin >= 0) {
                finalize.push_back(s);
                finish_slot(s, fin);
            } else {
                sl.out.sweeps += 1;
                sl.phase = Slot::NEED_INIT;
            }
        }
        if ((rc = launch_aux(finalize, AUX_X32))) return rc;
    }
    // 2) Systems (re)starting a PCG: state reset, init kernels.
    std::vector<uint32_t> init;
    for (uint32_t s = 0; s < slots_.size(); ++s)
        if (slots_[s] && slots_[s]->phase == Slot::NEED_INIT) init.push_back(s);
    uint32_t running = 0;
    for (auto &sl : slots_)
        if (sl && sl->phase == Slot::RUNNING) ++running;
    // Empty systems finish at once: b.b == 0 gives Ok(0) (compute.rs:252-254).
    for (auto it = init.begin(); it != init.end();) {
        Slot &sl = *slots_[*it];
        if (sl.A->n == 0) {
            sl.out = SolveOutcome();
            finish_slot(*it, WSB_OK);
            it = init.erase(it);
        } else {
            ++it;
        }
    }
    for (uint32_t s : init) {
        Slot &sl = *slots_[s];
        SysState &st = h_state_[s];
        std::memset(&st, 0, sizeof st);
        st.active = 1;
        st.status = ST_RUNNING;
        if (sl.mixed) {
            const uint64_t left = sl.cfg.max_iter > sl.iters_total ? sl.cfg.max_iter - sl.iters_total : 0;
            st.max_iter = (uint32_t)std::min<uint64_t>(left, 0xffffffffu);
            st.rel2 = (double)sl.cfg.inner_rel_tol * (double)sl.cfg.inner_rel_tol;
            st.abs2 = 0.0;
            // Record this sweep's residuals after the previous sweeps' ones.
            const uint64_t hoff = std::min<uint64_t>(sl.iters_total, sl.hist_cap);
            h_sys_[s].history = sl.hist ? sl.hist + hoff : nullptr;
            h_sys_[s].hist_cap = (uint32_t)std::min<uint64_t>(sl.hist_cap - hoff, 0xffffffffu);
            if ((rc = push_desc(s))) return rc;
        } else {
            st.max_iter = (uint32_t)std::min<uint64_t>(sl.cfg.max_iter, 0xffffffffu);
            st.rel2 = (double)sl.cfg.rel_tol * (double)sl.cfg.rel_tol;
            st.abs2 = (double)sl.cfg.abs_tol * (double)sl.cfg.abs_tol;
        }
        if ((rc = push_state(s))) return rc;
        sl.phase = Slot::RUNNING;
    }
    if (!init.empty()) work_dirty_ = true;
    if (work_dirty_ && (rc = rebuild_work())) return rc;
    if ((rc = launch_init(init))) return rc;
    num_active_ = running + (uint32_t)init.size();
    fill_list_ptrs();
    h_sp_->n_work_a = n_work_a_;
    h_sp_->n_work_b = n_work_b_;
    h_sp_->w_work_a = w_work_a_;
    h_sp_->w_work_b = w_work_b_;
    h_sp_->n_work_c = n_work_c_;
    h_sp_->error = 0;
    h_sp_->wait_cycles = ctx_->wait_cycles;
    // Bound the device loop by the largest remaining iteration budget: every
    // system stops by its own max_iter, so the loop ends even if one did not.
    uint64_t budget = 1;
    for (auto &sl : slots_)
        if (sl && sl->phase == Slot::RUNNING) {
            const uint64_t done = h_state_[&sl - &slots_[0]].iter;
            const uint64_t mx = sl->mixed ? (sl->cfg.max_iter > sl->iters_total ? sl->cfg.max_iter - sl->iters_total : 0)
                                          : sl->cfg.max_iter;
            budget = std::max<uint64_t>(budget, (mx > done ? mx - done : 0) + 1);
        }
    const uint32_t limit = (uint32_t)std::min<uint64_t>(loop_limit, std::min<uint64_t>(budget, 0xffffffffu));
    h_sp_->num_active = num_active_;
    h_sp_->loop_count = 0;
    h_sp_->loop_limit = limit;
    WSB_CUDA_TRY(ctx_, cudaMemcpyAsync(d_sp_, h_sp_, sizeof(StepParams), cudaMemcpyHostToDevice, stream_));
    if (!init.empty()) {
        const uint32_t ga = std::min<uint32_t>(h_sp_->w_init_a, (uint32_t)max_grid_a_);
        const uint32_t gb = std::min<uint32_t>(h_sp_->w_init_b, (uint32_t)max_grid_b_);
        const SysDesc *dsys = d_sys_;
        StepParams *dsp = d_sp_;
        if (ga) WSB_CUDA_TRY(ctx_, launch_pdl(k_spmv_init, ga, kSpmvThreads, kSpmvSmem, stream_, dsys, dsp));
        if (gb) WSB_CUDA_TRY(ctx_, launch_pdl(k_init, gb, kUpdThreads, kUpdSmem, stream_, dsys, dsp));
        launches_ += (ga ? 1 : 0) + (gb ? 1 : 0);
    }
    if (num_active_ > 0 && n_work_a_ > 0) {
        const uint32_t ga = std::max<uint32_t>(1, std::min<uint32_t>(w_work_a_, (uint32_t)max_grid_a_));
        const uint32_t gb = std::max<uint32_t>(1, std::min<uint32_t>(w_work_b_, (uint32_t)update_grid_max()));
        const uint32_t gc = std::max<uint32_t>(1, std::min<uint32_t>(n_work_c_, (uint32_t)max_grid_c_));
        if (use_graph_) {
            if (!exec_ || ga > graph_grid_a_ || gb > graph_grid_b_ || gc > graph_grid_c_ || 2 * ga < graph_grid_a_ ||
                2 * gb < graph_grid_b_ || 2 * gc < graph_grid_c_)
                if ((rc = capture_loop(ga, gb, gc))) return rc;
            WSB_CUDA_TRY(ctx_, cudaGraphLaunch(exec_, stream_));
        } else {
            // Plain launches, polling the device state every 16 iterations.
            uint32_t done_iters = 0;
            while (done_iters < limit) {
                const uint32_t burst = std::min<uint32_t>(16, limit - done_iters);
                const SysDesc *dsys = d_sys_;
                StepParams *dsp = d_sp_;
                const cudaGraphConditionalHandle none = 0;
                for (uint32_t i = 0; i < burst; ++i) {
                    WSB_CUDA_TRY(ctx_, launch_pdl(k_spmv_loop, ga, kSpmvThreads, kSpmvSmem, stream_, dsys, dsp));
                    if (algo_ == WSB_ALG_SINGLE_REDUCTION) {
                        WSB_CUDA_TRY(ctx_, launch_pdl(k_update_sr, gb, kUpdThreads, kUpdSmemSr, stream_, dsys, dsp, none));
                    } else {
                        WSB_CUDA_TRY(ctx_, launch_pdl(k_update, gb, kUpdThreads, kUpdSmem, stream_, dsys, dsp));
                        WSB_CUDA_TRY(ctx_, launch_pdl(k_pupdate, gc, kThreads, (size_t)0, stream_, dsys, dsp, none));
                    }
                }
                WSB_CUDA_TRY(ctx_, cudaGetLastError());
                done_iters += burst;
                WSB_CUDA_TRY(ctx_, cudaMemcpyAsync(h_sp_rb_, d_sp_, sizeof(StepParams), cudaMemcpyDeviceToHost, stream_));
                WSB_CUDA_TRY(ctx_, cudaStreamSynchronize(stream_));
                if (h_sp_rb_->num_active == 0 || h_sp_rb_->error) break;
            }
            h_sp_->loop_count = done_iters;
        }
    }
    if (timing) cudaEventRecord(ev1_, stream_);
    // 3) Read back states; retire or hand finished inner solves to refinement.
    std::vector<uint32_t> run_ids;
    for (uint32_t s = 0; s < slots_.size(); ++s)
        if (slots_[s] && slots_[s]->phase == Slot::RUNNING) run_ids.push_back(s);
    if ((rc = read_states(run_ids))) return rc;
    float ms = 0.f;
    if (timing && cudaEventElapsedTime(&ms, ev0_, ev1_) == cudaSuccess) last_device_ms_ = ms;
    uint64_t body_iters = 0;
    for (uint32_t s : run_ids) {
        Slot &sl = *slots_[s];
        const SysState &st = h_state_[s];
        body_iters = std::max<uint64_t>(body_iters, st.iter);
        if (st.active && st.iter >= st.max_iter) {
            // Past its own limit and still active: the device bookkeeping is
            // broken for this system; retire it with an error.
            sl.iters_total += st.iter;
            work_dirty_ = true;
            finish_slot(s, fail(ctx_, WSB_ERR_CUDA, "system %u did not stop at its iteration limit", s));
            continue;
        }
        if (st.active) continue;
        sl.iters_total += st.iter;
        sl.out.rr = st.rr;
        sl.out.breakdown = (int)st.breakdown;
        // Its device state is inactive, so the kernels skip its tiles: the
        // lists are re-laid out only once a quarter of their tiles belong to
        // systems that stopped (or when one joins), not at every retirement.
        retired_tiles_ += (uint64_t)sl.A->n_stiles + sl.M->n_utiles;
        if (sl.mixed) {
            if (st.status == ST_BREAKDOWN) sl.stalled = true;
            if (st.status == ST_MAXITER && sl.iters_total >= sl.cfg.max_iter) sl.stalled = true;
            sl.phase = Slot::NEED_REFINE;
        } else {
            sl.out.bb = st.bb;
            sl.out.relres = st.bb > 0.0 ? std::sqrt(st.rr / st.bb) : 0.0;
            finish_slot(s, map_status(st.status));
        }
    }
    (void)body_iters;
    if (retired_tiles_ * 4 > listed_tiles_) work_dirty_ = true;
    WSB_CUDA_TRY(ctx_, cudaMemcpyAsync(h_sp_rb_, d_sp_, sizeof(StepParams), cudaMemcpyDeviceToHost, stream_));
    WSB_CUDA_TRY(ctx_, cudaStreamSynchronize(stream_));
    // Graph: the gate kernel once, then three body kernels per loop pass.
    if (num_active_ > 0 && n_work_a_ > 0)
        launches_ += use_graph_ ? 1 + 3ull * h_sp_rb_->loop_count : 3ull * h_sp_->loop_count;
    if (h_sp_rb_->error) {
        // A bounded wait ran out inside a kernel: end every system in flight.
        const uint32_t code = h_sp_rb_->error;
        const int rc2 = (code & kErrWaitMask) ? fail(ctx_, WSB_ERR_TIMEOUT, "a device wait ran out (kernel code %u)", code)
                                    : fail(ctx_, WSB_ERR_CUDA, "a kernel met an invalid work item (code %u)", code);
        for (uint32_t s2 = 0; s2 < slots_.size(); ++s2)
            if (slots_[s2] && slots_[s2]->phase == Slot::RUNNING) finish_slot(s2, rc2);
        h_sp_->error = 0;
        WSB_CUDA_TRY(ctx_, cudaMemcpyAsync(d_sp_, h_sp_, sizeof(StepParams), cudaMemcpyHostToDevice, stream_));
        work_dirty_ = true;
        return rc2;
    }
    bool left = false;
    for (auto &sl : slots_)
        if (sl && (sl->phase == Slot::NEED_INIT || sl->phase == Slot::RUNNING || sl->phase == Slot::NEED_REFINE))
            left = true;
    *any_left = left;
    return WSB_OK;
}

int Engine::profile_kernels(uint32_t s, uint32_t iters, double ms[5]) {
    int rc;
    Slot &sl = *slots_[s];
    if (sl.A->n == 0 || iters == 0) return fail(ctx_, WSB_ERR_BAD_INPUT, "nothing to profile");
    SysState &st = h_state_[s];
    std::memset(&st, 0, sizeof st);
    st.active = 1;
    st.status = ST_RUNNING;
    st.max_iter = iters + 1;  // tolerances 0: runs all iterations
    if ((rc = push_state(s))) return rc;
    sl.phase = Slot::RUNNING;
    work_dirty_ = true;
    if ((rc = rebuild_work())) return rc;
    if ((rc = launch_init({s}))) return rc;
    fill_list_ptrs();
    h_sp_->n_work_a = n_work_a_;
    h_sp_->n_work_b = n_work_b_;
    h_sp_->w_work_a = w_work_a_;
    h_sp_->w_work_b = w_work_b_;
    h_sp_->n_work_c = n_work_c_;
    h_sp_->error = 0;
    h_sp_->wait_cycles = ctx_->wait_cycles;
    h_sp_->num_active = 1;
    h_sp_->loop_count = 0;
    h_sp_->loop_limit = iters;
    WSB_CUDA_TRY(ctx_, cudaMemcpyAsync(d_sp_, h_sp_, sizeof(StepParams), cudaMemcpyHostToDevice, stream_));
    const uint32_t ga = std::min<uint32_t>(w_work_a_, (uint32_t)max_grid_a_);
    const uint32_t gb = std::min<uint32_t>(w_work_b_, (uint32_t)update_grid_max());
    const uint32_t gc = std::min<uint32_t>(n_work_c_, (uint32_t)max_grid_c_);
    k_spmv_init<<<std::max<uint32_t>(1, std::min<uint32_t>(h_sp_->w_init_a, (uint32_t)max_grid_a_)), kSpmvThreads, kSpmvSmem, stream_>>>(d_sys_, d_sp_);
    k_init<<<std::max<uint32_t>(1, std::min<uint32_t>(h_sp_->w_init_b, (uint32_t)max_grid_b_)), kUpdThreads, kUpdSmem, stream_>>>(d_sys_, d_sp_);
    std::vector<cudaEvent_t> ev(4 * (size_t)iters);
    for (auto &e : ev) WSB_CUDA_TRY(ctx_, cudaEventCreate(&e));
    for (uint32_t i = 0; i < iters; ++i) {
        cudaEventRecord(ev[4 * i + 0], stream_);
        k_spmv_loop<<<ga, kSpmvThreads, kSpmvSmem, stream_>>>(d_sys_, d_sp_);
        cudaEventRecord(ev[4 * i + 1], stream_);
        if (algo_ == WSB_ALG_SINGLE_REDUCTION)
            k_update_sr<<<gb, kUpdThreads, kUpdSmemSr, stream_>>>(d_sys_, d_sp_, 0);
        else
            k_update<<<gb, kUpdThreads, kUpdSmem, stream_>>>(d_sys_, d_sp_);
        cudaEventRecord(ev[4 * i + 2], stream_);
        if (algo_ != WSB_ALG_SINGLE_REDUCTION) k_pupdate<<<gc, kThreads, 0, stream_>>>(d_sys_, d_sp_, 0);
        cudaEventRecord(ev[4 * i + 3], stream_);
    }
    WSB_CUDA_TRY(ctx_, cudaGetLastError());
    WSB_CUDA_TRY(ctx_, cudaMemcpyAsync(h_sp_rb_, d_sp_, sizeof(StepParams), cudaMemcpyDeviceToHost, stream_));
    WSB_CUDA_TRY(ctx_, cudaStreamSynchronize(stream_));
    if (h_sp_rb_->error) return fail(ctx_, (h_sp_rb_->error & kErrWaitMask) ? WSB_ERR_TIMEOUT : WSB_ERR_CUDA,
                                     "kernel error code %u during profiling", h_sp_rb_->error);
    double acc[3] = {0, 0, 0};
    for (uint32_t i = 0; i < iters; ++i)
        for (int k = 0; k < 3; ++k) {
            float t = 0.f;
            cudaEventElapsedTime(&t, ev[4 * i + k], ev[4 * i + k + 1]);
            acc[k] += t;
        }
    for (auto &e : ev) cudaEventDestroy(e);
    for (int k = 0; k < 3; ++k) ms[k] = acc[k] / iters;
    // The system must still be iterating after `iters` iterations, or the
    // later launches did no work and the means above are not kernel times.
    WSB_CUDA_TRY(ctx_, cudaMemcpyAsync(h_state_ + s, d_state_ + s, sizeof(SysState), cudaMemcpyDeviceToHost, stream_));
    WSB_CUDA_TRY(ctx_, cudaStreamSynchronize(stream_));
    ms[3] = (double)h_state_[s].iter;
    ms[4] = (double)h_state_[s].status;
    sl.phase = Slot::DONE;
    work_dirty_ = true;
    return WSB_OK;
}

int Engine::run() {
    bool left = true;
    double total = 0.0;
    while (left) {
        int rc = step(0xffffffffu, &left);
        if (rc) return rc;
        total += last_device_ms_;
    }
    last_device_ms_ = total;
    return WSB_OK;
}

int Engine::fetch(uint32_t s, float *x, bool dev, bool always_x, SolveOutcome *out, double *hist, uint64_t hist_cap,
                  uint64_t *hist_len, double *x64) {
    Slot &sl = *slots_[s];
    *out = sl.out;
    const size_t nb = sizeof(float) * sl.A->n;
    if (x && nb && (sl.out.status == WSB_OK || always_x))
        WSB_CUDA_TRY(ctx_, cudaMemcpyAsync(x, sl.x, nb, dev ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, stream_));
    if (x64 && sl.x64 && nb && (sl.out.status == WSB_OK || always_x))
        WSB_CUDA_TRY(ctx_, cudaMemcpyAsync(x64, sl.x64, sizeof(double) * sl.A->n,
                                           dev ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, stream_));
    uint64_t hl = std::min<uint64_t>(std::min<uint64_t>(sl.iters_total, sl.hist_cap), hist_cap);
    if (hist && hl) WSB_CUDA_TRY(ctx_, cudaMemcpyAsync(hist, sl.hist, sizeof(double) * hl, cudaMemcpyDeviceToHost, stream_));
    if (hist_len) *hist_len = hist ? hl : 0;
    WSB_CUDA_TRY(ctx_, cudaStreamSynchronize(stream_));
    return WSB_OK;
}

}  // namespace wsb
