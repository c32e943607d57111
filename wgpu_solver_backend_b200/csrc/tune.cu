// Tile-size autotuner.
//
// The SpMV and update kernels stream fixed-size tiles through shared memory;
// how many rows and nonzeros (6x6 blocks) a tile holds trades per-tile cost
// against parallelism: large tiles amortise the per-tile work of the
// pipeline, small tiles spread a small system over more SMs. The autotuner
// times the solver's own kernels on the matrix for a few candidate tilings
// (CUDA events around each launch, a short PCG run on a right-hand side of
// ones) and keeps the fastest SpMV tiling and the fastest update tiling.
// The choice is also recorded per shape class (layout, n to within a factor
// of 2, nonzeros per row), and matrices of that class created later start
// with it.
//
// A tiling changes how the per-tile FP64 partial sums of the dot products
// are grouped, so results of a retuned matrix agree with the untuned ones to
// FP64 rounding (not bit for bit); for a given tiling they are reproducible,
// alone and batched.
#include <algorithm>
#include <cmath>
#include <map>
#include <mutex>
#include <string>
#include <tuple>

#include "engine.h"

namespace wsb {

namespace {

std::mutex g_caps_mu;
std::map<std::tuple<uint32_t, int, uint32_t>, TileCaps> g_caps;

std::tuple<uint32_t, int, uint32_t> shape_key(uint32_t layout, uint32_t n, uint64_t nnz) {
    const int size_class = n ? (int)std::floor(std::log2((double)n)) : 0;
    const uint32_t per_row = n ? (uint32_t)std::lround((double)nnz / (double)n) : 0;
    return std::make_tuple(layout, size_class, per_row);
}

TileCaps default_caps(uint32_t layout) {
    TileCaps c;
    c.spmv_rows = layout == LAYOUT_BSR6 ? 6 * (kSpmvTileRows / 6) : kSpmvTileRows;
    c.spmv_cap = layout == LAYOUT_BSR6 ? kBsrCapBlocks : kCsrCap;
    c.upd_rows = kUpdTileRows;
    c.upd_blocks = kUpdBlocks;
    return c;
}

template <class T>
int upload_tiles(Context *ctx, const std::vector<T> &tiles, cudaStream_t st, T **dst, uint32_t *count,
                 uint64_t *bytes) {
    void *p = nullptr;
    const size_t nbytes = sizeof(T) * (tiles.size() + 1);
    int rc = dev_alloc(ctx, &p, nbytes, true, st);
    if (rc) return rc;
    if (!tiles.empty())
        WSB_CUDA_TRY(ctx, cudaMemcpyAsync(p, tiles.data(), sizeof(T) * tiles.size(), cudaMemcpyHostToDevice, st));
    WSB_CUDA_TRY(ctx, cudaStreamSynchronize(st));
    dev_free(*dst);
    *bytes = *bytes + nbytes - sizeof(T) * ((uint64_t)*count + 1);
    *dst = static_cast<T *>(p);
    *count = (uint32_t)tiles.size();
    return WSB_OK;
}

}  // namespace

TileCaps tile_caps_for(uint32_t layout, uint32_t n, uint64_t nnz) {
    std::lock_guard<std::mutex> lk(g_caps_mu);
    auto it = g_caps.find(shape_key(layout, n, nnz));
    return it != g_caps.end() ? it->second : default_caps(layout);
}

void tile_caps_record(uint32_t layout, uint32_t n, uint64_t nnz, const TileCaps &c) {
    std::lock_guard<std::mutex> lk(g_caps_mu);
    g_caps[shape_key(layout, n, nnz)] = c;
}

void tile_caps_clear() {
    std::lock_guard<std::mutex> lk(g_caps_mu);
    g_caps.clear();
}

int retile_spmv(MatA *A, uint32_t rows, uint32_t cap, cudaStream_t st) {
    std::vector<SpmvTile> tiles;
    if (A->layout == LAYOUT_BSR6) build_spmv_tiles_bsr(A->n / 6, A->h_rows.data(), &tiles, rows / 6, cap);
    else build_spmv_tiles_csr(A->n, A->h_rows.data(), &tiles, rows, cap);
    const int rc = upload_tiles(A->ctx, tiles, st, &A->stiles, &A->n_stiles, &A->bytes);
    if (!rc) {
        A->tile_rows = rows;
        A->tile_cap = cap;
    }
    return rc;
}

int retile_update(Precond *M, uint32_t rows, uint32_t blocks, cudaStream_t st) {
    std::vector<UpdTile> tiles;
    build_upd_tiles(M->n, M->h_bs.data(), M->nb, &tiles, rows, blocks);
    const int rc = upload_tiles(M->ctx, tiles, st, &M->utiles, &M->n_utiles, &M->bytes);
    if (!rc) {
        M->tile_rows = rows;
        M->tile_blocks = blocks;
    }
    return rc;
}

}  // namespace wsb

using namespace wsb;

// Mean per-launch time of the SpMV and update kernels over `iters` PCG
// iterations of the matrix with its current tiles (b = ones, x0 = 0).
static int time_tiling(Context *ctx, MatA *A, Precond *M, const float *d_b, uint32_t iters, double *spmv_ms,
                       double *upd_ms) {
    Engine E(ctx, ctx->stream);
    SolveCfg cfg;
    cfg.max_iter = iters + 1;
    uint32_t slot;
    int rc = E.add(A, M, cfg, &slot);
    if (rc) return rc;
    float *d_x0 = nullptr;
    const size_t xbytes = sizeof(float) * std::max<uint32_t>(A->n, 1);
    WSB_CUDA_TRY(ctx, cudaMallocAsync((void **)&d_x0, xbytes, ctx->stream));
    const cudaError_t me = cudaMemsetAsync(d_x0, 0, xbytes, ctx->stream);
    if (me != cudaSuccess) {
        cudaFreeAsync(d_x0, ctx->stream);
        return fail(ctx, WSB_ERR_CUDA, "autotune: cudaMemsetAsync failed: %s", cudaGetErrorString(me));
    }
    rc = E.set_rhs(slot, d_b, d_x0, true);
    double ms[5] = {0, 0, 0, 0, 0};
    if (!rc) rc = E.profile_kernels(slot, iters, ms);
    cudaFreeAsync(d_x0, ctx->stream);
    if (rc) return rc;
    if ((uint32_t)ms[3] != iters || ms[4] != 0.0)
        return fail(ctx, WSB_ERR_CUDA, "autotune: the timing run stopped after %u of %u iterations", (uint32_t)ms[3],
                    iters);
    *spmv_ms = ms[0];
    *upd_ms = ms[1];
    return WSB_OK;
}

int wsb::autotune_matrix(Context *ctx, MatA *A, Precond *M, uint32_t iters, wsb_tune_result *out) {
    if (A->n == 0) return fail(ctx, WSB_ERR_BAD_INPUT, "autotune: empty matrix");
    iters = std::max<uint32_t>(2, std::min<uint32_t>(iters, 64));
    std::vector<float> ones(A->n, 1.0f);
    float *d_b = nullptr;
    WSB_CUDA_TRY(ctx, cudaMalloc((void **)&d_b, sizeof(float) * A->n));
    std::unique_ptr<void, void (*)(void *)> guard(d_b, dev_free);
    WSB_CUDA_TRY(ctx, cudaMemcpyAsync(d_b, ones.data(), sizeof(float) * A->n, cudaMemcpyHostToDevice, ctx->stream));
    const bool bsr = A->layout == LAYOUT_BSR6;
    // SpMV candidates: (rows, cap) from the largest stage down.
    std::vector<std::pair<uint32_t, uint32_t>> sc;
    if (bsr) {
        const uint32_t br = kSpmvTileRows / 6;
        for (uint32_t d : {1u, 2u, 4u, 8u})
            if (br / d >= 1 && kBsrCapBlocks / d >= 4) sc.push_back({6 * std::max(1u, br / d), kBsrCapBlocks / d});
    } else {
        for (uint32_t d : {1u, 2u, 4u, 8u})
            if (kSpmvTileRows / d >= 8) sc.push_back({kSpmvTileRows / d, kCsrCap / d});
    }
    std::vector<std::pair<uint32_t, uint32_t>> uc;
    for (uint32_t d : {1u, 2u, 4u})
        if (kUpdTileRows / d >= 32) uc.push_back({kUpdTileRows / d, std::max(8u, (uint32_t)kUpdBlocks / d)});
    const TileCaps start{A->tile_rows, A->tile_cap, M->tile_rows, M->tile_blocks};
    // On any failure the matrix goes back to the tiling it came with (the
    // error of the failed step stays the reported one).
    auto give_up = [&](int err) {
        std::string msg;
        {
            std::lock_guard<std::mutex> lk(ctx->mu);
            msg = ctx->last_error;
        }
        const int r1 = retile_spmv(A, start.spmv_rows, start.spmv_cap, ctx->stream);
        const int r2 = retile_update(M, start.upd_rows, start.upd_blocks, ctx->stream);
        if (r1 || r2) fail(ctx, err, "%s", msg.c_str());
        return err;
    };
    wsb_tune_result r{};
    int rc;
    // Defaults first (also the baseline the result reports).
    const TileCaps def = default_caps(A->layout);
    if ((rc = retile_spmv(A, def.spmv_rows, def.spmv_cap, ctx->stream)) ||
        (rc = retile_update(M, def.upd_rows, def.upd_blocks, ctx->stream)))
        return give_up(rc);
    double best_s = 0, best_u = 0;
    if ((rc = time_tiling(ctx, A, M, d_b, iters, &best_s, &best_u))) return give_up(rc);
    r.default_spmv_ms = best_s;
    r.default_update_ms = best_u;
    r.candidates = 1;
    TileCaps best = def;
    for (const auto &c : sc) {
        if (c.first == def.spmv_rows && c.second == def.spmv_cap) continue;
        if ((rc = retile_spmv(A, c.first, c.second, ctx->stream))) return give_up(rc);
        double s = 0, u = 0;
        if ((rc = time_tiling(ctx, A, M, d_b, iters, &s, &u))) return give_up(rc);
        ++r.candidates;
        if (s < best_s) {
            best_s = s;
            best.spmv_rows = c.first;
            best.spmv_cap = c.second;
        }
    }
    if ((rc = retile_spmv(A, best.spmv_rows, best.spmv_cap, ctx->stream))) return give_up(rc);
    for (const auto &c : uc) {
        if (c.first == def.upd_rows && c.second == def.upd_blocks) continue;
        if ((rc = retile_update(M, c.first, c.second, ctx->stream))) return give_up(rc);
        double s = 0, u = 0;
        if ((rc = time_tiling(ctx, A, M, d_b, iters, &s, &u))) return give_up(rc);
        ++r.candidates;
        if (u < best_u) {
            best_u = u;
            best.upd_rows = c.first;
            best.upd_blocks = c.second;
        }
    }
    if ((rc = retile_update(M, best.upd_rows, best.upd_blocks, ctx->stream))) return give_up(rc);
    tile_caps_record(A->layout, A->n, A->nnz, best);
    r.spmv_rows = best.spmv_rows;
    r.spmv_cap = best.spmv_cap;
    r.update_rows = best.upd_rows;
    r.update_blocks = best.upd_blocks;
    r.spmv_ms = best_s;
    r.update_ms = best_u;
    if (out) *out = r;
    return WSB_OK;
}
