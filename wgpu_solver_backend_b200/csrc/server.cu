// Continuous-batching solve server.
//
// Three parties share a request table:
//  - wsb_server_submit (caller's thread) copies the arrays and queues them;
//  - the uploader thread validates a request, builds its block-Jacobi LU on
//    the host, reserves device memory against the budget and uploads the
//    matrix on its own stream while the GPU iterates other systems;
//  - the scheduler thread owns the Engine: at every step boundary it admits
//    uploaded systems (Krylov vectors allocated, b/x0 copied), runs
//    iters_per_step iterations of every active system in one graph launch,
//    then retires finished systems (x copied out, memory released).
// A request that cannot fit the budget even alone is rejected with
// WSB_ERR_OUT_OF_MEMORY; others wait until enough memory is released.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <thread>
#include <unordered_map>

#include "engine.h"

using namespace wsb;

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
    uint64_t id = 0;
    uint32_t n = 0;
    uint64_t nnz = 0;
    // The request's arrays: copies owned here, or (WSB_SERVER_BORROW_INPUTS)
    // the caller's arrays, read in place until the request is done. The
    // pointers below are the ones every stage uses.
    std::vector<uint32_t> row_ptr, col, bs;
    std::vector<float> val, b, x0;
    const uint32_t *p_row_ptr = nullptr, *p_col = nullptr, *p_bs = nullptr;
    const float *p_val = nullptr, *p_b = nullptr, *p_x0 = nullptr;
    uint64_t bs_len = 0;
    SolveCfg cfg;
    bool always_x = false;
    std::vector<double> hist;
    std::unique_ptr<MatA> A;
    std::unique_ptr<Precond> M;
    uint32_t slot = 0;
    uint64_t reserved = 0;
    enum State { QUEUED, UPLOADING, READY, ACTIVE, DONE } state = QUEUED;
    int status = WSB_PENDING;
    std::string error;
    std::vector<float> x;
    std::vector<double> x64;
    double *x64_out = nullptr;
    wsb_solve_result res{};
    Clock::time_point t_submit, t_done;
};

// Device bytes a request holds while resident (matrix, LU, vectors, partials).
uint64_t estimate_bytes(const Request &r) {
    const uint64_t n = r.n, nnz = r.nnz, nb = r.bs_len ? r.bs_len - 1 : 0;
    uint64_t a = 8 * nnz + 4 * (n + 1) + 8 * kPadElems + 8 * (n / 16 + 64);      // CSR (BSR6 is smaller)
    uint64_t m = 144 * nb + 4 * (nb + 1) + 16 * (n / 16 + 64) + 1024;            // LU, starts, tiles
    uint64_t v = 6 * 4 * (n + kPadElems) + 8 * (n / 16 + 64) + 16 * (n / 16 + 64) + 8 * 4096;
    if (r.cfg.precision == WSB_PREC_MIXED_F64_IR) v += 12 * (n + kPadElems);
    if (r.cfg.algorithm == WSB_ALG_SINGLE_REDUCTION) v += 4 * (n + kPadElems);
    v += 8 * std::min<uint64_t>(r.cfg.hist_cap, r.cfg.max_iter + 1);
    return a + m + v;
}

}  // namespace

struct wsb_server {
    Context *ctx = nullptr;
    wsb_server_opts opts{};
    cudaStream_t stream = nullptr;
    std::vector<cudaStream_t> upload_streams;
    // Device memory of the requests' matrices and factors: a stream-ordered
    // pool that keeps up to the budget cached, so that admitting and retiring
    // requests never calls cudaMalloc/cudaFree (a cudaFree waits for all work
    // in flight on the GPU, the uploads of other requests included).
    cudaMemPool_t pool = nullptr;
    std::unique_ptr<Engine> eng;
    std::mutex mu;
    std::condition_variable cv_upload, cv_sched, cv_done;
    std::deque<Request *> queued;   // waiting for the uploader
    std::deque<Request *> ready;    // uploaded, waiting for the scheduler
    std::vector<Request *> active;  // in the engine
    std::unordered_map<uint64_t, std::unique_ptr<Request>> table;
    uint64_t next_id = 1;
    uint64_t bytes_in_use = 0, bytes_peak = 0;
    uint32_t uploading = 0;          // requests an uploader is preparing
    wsb_server_stats stats{};
    bool stopping = false;
    std::vector<std::thread> uploaders;
    std::thread scheduler;
    std::string fatal;

    void finish(Request *r, int status, const std::string &err) {
        r->status = status;
        r->error = err;
        r->state = Request::DONE;
        r->t_done = Clock::now();
        r->res.status = status;
        r->res.total_ms = std::chrono::duration<double, std::milli>(r->t_done - r->t_submit).count();
        r->row_ptr.clear();
        r->row_ptr.shrink_to_fit();
        r->col.clear();
        r->col.shrink_to_fit();
        r->val.clear();
        r->val.shrink_to_fit();
        r->p_row_ptr = r->p_col = r->p_bs = nullptr;
        r->p_val = nullptr;
        if (status == WSB_OK) ++stats.completed;
        else ++stats.failed;
    }

    void upload_loop(cudaStream_t upload_stream) {
        cudaSetDevice(ctx->device);
        thread_alloc_pool() = pool;
        for (;;) {
            Request *r = nullptr;
            {
                std::unique_lock<std::mutex> lk(mu);
                cv_upload.wait(lk, [&] {
                    if (stopping) return true;
                    if (queued.empty()) return false;
                    const uint64_t need = estimate_bytes(*queued.front());
                    return need > opts.memory_budget_bytes || bytes_in_use + need <= opts.memory_budget_bytes;
                });
                if (stopping) return;
                r = queued.front();
                queued.pop_front();
                const uint64_t need = estimate_bytes(*r);
                if (need > opts.memory_budget_bytes) {
                    ++stats.rejected;
                    finish(r, WSB_ERR_OUT_OF_MEMORY, "request needs more device memory than the server budget");
                    cv_done.notify_all();
                    continue;
                }
                r->reserved = need;
                bytes_in_use += need;
                bytes_peak = std::max(bytes_peak, bytes_in_use);
                r->state = Request::UPLOADING;
                ++uploading;
            }
            std::string err;
            int rc = WSB_OK;
            const auto t0 = Clock::now();
            double prep_ms = 0.0;
            if (opts.flags & WSB_SERVER_DEVICE_PREP) {
                // O(n) checks and the tile lists on the host; the column
                // check, the BSR6 conversion and the LU on the GPU.
                new_parts(r, upload_stream);
                rc = prepare_system_device(ctx, r->n, r->p_row_ptr, r->p_col, r->p_val, r->nnz, r->p_bs, r->bs_len,
                                           WSB_LAYOUT_AUTO, upload_stream, r->A.get(), r->M.get());
                if (rc) err = thread_error();
            } else {
                rc = validate_system(r->n, r->p_row_ptr, r->p_col, r->nnz, r->p_bs, r->bs_len, &err);
                std::vector<float> lu;
                if (!rc) {
                    lu.resize((r->bs_len - 1) * 36 + 1);
                    rc = build_lu_blocks_6(r->n, r->p_row_ptr, (uint64_t)r->n + 1, r->p_col, r->nnz, r->p_val, r->nnz,
                                           r->p_bs, r->bs_len, lu.data(), &err);
                }
                prep_ms = std::chrono::duration<double, std::milli>(Clock::now() - t0).count();
                if (!rc) {
                    new_parts(r, upload_stream);
                    rc = upload_matA(ctx, r->n, r->p_row_ptr, r->p_col, r->p_val, r->nnz, r->p_bs, r->bs_len,
                                     WSB_LAYOUT_AUTO, upload_stream, r->A.get());
                    if (!rc) rc = upload_precond(ctx, r->n, lu.data(), r->p_bs, r->bs_len, upload_stream, r->M.get());
                    if (rc) err = thread_error();
                }
            }
            const double all_ms = std::chrono::duration<double, std::milli>(Clock::now() - t0).count();
            std::lock_guard<std::mutex> lk(mu);
            --uploading;
            stats.host_prep_ms += prep_ms;
            stats.upload_ms += all_ms - prep_ms;
            if (rc) {
                r->A.reset();
                r->M.reset();
                bytes_in_use -= r->reserved;
                finish(r, rc, err);
                cv_done.notify_all();
                cv_upload.notify_all();
                continue;
            }
            // From here on the scheduler's stream orders the release.
            r->A->free_stream = stream;
            r->M->free_stream = stream;
            r->state = Request::READY;
            ready.push_back(r);
            cv_sched.notify_all();
        }
    }

    // The request's matrix and factor objects; their memory comes from the
    // pool and is released on the upload stream until the request is ready.
    void new_parts(Request *r, cudaStream_t upload_stream) {
        r->A.reset(new MatA());
        r->M.reset(new Precond());
        r->A->pooled = r->M->pooled = pool != nullptr;
        r->A->free_stream = r->M->free_stream = upload_stream;
    }

    void sched_loop() {
        cudaSetDevice(ctx->device);
        for (;;) {
            std::vector<Request *> admit;
            bool more_coming = false;
            {
                std::unique_lock<std::mutex> lk(mu);
                const auto tw = Clock::now();
                cv_sched.wait(lk, [&] { return stopping || !ready.empty() || !active.empty(); });
                stats.sched_idle_ms += std::chrono::duration<double, std::milli>(Clock::now() - tw).count();
                if (stopping && active.empty() && ready.empty()) return;
                while (!ready.empty() && (opts.max_active == 0 || active.size() + admit.size() < opts.max_active)) {
                    admit.push_back(ready.front());
                    ready.pop_front();
                }
                // Requests still on their way to the GPU: keep steps short so
                // they join soon; otherwise longer steps (fewer host turnarounds).
                more_coming = !queued.empty() || !ready.empty() || uploading > 0;
            }
            const auto ta = Clock::now();
            for (Request *r : admit) {
                int rc = eng->add(r->A.get(), r->M.get(), r->cfg, &r->slot);
                if (!rc) rc = eng->set_rhs(r->slot, r->p_b, r->p_x0, false);
                std::lock_guard<std::mutex> lk(mu);
                if (rc) {
                    r->A.reset();
                    r->M.reset();
                    bytes_in_use -= r->reserved;
                    finish(r, rc, thread_error());
                    cv_done.notify_all();
                    cv_upload.notify_all();
                } else {
                    r->state = Request::ACTIVE;
                    active.push_back(r);
                }
            }
            const double admit_ms = std::chrono::duration<double, std::milli>(Clock::now() - ta).count();
            if (active.empty()) continue;
            const auto t0 = Clock::now();
            bool left = false;
            const uint32_t iters = more_coming ? opts.iters_per_step : 4 * opts.iters_per_step;
            int rc = eng->step(iters, &left);
            const double ms = std::chrono::duration<double, std::milli>(Clock::now() - t0).count();
            std::vector<Request *> finished;
            std::unique_lock<std::mutex> lk(mu);
            const auto tr = Clock::now();
            stats.steps += 1;
            stats.busy_ms += ms;
            stats.admit_ms += admit_ms;
            stats.kernel_launches = eng->launches();
            if (rc) {
                // A device error ends every active request.
                fatal = thread_error();
                for (Request *r : active) finished.push_back(r);
            } else {
                for (Request *r : active)
                    if (eng->done(r->slot)) finished.push_back(r);
            }
            for (Request *r : finished) {
                SolveOutcome out;
                uint64_t hl = 0;
                int frc = WSB_ERR_CUDA;
                if (!rc) {
                    r->x.resize(r->n);
                    if (r->x64_out) r->x64.resize(r->n);
                    frc = eng->fetch(r->slot, r->x.data(), false, true, &out, r->hist.empty() ? nullptr : r->hist.data(),
                                     r->hist.size(), &hl, r->x64_out ? r->x64.data() : nullptr);
                }
                eng->remove(r->slot);
                r->A.reset();
                r->M.reset();
                bytes_in_use -= r->reserved;
                std::memset(&r->res, 0, sizeof r->res);
                r->res.breakdown_kind = out.breakdown;
                r->res.iterations = out.iterations;
                r->res.refine_sweeps = out.sweeps;
                r->res.b_norm2 = out.bb;
                r->res.final_r_norm2 = out.rr;
                r->res.final_relres = out.relres;
                r->res.history_len = hl;
                const int st = rc ? rc : frc ? frc : out.status;
                finish(r, st, rc ? fatal : "");
                active.erase(std::find(active.begin(), active.end(), r));
            }
            stats.retire_ms += std::chrono::duration<double, std::milli>(Clock::now() - tr).count();
            if (!finished.empty()) {
                cv_done.notify_all();
                cv_upload.notify_all();
            }
        }
    }
};

extern "C" int wsb_server_create(wsb_context *ctx_in, const wsb_server_opts *opts, wsb_server **out) {
    Context *ctx = reinterpret_cast<Context *>(ctx_in);
    if (!ctx || !out) return fail(ctx, WSB_ERR_BAD_INPUT, "bad arguments");
    cudaSetDevice(ctx->device);
    auto *s = new wsb_server();
    s->ctx = ctx;
    if (opts) s->opts = *opts;
    if (s->opts.memory_budget_bytes == 0) s->opts.memory_budget_bytes = 120ull << 30;
    if (s->opts.iters_per_step == 0) s->opts.iters_per_step = 16;
    cudaError_t e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete s;
        return fail(ctx, WSB_ERR_CUDA, "server stream creation failed: %s", cudaGetErrorString(e));
    }
    s->eng.reset(new Engine(ctx, s->stream));
    cudaMemPoolProps pp = {};
    pp.allocType = cudaMemAllocationTypePinned;
    pp.location.type = cudaMemLocationTypeDevice;
    pp.location.id = ctx->device;
    if (cudaMemPoolCreate(&s->pool, &pp) == cudaSuccess) {
        uint64_t keep = s->opts.memory_budget_bytes;
        cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrReleaseThreshold, &keep);
    } else {
        s->pool = nullptr;  // plain cudaMalloc/cudaFree then
    }
    // Several uploaders: host preparation of one large request (validation,
    // LU, BSR6 conversion, copies) overlaps with that of the next ones.
    const unsigned n_up = std::max(1u, std::min(4u, std::thread::hardware_concurrency() / 2));
    for (unsigned i = 0; i < n_up; ++i) {
        cudaStream_t us = nullptr;
        if (cudaStreamCreateWithFlags(&us, cudaStreamNonBlocking) != cudaSuccess) break;
        s->upload_streams.push_back(us);
    }
    for (cudaStream_t us : s->upload_streams) s->uploaders.emplace_back([s, us] { s->upload_loop(us); });
    s->scheduler = std::thread([s] { s->sched_loop(); });
    *out = s;
    return WSB_OK;
}

extern "C" int wsb_server_submit(wsb_server *s, uint32_t n, const uint32_t *row_ptr, const uint32_t *col, const float *val,
                                 uint64_t nnz, const uint32_t *bs, uint64_t bs_len, const float *b, const float *x0,
                                 uint64_t max_iter, float rel_tol, float abs_tol, const wsb_solve_opts *o, uint64_t *id) {
    if (!s || !id) return fail(nullptr, WSB_ERR_BAD_INPUT, "bad arguments");
    if (!row_ptr || (nnz && (!col || !val)) || !bs || bs_len < 1 || (n && (!b || !x0)))
        return fail(s->ctx, WSB_ERR_BAD_INPUT, "null array");
    if (o && o->precision != WSB_PREC_F32_F64DOT && o->precision != WSB_PREC_MIXED_F64_IR)
        return fail(s->ctx, WSB_ERR_UNSUPPORTED, "the server uses FP64 reductions (F32_F64DOT or MIXED_F64_IR)");
    auto r = std::make_unique<Request>();
    r->n = n;
    r->nnz = nnz;
    r->bs_len = bs_len;
    if (s->opts.flags & WSB_SERVER_BORROW_INPUTS) {
        r->p_row_ptr = row_ptr;
        r->p_col = col;
        r->p_val = val;
        r->p_bs = bs;
        r->p_b = b;
        r->p_x0 = x0;
    } else {
        r->row_ptr.assign(row_ptr, row_ptr + (size_t)n + 1);
        r->col.assign(col, col + nnz);
        r->val.assign(val, val + nnz);
        r->bs.assign(bs, bs + bs_len);
        r->b.assign(b, b + n);
        r->x0.assign(x0, x0 + n);
        r->p_row_ptr = r->row_ptr.data();
        r->p_col = r->col.data();
        r->p_val = r->val.data();
        r->p_bs = r->bs.data();
        r->p_b = r->b.data();
        r->p_x0 = r->x0.data();
    }
    SolveCfg c;
    c.max_iter = max_iter;
    c.rel_tol = rel_tol;
    c.abs_tol = abs_tol;
    if (o) {
        c.precision = o->precision;
        if (o->target_relres > 0) c.target_relres = o->target_relres;
        if (o->inner_rel_tol > 0) c.inner_rel_tol = o->inner_rel_tol;
        if (o->max_refine > 0) c.max_refine = o->max_refine;
        c.hist_cap = o->history_capacity;
        c.algorithm = o->algorithm;
        r->always_x = o->always_write_x != 0;
        r->x64_out = o->x64_out;
    }
    r->cfg = c;
    if (c.hist_cap) r->hist.assign(std::min<uint64_t>(c.hist_cap, max_iter + 1), 0.0);
    r->t_submit = Clock::now();
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stopping) return fail(s->ctx, WSB_ERR_BAD_INPUT, "server is stopping");
    r->id = s->next_id++;
    *id = r->id;
    s->queued.push_back(r.get());
    s->table.emplace(r->id, std::move(r));
    ++s->stats.submitted;
    s->cv_upload.notify_all();
    return WSB_OK;
}

static int take_result(wsb_server *s, Request *r, float *x, wsb_solve_result *res) {
    const int st = r->status;
    if (res) *res = r->res;
    if (x && !r->x.empty() && (st == WSB_OK || r->always_x)) std::memcpy(x, r->x.data(), sizeof(float) * r->n);
    if (r->x64_out && !r->x64.empty() && (st == WSB_OK || r->always_x))
        std::memcpy(r->x64_out, r->x64.data(), sizeof(double) * r->n);
    if (st != WSB_OK) {
        if (st == WSB_ERR_NOT_CONVERGED)
            fail(s->ctx, st, "PCG(BlockJacobiGpu): did not converge in %llu iterations", (unsigned long long)r->cfg.max_iter);
        else if (st == WSB_ERR_BREAKDOWN)
            fail(s->ctx, st, r->res.breakdown_kind == 2 ? "PCG(BlockJacobiGpu): rz_old is zero (breakdown)"
                                                         : "PCG(BlockJacobiGpu): dot(p,Ap) is zero (breakdown)");
        else
            fail(s->ctx, st, "%s", r->error.c_str());
    }
    s->table.erase(r->id);
    return st;
}

extern "C" int wsb_server_poll(wsb_server *s, uint64_t id, float *x, wsb_solve_result *res) {
    if (!s) return fail(nullptr, WSB_ERR_BAD_INPUT, "server is null");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->table.find(id);
    if (it == s->table.end()) return fail(s->ctx, WSB_ERR_BAD_INPUT, "unknown request id %llu", (unsigned long long)id);
    Request *r = it->second.get();
    if (r->state != Request::DONE) return WSB_PENDING;
    return take_result(s, r, x, res);
}

extern "C" int wsb_server_wait(wsb_server *s, uint64_t id, float *x, wsb_solve_result *res, double timeout_s) {
    if (!s) return fail(nullptr, WSB_ERR_BAD_INPUT, "server is null");
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->table.find(id);
    if (it == s->table.end()) return fail(s->ctx, WSB_ERR_BAD_INPUT, "unknown request id %llu", (unsigned long long)id);
    Request *r = it->second.get();
    const auto deadline = Clock::now() + std::chrono::duration_cast<Clock::duration>(std::chrono::duration<double>(timeout_s));
    if (!s->cv_done.wait_until(lk, deadline, [&] { return r->state == Request::DONE; }))
        return fail(s->ctx, WSB_ERR_TIMEOUT, "request %llu not finished after %.3f s", (unsigned long long)id, timeout_s);
    return take_result(s, r, x, res);
}

extern "C" int wsb_server_stats_get(wsb_server *s, wsb_server_stats *out) {
    if (!s || !out) return fail(nullptr, WSB_ERR_BAD_INPUT, "bad arguments");
    std::lock_guard<std::mutex> lk(s->mu);
    *out = s->stats;
    out->active = s->active.size();
    out->pending = s->queued.size() + s->ready.size();
    out->device_bytes_in_use = s->bytes_in_use;
    out->device_bytes_peak = s->bytes_peak;
    return WSB_OK;
}

extern "C" void wsb_server_destroy(wsb_server *s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stopping = true;
        // Queued requests never start.
        for (Request *r : s->queued) s->finish(r, WSB_ERR_TIMEOUT, "server stopped before the request started");
        s->queued.clear();
    }
    s->cv_upload.notify_all();
    s->cv_sched.notify_all();
    for (auto &t : s->uploaders)
        if (t.joinable()) t.join();
    if (s->scheduler.joinable()) s->scheduler.join();
    cudaSetDevice(s->ctx->device);
    s->eng.reset();
    s->table.clear();
    cudaStreamSynchronize(s->stream);
    for (cudaStream_t us : s->upload_streams) cudaStreamSynchronize(us);
    if (s->pool) cudaMemPoolDestroy(s->pool);
    cudaStreamDestroy(s->stream);
    for (cudaStream_t us : s->upload_streams) cudaStreamDestroy(us);
    delete s;
}
