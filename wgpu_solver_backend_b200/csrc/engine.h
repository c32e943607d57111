// Host-side solver objects: device-resident matrix parts and the engine that
// iterates any number of independent systems with the fused kernels.
#pragma once
#include <memory>

#include "kernels_fused.cuh"

namespace wsb {

// The operator A on the device (the part SpmvExecutor::create uploads,
// spmv_exec.rs:38-118), in CSR or BSR6 layout, with its SpMV tile list.
struct MatA {
    Context *ctx = nullptr;
    uint32_t n = 0;
    uint64_t nnz = 0;
    uint32_t layout = LAYOUT_CSR;
    uint32_t *row_ptr = nullptr, *col = nullptr;
    float *val = nullptr;
    uint32_t *brow_ptr = nullptr, *bcol = nullptr;
    float *bval = nullptr;
    uint64_t nbsr = 0;
    SpmvTile *stiles = nullptr;
    uint32_t n_stiles = 0;
    uint64_t bytes = 0;
    // Host copy of the row structure the SpMV tiles are cut from (row_ptr,
    // or brow_ptr for BSR6) and the caps the current tiles were built with.
    std::vector<uint32_t> h_rows;
    uint32_t tile_rows = 0, tile_cap = 0;
    // Memory drawn from a stream-ordered pool (thread_alloc_pool): released
    // with cudaFreeAsync on free_stream, which must order after its last use.
    bool pooled = false;
    cudaStream_t free_stream = nullptr;
    ~MatA();
};

// The block-Jacobi preconditioner on the device (BlockJacobiExecutor::create,
// block_jacobi_exec.rs:48-91): LU factors, block starts, update tile list.
struct Precond {
    Context *ctx = nullptr;
    uint32_t n = 0, nb = 0;
    float *lu = nullptr;
    uint32_t *bs = nullptr;
    UpdTile *utiles = nullptr;
    uint32_t n_utiles = 0;
    uint64_t bytes = 0;
    std::vector<uint32_t> h_bs;                 // host copy of the block starts
    uint32_t tile_rows = 0, tile_blocks = 0;    // caps of the current update tiles
    bool pooled = false;                        // as MatA::pooled
    cudaStream_t free_stream = nullptr;
    ~Precond();
};

// SpMV and update tile caps (rows are rows for CSR and 6 x block rows for
// BSR6; cap is nonzeros for CSR and 6x6 blocks for BSR6).
struct TileCaps {
    uint32_t spmv_rows, spmv_cap, upd_rows, upd_blocks;
};
// The caps recorded for matrices of this shape by the autotuner, or the
// largest tiles the kernels stage.
TileCaps tile_caps_for(uint32_t layout, uint32_t n, uint64_t nnz);
void tile_caps_record(uint32_t layout, uint32_t n, uint64_t nnz, const TileCaps &c);
void tile_caps_clear();
// Rebuild a matrix's SpMV tiles or a preconditioner's update tiles with new
// caps (device tile lists replaced; no solve may be running on them).
int retile_spmv(MatA *A, uint32_t rows, uint32_t cap, cudaStream_t st);
int retile_update(Precond *M, uint32_t rows, uint32_t blocks, cudaStream_t st);
// Times candidate tilings of the matrix's SpMV and update kernels, keeps the
// fastest of each and records them for the matrix's shape class (tune.cu).
int autotune_matrix(Context *ctx, MatA *A, Precond *M, uint32_t iters, wsb_tune_result *out);

// Host arrays of a system; csr is always given, the rest is derived.
int upload_matA(Context *ctx, uint32_t n, const uint32_t *row_ptr, const uint32_t *col, const float *val,
                uint64_t nnz, const uint32_t *bs, uint64_t bs_len, int layout_req, cudaStream_t st, MatA *out);
int upload_precond(Context *ctx, uint32_t n, const float *lu, const uint32_t *bs, uint64_t bs_len,
                   cudaStream_t st, Precond *out);
// Uploads a system's CSR arrays and block starts and prepares the rest on the
// device (column check, BSR6 test and conversion, block-Jacobi LU); host
// work is limited to O(n) checks and the tile lists. Status and message as
// the host path (validate_system, build_lu_blocks_6, upload_matA).
int prepare_system_device(Context *ctx, uint32_t n, const uint32_t *row_ptr, const uint32_t *col, const float *val,
                          uint64_t nnz, const uint32_t *bs, uint64_t bs_len, int layout_req, cudaStream_t st,
                          MatA *A, Precond *M);
uint64_t spmv_algorithmic_bytes(const MatA &A);
uint64_t iteration_algorithmic_bytes(const MatA &A, const Precond &M);

struct SolveCfg {
    uint64_t max_iter = 0;
    float rel_tol = 0.0f, abs_tol = 0.0f;
    int precision = WSB_PREC_F32_F64DOT;
    double target_relres = 1e-10;
    float inner_rel_tol = 1e-4f;
    uint32_t max_refine = 50;
    uint64_t hist_cap = 0;
    int algorithm = WSB_ALG_CLASSIC;  // the PCG recurrence (wsb_algorithm)
};

struct SolveOutcome {
    int status = WSB_OK;
    int breakdown = 0;
    uint64_t iterations = 0;
    uint32_t sweeps = 0;
    double bb = 0.0, rr = 0.0, relres = 0.0;
};


// Multi-system PCG engine. Systems are slots; each owns its Krylov vectors,
// partial buffers and state in HBM. run()/step() iterate all active slots
// together with one captured graph: a gate kernel, then a while loop of
// {k_spmv, k_update, k_pupdate} that ends when no slot is active or after
// loop_limit iterations. Between steps the host retires finished slots,
// restarts refinement sweeps and rebuilds the work lists.
class Engine {
  public:
    Engine(Context *ctx, cudaStream_t stream);
    ~Engine();
    int add(const MatA *A, const Precond *M, const SolveCfg &cfg, uint32_t *slot);
    // b, x0: n floats each, host (pinned or pageable) or device memory.
    int set_rhs(uint32_t slot, const float *b, const float *x0, bool device_ptrs);
    int run();                                       // all slots to completion
    int step(uint32_t loop_limit, bool *any_left);   // one scheduler step
    int fetch(uint32_t slot, float *x, bool device_ptr, bool always_x, SolveOutcome *out, double *hist,
              uint64_t hist_cap, uint64_t *hist_len, double *x64 = nullptr);
    int reset_slot(uint32_t slot, const SolveCfg &cfg);  // reuse for another solve
    // Runs the init kernels and then `iters` loop iterations of one slot
    // outside the graph with CUDA events around every launch; ms[0..2] get
    // the mean duration of k_spmv_loop, k_update and k_pupdate; ms[3] and
    // ms[4] the system's iteration count and status afterwards.
    int profile_kernels(uint32_t slot, uint32_t iters, double ms[5]);
    void remove(uint32_t slot);
    bool done(uint32_t slot) const;
    uint64_t slot_bytes(uint32_t slot) const;
    uint32_t active_count() const;
    double last_device_ms() const { return last_device_ms_; }
    cudaStream_t stream() const { return stream_; }
    // Number of fused-kernel launches issued so far (3 per iteration step).
    uint64_t launches() const { return launches_; }

  public:
    struct Slot;

  private:
    int ensure_capacity(uint32_t need);
    int capture_loop(uint32_t grid_a, uint32_t grid_b, uint32_t grid_c);
    void fill_list_ptrs();
    static uint32_t chunks_of(uint32_t n) { return (n + kChunkRows - 1) / kChunkRows; }
    // Work-list regions in d_work_ / h_work_ (work_cap_ items each).
    enum { L_A = 0, L_B = 1, L_C = 2, L_IA = 3, L_IB = 4, L_X = 5, kLists = 6 };
    int push_desc(uint32_t slot);
    int push_state(uint32_t slot);
    int launch_init(const std::vector<uint32_t> &slots);
    int launch_aux(const std::vector<uint32_t> &slots, int which);
    int rebuild_work();
    int read_states(const std::vector<uint32_t> &slots);
    int finish_slot(uint32_t slot, int status);

    Context *ctx_;
    cudaStream_t stream_;
    std::vector<std::unique_ptr<Slot>> slots_;
    uint32_t cap_ = 0;
    SysDesc *d_sys_ = nullptr, *h_sys_ = nullptr;      // device array + pinned mirror
    SysState *d_state_ = nullptr, *h_state_ = nullptr;
    StepParams *d_sp_ = nullptr, *h_sp_ = nullptr, *h_sp_rb_ = nullptr;
    WorkItem *d_work_ = nullptr, *h_work_ = nullptr;  // kLists regions
    size_t work_cap_ = 0;
    uint32_t n_work_a_ = 0, n_work_b_ = 0, n_work_c_ = 0;
    uint32_t w_work_a_ = 0, w_work_b_ = 0;  // column counts of the loop SpMV and update lists
    int ensure_work_cap(size_t per);
    std::vector<uint32_t> layout_tmp_;  // scratch of the work-list layout (column lengths / cursors)
    uint64_t listed_tiles_ = 0, retired_tiles_ = 0;  // tiles in the lists; of systems stopped since
    bool work_dirty_ = true;
    bool use_graph_ = true;   // WSB_LOOP=launch: plain launches + host polling
    cudaGraph_t graph_ = nullptr;
    cudaGraphExec_t exec_ = nullptr;
    uint32_t graph_grid_a_ = 0, graph_grid_b_ = 0, graph_grid_c_ = 0;
    int max_grid_a_ = 0, max_grid_b_ = 0, max_grid_c_ = 0;
    int max_grid_sr_ = 0;                   // resident CTAs of k_update_sr
    uint32_t algo_ = WSB_ALG_CLASSIC;       // the recurrence of every system in this engine
    int update_grid_max() const { return algo_ == WSB_ALG_SINGLE_REDUCTION ? max_grid_sr_ : max_grid_b_; }
    uint32_t num_active_ = 0;
    double last_device_ms_ = 0.0;
    uint64_t launches_ = 0;
    cudaEvent_t ev0_ = nullptr, ev1_ = nullptr;
};

}  // namespace wsb
