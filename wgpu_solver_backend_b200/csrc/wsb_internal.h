// Internal declarations shared by the host library (.cpp) and the kernels (.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <cstdarg>
#include <cstdio>
#include <functional>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/wsb.h"

namespace wsb {

// ---------------------------------------------------------------------------
// Launch geometry shared by host and device code.
// ---------------------------------------------------------------------------
// The SpMV tile caps and ring depth can be overridden at build time
// (-DWSB_CSR_CAP=..., -DWSB_BSR_CAP=..., -DWSB_SPMV_STAGES=...) for tuning
// sweeps; the host tiling and the kernels always use the same values.
#ifndef WSB_CSR_CAP
#define WSB_CSR_CAP 2048
#endif
#ifndef WSB_BSR_CAP
#define WSB_BSR_CAP 128
#endif
#ifndef WSB_SPMV_STAGES
#define WSB_SPMV_STAGES 3
#endif
#ifndef WSB_UPD_STAGES
#define WSB_UPD_STAGES 2
#endif
#ifndef WSB_SPMV_CONSUMERS
#define WSB_SPMV_CONSUMERS 128
#endif
#ifndef WSB_UPD_CONSUMERS
#define WSB_UPD_CONSUMERS 128
#endif
constexpr int kThreads = 256;        // threads per CTA of the vector and refinement kernels
constexpr int kUpdConsumers = WSB_UPD_CONSUMERS;   // consumer threads per CTA of the update kernels
static_assert(kUpdConsumers % 32 == 0 && kUpdConsumers <= 1024, "update consumers");
constexpr int kUpdTileRows = 6 * kUpdConsumers;    // rows per update tile (6 per block)
constexpr int kSpmvConsumers = WSB_SPMV_CONSUMERS;  // consumer threads per CTA of the SpMV kernels
constexpr int kSpmvTileRows = kSpmvConsumers;       // rows (or block rows x 6) per SpMV tile
constexpr int kCsrCap = WSB_CSR_CAP;         // CSR nonzeros per SpMV tile (one TMA stage)
constexpr int kBsrCapBlocks = WSB_BSR_CAP;   // BSR 6x6 blocks per SpMV tile (144 B each)
constexpr int kSpmvStages = WSB_SPMV_STAGES; // depth of the SpMV shared-memory ring
constexpr int kUpdBlocks = kUpdConsumers;          // block-Jacobi blocks per update tile (one per consumer)
constexpr int kUpdStages = WSB_UPD_STAGES;   // depth of the update shared-memory ring
static_assert(kCsrCap % 4 == 0 && kBsrCapBlocks % 4 == 0 && kSpmvStages >= 2, "SpMV tile caps");
constexpr int kChunkRows = 4096;     // rows per work item of the vector kernels
constexpr int kPadElems = 64;        // tail padding of streamed arrays (elements)

enum SysStatus : uint32_t {
    ST_RUNNING = 0,
    ST_CONVERGED = 1,
    ST_BREAKDOWN = 2,
    ST_MAXITER = 3,
};

enum Layout : uint32_t { LAYOUT_CSR = 1, LAYOUT_BSR6 = 2 };

// The PCG recurrence of a system (WSB_ALG_*): the reference's classic one, or
// the single-reduction recurrence of Chronopoulos and Gear, whose SpMV
// multiplies u = M r (w = A u) and keeps s = A p by recurrence, so that the
// direction update p = u + beta p moves into the update kernel.
enum Algo : uint32_t { ALGO_CLASSIC = 0, ALGO_SINGLE_REDUCTION = 1 };

// Row tile of the SpMV: rows [row0, row1) (CSR) or block rows (BSR6), and
// their nonzero (or 6x6 block) range [k0, k1). A tile holds at most
// kCsrCap nonzeros (kBsrCapBlocks blocks) unless it is a single longer row.
struct SpmvTile {
    uint32_t row0, row1, k0, k1;
};
// Row tile of the update kernels; never cuts the first 6 rows of a block and
// holds at most kUpdBlocks block starts. Blocks whose first row lies in
// [row0, row1) are [blk0, blk1).
struct UpdTile {
    uint32_t row0, row1, blk0, blk1;
};
// One tile of a system (a list position that carries no tile has sys ==
// kNoSys; the SpMV and update lists are laid out in columns, see
// StepParams). A tile's reduction group and whether it opens or closes it
// follow from the tile index: with G groups, tile t is in group t mod G,
// opens it when t < G and closes it when t + G >= T.
struct WorkItem {
    uint32_t sys, tile;
};
constexpr uint32_t kNoSys = 0xffffffffu;
constexpr uint32_t kGroupFirst = 1u, kGroupLast = 2u;

// Mutable per-system scalars; written only by the last CTA of a reduction.
struct alignas(64) SysState {
    double bb, rz_old, pap, rr, rz_new, alpha, beta;
    double rel2, abs2;
    float alpha_f, beta_f;
    uint32_t iter, max_iter, status, active;
    uint32_t cnt_a, cnt_b;      // last-CTA tickets of the two reductions
    uint32_t breakdown;         // 1: pAp == 0, 2: rz_old == 0
    uint32_t pad0;
    double rr64, bb64;          // FP64 true residual and ||b||^2 (mixed precision)
    uint32_t cnt_c, pad1;
    double gamma_prev;          // single reduction: (r, u) of the previous iteration
};

// Read-mostly description of one system in device memory.
struct SysDesc {
    uint32_t n, nb, layout, hist_cap;
    const uint32_t *row_ptr, *col;
    const float *val;
    const uint32_t *brow_ptr, *bcol;   // BSR6: block rows = n/6
    const float *bval;                 // 36 floats per block, row-major
    const float *lu;                   // 36 floats per diagonal block
    const uint32_t *bstart;            // nb + 1
    const float *b;                    // right-hand side of the (inner) PCG
    float *x, *r, *z, *p, *ap;
    const float *b_orig;               // mixed precision: the caller's b
    double *x64;                       // mixed precision: FP64 solution
    const SpmvTile *stiles;
    const UpdTile *utiles;
    uint32_t n_stiles, n_utiles;
    uint32_t n_sgroups, n_ugroups;     // reduction groups of the SpMV and update tiles
    double *part_a;                    // p.Ap (u.w) partial of each SpMV tile group
    double2 *part_b;                   // (r.r, r.z) partials of each update tile group (refinement: of each tile)
    SysState *st;
    double *history;                   // hist_cap entries or null
    uint32_t algo, pad_algo;           // Algo
    float *s;                          // single reduction: s = A p (by recurrence)
};

// Bits of StepParams::error. The wait bits mean a bounded mbarrier wait ran
// out (the kernel recorded the bit, drained its own copies and returned); the
// host reports them as WSB_ERR_TIMEOUT. kErrBadItem marks a work item that
// names a system or tile that does not exist (the item was skipped).
constexpr uint32_t kErrSpmvConsumerWait = 1u;   // SpMV consumers: stage data
constexpr uint32_t kErrUpdConsumerWait = 2u;    // update consumers (loop kernel)
constexpr uint32_t kErrInitConsumerWait = 4u;   // update consumers (init kernel)
constexpr uint32_t kErrBadItem = 8u;            // invalid work item
constexpr uint32_t kErrSpmvProducerWait = 16u;  // SpMV producer: a free stage
constexpr uint32_t kErrUpdProducerWait = 32u;   // update producer: a free stage
constexpr uint32_t kErrGatherWait = 64u;        // SpMV gather warp: a tile descriptor
constexpr uint32_t kErrWaitMask = kErrSpmvConsumerWait | kErrUpdConsumerWait | kErrInitConsumerWait |
                                  kErrSpmvProducerWait | kErrUpdProducerWait | kErrGatherWait;

// Kernel parameters of one loop step that the host may change between graph
// launches (work lists, counts); lives in device memory so a captured graph
// stays valid.
struct StepParams {
    const WorkItem *work_a;            // loop: SpMV tiles of active systems
    const WorkItem *work_b;            // loop: update tiles of active systems
    const WorkItem *work_c;            // loop: kChunkRows row chunks of active systems
    const WorkItem *init_a;            // init: SpMV tiles of systems (re)starting
    const WorkItem *init_b;            // init: update tiles of systems (re)starting
    const WorkItem *aux_b;             // refinement kernels: update tiles
    uint32_t n_work_a, n_work_b, n_work_c;
    uint32_t n_init_a, n_init_b;
    // Column counts of the grouped lists (loop and init SpMV / update lists):
    // a list of n items is w columns of n / w consecutive positions each
    // (position c + w j is item j of column c); a CTA walks columns
    // blockIdx.x, blockIdx.x + gridDim.x, ..., each from its first item to
    // its last, so a reduction group (consecutive items of one column) is
    // always processed by one CTA, in order, whatever the grid.
    uint32_t w_work_a, w_work_b, w_init_a, w_init_b;
    uint32_t n_aux_b;
    uint32_t num_active;               // systems still iterating
    uint32_t loop_count;               // body executions in this launch
    uint32_t loop_limit;               // stop the while loop after this many
    uint32_t error;                    // nonzero: a bounded wait ran out or a work item was invalid
    uint32_t num_sys;                  // entries of the SysDesc array (work items are checked against it)
    uint32_t tail_ticket;              // single reduction: CTAs of the update kernel done (last one ends the step)
    unsigned long long wait_cycles;    // limit of one pipeline wait in SM clock cycles; 0: the default (~2 s)
};

// ---------------------------------------------------------------------------
// Errors
// ---------------------------------------------------------------------------
void set_thread_error(const std::string &msg);
const char *thread_error();

struct Context;
int fail(Context *ctx, int status, const char *fmt, ...);

#define WSB_CUDA_TRY(ctx, expr)                                                              \
    do {                                                                                     \
        cudaError_t _e = (expr);                                                             \
        if (_e != cudaSuccess)                                                               \
            return ::wsb::fail((ctx), _e == cudaErrorMemoryAllocation ? WSB_ERR_OUT_OF_MEMORY \
                                                                      : WSB_ERR_CUDA,          \
                               "%s failed: %s (%s:%d)", #expr, cudaGetErrorString(_e),       \
                               __FILE__, __LINE__);                                          \
    } while (0)

// ---------------------------------------------------------------------------
// Context
// ---------------------------------------------------------------------------
struct Context {
    int device = 0;
    unsigned long long wait_cycles = 0;  // StepParams::wait_cycles of this context's launches (0: default)
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;     // own_stream or the caller's
    cudaDeviceProp prop{};
    int sm_count = 0;
    std::string last_error;
    std::mutex mu;
};

struct Buffer {
    Context *ctx = nullptr;
    void *ptr = nullptr;
    size_t bytes = 0;
};

// Device allocation; when `zero`, the zero fill is enqueued on `stream`, so
// it is ordered before every later copy or kernel on that stream (a plain
// cudaMemset would run on the legacy default stream, unordered with work on
// non-blocking streams).
int dev_alloc(Context *ctx, void **p, size_t bytes, bool zero, cudaStream_t stream);
void dev_free(void *p);
// A memory pool that dev_alloc draws from on the calling thread (stream
// ordered, cudaMallocFromPoolAsync on the given stream) instead of
// cudaMalloc, or null. The server's uploader threads set it, so that
// retiring a request frees its matrix with cudaFreeAsync instead of a
// cudaFree, which would wait for every copy and kernel in flight on the GPU.
cudaMemPool_t &thread_alloc_pool();

// ---------------------------------------------------------------------------
// Host-side setup helpers (host_setup.cpp)
// ---------------------------------------------------------------------------
int lu_factor_inplace_6(float *mat, uint32_t n, uint32_t *pivot_k);
// Returns WSB_OK / WSB_ERR_BAD_INPUT / WSB_ERR_ZERO_PIVOT with message in *err.
int build_lu_blocks_6(uint32_t n, const uint32_t *row_ptr, uint64_t row_ptr_len, const uint32_t *col,
                      uint64_t col_len, const float *val, uint64_t val_len, const uint32_t *bs,
                      uint64_t bs_len, float *out, std::string *err);
// Validation of a CSR matrix + block partition (loaders.rs:44-212 rules).
// With check_cols false the O(nnz) column-range scan is left to the caller
// (the device-side preparation does it on the GPU).
int validate_system(uint32_t n, const uint32_t *row_ptr, const uint32_t *col, uint64_t nnz,
                    const uint32_t *bs, uint64_t bs_len, std::string *err, bool check_cols = true);

// Tile builders; the caps default to the largest tiles the kernels stage.
void build_spmv_tiles_csr(uint32_t n, const uint32_t *row_ptr, std::vector<SpmvTile> *out,
                          uint32_t max_rows = kSpmvTileRows, uint32_t max_nnz = kCsrCap);
void build_spmv_tiles_bsr(uint32_t nbrows, const uint32_t *brow_ptr, std::vector<SpmvTile> *out,
                          uint32_t max_brows = kSpmvTileRows / 6, uint32_t max_blocks = kBsrCapBlocks);
void build_upd_tiles(uint32_t n, const uint32_t *bs, uint32_t nb, std::vector<UpdTile> *out,
                     uint32_t max_rows = kUpdTileRows, uint32_t max_blocks = kUpdBlocks);
// True when every block has 6 rows and every touched 6x6 block is fully stored.
bool bsr6_convertible(uint32_t n, const uint32_t *row_ptr, const uint32_t *col, const uint32_t *bs,
                      uint64_t bs_len);
// CSR -> BSR6 (requires bsr6_convertible). Returns block count.
uint64_t csr_to_bsr6(uint32_t n, const uint32_t *row_ptr, const uint32_t *col, const float *val,
                     std::vector<uint32_t> *brow_ptr, std::vector<uint32_t> *bcol, std::vector<float> *bval);

void parallel_for(int64_t n, int64_t grain, const std::function<void(int64_t, int64_t)> &fn);

}  // namespace wsb
