/*
 * wsb.h - C ABI of the B200-native block-Jacobi preconditioned CG library.
 *
 * This is the drop-in boundary for the solve path of the Rust crate
 * `wgpu_solver_backend` (crates/wgpu_solver_backend). Each entry point names
 * the reference item it replaces as path:line inside that crate.
 *
 * Conventions
 *  - Every call returns an int status (wsb_status); 0 is success.
 *  - On failure the message is available from wsb_last_error(ctx) (or
 *    wsb_last_error(NULL) for calls that take no context). Where the reference
 *    returns Err(String), the message text follows the reference's.
 *  - Handles are opaque. Host arrays are owned by the caller and copied; the
 *    library never keeps a caller pointer after a call returns.
 *  - One context is used by one host thread at a time (the reference's
 *    executors are !Sync). A server object runs its own internal thread.
 *  - All device work is ordered on the context's stream (its own, or one given
 *    with wsb_context_set_stream).
 */
#ifndef WSB_H
#define WSB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define WSB_ABI_VERSION 1

typedef enum wsb_status {
    WSB_OK = 0,
    WSB_ERR_BAD_INPUT = 1,      /* validation failures: compute.rs:210-217, compute.rs:93-131, loaders.rs:8-212 */
    WSB_ERR_ZERO_PIVOT = 2,     /* "LU zero pivot at k = ..." compute.rs:50-52 */
    WSB_ERR_BREAKDOWN = 3,      /* dot(p,Ap)==0 or rz_old==0, compute.rs:473-478 */
    WSB_ERR_NOT_CONVERGED = 4,  /* "did not converge in N iterations", compute.rs:491-494 */
    WSB_ERR_CUDA = 5,           /* a CUDA runtime error (GpuError::RequestDevice analogue) */
    WSB_ERR_OUT_OF_MEMORY = 6,  /* device allocation failed or a request exceeds the memory budget */
    WSB_ERR_TIMEOUT = 7,        /* a bounded wait ran out */
    WSB_ERR_NO_DEVICE = 8,      /* GpuError::NoAdapter, context.rs:14-20 */
    WSB_ERR_UNSUPPORTED = 9,
    WSB_PENDING = 10            /* server: request accepted but not finished */
} wsb_status;

/* ------------------------------------------------------------------------- */
/* Context (replaces GpuContext, gpu/context.rs:40-178)                       */
/* ------------------------------------------------------------------------- */
typedef struct wsb_context wsb_context;

typedef struct wsb_adapter_info {   /* AdapterInfo, gpu/context.rs:31-37 */
    char name[256];
    char backend[16];               /* always "Cuda" */
    char device_type[32];           /* "DiscreteGpu" */
    uint32_t vendor;                /* PCI vendor id (0x10de) */
    uint32_t device;                /* PCI device id when known, else 0 */
    uint32_t sm_count;
    int cc_major, cc_minor;
    uint64_t total_mem_bytes;
} wsb_adapter_info;

/* GpuContext::create(GpuBackend), gpu/context.rs:60-109. `device` is a CUDA
 * ordinal; the reference's backend choice (Auto/Vulkan/Dx12/Metal) has no
 * counterpart: this library runs only on CUDA sm_100a devices. */
int wsb_context_create(int device, wsb_context **out);
void wsb_context_destroy(wsb_context *ctx);
/* Last error message of this context (or of the calling thread when ctx is NULL). */
const char *wsb_last_error(const wsb_context *ctx);
/* GpuContext::describe, gpu/context.rs:111-120. */
int wsb_context_describe(const wsb_context *ctx, char *buf, size_t cap);
int wsb_context_adapter_info(const wsb_context *ctx, wsb_adapter_info *out);
/* Order all further work of this context on the caller's cudaStream_t
 * (passed as void*); NULL restores the context's own stream. */
int wsb_context_set_stream(wsb_context *ctx, void *cuda_stream);
int wsb_context_synchronize(wsb_context *ctx);
/* Failure detection (no counterpart in the reference, which blocks on
 * futures without a limit): every wait of the pipelined solver kernels gives
 * up after `cycles` SM clock cycles (0 restores the default of about 2 s);
 * the kernel then records the wait, drains its own copies in flight and
 * returns, and the solve reports WSB_ERR_TIMEOUT for every system in flight.
 * Applies to solves, batches and servers started on this context afterwards. */
int wsb_context_set_wait_limit(wsb_context *ctx, uint64_t cycles);

/* ------------------------------------------------------------------------- */
/* Device buffers (GpuBuffer<T>, gpu/buffer.rs:6-17)                          */
/* ------------------------------------------------------------------------- */
typedef struct wsb_buffer wsb_buffer;
/* create_storage_buffer (context.rs:122-142) when data != NULL, else
 * create_storage_buffer_uninit (context.rs:144-166); like wgpu, a buffer
 * created without data is zero-filled. */
int wsb_buffer_create(wsb_context *ctx, const void *data, size_t bytes, wsb_buffer **out);
int wsb_buffer_write(wsb_context *ctx, wsb_buffer *buf, size_t offset, const void *src, size_t bytes);
/* GpuContext::readback / readback_to_vec, context.rs:168-177, readback.rs:9-54. Blocking. */
int wsb_buffer_read(wsb_context *ctx, const wsb_buffer *buf, size_t offset, void *dst, size_t bytes);
size_t wsb_buffer_size(const wsb_buffer *buf);
void *wsb_buffer_device_ptr(const wsb_buffer *buf);
void wsb_buffer_destroy(wsb_buffer *buf);

/* ------------------------------------------------------------------------- */
/* Executors: the reference's per-pass building blocks, on the GPU with the   */
/* reference's arithmetic (sequential row sums, 256-wide FP32 tree dots).     */
/* ------------------------------------------------------------------------- */
typedef struct wsb_spmv_executor wsb_spmv_executor;
/* SpmvExecutor::create(ctx, n_rows, row_ptr, col_idx, values), spmv_exec.rs:38-118. */
int wsb_spmv_executor_create(wsb_context *ctx, uint32_t n_rows, const uint32_t *row_ptr,
                             const uint32_t *col_idx, const float *values, uint64_t nnz,
                             wsb_spmv_executor **out);
/* encode_copy_x_from + encode_spmv, spmv_exec.rs:122-147: y = A x. */
int wsb_spmv_executor_spmv(wsb_spmv_executor *ex, const wsb_buffer *x, wsb_buffer *y);
void wsb_spmv_executor_destroy(wsb_spmv_executor *ex);

typedef struct wsb_dot_scalar_executor wsb_dot_scalar_executor;
/* DotScalarExecutor::create(ctx, n_max, scalar_results_len), dot_scalar_exec.rs:42-123. */
int wsb_dot_scalar_executor_create(wsb_context *ctx, uint64_t n_max, uint32_t scalar_results_len,
                                   wsb_dot_scalar_executor **out);
/* encode_dot_scalar_into, dot_scalar_exec.rs:151-247: scalar_results[out_index] = a.b */
int wsb_dot_scalar_executor_dot_into(wsb_dot_scalar_executor *ex, const wsb_buffer *a, const wsb_buffer *b,
                                     uint32_t n, uint32_t out_index);
/* scalar_results_buffer, dot_scalar_exec.rs:125-127 (owned by the executor). */
wsb_buffer *wsb_dot_scalar_executor_scalar_results(wsb_dot_scalar_executor *ex);
/* encode_copy_scalar_results_to_readback + readback_scalar_results, dot_scalar_exec.rs:251-270. */
int wsb_dot_scalar_executor_readback(wsb_dot_scalar_executor *ex, float *out, uint32_t len);
void wsb_dot_scalar_executor_destroy(wsb_dot_scalar_executor *ex);

/* VecOpsExecutor (vec_ops_exec.rs:23-239); stateless here, so context-level. */
/* encode_axpy_inplace, vec_ops_exec.rs:130-161: y = y + alpha*x */
int wsb_vec_axpy_inplace(wsb_context *ctx, const wsb_buffer *x, wsb_buffer *y, uint32_t n, float alpha);
/* encode_axpy_inplace_from_scalar_results, vec_ops_exec.rs:163-198: y = y + s[idx]*x */
int wsb_vec_axpy_inplace_from_scalar_results(wsb_context *ctx, const wsb_buffer *x, wsb_buffer *y, uint32_t n,
                                             const wsb_buffer *scalar_results, uint32_t scalar_index);
/* encode_scale_inplace_from_scalar_results, vec_ops_exec.rs:200-232: x = x*s[idx] */
int wsb_vec_scale_inplace_from_scalar_results(wsb_context *ctx, wsb_buffer *x, uint32_t n,
                                              const wsb_buffer *scalar_results, uint32_t scalar_index);

typedef struct wsb_block_jacobi_executor wsb_block_jacobi_executor;
/* BlockJacobiExecutor::create(ctx, n, lu_blocks, block_starts), block_jacobi_exec.rs:48-91. */
int wsb_block_jacobi_executor_create(wsb_context *ctx, uint32_t n, const float *lu_blocks, uint64_t lu_len,
                                     const uint32_t *block_starts, uint64_t block_starts_len,
                                     wsb_block_jacobi_executor **out);
/* encode_apply, block_jacobi_exec.rs:96-124: z = M^-1 r */
int wsb_block_jacobi_executor_apply(wsb_block_jacobi_executor *ex, const wsb_buffer *r, wsb_buffer *z);
void wsb_block_jacobi_executor_destroy(wsb_block_jacobi_executor *ex);

/* PcgUpdateScalarsExecutor::encode_update_scalars, pcg_update_scalars_exec.rs:72-118. */
int wsb_pcg_update_scalars(wsb_context *ctx, wsb_buffer *scalar_results, uint32_t p_ap_index,
                           uint32_t rz_new_index, uint32_t rz_old_index, uint32_t alpha_index,
                           uint32_t minus_alpha_index, uint32_t beta_index);

/* Allocation-free dot product. No counterpart in the reference: it is the
 * dot pass structure above (256-wide FP32 tree, result identical to
 * wsb_dot_scalar_executor_dot_into) for callers that cannot allocate device
 * memory where they need it (a spent memory budget, no tolerance for the
 * synchronisation cudaMalloc can cause). d_a, d_b: n floats and d_out: one
 * float, all device memory owned by the caller. Scratch between passes is a
 * static device array of this library (held by every GPU that loads it until
 * exit), which limits n to WSB_NOALLOC_DOT_MAX_N; larger n returns
 * WSB_ERR_BAD_INPUT. The first call on a device resolves that array's
 * address and keeps it for the life of the process; make it before any
 * stream capture. The kept address assumes the device's primary context is
 * never torn down (no cudaDeviceReset while the library is in use). Calls
 * that overlap on the GPU share the array and race. Enqueued on the
 * context's stream; not waited for. */
#define WSB_NOALLOC_DOT_MAX_N 16777216u
int wsb_dot_tree256_noalloc(wsb_context *ctx, const float *d_a, const float *d_b, uint32_t n, float *d_out);

/* ------------------------------------------------------------------------- */
/* Host-side block-Jacobi setup (no GPU needed)                              */
/* ------------------------------------------------------------------------- */
/* lu_factor_inplace_6(mat, n), compute.rs:37-71. mat: row-major 6x6 (>= 36 floats). */
int wsb_lu_factor_inplace_6(float *mat, uint64_t mat_len, uint32_t n);
/* build_lu_blocks_from_csr_block_starts_6, compute.rs:84-181.
 * out_lu receives (block_starts_len-1)*36 floats (0 floats when block_starts_len < 2). */
int wsb_build_lu_blocks_from_csr_block_starts_6(uint32_t n, const uint32_t *row_ptr, uint64_t row_ptr_len,
                                                const uint32_t *col_idx, uint64_t col_idx_len,
                                                const float *values, uint64_t values_len,
                                                const uint32_t *block_starts, uint64_t block_starts_len,
                                                float *out_lu);

/* ------------------------------------------------------------------------- */
/* Solver options and results                                                */
/* ------------------------------------------------------------------------- */
typedef enum wsb_precision {
    /* FP32 matrix and vectors, FP64 dot products and scalars (default). */
    WSB_PREC_F32_F64DOT = 0,
    /* The reference's arithmetic exactly: FP32 256-wide tree dots, FP32
     * scalars and stop test (compute.rs:189-495), scalars kept on the device. */
    WSB_PREC_REFERENCE_F32 = 1,
    /* FP64 outer iterative refinement around an inner F32_F64DOT PCG. */
    WSB_PREC_MIXED_F64_IR = 2
} wsb_precision;

typedef enum wsb_layout {
    WSB_LAYOUT_AUTO = 0,  /* BSR6 when every block is 6 rows and the 6x6 fill is complete, else CSR */
    WSB_LAYOUT_CSR = 1,
    WSB_LAYOUT_BSR6 = 2
} wsb_layout;

/* The PCG recurrence (wsb_solve_opts.algorithm). No counterpart in the
 * reference, which has the classic one only. */
typedef enum wsb_algorithm {
    /* The reference's recurrence (compute.rs:336-489): SpMV of p, then x, r and
     * z = M r, then p = z + beta p; three fused kernels per iteration. */
    WSB_ALG_CLASSIC = 0,
    /* The single-reduction recurrence of Chronopoulos and Gear (J. Comput.
     * Appl. Math. 25, 1989): w = A u with u = M r, s = A p kept by recurrence,
     * and the iteration's two dots, (r, u) and (A u, u), formed in the update
     * and SpMV epilogues; the direction update moves into the update kernel,
     * so an iteration is two fused kernels. Same stop test on the recursive
     * residual; iterates agree with the classic ones to rounding. FP64
     * reductions only (F32_F64DOT and MIXED_F64_IR); systems solved together
     * (a batch, a server) all use one recurrence. */
    WSB_ALG_SINGLE_REDUCTION = 1
} wsb_algorithm;

typedef struct wsb_solve_opts {
    uint32_t struct_size;        /* sizeof(wsb_solve_opts) */
    int32_t precision;           /* wsb_precision */
    double target_relres;        /* MIXED: stop when ||b-Ax||_2/||b||_2 (FP64) <= this; default 1e-10 */
    float inner_rel_tol;         /* MIXED: relative tolerance of each inner PCG; default 1e-4 */
    uint32_t max_refine;         /* MIXED: maximum outer sweeps; default 50 */
    uint64_t history_capacity;   /* entries available in history_out */
    double *history_out;         /* r.r after each PCG iteration (host memory), or NULL */
    int32_t always_write_x;      /* 0: x written only on success, as compute.rs:482-484 */
    int32_t algorithm;           /* wsb_algorithm; default WSB_ALG_CLASSIC */
    double *x64_out;             /* MIXED: receives the FP64 solution (n doubles, host), or NULL.
                                    For server requests it is filled by wsb_server_poll/wait. */
} wsb_solve_opts;

/* Fill *opts with the defaults above. */
void wsb_solve_opts_default(wsb_solve_opts *opts);

typedef struct wsb_solve_result {
    int32_t status;              /* wsb_status of the solve */
    int32_t breakdown_kind;      /* 1: dot(p,Ap)==0, 2: rz_old==0 */
    uint64_t iterations;         /* PCG iterations (all inner iterations for MIXED) */
    uint32_t refine_sweeps;      /* MIXED: outer sweeps */
    uint32_t reserved;
    double b_norm2;              /* ||b||^2 */
    double final_r_norm2;        /* last r.r of the (inner) recursion */
    double final_relres;         /* MIXED: FP64 true ||b-Ax||/||b||; else sqrt(final_r_norm2/b_norm2) */
    double device_ms;            /* device time of the solve (CUDA events), excludes host copies */
    double total_ms;             /* host wall time of the call */
    uint64_t history_len;        /* entries written to history_out */
    uint64_t kernel_launches;    /* kernels this library launched for the solve (0 for REFERENCE_F32) */
} wsb_solve_result;

/* ------------------------------------------------------------------------- */
/* The reference's driver (compute.rs:189-206):                              */
/*   pcg_block_jacobi_csr_wgpu(n, b, x, max_iter, rel_tol, abs_tol, ctx,     */
/*                             spmv, vec_ops, dot, block_jacobi, scalars)     */
/* The vector, dot and scalar executors have no separate role here: their    */
/* passes are fused into the solver's kernels. x: in x0, out solution,       */
/* written only on success unless opts->always_write_x. *iterations gets     */
/* Ok(iterations).                                                           */
/* ------------------------------------------------------------------------- */
int wsb_pcg_block_jacobi_csr(wsb_context *ctx, uint64_t n, const float *b, uint64_t b_len, float *x,
                             uint64_t x_len, uint64_t max_iter, float rel_tol, float abs_tol,
                             wsb_spmv_executor *spmv, wsb_block_jacobi_executor *block_jacobi,
                             const wsb_solve_opts *opts, uint64_t *iterations, wsb_solve_result *result);

/* ------------------------------------------------------------------------- */
/* Matrix handle: CSR (+ optional BSR6 copy), block_starts and LU resident   */
/* in HBM; it combines SpmvExecutor::create, build_lu_blocks_... and          */
/* BlockJacobiExecutor::create as run_pcg_case does (cli main.rs:490-538).   */
/* ------------------------------------------------------------------------- */
typedef struct wsb_matrix wsb_matrix;
typedef struct wsb_matrix_info {
    uint64_t n, nnz, num_blocks;
    int32_t layout;              /* layout in use: WSB_LAYOUT_CSR or WSB_LAYOUT_BSR6 */
    int32_t reserved;
    uint64_t device_bytes;       /* bytes held on the device */
    uint64_t spmv_bytes;         /* algorithmic bytes of one SpMV */
    uint64_t iteration_bytes;    /* algorithmic bytes of one PCG iteration */
} wsb_matrix_info;

int wsb_matrix_create(wsb_context *ctx, uint32_t n, const uint32_t *row_ptr, const uint32_t *col_idx,
                      const float *values, uint64_t nnz, const uint32_t *block_starts,
                      uint64_t block_starts_len, int32_t layout, wsb_matrix **out);
int wsb_matrix_info_get(const wsb_matrix *m, wsb_matrix_info *out);
void wsb_matrix_destroy(wsb_matrix *m);
/* Tile autotuner (no counterpart in the reference, whose kernels have one  */
/* fixed launch shape): times the solver's SpMV and update kernels on this  */
/* matrix for a few tile sizes (a short PCG run on b = ones), keeps the     */
/* fastest of each, and records the choice for matrices of the same shape   */
/* class (layout, n within a factor of 2, nonzeros per row) created later   */
/* in this process. Retuned tiles regroup the FP64 partial sums of the dot  */
/* products: results agree with the untuned ones to FP64 rounding.          */
typedef struct wsb_tune_result {
    uint32_t spmv_rows;          /* rows per SpMV tile (6 x block rows for BSR6) */
    uint32_t spmv_cap;           /* nonzeros (CSR) or 6x6 blocks (BSR6) per SpMV tile */
    uint32_t update_rows;        /* rows per update tile */
    uint32_t update_blocks;      /* block starts per update tile */
    double spmv_ms, update_ms;   /* mean kernel time with the chosen tiles */
    double default_spmv_ms, default_update_ms;  /* ... with the largest tiles */
    uint32_t candidates;         /* tilings timed */
    uint32_t reserved;
} wsb_tune_result;
int wsb_matrix_autotune(wsb_context *ctx, wsb_matrix *m, uint32_t iterations, wsb_tune_result *out);
/* Forgets the tilings the autotuner recorded per shape class. */
void wsb_autotune_clear(void);

/* Copies the block-Jacobi factors the handle holds (built on the device,   */
/* num_blocks * 36 floats, the layout and bits of the Vec<f32> that         */
/* build_lu_blocks_from_csr_block_starts_6 returns, compute.rs:84-181)      */
/* into out; out_len must be at least num_blocks * 36.                      */
int wsb_matrix_read_lu(wsb_context *ctx, const wsb_matrix *m, float *out, uint64_t out_len);

/* Solve A x = b with host arrays (copies inside the call). */
int wsb_solve(wsb_context *ctx, wsb_matrix *m, const float *b, float *x, uint64_t max_iter, float rel_tol,
              float abs_tol, const wsb_solve_opts *opts, wsb_solve_result *result);
/* Same with device pointers (d_b: n floats, d_x: n floats in/out). */
int wsb_solve_device(wsb_context *ctx, wsb_matrix *m, const float *d_b, float *d_x, uint64_t max_iter,
                     float rel_tol, float abs_tol, const wsb_solve_opts *opts, wsb_solve_result *result);
/* y = A x with the product SpMV kernel of the matrix's layout (device
 * pointers), as SpmvExecutor::encode_spmv does for its own buffers
 * (spmv_exec.rs:120-147). Enqueued on the context's stream, not waited for.
 * The kernel's descriptor and error word belong to the matrix; a kernel error
 * (a device wait that ran out) is reported by a later wsb_matrix_spmv_device
 * call on the matrix once its read-back has completed, or by
 * wsb_matrix_spmv_check. Calls on one matrix from several streams share the
 * descriptor and the error word. */
int wsb_matrix_spmv_device(wsb_context *ctx, wsb_matrix *m, const float *d_x, float *d_y);
/* Waits for the last wsb_matrix_spmv_device launch on m and returns the
 * status of the launches since the last reported error (WSB_OK, or
 * WSB_ERR_TIMEOUT / WSB_ERR_CUDA with wsb_last_error). No counterpart in the
 * reference, whose SpMV executor blocks on every submission. */
int wsb_matrix_spmv_check(wsb_context *ctx, wsb_matrix *m);

/* Measurement aid (no counterpart in the reference): runs `iterations` PCG
 * iterations of this matrix with right-hand side d_b (device) outside the
 * CUDA graph, CUDA events around each launch, and writes the mean duration
 * in ms of the SpMV+p.Ap kernel, the update+preconditioner kernel and the
 * p-update kernel to ms[0..2]; ms[3] and ms[4] receive the iteration count
 * and status code of the system afterwards (a valid measurement has
 * ms[3] == iterations and status 0, still running). ms holds 5 doubles. */
int wsb_matrix_kernel_times(wsb_context *ctx, wsb_matrix *m, const float *d_b, uint32_t iterations, double *ms);

/* ------------------------------------------------------------------------- */
/* Batched solve of many independent systems                                 */
/* ------------------------------------------------------------------------- */
typedef struct wsb_batch wsb_batch;
int wsb_batch_create(wsb_context *ctx, wsb_batch **out);
/* Adds one system; the matrix must outlive the batch. *id is its index. The
 * host buffers named in opts (history_out, x64_out) must stay valid until
 * wsb_batch_result for this id, which fills them. */
int wsb_batch_add(wsb_batch *bt, wsb_matrix *m, const float *b, const float *x0, uint64_t max_iter,
                  float rel_tol, float abs_tol, const wsb_solve_opts *opts, uint32_t *id);
/* Solves all added systems together; converged systems retire in place. */
int wsb_batch_solve(wsb_batch *bt);
int wsb_batch_result(wsb_batch *bt, uint32_t id, float *x, wsb_solve_result *result);
void wsb_batch_destroy(wsb_batch *bt);

/* ------------------------------------------------------------------------- */
/* Serving: continuous batching of solve requests                            */
/* ------------------------------------------------------------------------- */
typedef struct wsb_server wsb_server;
/* wsb_server_opts.flags */
#define WSB_SERVER_BORROW_INPUTS 1u /* submit does not copy: the caller's arrays (row_ptr, col_idx,
                                       values, block_starts, b, x0) are read in place and must stay
                                       valid and unchanged until poll/wait reports the request done */
#define WSB_SERVER_DEVICE_PREP 2u   /* the column check, BSR6 conversion and block LU of each request
                                       run on the GPU (as wsb_matrix_create does) instead of the
                                       uploader threads' host builders */
typedef struct wsb_server_opts {
    uint32_t struct_size;
    uint32_t max_active;          /* systems iterated together (0: no limit) */
    uint64_t memory_budget_bytes; /* device bytes for resident systems (0: 120 GB) */
    uint32_t iters_per_step;      /* PCG iterations between scheduler steps while requests are still
                                     arriving (0: 16); 4x that when none is on its way */
    uint32_t flags;               /* WSB_SERVER_* above */
} wsb_server_opts;
typedef struct wsb_server_stats {
    uint64_t submitted, completed, failed, rejected;
    uint64_t active, pending;
    uint64_t steps;
    uint64_t device_bytes_in_use, device_bytes_peak;
    double busy_ms;             /* scheduler: time inside engine steps (graph launch to state read-back) */
    uint64_t kernel_launches;   /* kernels the scheduler has launched so far */
    double host_prep_ms;        /* uploaders: host validation and LU (summed over threads) */
    double upload_ms;           /* uploaders: copies and device-side preparation (summed over threads) */
    double admit_ms;            /* scheduler: adding ready requests to the engine (b, x0 uploads) */
    double retire_ms;           /* scheduler: reading results back and releasing finished requests */
    double sched_idle_ms;       /* scheduler: waiting for work */
} wsb_server_stats;

int wsb_server_create(wsb_context *ctx, const wsb_server_opts *opts, wsb_server **out);
/* Queues one solve; all arrays are copied before the call returns. */
int wsb_server_submit(wsb_server *s, uint32_t n, const uint32_t *row_ptr, const uint32_t *col_idx,
                      const float *values, uint64_t nnz, const uint32_t *block_starts, uint64_t block_starts_len,
                      const float *b, const float *x0, uint64_t max_iter, float rel_tol, float abs_tol,
                      const wsb_solve_opts *opts, uint64_t *request_id);
/* WSB_PENDING while running; else the solve's status, with x (n floats, may be
 * NULL) and *result filled. A finished request is released after this call. */
int wsb_server_poll(wsb_server *s, uint64_t request_id, float *x, wsb_solve_result *result);
/* Blocks until the request finishes or timeout_s passes (WSB_ERR_TIMEOUT). */
int wsb_server_wait(wsb_server *s, uint64_t request_id, float *x, wsb_solve_result *result, double timeout_s);
int wsb_server_stats_get(wsb_server *s, wsb_server_stats *out);
void wsb_server_destroy(wsb_server *s);

/* ------------------------------------------------------------------------- */
/* Synthetic 3-D lattice systems (6 unknowns per node, 6x6 blocks)           */
/* ------------------------------------------------------------------------- */
typedef struct wsb_lattice_sizes {
    uint64_t nodes, edges, n, nnz, num_blocks, bsr_blocks;
} wsb_lattice_sizes;
int wsb_lattice_sizes_get(uint32_t side, wsb_lattice_sizes *out);
/* Fills CSR (sorted columns), block_starts (0,6,...,n) and b ~ U[-1,1].
 * Each edge stiffness is S = R R^T/6 + 0.1 I with R ~ N(0,1) 6x6, scaled by
 * 10^U(-aniso_log10, aniso_log10); 1e-3 I is added on the diagonal. */
int wsb_lattice_generate(uint32_t side, uint64_t seed, double aniso_log10, uint32_t *row_ptr, uint32_t *col_idx,
                         float *values, uint32_t *block_starts, float *b);

#ifdef __cplusplus
}
#endif
#endif /* WSB_H */
