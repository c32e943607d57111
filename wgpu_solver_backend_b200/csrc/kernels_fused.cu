// Fused, batch-native PCG kernels for B200 (sm_100a).
//
// Memory-bound design (no dense contraction on this path, so no tensor
// cores). Every CTA is persistent over a device work list of row tiles (grid
// = SMs x resident CTAs, grid-stride over the list), so one captured CUDA
// graph serves any number of systems. The matrix and vector slices of a tile
// are brought into shared memory with TMA bulk copies (cp.async.bulk +
// mbarrier transaction counts) into a ring of kSpmvStages (SpMV) or
// kUpdStages (update) stages: while a CTA computes tile k, the next tiles
// are already streaming in. The gathered vector is read through the read-only path and stays
// in the 126 MB L2. Per-system reductions are deterministic: every tile
// writes one FP64 partial and the last CTA of a system (ticket counter) sums
// them in a fixed order, so a system's arithmetic does not depend on what
// else shares the launch.
//
// Arithmetic parity with the reference: SpMV rows are summed sequentially in
// index order with separately rounded multiply and add (spmv.wgsl:58-61); the
// vector updates are y + a*x without contraction (axpy*.wgsl); the block
// solve is block_jacobi.wgsl:93-126 operation by operation; p = p*beta + z is
// scale_from_scalar_results.wgsl then axpy.wgsl.
//
// Every mbarrier wait is bounded (about 2 s of clock); a wait that runs out
// records an error code in StepParams::error, waits (bounded) for the CTA's
// own copies in flight and returns, and the host reports WSB_ERR_TIMEOUT.
#include "kernels_fused.cuh"

namespace wsb {

namespace {

// ---------------------------------------------------------------------------
// TMA bulk copies and mbarriers (inline PTX).
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_barrier_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// Orders this thread's generic-proxy shared-memory accesses before later
// async-proxy (TMA) writes to the same buffers.
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 1-D bulk store shared -> global (no multicast), tracked by this thread's
// bulk async-groups: dst and src 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_store(void *dst, const void *src, uint32_t bytes) {
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst), "r"(smem_u32(src)),
                 "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
// The shared-memory sources of this thread's bulk stores have been read.
__device__ __forceinline__ void bulk_wait_read() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
// This thread's bulk stores are complete (their global writes performed).
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

// 1-D bulk copy global -> shared; 16-byte aligned addresses, size % 16 == 0.
__device__ __forceinline__ void tma_load(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

// 1-D bulk copy with an L2 evict-first hint, for data streamed once per
// iteration (matrix values and indices, LU factors): it leaves the L2 to the
// Krylov vectors, which the next kernels read again.
__device__ __forceinline__ uint64_t l2_evict_first_policy() {
    uint64_t pol;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}

__device__ __forceinline__ void tma_load_stream(void *dst, const void *src, uint32_t bytes, uint64_t *bar,
                                                uint64_t pol) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar)), "l"(pol)
        : "memory");
}

// Two FP32 products in one packed instruction (mul.rn.f32x2, sm_100): each
// lane is rounded to nearest on its own, exactly as two __fmul_rn.
__device__ __forceinline__ float2 mul2_rn(float2 a, float2 b) {
    float2 r;
    asm("{\n\t.reg .b64 ra, rb, rc;\n\tmov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
        "mul.rn.f32x2 rc, ra, rb;\n\tmov.b64 {%0, %1}, rc;\n}"
        : "=f"(r.x), "=f"(r.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return r;
}

// Bulk prefetch of a global range into the L2 (no completion tracking). The
// range is widened to 16-byte boundaries; every array it is used on has tail
// padding, so the widened range stays inside its allocation.
__device__ __forceinline__ void l2_prefetch(const void *p, uint32_t bytes) {
    const uintptr_t a = reinterpret_cast<uintptr_t>(p) & ~uintptr_t(15);
    const uintptr_t e = (reinterpret_cast<uintptr_t>(p) + bytes + 15) & ~uintptr_t(15);
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(a), "r"((uint32_t)(e - a)) : "memory");
}

// Read-only 4-byte load of the index data the gather warps read every
// iteration (row pointers, BSR6 block columns). With WSB_GATHER_KEEP_L2 it
// carries an L2 evict-last hint: that data is small next to the block values
// and can stay in the L2 between iterations.
__device__ __forceinline__ uint32_t ldg_index(const uint32_t *p) {
#if WSB_GATHER_KEEP_L2
    uint64_t pol;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
    uint32_t v;
    asm volatile("ld.global.nc.L2::cache_hint.u32 %0, [%1], %2;" : "=r"(v) : "l"(p), "l"(pol));
    return v;
#else
    return __ldg(p);
#endif
}

// Asynchronous 4- and 8-byte copies global -> shared (cp.async): the
// gathered x values go straight into the stage without holding registers.
__device__ __forceinline__ void cp_async4(void *dst, const void *src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async8(void *dst, const void *src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}
// Arrive on an mbarrier once all of this thread's earlier cp.async copies
// have landed (the barrier's expected count covers the arrival).
__device__ __forceinline__ void cp_async_mbar_arrive(uint64_t *bar) {
    asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Non-blocking probe of a phase.
__device__ __forceinline__ bool mbar_test_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred P;\n\tmbarrier.test_wait.parity.shared::cta.b64 P, [%1], %2;\n\tselp.u32 %0, 1, 0, P;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred P;\n\tmbarrier.try_wait.parity.shared::cta.b64 P, [%1], %2;\n\tselp.u32 %0, 1, 0, P;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

constexpr long long kWaitCycles = 4000000000ll;  // about 2 s at 1.9 GHz

// The limit of the pipeline waits of one launch: StepParams::wait_cycles, or
// kWaitCycles when that is 0. The drains of a CTA's own copies in flight
// always use kWaitCycles (a CTA must not leave while a copy into its shared
// memory may still land).
__device__ __forceinline__ long long wait_limit(const StepParams *sp) {
    const unsigned long long w = sp->wait_cycles;
    return w == 0 ? kWaitCycles : (long long)(w > (unsigned long long)kWaitCycles ? kWaitCycles : w);
}

__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, long long lim = kWaitCycles) {
    if (mbar_try_wait(bar, parity)) return true;
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity))
        if (clock64() - t0 > lim) return false;
    return true;
}

// A phase that another thread of the CTA has already seen complete: a
// non-blocking check (which also makes the phase's data visible to this
// thread), with the bounded wait as a fallback.
__device__ __forceinline__ void mbar_observe(uint64_t *bar, uint32_t parity, long long lim) {
    if (!mbar_test_wait(bar, parity)) mbar_wait(bar, parity, lim);
}

// Programmatic dependent launch: the next kernel in the stream may start
// launching its CTAs now (they occupy SMs only as this kernel's CTAs leave);
// and this kernel waits until the previous one has completed and its memory
// is visible. Both are no-ops for a launch without the attribute.
__device__ __forceinline__ void pdl_start() {
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    asm volatile("griddepcontrol.wait;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// One arrival per warp (the barrier counts warps): the warp's lanes converge
// first, so all of their earlier shared-memory reads are done, then lane 0
// arrives. A per-thread arrival would put 32 atomic updates of one
// shared-memory word behind every warp.
__device__ __forceinline__ void mbar_arrive_warp(uint64_t *bar) {
    __syncwarp();
    if ((threadIdx.x & 31u) == 0) mbar_arrive(bar);
}

// The pipelined kernels run their consumer threads in the low warps
// (kSpmvConsumers in the SpMV, kUpdConsumers in the update kernels), then one
// producer warp (plus the gather warps in the SpMV). Consumers synchronise
// among themselves on named barrier 1 so the other warps never have to join. Kernels without a producer warp launch exactly kThreads
// threads and use barrier 1.

template <int N = kThreads>
__device__ __forceinline__ void csync() {
    asm volatile("bar.sync 1, %0;" ::"n"(N) : "memory");
}

// ---------------------------------------------------------------------------
// Reductions
// ---------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// Fixed-shape block reduction over the N consumer threads (result valid in
// thread 0). red: >= 32 doubles.
template <int N = kThreads>
__device__ __forceinline__ double block_sum(double v, double *red) {
    v = warp_sum(v);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) red[w] = v;
    csync<N>();
    double s = 0.0;
    if (w == 0) {
        s = lane < (N >> 5) ? red[lane] : 0.0;
        s = warp_sum(s);
    }
    csync<N>();
    return s;
}

template <int N = kThreads>
__device__ __forceinline__ double2 block_sum2(double a, double b, double *red) {
    a = warp_sum(a);
    b = warp_sum(b);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) {
        red[w] = a;
        red[32 + w] = b;
    }
    csync<N>();
    double sa = 0.0, sb = 0.0;
    if (w == 0) {
        sa = lane < (N >> 5) ? red[lane] : 0.0;
        sb = lane < (N >> 5) ? red[32 + lane] : 0.0;
        sa = warp_sum(sa);
        sb = warp_sum(sb);
    }
    csync<N>();
    return make_double2(sa, sb);
}

// Sum of n FP64 partials over the N consumer threads: thread t adds
// elements t, t + N, t + 2N, ... in that order (16 loads in flight), then the
// fixed-shape block sum. Result valid in thread 0.
template <int N = kThreads>
__device__ __forceinline__ double sum_partials(const double *__restrict__ p, uint32_t n, double *red) {
    double v = 0.0;
    uint32_t i = threadIdx.x;
    for (; i + 15u * N < n; i += 16u * N) {
        double q[16];
#pragma unroll
        for (int u = 0; u < 16; ++u) q[u] = __ldcg(p + i + u * N);
#pragma unroll
        for (int u = 0; u < 16; ++u) v += q[u];
    }
    for (; i < n; i += N) v += __ldcg(p + i);
    return block_sum<N>(v, red);
}

// Ticket on a per-system counter: this CTA adds the number of tiles whose
// partials it has published (thread `who` wrote them and takes the ticket);
// true in every thread of the CTA whose tickets complete the system's total.
template <int N = kThreads>
__device__ __forceinline__ bool take_ticket(uint32_t *counter, uint32_t cnt, uint32_t total, int *s_last,
                                            uint32_t who = 0) {
    if (threadIdx.x == who) {
        __threadfence();
        const uint32_t t = atomicAdd(counter, cnt);
        *s_last = (t + cnt == total);
    }
    csync<N>();
    const bool last = *s_last != 0;
    if (last) __threadfence();
    return last;
}

// ---------------------------------------------------------------------------
// SpMV tiles
// ---------------------------------------------------------------------------
enum SpmvMode { M_LOOP = 0, M_INIT = 1, M_PLAIN = 2 };

// The list positions a CTA takes, in order. A list of n items laid out in w
// columns (StepParams) is walked column by column: columns blockIdx.x,
// blockIdx.x + gridDim.x, ..., each from its first position (c) to its last
// (c + w (n/w - 1)). w == 0: plain grid-stride over n items.
constexpr uint32_t kNoPos = 0xffffffffu;
struct ListWalk {
    uint32_t n, w;
    __device__ __forceinline__ uint32_t pos(uint32_t k) const {
        if (w == 0) {
            const uint64_t p = blockIdx.x + (uint64_t)k * gridDim.x;
            return p < n ? (uint32_t)p : kNoPos;
        }
        const uint32_t len = n / w;
        if (len == 0) return kNoPos;
        const uint64_t c = blockIdx.x + (uint64_t)(k / len) * gridDim.x;
        return c < w ? (uint32_t)(c + (uint64_t)w * (k % len)) : kNoPos;
    }
};

// Stage layout (floats), from kernels_fused.cuh: CSR values [0, kCsrCap+8),
// the gathered x[col] of every staged value at kColOff (same index as the
// value); BSR6 block values [0, 36 kBsrCapBlocks), block columns
// at kBcolOff, gathered x at kXgOff (float2, 3 per block); row pointers at
// kRpOff.
constexpr int NC = kSpmvConsumers;  // consumer threads of the SpMV kernels
constexpr int kValCap = kCsrCap + 8;
constexpr int kColOff = kValCap;
constexpr int kBcolOff = kSpmvBcolOff;
constexpr int kXgOff = kSpmvXgOff;
constexpr int kRpOff = kSpmvRpOff;
static_assert((kColOff * 4) % 16 == 0 && (kBcolOff * 4) % 16 == 0 && (kXgOff * 4) % 16 == 0 &&
                  (kRpOff * 4) % 16 == 0 && (kSpmvStageFloats * 4) % 128 == 0,
              "TMA alignment");
static_assert(kSpmvStageFloats >= kRpOff + kSpmvTileRows + 8, "stage size");
// bsr_stage reads the operands of one block past a tile's last (unused).
static_assert(36 * (kBsrCapBlocks + 1) <= kXgOff && kXgOff + 6 * (kBsrCapBlocks + 1) <= kSpmvStageFloats,
              "one block past a tile's last stays inside the stage");

struct SpmvDesc {
    uint32_t valid, sys, tile, layout;
    uint32_t r0, nr;  // tile rows in layout units (rows, or block rows)
    uint32_t k0, k1;  // nonzero (block) range
    uint32_t ka;      // 4-aligned start of the staged CSR value / column range
    uint32_t lng;     // a single row longer than a stage: synchronous path
    const float *x;   // the vector multiplied: p (loop), x0 (init) or the caller's x
    float *y;         // Ap (loop, init) or the caller's y
    double *part;     // the system's per-group p.Ap partials (loop)
    uint32_t grp;     // the tile's reduction group
    uint32_t gflags;  // kGroupFirst / kGroupLast
    const uint32_t *rptr;  // the tile's row pointers: row_ptr + r0 or brow_ptr + r0
    const uint32_t *cols;  // BSR6: the tile's block columns, bcol + k0
    const float *vsrc;     // bulk-copy source of the values: bval + 36 k0, or val + ka
    const uint32_t *csrc;  // CSR: the staged range's columns, col + ka (read by the gather warp)
};

// The vector the SpMV multiplies: p (classic loop), u = z (single-reduction
// loop), x0 (init) or the caller's x (plain).
template <int kMode>
__device__ __forceinline__ const float *spmv_input(const SysDesc &S, const float *__restrict__ xplain) {
    return kMode == M_PLAIN ? xplain : kMode == M_INIT ? S.x : (S.algo == ALGO_SINGLE_REDUCTION ? S.z : S.p);
}

// Checks one work index of the SpMV work list (one producer lane): false
// for an index past the end, an invalid item (which also sets an error code)
// and, in the loop kernel, a system that is no longer active. *it is set to
// the (system, tile) the index stands for.
template <int kMode>
__device__ __forceinline__ bool check_spmv(const SysDesc *__restrict__ sys, const StepParams *sp, uint32_t idx,
                                           WorkItem *it) {
    if (idx == kNoPos) return false;
    if (kMode == M_PLAIN) {
        it->sys = 0;
        it->tile = idx;
        return true;
    }
    if (it->sys == kNoSys) return false;  // a position that carries no tile
    if (it->sys >= sp->num_sys || it->tile >= sys[it->sys].n_stiles) {
        atomicOr(const_cast<uint32_t *>(&sp->error), kErrBadItem);  // invalid work item: skipped
        return false;
    }
    return !(kMode == M_LOOP && !sys[it->sys].st->active);
}

// Fills the descriptor of a checked work item, field by field, in shared memory.
template <int kMode>
__device__ __forceinline__ void fill_spmv(const SysDesc *__restrict__ sys, WorkItem it, const float *xplain,
                                          float *yplain, SpmvDesc *d) {
    const SysDesc &S = sys[it.sys];
    const SpmvTile T = S.stiles[it.tile];
    const bool bsr = S.layout == LAYOUT_BSR6;
    const uint32_t ka = T.k0 & ~3u;
    d->valid = 1;
    d->sys = it.sys;
    d->tile = it.tile;
    d->layout = S.layout;
    d->r0 = T.row0;
    d->nr = T.row1 - T.row0;
    d->k0 = T.k0;
    d->k1 = T.k1;
    d->ka = ka;
    d->lng = bsr ? (T.k1 - T.k0 > (uint32_t)kBsrCapBlocks) : (T.k1 - T.k0 > (uint32_t)kCsrCap);
    d->x = spmv_input<kMode>(S, xplain);
    d->y = kMode == M_PLAIN ? yplain : S.ap;
    d->part = S.part_a;
    if (kMode == M_LOOP) {
        const uint32_t G = S.n_sgroups;
        d->grp = it.tile % G;
        d->gflags = (it.tile < G ? kGroupFirst : 0u) | (it.tile + G >= S.n_stiles ? kGroupLast : 0u);
    } else {
        d->grp = 0;
        d->gflags = 0;
    }
    d->rptr = (bsr ? S.brow_ptr : S.row_ptr) + T.row0;
    d->cols = bsr ? S.bcol + T.k0 : nullptr;
    d->vsrc = bsr ? S.bval + (size_t)T.k0 * 36u : S.val + ka;
    d->csrc = bsr ? nullptr : S.col + ka;
}

// Issues the bulk copies of a resolved tile into a stage (producer lane 0):
// the block values (BSR6) or the values and columns (CSR). Row pointers and
// block columns are read by the gather warps.
__device__ __forceinline__ void issue_spmv(const SpmvDesc &d, float *stage, uint64_t *bar, uint64_t pol) {
    if (d.lng) {
        mbar_expect_tx(bar, 0);
        return;
    }
    if (d.layout == LAYOUT_BSR6) {
        const uint32_t vb = (d.k1 - d.k0) * 144u;
        mbar_expect_tx(bar, vb);
        if (vb) tma_load_stream(stage, d.vsrc, vb, bar, pol);
    } else {
        const uint32_t cc = ((d.k1 - d.ka) + 3) & ~3u;
        mbar_expect_tx(bar, 4u * cc);
        if (cc) tma_load_stream(stage, d.vsrc, 4u * cc, bar, pol);
    }
}

// Gather warp, CSR tile: x[col[j]] for every staged index j of [ka, ka + cc)
// into xg[j - ka] by 4-byte cp.async. The columns are read here with
// streaming 16-byte loads (8 in flight per lane) and never staged; indices
// outside [k0, k1) belong to neighbouring tiles or the zero padding of the
// column array, so every gathered address is a valid row of x. Each lane
// keeps WSB_CSR_GATHER_BATCH column loads in flight per round.
__device__ __forceinline__ void gather_csr(const SpmvDesc &d, float *stage, uint32_t lane) {
    const float *__restrict__ xin = d.x;
    float *xg = stage + kColOff;
    const uint4 *__restrict__ c4 = reinterpret_cast<const uint4 *>(d.csrc);
    const uint32_t nq = (((d.k1 - d.ka) + 3) & ~3u) >> 2;  // 16-byte groups of columns
    constexpr uint32_t kBatch = WSB_CSR_GATHER_BATCH;
    for (uint32_t q0 = 0; q0 < nq; q0 += 32u * kBatch) {
        uint4 c[kBatch];
#pragma unroll
        for (uint32_t u = 0; u < kBatch; ++u) {
            const uint32_t q = q0 + lane + 32u * u;
            c[u] = q < nq ? __ldcs(c4 + q) : make_uint4(0u, 0u, 0u, 0u);
        }
#pragma unroll
        for (uint32_t u = 0; u < kBatch; ++u) {
            const uint32_t q = q0 + lane + 32u * u;
            if (q < nq) {
                float *dst = xg + 4u * q;
                cp_async4(dst + 0, xin + c[u].x);
                cp_async4(dst + 1, xin + c[u].y);
                cp_async4(dst + 2, xin + c[u].z);
                cp_async4(dst + 3, xin + c[u].w);
            }
        }
    }
}

// Gather warp, one tile (32 lanes): the tile's row pointers into the stage
// (rp[i] = row_ptr[r0 + i], i <= nr); for CSR the x value of every staged
// nonzero (gather_csr); for BSR6 its block columns (bcol[i] = block column of
// block k0 + i) and the 6 x values of every block column, as 3 float2 per
// block, by cp.async. None of this waits for the tile's bulk copy, so the
// gathers run while the values stream in.
__device__ __forceinline__ void gather_tile(const SpmvDesc &d, float *stage, uint32_t lane) {
    uint32_t *rp = reinterpret_cast<uint32_t *>(stage + kRpOff);
    for (uint32_t i = lane; i <= d.nr; i += 32u) rp[i] = ldg_index(d.rptr + i);
    if (d.layout != LAYOUT_BSR6) {
        gather_csr(d, stage, lane);
        return;
    }
    const float *__restrict__ xin = d.x;
    const bool al8 = (reinterpret_cast<uintptr_t>(xin) & 7u) == 0;
    float *xg = stage + kXgOff;
    const uint32_t nb = d.k1 - d.k0;
    // All block columns of this lane first (independent loads), then the
    // copies that depend on them.
    constexpr int kPer = (kBsrCapBlocks + 31) / 32;
    uint32_t c[kPer];
#pragma unroll
    for (int q = 0; q < kPer; ++q) {
        const uint32_t blk = lane + 32u * q;
        c[q] = blk < nb ? ldg_index(d.cols + blk) : 0u;
    }
#pragma unroll
    for (int q = 0; q < kPer; ++q) {
        const uint32_t blk = lane + 32u * q;
        if (blk < nb) {
            const float *src = xin + 6u * (size_t)c[q];
            float *dst = xg + 6u * blk;
            if (al8) {
                cp_async8(dst, src);
                cp_async8(dst + 2, src + 2);
                cp_async8(dst + 4, src + 4);
            } else {  // a caller's x that is only 4-byte aligned (plain SpMV entry point)
#pragma unroll
                for (int h = 0; h < 6; ++h) cp_async4(dst + h, src + h);
            }
        }
    }
}

// CSR tile from a filled and gathered stage: one thread per row adds
// val[j] * x[col[j]] over its nonzeros in index order, each product rounded
// before the add (spmv.wgsl:58-61); both factors come from the stage.
__device__ __forceinline__ float csr_stage(const SpmvDesc &d, const float *stage) {
    const float *val = stage;
    const float *xg = stage + kColOff;
    const uint32_t *rp = reinterpret_cast<const uint32_t *>(stage + kRpOff);
    float acc = 0.0f;
    if (threadIdx.x < d.nr) {
        const uint32_t o = threadIdx.x;
        const uint32_t s = rp[o] - d.ka, e = rp[o + 1] - d.ka;
        uint32_t q = s;
        // Operands two products ahead, so shared-memory latency overlaps the add chain.
        for (; q + 4u <= e; q += 4u) {
            const float2 p01 = mul2_rn(make_float2(val[q], val[q + 1]), make_float2(xg[q], xg[q + 1]));
            const float2 p23 = mul2_rn(make_float2(val[q + 2], val[q + 3]), make_float2(xg[q + 2], xg[q + 3]));
            acc = __fadd_rn(acc, p01.x);
            acc = __fadd_rn(acc, p01.y);
            acc = __fadd_rn(acc, p23.x);
            acc = __fadd_rn(acc, p23.y);
        }
        for (; q < e; ++q) acc = __fadd_rn(acc, __fmul_rn(val[q], xg[q]));
    }
    return acc;
}

// BSR6 tile from a filled and gathered stage: thread t owns row (t/6, t%6) of
// the tile and walks its block row's blocks in column order, six products
// each from shared memory, added in index order (for complete 6x6 blocks
// with sorted columns this is the CSR order). (The row's own p value for
// p.Ap is loaded by the caller: testing every block for the diagonal one
// cost the 80^3 SpMV 6 % of its time.)
__device__ __forceinline__ float bsr_stage(const SpmvDesc &d, const float *stage) {
    const uint32_t *rp = reinterpret_cast<const uint32_t *>(stage + kRpOff);
    const float2 *xg = reinterpret_cast<const float2 *>(stage + kXgOff);
    float acc = 0.0f;
    const uint32_t t = threadIdx.x;
    if (t < 6u * d.nr) {
        const uint32_t br = t / 6u, a = t - 6u * br;
        const uint32_t s0 = rp[br] - d.k0, s1 = rp[br + 1] - d.k0;
        // The next block's operands are loaded before this block's products
        // are added, so shared-memory latency overlaps the add chain.
        float2 b0, b1, b2, x0, x1, x2;
        if (s0 < s1) {
            const float2 *B = reinterpret_cast<const float2 *>(stage + s0 * 36u + a * 6u);
            const float2 *X = xg + s0 * 3u;
            b0 = B[0], b1 = B[1], b2 = B[2], x0 = X[0], x1 = X[1], x2 = X[2];
        }
#pragma unroll 2
        for (uint32_t blk = s0; blk < s1; ++blk) {
            // Block blk + 1 <= the tile's block count stays inside the stage
            // (the block-column and row-pointer areas follow the values and
            // the gathered x), so it is loaded without a test; past the block
            // row's end the values are never used.
            const float2 *B = reinterpret_cast<const float2 *>(stage + (blk + 1) * 36u + a * 6u);
            const float2 *X = xg + (blk + 1) * 3u;
            const float2 nb0 = B[0], nb1 = B[1], nb2 = B[2], nx0 = X[0], nx1 = X[1], nx2 = X[2];
            // The six products (packed two at a time), then the adds in
            // index order.
            const float2 q0 = mul2_rn(b0, x0), q1 = mul2_rn(b1, x1), q2 = mul2_rn(b2, x2);
            acc = __fadd_rn(acc, q0.x);
            acc = __fadd_rn(acc, q0.y);
            acc = __fadd_rn(acc, q1.x);
            acc = __fadd_rn(acc, q1.y);
            acc = __fadd_rn(acc, q2.x);
            acc = __fadd_rn(acc, q2.y);
            b0 = nb0, b1 = nb1, b2 = nb2, x0 = nx0, x1 = nx1, x2 = nx2;
        }
    }
    return acc;
}

// A tile whose single row (or block row) exceeds a stage: staged in chunks
// with plain loads, using the stage as scratch (no copy is in flight into it).
__device__ __forceinline__ float long_tile(const SysDesc &S, const SpmvDesc &d, const float *__restrict__ xin, float *stage) {
    const uint32_t t = threadIdx.x;
    float acc = 0.0f;
    if (d.layout == LAYOUT_BSR6) {
        // One block row of 6 rows, blocks [k0, k1) in chunks of kBsrCapBlocks.
        uint32_t *bcol = reinterpret_cast<uint32_t *>(stage + kBcolOff);
        for (uint32_t c0 = d.k0; c0 < d.k1; c0 += kBsrCapBlocks) {
            const uint32_t nb = min(d.k1 - c0, (uint32_t)kBsrCapBlocks);
            const float4 *src = reinterpret_cast<const float4 *>(S.bval) + (size_t)c0 * 9u;
            float4 *dst = reinterpret_cast<float4 *>(stage);
            for (uint32_t q = t; q < nb * 9u; q += NC) dst[q] = __ldcs(src + q);
            for (uint32_t q = t; q < nb; q += NC) bcol[q] = __ldcs(S.bcol + c0 + q);
            csync<NC>();
            if (t < 6u) {
                for (uint32_t blk = 0; blk < nb; ++blk) {
                    const float *B = stage + blk * 36u + t * 6u;
                    const float *xx = xin + 6u * (size_t)bcol[blk];
#pragma unroll
                    for (int jj = 0; jj < 6; ++jj) acc = __fadd_rn(acc, __fmul_rn(B[jj], __ldg(xx + jj)));
                }
            }
            csync<NC>();
        }
        return acc;
    }
    // One CSR row, nonzeros [k0, k1) in chunks of 2 kCsrCap products.
    constexpr uint32_t kChunk = 2 * kCsrCap;
    for (uint32_t c0 = d.k0; c0 < d.k1; c0 += kChunk) {
        const uint32_t c1 = min(d.k1, c0 + kChunk);
        for (uint32_t q = c0 + t; q < c1; q += NC)
            stage[q - c0] = __fmul_rn(__ldcs(S.val + q), __ldg(xin + __ldcs(S.col + q)));
        csync<NC>();
        if (t == 0)
            for (uint32_t q = c0; q < c1; ++q) acc = __fadd_rn(acc, stage[q - c0]);
        csync<NC>();
    }
    return acc;
}

// The consumer thread that publishes the per-tile p.Ap partials and takes the
// system tickets: lane 0 of the last consumer warp, which has no rows in
// most BSR6 tiles and so is free while the others compute.
constexpr uint32_t kPublisher = NC - 32;

// The last CTA of a system's SpMV tiles. Classic: p.Ap from the per-tile
// partials in tile order, alpha = rz_old / pAp (0 when pAp == 0, as
// pcg_update_scalars.wgsl:59-62). Single reduction (the SpMV multiplied u, so
// the partials sum to delta = (A u, u)), with gamma = (r, u) from the update
// kernel: beta = gamma / gamma_prev and alpha = gamma / (delta - beta gamma /
// alpha_prev), or beta = 0 and alpha = gamma / delta in the first iteration;
// the denominator is kept in pap for the update kernel's breakdown check.
__device__ __forceinline__ void flush_spmv(const SysDesc *__restrict__ sys, uint32_t s, uint32_t cnt, double *red,
                                           int *s_last) {
    if (cnt == 0) return;
    const SysDesc &S = sys[s];
    SysState *st = S.st;
    if (!take_ticket<NC>(&st->cnt_a, cnt, S.n_stiles, s_last, kPublisher)) return;
    const double pap = sum_partials<NC>(S.part_a, S.n_sgroups, red);
    if (threadIdx.x == 0) {
        if (S.algo == ALGO_SINGLE_REDUCTION) {
            const double gamma = st->rz_old;
            double beta = 0.0, den = pap;
            if (st->iter > 0) {
                beta = st->gamma_prev != 0.0 ? gamma / st->gamma_prev : 0.0;
                den = st->alpha != 0.0 ? pap - beta * gamma / st->alpha : 0.0;
            }
            const double alpha = den != 0.0 ? gamma / den : 0.0;
            st->pap = den;
            st->alpha = alpha;
            st->alpha_f = (float)alpha;
            st->beta = beta;
            st->beta_f = (float)beta;
        } else {
            const double alpha = pap != 0.0 ? st->rz_old / pap : 0.0;
            st->pap = pap;
            st->alpha = alpha;
            st->alpha_f = (float)alpha;
        }
        st->cnt_a = 0;
    }
}



// The index data a gather warp will read for tile d (its row pointers, and
// its block columns or, for CSR, its columns), prefetched into the L2 by the
// producer a few tiles ahead, so that the gather warp's first, dependent
// round trip is served from the L2 rather than from DRAM.
__device__ __forceinline__ void prefetch_gather(const SpmvDesc &d) {
    if (d.lng) return;
    l2_prefetch(d.rptr, 4u * (d.nr + 1));
    if (d.layout == LAYOUT_BSR6) l2_prefetch(d.cols, 4u * (d.k1 - d.k0));
    else l2_prefetch(d.csrc, 4u * ((d.k1 - d.ka + 3) & ~3u));
}

// Producer warp of the SpMV ring. The warp resolves 32 work items at once
// (one lane each: work item -> system -> tile), so the chain of dependent
// loads behind a tile is paid once per 32 tiles, and keeps the work items of
// the next batch in flight meanwhile. Lane 0 then walks the batch in order:
// it claims stage k % NS once the consumers released tile k - NS, publishes
// the tile's descriptor (meta barrier) and issues its bulk copies. After the
// last tile it publishes one end marker per gather warp. Every wait is bounded; on a timeout lane 0 records
// an error, waits (bounded) for its copies still in flight and returns.
template <int kMode>
__device__ __forceinline__ void spmv_producer(const SysDesc *__restrict__ sys, StepParams *sp,
                                              const float *xplain, float *yplain, float *smem, uint64_t *full,
                                              uint64_t *meta, uint64_t *empty, SpmvDesc *desc, SpmvDesc *bdesc,
                                              long long lim) {
    constexpr uint32_t NS = kSpmvStages;
    const uint32_t lane = threadIdx.x & 31u;
    const ListWalk walk = kMode == M_PLAIN  ? ListWalk{sys[0].n_stiles, 0u}
                          : kMode == M_INIT ? ListWalk{sp->n_init_a, sp->w_init_a}
                                            : ListWalk{sp->n_work_a, sp->w_work_a};
    const WorkItem *__restrict__ work = kMode == M_INIT ? sp->init_a : sp->work_a;
    uint32_t base = 0;  // walk index of lane 0's item in the current batch
    uint32_t ipos = walk.pos(lane);
    WorkItem it = {0u, 0u};
    if (kMode != M_PLAIN && ipos != kNoPos) it = work[ipos];
    uint32_t k = 0, issued = 0;
    bool err = false;
    const uint64_t pol = l2_evict_first_policy();
    for (;;) {
        const bool ok = check_spmv<kMode>(sys, sp, ipos, &it);
        const uint32_t m = __ballot_sync(0xffffffffu, ok);
        if (ok) fill_spmv<kMode>(sys, it, xplain, yplain, &bdesc[__popc(m & ((1u << lane) - 1u))]);
        const uint32_t cnt = __popc(m);
        base += 32u;
        const bool more = walk.pos(base) != kNoPos;
        ipos = walk.pos(base + lane);
        if (kMode != M_PLAIN && ipos != kNoPos) it = work[ipos];  // next batch, in flight
        __syncwarp();
        if (lane == 0) {
            // After the last tile: one end marker for each gather warp.
            const uint32_t n_out = more ? cnt : cnt + kGatherWarps;
            for (uint32_t i = 0; i < n_out; ++i) {
                const uint32_t s = k % NS;
                if (k >= NS && !mbar_wait(&empty[s], ((k / NS) - 1) & 1u, lim)) {
                    atomicOr(&sp->error, kErrSpmvProducerWait);
                    err = true;
                    break;
                }
                if (i < cnt) {
                    desc[s] = bdesc[i];
                    mbar_arrive(&meta[s]);  // the gather warps may start on this tile
                    issue_spmv(desc[s], smem + s * kSpmvStageFloats, &full[s], pol);
                    issued = k + 1;
                    if (kSpmvPrefetchAhead > 0 && i + kSpmvPrefetchAhead < cnt)
                        prefetch_gather(bdesc[i + kSpmvPrefetchAhead]);
                } else {  // end marker
                    desc[s].valid = 0;
                    mbar_arrive(&meta[s]);
                    mbar_expect_tx(&full[s], 0);
                }
                ++k;
            }
        }
        err = __shfl_sync(0xffffffffu, err ? 1u : 0u, 0) != 0;
        __syncwarp();  // lane 0 is done with bdesc before the next batch overwrites it
        if (err || !more) break;
    }
    if (err && lane == 0) {
        // Bounded drain of the copies that may still be in flight.
        for (uint32_t j = issued > NS ? issued - NS : 0; j < issued; ++j) mbar_wait(&full[j % NS], (j / NS) & 1u);
    }
}

// Gather warps of the SpMV ring (warp g takes tiles g, g + kGatherWarps, ...): as soon
// as the producer publishes a tile's descriptor, the warp reads its row
// pointers and block columns and issues the x gathers (cp.async), in
// parallel with the tile's bulk copy. The stage's gather barrier completes
// when the warp's stores are done (a release arrival per lane) and its
// cp.async copies have landed (an asynchronous arrival per lane).
template <int kMode>
__device__ __forceinline__ void spmv_gatherer(const SysDesc *__restrict__ sys, StepParams *sp,
                                              const float *__restrict__ xplain, float *smem, uint64_t *meta,
                                              uint64_t *gath, const SpmvDesc *desc, uint32_t g, long long lim) {
    constexpr uint32_t NS = kSpmvStages;
    const uint32_t lane = threadIdx.x & 31u;
    for (uint32_t j = g;; j += kGatherWarps) {
        const uint32_t s = j % NS, par = (j / NS) & 1u;
        uint32_t ok = 1;
        if (lane == 0) ok = mbar_wait(&meta[s], par, lim) ? 1u : 0u;
        ok = __shfl_sync(0xffffffffu, ok, 0);
        if (!ok) {
            if (lane == 0) atomicOr(&sp->error, kErrGatherWait);
            break;
        }
        mbar_observe(&meta[s], par, lim);  // completed: the descriptor is visible
        const SpmvDesc d = desc[s];
        if (d.valid && !d.lng) gather_tile(d, smem + s * kSpmvStageFloats, lane);
        mbar_arrive(&gath[s]);
        cp_async_mbar_arrive(&gath[s]);
        if (!d.valid) break;
    }
    cp_async_wait<0>();
}

// The SpMV pipeline shared by the loop, init and plain kernels: NC
// consumer threads compute tile after tile from the ring that the producer
// warp fills and the gather warps complete. Per tile the consumers pass one
// barrier (the stage wait, which also separates the previous tile's warp
// partials from their publication by thread 0).
template <int kMode>
__device__ __forceinline__ void spmv_pipeline(const SysDesc *__restrict__ sys, StepParams *sp,
                                              const float *__restrict__ xplain, float *__restrict__ yplain,
                                              float *smem) {
    constexpr uint32_t NS = kSpmvStages;
    __shared__ __align__(8) uint64_t full[NS], meta[NS], gath[NS], empty[NS];
    __shared__ SpmvDesc desc[NS];
    __shared__ SpmvDesc bdesc[32];
    __shared__ double red[64];
    __shared__ double wred[2 * (NC / 32)];
    __shared__ int s_last, s_ok[2];
    const uint32_t tid = threadIdx.x;
    if (tid == 0) {
        for (uint32_t i = 0; i < NS; ++i) {
            mbar_init(&full[i], 1);
            mbar_init(&meta[i], 1);
            mbar_init(&gath[i], 64);
            mbar_init(&empty[i], NC / 32);
        }
        fence_barrier_init();
    }
    __syncthreads();
    pdl_start();
    const long long lim = wait_limit(sp);
    if (tid >= NC) {
        if (tid < NC + 32) spmv_producer<kMode>(sys, sp, xplain, yplain, smem, full, meta, empty, desc, bdesc, lim);
        else spmv_gatherer<kMode>(sys, sp, xplain, smem, meta, gath, desc, (tid - NC - 32) >> 5, lim);
        return;
    }
    uint32_t run_sys = 0xffffffffu, run_cnt = 0;  // tiles of run_sys published since the last ticket
    // Publisher: the group partial array of the group the previous tile
    // closed (null: nothing pending) and the group. Every thread: its rows'
    // p.Ap products summed over the current group's tiles (which come one
    // after another in this CTA's walk), so that the FP64 warp and CTA sums
    // run once per group, not once per tile.
    double *pend_part = nullptr, gpart = 0.0;
    uint32_t pend_grp = 0;
    for (uint32_t k = 0;; ++k) {
        const uint32_t s = k % NS, par = (k / NS) & 1u;
        // Thread 0 waits (bounded) and shares the outcome through a flag that
        // alternates with k, so a later write never meets an earlier read.
        if (tid == 0) s_ok[k & 1u] = (mbar_wait(&gath[s], par, lim) && mbar_wait(&full[s], par, lim)) ? 1 : 0;
        csync<NC>();
        if (!s_ok[k & 1u]) {
            if (tid == 0) atomicOr(&sp->error, kErrSpmvConsumerWait);
            return;
        }
        mbar_observe(&gath[s], par, lim);
        mbar_observe(&full[s], par, lim);
        // The descriptor is read in place: it stays valid until this stage
        // is handed back; what is needed after that is copied first.
        const SpmvDesc &d = desc[s];
        // The group that the previous tile closed: its warps' sums in warp
        // order.
        if (kMode == M_LOOP && tid == kPublisher && pend_part) {
            const double *wr = wred + (NC / 32) * ((k - 1) & 1u);
            double v = 0.0;
#pragma unroll
            for (int q = 0; q < NC / 32; ++q) v += wr[q];
            pend_part[pend_grp] = v;
            pend_part = nullptr;
        }
        if (!d.valid) break;
        float *stage = smem + s * kSpmvStageFloats;
        if (kMode == M_LOOP && d.sys != run_sys) {
            flush_spmv(sys, run_sys, run_cnt, red, &s_last);
            run_sys = d.sys;
            run_cnt = 0;
        }
        const uint32_t row0 = d.layout == LAYOUT_BSR6 ? 6u * d.r0 : d.r0;
        const uint32_t nrows = d.layout == LAYOUT_BSR6 ? 6u * d.nr : d.nr;
        const bool bsr_gathered = !d.lng && d.layout == LAYOUT_BSR6;
        // The row's own p value for p.Ap, read before the row's sum (an L2
        // hit: the gather has just read it).
        float acc, p_own = 0.0f;
        if (kMode == M_LOOP && tid < nrows) p_own = __ldg(d.x + row0 + tid);
        if (bsr_gathered) {
            acc = bsr_stage(d, stage);
        } else {
            if (d.lng) {
                acc = long_tile(sys[d.sys], d, d.x, stage);
                // That path wrote into the stage: order those writes before
                // the bulk copy that will next fill it.
                fence_proxy_async();
            } else {
                acc = csr_stage(d, stage);
            }
        }
        float *const yv = d.y;
        double *const part_arr = d.part;
        const uint32_t tgrp = d.grp, tflags = d.gflags;
        // Done reading the stage: hand it back to the producer.
        mbar_arrive_warp(&empty[s]);
        if (kMode == M_PLAIN) {
            if (tid < nrows) yv[row0 + tid] = acc;
        } else {
            double part = 0.0;
            if (tid < nrows) {
                const uint32_t i = row0 + tid;
                yv[i] = acc;
                if (kMode == M_LOOP) part = (double)p_own * (double)acc;
            }
            if (kMode == M_LOOP) {
                gpart = (tflags & kGroupFirst) ? part : gpart + part;
                if (tflags & kGroupLast) {
                    const double w = warp_sum(gpart);
                    if ((tid & 31u) == 0) wred[(NC / 32) * (k & 1u) + (tid >> 5)] = w;
                    pend_part = part_arr;
                    pend_grp = tgrp;
                }
                ++run_cnt;
            }
        }
    }
    if (kMode == M_LOOP && run_sys != 0xffffffffu) flush_spmv(sys, run_sys, run_cnt, red, &s_last);
}

// ---------------------------------------------------------------------------
// Update tiles (x, r, z and the block-Jacobi solve)
// ---------------------------------------------------------------------------
// Three kernels share this pipeline (kK):
//   K_INIT  k_init       r = b + (-1)(A x0); z = M r; p = z; FP64 b.b, r.z
//   K_LOOP  k_update     x += alpha p; r += (-alpha) Ap; z = M r; FP64 r.r, r.z
//   K_SR    k_update_sr  single reduction: p = u + beta p; s = w + beta s;
//                        x += alpha p; r += (-alpha) s; u = M r; FP64 r.r, r.u
//                        (u lives in z, w = A u in ap)
// Stage slots (kVecCap floats each): 0 = x (init: b), 1 = p, 2 = r, 3 = Ap
// (w), and for K_SR 4 = z (u), 5 = s; then the tile's LU blocks and block
// starts.
enum UpdKind { K_INIT = 0, K_LOOP = 1, K_SR = 2 };
constexpr int NU = kUpdConsumers;  // consumer threads of the update kernels
constexpr uint32_t kBulkIssuer = 32;  // the consumer thread that issues a tile's bulk stores
constexpr int kVecCap = kUpdTileRows + 8;  // floats per staged vector slice
template <int kK>
struct UpdLayout {
    static constexpr int kSlots = kK == K_SR ? 6 : 4;
    static constexpr int kLuOff = kSlots * kVecCap;          // LU blocks
    static constexpr int kBsOff = kLuOff + kUpdBlocks * 36;  // block starts slice
    static constexpr int kStageFloats = kK == K_SR ? kUpdStageFloatsSr : kUpdStageFloats;
    static_assert((kLuOff * 4) % 16 == 0 && (kBsOff * 4) % 16 == 0 && (kVecCap * 4) % 16 == 0, "TMA alignment");
    static_assert(kStageFloats >= kBsOff + kUpdBlocks + 8 && (kStageFloats * 4) % 128 == 0, "stage size");
};

struct UpdDesc {
    uint32_t valid, sys, tile;
    uint32_t row0, rows, blk0, nblk;
    uint32_t ra, ba;  // 4-aligned starts of the staged row / block-start ranges
    float alpha;      // the system's alpha (loop kernels), read by the producer
    float beta;       // single reduction: the system's beta
    uint32_t first;   // single reduction: the system's first iteration (p = u, s = w)
    float *x, *r, *z, *p, *s;
    double2 *part;    // the system's per-group (r.r, r.z) partials
    uint32_t grp;     // the tile's reduction group
    uint32_t gflags;  // kGroupFirst / kGroupLast
    const float *v[6];  // bulk-copy sources of the staged vector slots (from ra)
    const float *lu;    // bulk-copy source of the tile's LU blocks
    const uint32_t *bs; // bulk-copy source of the tile's block starts (from ba)
};

// Checks one work index of the update work list (one producer lane); false
// past the end, for an invalid item (error code set) and, in the loop kernels,
// for a system that is no longer active.
template <int kK>
__device__ __forceinline__ bool check_upd(const SysDesc *__restrict__ sys, const StepParams *sp, uint32_t idx,
                                          WorkItem it) {
    if (idx == kNoPos || it.sys == kNoSys) return false;
    if (it.sys >= sp->num_sys || it.tile >= sys[it.sys].n_utiles) {
        atomicOr(const_cast<uint32_t *>(&sp->error), kErrBadItem);  // invalid work item: skipped
        return false;
    }
    return kK == K_INIT || sys[it.sys].st->active;
}

// Fills the descriptor of a checked work item, field by field, in shared memory.
template <int kK>
__device__ __forceinline__ void fill_upd(const SysDesc *__restrict__ sys, WorkItem it, UpdDesc *d) {
    const SysDesc &S = sys[it.sys];
    const UpdTile T = S.utiles[it.tile];
    const uint32_t ra = T.row0 & ~3u, ba = T.blk0 & ~3u;
    d->valid = 1;
    d->sys = it.sys;
    d->tile = it.tile;
    d->row0 = T.row0;
    d->rows = T.row1 - T.row0;
    d->blk0 = T.blk0;
    d->nblk = T.blk1 - T.blk0;
    d->ra = ra;
    d->ba = ba;
    d->alpha = kK == K_INIT ? 0.0f : S.st->alpha_f;
    d->beta = kK == K_SR ? S.st->beta_f : 0.0f;
    d->first = kK == K_SR ? (S.st->iter == 0) : 0u;
    d->x = S.x;
    d->r = S.r;
    d->z = S.z;
    d->p = S.p;
    d->s = S.s;
    d->part = S.part_b;
    {
        const uint32_t G = S.n_ugroups;
        d->grp = it.tile % G;
        d->gflags = (it.tile < G ? kGroupFirst : 0u) | (it.tile + G >= S.n_utiles ? kGroupLast : 0u);
    }
    d->v[0] = (kK == K_INIT ? S.b : S.x) + ra;
    d->v[1] = S.p + ra;
    d->v[2] = S.r + ra;
    d->v[3] = S.ap + ra;
    d->v[4] = kK == K_SR ? S.z + ra : nullptr;
    d->v[5] = kK == K_SR ? S.s + ra : nullptr;
    d->lu = S.lu + (size_t)T.blk0 * 36u;
    d->bs = S.bstart + ba;
}

template <int kK>
__device__ __forceinline__ void issue_upd(const UpdDesc &d, float *stage, uint64_t *bar, uint64_t pol) {
    using Lay = UpdLayout<kK>;
    const uint32_t vc = ((d.row0 + d.rows - d.ra) + 3) & ~3u;
    const uint32_t bc = ((d.blk0 + d.nblk + 1 - d.ba) + 3) & ~3u;
    const uint32_t lub = d.nblk * 144u;
    const uint32_t nvec = kK == K_INIT ? 2u : kK == K_SR ? 6u : 4u;
    mbar_expect_tx(bar, nvec * 4u * vc + lub + 4u * bc);
    tma_load(stage, d.v[0], 4u * vc, bar);
    if (kK != K_INIT) {
        tma_load(stage + kVecCap, d.v[1], 4u * vc, bar);
        tma_load(stage + 2 * kVecCap, d.v[2], 4u * vc, bar);
    }
    tma_load(stage + 3 * kVecCap, d.v[3], 4u * vc, bar);
    if (kK == K_SR) {
        tma_load(stage + 4 * kVecCap, d.v[4], 4u * vc, bar);
        tma_load(stage + 5 * kVecCap, d.v[5], 4u * vc, bar);
    }
    if (lub) tma_load_stream(stage + Lay::kLuOff, d.lu, lub, bar, pol);
    tma_load_stream(stage + Lay::kBsOff, d.bs, 4u * bc, bar, pol);
}

// The row update of staged row o before the block solve: the new residual
// (returned), and in the stage the row's new x (slot 0) and, for K_SR, its
// new p (slot 1) and s (slot 5); the new r is written by the caller.
//   K_INIT r = b + (-1)(A x0)          (the reference's r = b, r += -1 * Ax)
//   K_LOOP r = r + (-alpha) Ap, x = x + alpha p                (axpy*.wgsl)
//   K_SR   p = p*beta + u, s = s*beta + w (p = u, s = w in the first
//          iteration), x = x + alpha p, r = r + (-alpha) s
// Each thread touches only its own rows, after reading them.
template <int kK>
__device__ __forceinline__ float row_update(const UpdDesc &d, float *stage, uint32_t o) {
    if (kK == K_INIT) return __fsub_rn(stage[o], stage[3 * kVecCap + o]);
    const float a = d.alpha, ma = -a;
    if (kK == K_LOOP) {
        const float ri = __fadd_rn(stage[2 * kVecCap + o], __fmul_rn(ma, stage[3 * kVecCap + o]));
        stage[o] = __fadd_rn(stage[o], __fmul_rn(a, stage[kVecCap + o]));
        return ri;
    }
    const float u = stage[4 * kVecCap + o], w = stage[3 * kVecCap + o];
    const float pi = d.first ? u : __fadd_rn(__fmul_rn(stage[kVecCap + o], d.beta), u);
    const float si = d.first ? w : __fadd_rn(__fmul_rn(stage[5 * kVecCap + o], d.beta), w);
    stage[kVecCap + o] = pi;
    stage[5 * kVecCap + o] = si;
    stage[o] = __fadd_rn(stage[o], __fmul_rn(a, pi));
    return __fadd_rn(stage[2 * kVecCap + o], __fmul_rn(ma, si));
}

// Stage slot that receives the new z (u): slot 1 for the classic kernels (p
// is not needed after the row update; the copy-out writes it to z, and to p
// in k_init), slot 4 for K_SR.
template <int kK>
constexpr int z_slot() {
    return kK == K_SR ? 4 : 1;
}

// Block solve of one thread: block blk0 + j of the tile, rows [off, off + m)
// of the stage (m = min(6, block length)). The thread forms its rows' row
// update (row_update) itself, runs z = U^-1 L^-1 r in registers with the
// reference's operation order (block_jacobi.wgsl: unit-L forward solve lines
// 93-101, U backward solve dividing by U(i,i) lines 103-122, rows i < m only,
// lines 79 and 124-126), and writes its rows' new r and z back into the
// stage. FP64 r.r (init: b.b) and r.z of the rows go to da and rz.
template <int kK, bool kFull>
__device__ __forceinline__ void bj_block(const UpdDesc &d, float *stage, uint32_t j, double &da, double &rz) {
    using Lay = UpdLayout<kK>;
    const uint32_t *bs = reinterpret_cast<const uint32_t *>(stage + Lay::kBsOff);
    const uint32_t off = bs[d.blk0 + j - d.ba], nxt = bs[d.blk0 + j + 1 - d.ba];
    const uint32_t m = kFull ? 6u : min(nxt - off, 6u);  // kFull: a block of 6 or more rows
    const uint32_t ro = off - d.ra;
    const float2 *L2 = reinterpret_cast<const float2 *>(stage + Lay::kLuOff + j * 36u);
    float L[36];
#pragma unroll
    for (int q = 0; q < 18; ++q) {
        const float2 v = L2[q];
        L[2 * q] = v.x;
        L[2 * q + 1] = v.y;
    }
    float rv[6], y[6], xs[6];
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        if ((uint32_t)i < m) {
            if (kK == K_INIT) {
                const float bi = stage[ro + i];
                da += (double)bi * (double)bi;
            }
            rv[i] = row_update<kK>(d, stage, ro + i);
            if (kK != K_INIT) da += (double)rv[i] * (double)rv[i];
        } else {
            rv[i] = 0.0f;
        }
        y[i] = 0.0f;
        xs[i] = 0.0f;
    }
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        if ((uint32_t)i < m) {
            float t = rv[i];
#pragma unroll
            for (int q = 0; q < i; ++q) t = __fsub_rn(t, __fmul_rn(L[i * 6 + q], y[q]));
            y[i] = t;
        }
    }
#pragma unroll
    for (int i = 5; i >= 0; --i) {
        if ((uint32_t)i < m) {
            float t = y[i];
#pragma unroll
            for (int q = i + 1; q < 6; ++q)
                if ((uint32_t)q < m) t = __fsub_rn(t, __fmul_rn(L[i * 6 + q], xs[q]));
            xs[i] = __fdiv_rn(t, L[i * 6 + i]);
        }
    }
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        if ((uint32_t)i < m) {
            const uint32_t o = ro + i;
            stage[2 * kVecCap + o] = rv[i];
            stage[z_slot<kK>() * kVecCap + o] = xs[i];
            rz += (double)rv[i] * (double)xs[i];
        }
    }
}

// A row the block solve leaves alone (position >= 6 in its block): the row
// update applies, z (u) keeps its value and enters r.z as it is.
template <int kK>
__device__ __forceinline__ void passive_row(const UpdDesc &d, float *stage, uint32_t row, double &da, double &rz) {
    const uint32_t o = row - d.ra;
    if (kK == K_INIT) {
        const float bi = stage[o];
        da += (double)bi * (double)bi;
    }
    const float ri = row_update<kK>(d, stage, o);
    if (kK != K_INIT) da += (double)ri * (double)ri;
    const float zi = kK == K_SR ? stage[4 * kVecCap + o] : d.z[row];
    stage[2 * kVecCap + o] = ri;
    stage[z_slot<kK>() * kVecCap + o] = zi;
    rz += (double)ri * (double)zi;
}

// Barrier, reductions and ticket of the update consumers: GT threads (local
// index lt) on named barrier BAR.
template <int GT, int BAR>
__device__ __forceinline__ void gsync() {
    asm volatile("bar.sync %0, %1;" ::"n"(BAR), "n"(GT) : "memory");
}

template <int GT, int BAR>
__device__ __forceinline__ double2 group_sum2(double a, double b, double *red, uint32_t lt) {
    a = warp_sum(a);
    b = warp_sum(b);
    const uint32_t lane = lt & 31u, w = lt >> 5;
    if (lane == 0) {
        red[w] = a;
        red[32 + w] = b;
    }
    gsync<GT, BAR>();
    double sa = 0.0, sb = 0.0;
    if (w == 0) {
        sa = lane < (uint32_t)(GT >> 5) ? red[lane] : 0.0;
        sb = lane < (uint32_t)(GT >> 5) ? red[32 + lane] : 0.0;
        sa = warp_sum(sa);
        sb = warp_sum(sb);
    }
    gsync<GT, BAR>();
    return make_double2(sa, sb);
}

// Sum of n pairs of FP64 partials over the group: thread lt adds elements
// lt, lt + GT, ... in that order (16 loads in flight: the last CTA's sum is
// bound by the bytes it keeps in flight), then the group sum.
template <int GT, int BAR>
__device__ __forceinline__ double2 group_sum_partials2(const double2 *__restrict__ p, uint32_t n, double *red,
                                                       uint32_t lt) {
    double va = 0.0, vb = 0.0;
    uint32_t i = lt;
    for (; i + 15u * GT < n; i += 16u * GT) {
        double2 q[16];
#pragma unroll
        for (int u = 0; u < 16; ++u) q[u] = __ldcg(p + i + u * GT);
#pragma unroll
        for (int u = 0; u < 16; ++u) {
            va += q[u].x;
            vb += q[u].y;
        }
    }
    for (; i < n; i += GT) {
        const double2 q = __ldcg(p + i);
        va += q.x;
        vb += q.y;
    }
    return group_sum2<GT, BAR>(va, vb, red, lt);
}

template <int GT, int BAR>
__device__ __forceinline__ bool group_ticket(uint32_t *counter, uint32_t cnt, uint32_t total, int *s_last,
                                             uint32_t lt) {
    if (lt == 0) {
        __threadfence();
        const uint32_t t = atomicAdd(counter, cnt);
        *s_last = (t + cnt == total);
    }
    gsync<GT, BAR>();
    const bool last = *s_last != 0;
    if (last) __threadfence();
    return last;
}

// The last CTA of a system's update tiles: the FP64 sums of the per-tile
// partials in tile order, then the host-side logic of compute.rs:466-488 on
// the device. K_LOOP: breakdown checks (pAp == 0, then rz_old == 0), stop
// test r.r <= abs^2 or r.r <= rel^2 b.b, iteration limit, beta = rz_new /
// rz_old, residual history entry. K_SR: the same checks and stop test (pap
// holds the SpMV epilogue's alpha denominator); the scalars of the next
// iteration come from the next SpMV epilogue. K_INIT: b.b and rz_old; b.b ==
// 0 finishes the system with 0 iterations and x untouched
// (compute.rs:252-254), max_iter == 0 finishes it as not converged.
template <int kK, int GT, int BAR>
__device__ __forceinline__ void flush_upd(const SysDesc *__restrict__ sys, StepParams *sp, uint32_t s, uint32_t cnt,
                                          double *red, int *s_last, uint32_t lt) {
    if (cnt == 0) return;
    const SysDesc &S = sys[s];
    SysState *st = S.st;
    if (!group_ticket<GT, BAR>(&st->cnt_b, cnt, S.n_utiles, s_last, lt)) return;
    const double2 sum = group_sum_partials2<GT, BAR>(S.part_b, S.n_ugroups, red, lt);
    if (lt != 0) return;
    if (kK == K_INIT) {
        st->bb = sum.x;
        st->rz_old = sum.y;
        uint32_t status = ST_RUNNING;
        if (sum.x == 0.0) status = ST_CONVERGED;
        else if (st->max_iter == 0) status = ST_MAXITER;
        if (status != ST_RUNNING) {
            st->status = status;
            st->active = 0;
            atomicSub(&sp->num_active, 1u);
        }
    } else {
        const double rr_t = sum.x, rz_new = sum.y;
        const uint32_t it = st->iter;
        const double pap = st->pap, rz_old = st->rz_old;
        if (S.history && it < S.hist_cap) S.history[it] = rr_t;
        st->rr = rr_t;
        st->rz_new = rz_new;
        st->iter = it + 1;
        uint32_t status = ST_RUNNING;
        if (pap == 0.0) {
            status = ST_BREAKDOWN;
            st->breakdown = 1;
        } else if (rz_old == 0.0) {
            status = ST_BREAKDOWN;
            st->breakdown = 2;
        } else if (rr_t <= st->abs2 || rr_t <= st->rel2 * st->bb) {
            status = ST_CONVERGED;
        } else if (it + 1 >= st->max_iter) {
            status = ST_MAXITER;
        }
        if (kK == K_LOOP) {
            const double beta = rz_old != 0.0 ? rz_new / rz_old : 0.0;
            st->beta = beta;
            st->beta_f = (float)beta;
        }
        if (status != ST_RUNNING) {
            st->status = status;
            st->active = 0;
            atomicSub(&sp->num_active, 1u);
        } else {
            if (kK == K_SR) st->gamma_prev = rz_old;
            st->rz_old = rz_new;
        }
    }
    st->cnt_b = 0;
}

// Producer warp of the update ring: the same batched resolution and ring
// discipline as the SpMV producer.
template <int kK>
__device__ __forceinline__ void upd_producer(const SysDesc *__restrict__ sys, StepParams *sp, float *smem,
                                             uint64_t *full, uint64_t *empty, UpdDesc *desc, UpdDesc *bdesc,
                                             long long lim) {
    constexpr uint32_t NS = kUpdStages;
    const uint32_t lane = threadIdx.x & 31u;
    const ListWalk walk = kK == K_INIT ? ListWalk{sp->n_init_b, sp->w_init_b} : ListWalk{sp->n_work_b, sp->w_work_b};
    const WorkItem *__restrict__ work = kK == K_INIT ? sp->init_b : sp->work_b;
    uint32_t base = 0;  // walk index of lane 0's item in the current batch
    uint32_t ipos = walk.pos(lane);
    WorkItem it = {0u, 0u};
    if (ipos != kNoPos) it = work[ipos];
    uint32_t k = 0, issued = 0;
    bool err = false;
    const uint64_t pol = l2_evict_first_policy();
    for (;;) {
        const bool ok = check_upd<kK>(sys, sp, ipos, it);
        const uint32_t m = __ballot_sync(0xffffffffu, ok);
        if (ok) fill_upd<kK>(sys, it, &bdesc[__popc(m & ((1u << lane) - 1u))]);
        const uint32_t cnt = __popc(m);
        base += 32u;
        const bool more = walk.pos(base) != kNoPos;
        ipos = walk.pos(base + lane);
        if (ipos != kNoPos) it = work[ipos];  // next batch, in flight
        __syncwarp();
        if (lane == 0) {
            // After the last tile: one end marker for the consumers.
            const uint32_t n_out = more ? cnt : cnt + 1;
            for (uint32_t i = 0; i < n_out; ++i) {
                const uint32_t s = k % NS;
                if (k >= NS && !mbar_wait(&empty[s], ((k / NS) - 1) & 1u, lim)) {
                    atomicOr(&sp->error, kErrUpdProducerWait);
                    err = true;
                    break;
                }
                if (i < cnt) {
                    desc[s] = bdesc[i];
                    issue_upd<kK>(desc[s], smem + s * UpdLayout<kK>::kStageFloats, &full[s], pol);
                    issued = k + 1;
                } else {  // end marker
                    desc[s].valid = 0;
                    mbar_expect_tx(&full[s], 0);
                }
                ++k;
            }
        }
        err = __shfl_sync(0xffffffffu, err ? 1u : 0u, 0) != 0;
        __syncwarp();
        if (err || !more) break;
    }
    if (err && lane == 0) {
        for (uint32_t j = issued > NS ? issued - NS : 0; j < issued; ++j) mbar_wait(&full[j % NS], (j / NS) & 1u);
    }
}

// Consumers of the update kernels (see UpdKind). Per-system results are
// formed by flush_upd. A tile holds at most NU blocks: consumer j solves
// block j of the tile (bj_block; its rows >= 6, if any, are passive rows)
// and the rows in front of the tile's first block start (continuation rows
// of a long block) are shared out. The new vectors go back into the stage,
// and after one barrier all consumers copy the tile's rows out with
// consecutive threads on consecutive rows. Per tile the consumers pass two
// barriers: the stage wait (which also keeps the next tile's warp partials
// out of wred until thread 0 has published this tile's) and the one before
// the copy-out.
template <int kK>
__device__ __forceinline__ void upd_consumers(const SysDesc *__restrict__ sys, StepParams *sp, float *smem,
                                              uint64_t *full, uint64_t *empty, const UpdDesc *desc, double *red,
                                              double2 *wred, int *s_last, int *s_ok, long long lim) {
    using Lay = UpdLayout<kK>;
    constexpr uint32_t NS = kUpdStages;
    constexpr int BAR = 1;
    const uint32_t lt = threadIdx.x;
    uint32_t run_sys = 0xffffffffu, run_cnt = 0;  // tiles of run_sys published since the last ticket
    double da = 0.0, rz = 0.0;  // this thread's sums over the current group
    for (uint32_t k = 0;; ++k) {
        const uint32_t s = k % NS, par = (k / NS) & 1u;
        if (lt == 0) s_ok[k & 1u] = mbar_wait(&full[s], par, lim) ? 1 : 0;
        gsync<NU, BAR>();
        if (!s_ok[k & 1u]) {
            if (lt == 0) atomicOr(&sp->error, kK == K_INIT ? kErrInitConsumerWait : kErrUpdConsumerWait);
            if (lt == kBulkIssuer) bulk_wait_all();
            return;
        }
        mbar_observe(&full[s], par, lim);
        const UpdDesc &d = desc[s];
        if (!d.valid) break;
        if (d.sys != run_sys) {
            flush_upd<kK, NU, BAR>(sys, sp, run_sys, run_cnt, red, s_last, lt);
            run_sys = d.sys;
            run_cnt = 0;
        }
        float *stage = smem + s * Lay::kStageFloats;
        // Loops: r.r and r.z (r.u); init: b.b and r.z; each thread's rows
        // summed over the current group's tiles (consecutive in this CTA's
        // walk), so that the FP64 warp and CTA sums run once per group.
        if (d.gflags & kGroupFirst) da = rz = 0.0;
        const uint32_t *bs = reinterpret_cast<const uint32_t *>(stage + Lay::kBsOff);
        const uint32_t row1 = d.row0 + d.rows;
        // Continuation rows of a long block that started in an earlier tile.
        const uint32_t lead_end = d.nblk ? bs[d.blk0 - d.ba] : row1;
        for (uint32_t row = d.row0 + lt; row < lead_end; row += NU) passive_row<kK>(d, stage, row, da, rz);
        if (lt < d.nblk) {
            const uint32_t off = bs[d.blk0 + lt - d.ba], nxt = bs[d.blk0 + lt + 1 - d.ba];
            // Blocks of 6 or more rows (all of them in a 6-DOF lattice) take a
            // copy of the solve without the row-count tests (80^3 k_update
            // 34.9 -> 32.8 us).
            if (nxt - off >= 6u) bj_block<kK, true>(d, stage, lt, da, rz);
            else bj_block<kK, false>(d, stage, lt, da, rz);
            // The block's rows >= 6 inside this tile.
            const uint32_t end = min(nxt, row1);
            for (uint32_t row = off + 6u; row < end; ++row) passive_row<kK>(d, stage, row, da, rz);
        }
        const bool closes = (d.gflags & kGroupLast) != 0;
        if (closes) {
            const double wa = warp_sum(da), wb = warp_sum(rz);
            if ((lt & 31u) == 0) wred[lt >> 5] = make_double2(wa, wb);
        }
        // The consumers wrote their rows into the stage: make those writes
        // visible to the bulk stores below and order them before the bulk
        // loads that will next fill the stage.
        fence_proxy_async();
        gsync<NU, BAR>();
        // Copy-out of the tile's rows: x (loops), r, z (u), and p (init: p =
        // z; single reduction: the new p) and s (single reduction). The
        // 16-byte aligned middle of each slice goes out by bulk stores that
        // one thread issues (thread kBulkIssuer, not in warp 0, which
        // publishes the partials meanwhile); the up to 3 rows before and
        // after it by plain stores. (128 threads storing every row took 0.8
        // us of a 2.6 us tile.)
        {
            const uint32_t r0 = d.row0, r1 = d.row0 + d.rows;
            const uint32_t a0 = min((r0 + 3u) & ~3u, r1), a1 = max(r1 & ~3u, a0);
            if (lt == kBulkIssuer && a1 > a0) {
                const uint32_t so = a0 - d.ra, nbytes = 4u * (a1 - a0);
                if (kK != K_INIT) bulk_store(d.x + a0, stage + so, nbytes);
                bulk_store(d.r + a0, stage + 2 * kVecCap + so, nbytes);
                bulk_store(d.z + a0, stage + z_slot<kK>() * kVecCap + so, nbytes);
                if (kK == K_INIT) bulk_store(d.p + a0, stage + z_slot<kK>() * kVecCap + so, nbytes);
                if (kK == K_SR) {
                    bulk_store(d.p + a0, stage + kVecCap + so, nbytes);
                    bulk_store(d.s + a0, stage + 5 * kVecCap + so, nbytes);
                }
                bulk_commit();
            }
            const uint32_t nh = a0 - r0, nt = r1 - a1;
            float *const xv = d.x, *const rv = d.r, *const zv = d.z, *const pv = d.p, *const sv = d.s;
            if (lt < nh + nt) {
                const uint32_t i = lt < nh ? r0 + lt : a1 + (lt - nh), o = i - d.ra;
                if (kK != K_INIT) xv[i] = stage[o];
                rv[i] = stage[2 * kVecCap + o];
                const float zi = stage[z_slot<kK>() * kVecCap + o];
                zv[i] = zi;
                if (kK == K_INIT) pv[i] = zi;
                if (kK == K_SR) {
                    pv[i] = stage[kVecCap + o];
                    sv[i] = stage[5 * kVecCap + o];
                }
            }
        }
        if (lt == 0 && closes) {
            double va = 0.0, vb = 0.0;
#pragma unroll
            for (int q = 0; q < NU / 32; ++q) {
                va += wred[q].x;
                vb += wred[q].y;
            }
            d.part[d.grp] = make_double2(va, vb);
        }
        // The bulk stores have read the stage: hand it back.
        if (lt == kBulkIssuer) bulk_wait_read();
        mbar_arrive_warp(&empty[s]);
        ++run_cnt;
    }
    // This CTA's bulk stores are complete before it leaves.
    if (lt == kBulkIssuer) bulk_wait_all();
    if (run_sys != 0xffffffffu) flush_upd<kK, NU, BAR>(sys, sp, run_sys, run_cnt, red, s_last, lt);
}

template <int kK>
__device__ __forceinline__ void upd_pipeline(const SysDesc *__restrict__ sys, StepParams *sp, float *smem,
                                             cudaGraphConditionalHandle h = 0) {
    constexpr uint32_t NS = kUpdStages;
    __shared__ __align__(8) uint64_t full[NS], empty[NS];
    __shared__ UpdDesc desc[NS];
    __shared__ UpdDesc bdesc[32];
    __shared__ double red[64];
    __shared__ double2 wred[NU / 32];
    __shared__ int s_last, s_ok[2];
    const uint32_t tid = threadIdx.x;
    if (tid == 0) {
        for (uint32_t i = 0; i < NS; ++i) {
            mbar_init(&full[i], 1);
            mbar_init(&empty[i], NU / 32);  // one arrival per consumer warp
        }
        fence_barrier_init();
    }
    __syncthreads();
    pdl_start();
    const long long lim = wait_limit(sp);
    if (tid >= NU) {
        if (tid < NU + 32) upd_producer<kK>(sys, sp, smem, full, empty, desc, bdesc, lim);
        return;
    }
    upd_consumers<kK>(sys, sp, smem, full, empty, desc, red, wred, &s_last, s_ok, lim);
    if (kK == K_SR) {
        // The end of the loop body (there is no p-update kernel in this
        // recurrence): the last CTA to finish counts the pass and ends the
        // graph's while loop when no system is active, the step's iteration
        // budget is used, or a kernel reported an error.
        if (tid == 0) {
            __threadfence();
            if (atomicAdd(&sp->tail_ticket, 1u) + 1u == gridDim.x) {
                __threadfence();
                sp->tail_ticket = 0;
                const uint32_t c = sp->loop_count + 1;
                sp->loop_count = c;
                if (h != 0 && (sp->num_active == 0 || c >= sp->loop_limit || sp->error != 0))
                    cudaGraphSetConditional(h, 0);
            }
        }
    }
}

}  // namespace

__global__ void __launch_bounds__(kSpmvThreads, kSpmvMinCtas) k_spmv_loop(const SysDesc *__restrict__ sys, StepParams *sp) {
    extern __shared__ __align__(128) float smem[];
    spmv_pipeline<M_LOOP>(sys, sp, nullptr, nullptr, smem);
}

__global__ void __launch_bounds__(kSpmvThreads, kSpmvMinCtas) k_spmv_init(const SysDesc *__restrict__ sys, StepParams *sp) {
    extern __shared__ __align__(128) float smem[];
    spmv_pipeline<M_INIT>(sys, sp, nullptr, nullptr, smem);
}

__global__ void __launch_bounds__(kSpmvThreads, kSpmvMinCtas) k_spmv_plain(const SysDesc *__restrict__ sys, StepParams *sp,
                                                         const float *__restrict__ x, float *__restrict__ y) {
    extern __shared__ __align__(128) float smem[];
    spmv_pipeline<M_PLAIN>(sys, sp, x, y, smem);
}

__global__ void __launch_bounds__(kUpdThreads, kUpdMinCtas) k_update(const SysDesc *__restrict__ sys, StepParams *sp) {
    extern __shared__ __align__(128) float smem[];
    upd_pipeline<K_LOOP>(sys, sp, smem);
}

__global__ void __launch_bounds__(kUpdThreads, kUpdMinCtas) k_update_sr(const SysDesc *__restrict__ sys, StepParams *sp,
                                                                         cudaGraphConditionalHandle h) {
    extern __shared__ __align__(128) float smem[];
    upd_pipeline<K_SR>(sys, sp, smem, h);
}

__global__ void __launch_bounds__(kUpdThreads, kUpdMinCtas) k_init(const SysDesc *__restrict__ sys, StepParams *sp) {
    extern __shared__ __align__(128) float smem[];
    upd_pipeline<K_INIT>(sys, sp, smem);
}

// ---------------------------------------------------------------------------
// k_pupdate: p = p*beta + z over kChunkRows row chunks with float4 accesses
// (scale_from_scalar_results.wgsl then axpy.wgsl with alpha 1). CTA 0 then
// ends the graph's while loop when no system is active, the step's iteration
// budget is used, or a kernel reported an error.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads) k_pupdate(const SysDesc *__restrict__ sys, StepParams *sp,
                                                      cudaGraphConditionalHandle h) {
    pdl_start();
    const uint32_t nw = sp->n_work_c;
    const WorkItem *__restrict__ work = sp->work_c;
    for (uint32_t w = blockIdx.x; w < nw; w += gridDim.x) {
        const WorkItem it = work[w];
        if (it.sys >= sp->num_sys || it.tile * (uint32_t)kChunkRows >= sys[it.sys].n) {
            if (threadIdx.x == 0) atomicOr(&sp->error, kErrBadItem);
            continue;
        }
        const SysDesc &S = sys[it.sys];
        const SysState *st = S.st;
        if (!st->active || S.algo != ALGO_CLASSIC) continue;
        const float bf = st->beta_f;
        const uint32_t r0 = it.tile * (uint32_t)kChunkRows;
        const uint32_t r1 = min(S.n, r0 + (uint32_t)kChunkRows);
        float *__restrict__ p = S.p;
        const float *__restrict__ z = S.z;
        uint32_t q = r0 + 4u * threadIdx.x;
        for (; q + 4u * kThreads + 3u < r1; q += 8u * kThreads) {
            float4 p0 = *reinterpret_cast<const float4 *>(p + q);
            float4 p1 = *reinterpret_cast<const float4 *>(p + q + 4u * kThreads);
            const float4 z0 = *reinterpret_cast<const float4 *>(z + q);
            const float4 z1 = *reinterpret_cast<const float4 *>(z + q + 4u * kThreads);
            p0.x = __fadd_rn(__fmul_rn(p0.x, bf), z0.x);
            p0.y = __fadd_rn(__fmul_rn(p0.y, bf), z0.y);
            p0.z = __fadd_rn(__fmul_rn(p0.z, bf), z0.z);
            p0.w = __fadd_rn(__fmul_rn(p0.w, bf), z0.w);
            p1.x = __fadd_rn(__fmul_rn(p1.x, bf), z1.x);
            p1.y = __fadd_rn(__fmul_rn(p1.y, bf), z1.y);
            p1.z = __fadd_rn(__fmul_rn(p1.z, bf), z1.z);
            p1.w = __fadd_rn(__fmul_rn(p1.w, bf), z1.w);
            *reinterpret_cast<float4 *>(p + q) = p0;
            *reinterpret_cast<float4 *>(p + q + 4u * kThreads) = p1;
        }
        for (; q < r1; q += 4u * kThreads) {
            if (q + 3u < r1) {
                float4 p0 = *reinterpret_cast<const float4 *>(p + q);
                const float4 z0 = *reinterpret_cast<const float4 *>(z + q);
                p0.x = __fadd_rn(__fmul_rn(p0.x, bf), z0.x);
                p0.y = __fadd_rn(__fmul_rn(p0.y, bf), z0.y);
                p0.z = __fadd_rn(__fmul_rn(p0.z, bf), z0.z);
                p0.w = __fadd_rn(__fmul_rn(p0.w, bf), z0.w);
                *reinterpret_cast<float4 *>(p + q) = p0;
            } else {
                for (uint32_t i = q; i < r1; ++i) p[i] = __fadd_rn(__fmul_rn(p[i], bf), z[i]);
            }
        }
    }
    if (h != 0 && blockIdx.x == 0 && threadIdx.x == 0) {
        const uint32_t c = sp->loop_count + 1;
        sp->loop_count = c;
        if (sp->num_active == 0 || c >= sp->loop_limit || sp->error != 0) cudaGraphSetConditional(h, 0);
    }
}

// Parent-graph node in front of the while loop: resets the step's iteration
// count and skips the loop when nothing is active.
__global__ void k_loop_gate(StepParams *sp, cudaGraphConditionalHandle h) {
    pdl_start();
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        sp->loop_count = 0;
        cudaGraphSetConditional(h, (sp->num_active > 0 && sp->loop_limit > 0 && sp->error == 0) ? 1u : 0u);
    }
}

// ---------------------------------------------------------------------------
// Mixed precision (FP64 outer iterative refinement).
// k_resid64: r64 = b - A x64 with FP32 matrix entries and FP64 accumulation;
// the inner right-hand side becomes (float) r64; FP64 ||r64||^2 and ||b||^2.
// One work item is one update tile (kUpdTileRows rows at most). BSR6: one thread per row,
// which walks its block row four blocks at a time with every load of the four
// issued before the first multiply (block columns, then 3 float2 of the row's
// block values and 3 double2 of x64 per block). CSR: eight lanes per row,
// striding over the row's nonzeros (32-byte coalesced runs of values and
// columns), then a fixed shuffle tree. FP64 sums need no particular order
// here (the result only has to be an accurate FP64 residual), but the order
// is fixed, so a system's residual does not depend on what else runs.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double resid_row_bsr6(const SysDesc &S, uint32_t i) {
    const uint32_t br = i / 6u, a = i - 6u * br;
    const uint32_t k0 = __ldg(S.brow_ptr + br), k1 = __ldg(S.brow_ptr + br + 1);
    const double2 *__restrict__ x2 = reinterpret_cast<const double2 *>(S.x64);
    double s = 0.0;
    for (uint32_t k = k0; k < k1; k += 4u) {
        uint32_t c[4];
        float2 v[4][3];
#pragma unroll
        for (uint32_t u = 0; u < 4; ++u) c[u] = k + u < k1 ? __ldg(S.bcol + k + u) : 0u;
#pragma unroll
        for (uint32_t u = 0; u < 4; ++u) {
            if (k + u < k1) {
                const float2 *B = reinterpret_cast<const float2 *>(S.bval + (size_t)(k + u) * 36u + a * 6u);
                v[u][0] = __ldcs(B);
                v[u][1] = __ldcs(B + 1);
                v[u][2] = __ldcs(B + 2);
            }
        }
#pragma unroll
        for (uint32_t u = 0; u < 4; ++u) {
            if (k + u < k1) {
                const double2 *X = x2 + 3u * (size_t)c[u];
                const double2 y0 = X[0], y1 = X[1], y2 = X[2];
                s += (double)v[u][0].x * y0.x;
                s += (double)v[u][0].y * y0.y;
                s += (double)v[u][1].x * y1.x;
                s += (double)v[u][1].y * y1.y;
                s += (double)v[u][2].x * y2.x;
                s += (double)v[u][2].y * y2.y;
            }
        }
    }
    return s;
}

__global__ void __launch_bounds__(kThreads) k_resid64(const SysDesc *__restrict__ sys, StepParams *sp) {
    __shared__ double red[64];
    __shared__ int s_last;
    const uint32_t nw = sp->n_aux_b;
    const WorkItem *__restrict__ work = sp->aux_b;
    const uint32_t t = threadIdx.x;
    for (uint32_t w = blockIdx.x; w < nw; w += gridDim.x) {
        const WorkItem it = work[w];
        if (it.sys >= sp->num_sys || it.tile >= sys[it.sys].n_utiles) {
            if (threadIdx.x == 0) atomicOr(&sp->error, kErrBadItem);
            continue;
        }
        const SysDesc &S = sys[it.sys];
        SysState *st = S.st;
        const UpdTile T = S.utiles[it.tile];
        const uint32_t rows = T.row1 - T.row0;
        float *const bin = const_cast<float *>(S.b);
        double rr = 0.0, bb = 0.0;
        if (S.layout == LAYOUT_BSR6) {
            for (uint32_t o = t; o < rows; o += kThreads) {
                const uint32_t i = T.row0 + o;
                const double bi = (double)__ldg(S.b_orig + i);
                const double r64 = bi - resid_row_bsr6(S, i);
                bin[i] = (float)r64;
                rr += r64 * r64;
                bb += bi * bi;
            }
        } else {
            constexpr uint32_t kLanes = 8, kRowsPerPass = kThreads / kLanes;
            const uint32_t sub = t / kLanes, l = t % kLanes;
            const double *__restrict__ x64 = S.x64;
            for (uint32_t r0 = 0; r0 < rows; r0 += kRowsPerPass) {
                const uint32_t o = r0 + sub;
                double sum = 0.0;
                if (o < rows) {
                    const uint32_t i = T.row0 + o;
                    const uint32_t k0 = __ldg(S.row_ptr + i), k1 = __ldg(S.row_ptr + i + 1);
                    uint32_t k = k0 + l;
                    for (; k + kLanes < k1; k += 2 * kLanes) {
                        const float v0 = __ldcs(S.val + k), v1 = __ldcs(S.val + k + kLanes);
                        const uint32_t c0 = __ldcs(S.col + k), c1 = __ldcs(S.col + k + kLanes);
                        sum += (double)v0 * x64[c0];
                        sum += (double)v1 * x64[c1];
                    }
                    if (k < k1) sum += (double)__ldcs(S.val + k) * x64[__ldcs(S.col + k)];
                }
                sum += __shfl_xor_sync(0xffffffffu, sum, 4);
                sum += __shfl_xor_sync(0xffffffffu, sum, 2);
                sum += __shfl_xor_sync(0xffffffffu, sum, 1);
                if (o < rows && l == 0) {
                    const uint32_t i = T.row0 + o;
                    const double bi = (double)__ldg(S.b_orig + i);
                    const double r64 = bi - sum;
                    bin[i] = (float)r64;
                    rr += r64 * r64;
                    bb += bi * bi;
                }
            }
        }
        const double2 tot = block_sum2(rr, bb, red);
        if (t == 0) S.part_b[it.tile] = tot;
        if (take_ticket(&st->cnt_c, 1u, S.n_utiles, &s_last)) {
            double va = 0.0, vb = 0.0;
            for (uint32_t i = t; i < S.n_utiles; i += kThreads) {
                const double2 q = __ldcg(S.part_b + i);
                va += q.x;
                vb += q.y;
            }
            const double2 sum = block_sum2(va, vb, red);
            if (t == 0) {
                st->rr64 = sum.x;
                st->bb64 = sum.y;
                st->cnt_c = 0;
            }
        }
        csync();
    }
}

// x64 += d (the inner solution in x), then d = 0 for the next inner solve.
__global__ void __launch_bounds__(kThreads) k_refine(const SysDesc *__restrict__ sys, StepParams *sp) {
    const uint32_t nw = sp->n_aux_b;
    const WorkItem *__restrict__ work = sp->aux_b;
    for (uint32_t w = blockIdx.x; w < nw; w += gridDim.x) {
        const WorkItem it = work[w];
        if (it.sys >= sp->num_sys || it.tile >= sys[it.sys].n_utiles) {
            if (threadIdx.x == 0) atomicOr(&sp->error, kErrBadItem);
            continue;
        }
        const SysDesc &S = sys[it.sys];
        const UpdTile T = S.utiles[it.tile];
        for (uint32_t i = T.row0 + threadIdx.x; i < T.row1; i += kThreads) {
            S.x64[i] += (double)S.x[i];
            S.x[i] = 0.0f;
        }
    }
}

// x = (float) x64: the mixed-precision result in the FP32 output vector.
__global__ void __launch_bounds__(kThreads) k_x64_to_x32(const SysDesc *__restrict__ sys, StepParams *sp) {
    const uint32_t nw = sp->n_aux_b;
    const WorkItem *__restrict__ work = sp->aux_b;
    for (uint32_t w = blockIdx.x; w < nw; w += gridDim.x) {
        const WorkItem it = work[w];
        if (it.sys >= sp->num_sys || it.tile >= sys[it.sys].n_utiles) {
            if (threadIdx.x == 0) atomicOr(&sp->error, kErrBadItem);
            continue;
        }
        const SysDesc &S = sys[it.sys];
        const UpdTile T = S.utiles[it.tile];
        for (uint32_t i = T.row0 + threadIdx.x; i < T.row1; i += kThreads) S.x[i] = (float)S.x64[i];
    }
}

}  // namespace wsb
