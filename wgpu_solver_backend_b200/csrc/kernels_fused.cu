// Fused, batch-native PCG kernels for B200 (sm_100a).
//
// Memory-bound design notes (no dense contraction on this path, so no tensor
// cores): every CTA works on row tiles taken from a device work list in a
// grid-stride loop, so one captured CUDA graph serves any number of systems.
// Matrix values/columns are streamed once per iteration with 128-bit
// evict-first loads (ld.global.cs) into shared memory; the gathered vector is
// read through the read-only path (ld.global.nc) and stays in the 126 MB L2.
// Per-system reductions are deterministic: each tile writes one FP64 partial,
// and the last CTA of a system (ticket counter) sums the partials in a fixed
// order, so a system's arithmetic does not depend on how many other systems
// share the launch.
//
// Arithmetic parity with the reference: SpMV rows are summed sequentially in
// index order with separately rounded multiply and add (spmv.wgsl:58-61), the
// vector updates are y + a*x without contraction (axpy*.wgsl), the block solve
// is block_jacobi.wgsl:93-126 operation by operation, and p = p*beta + z
// follows scale_from_scalar_results.wgsl then axpy.wgsl.
#include "kernels_fused.cuh"

namespace wsb {

namespace {

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// Fixed-shape block reduction (result valid in thread 0). red: >= 32 doubles.
__device__ __forceinline__ double block_sum(double v, double *red) {
    v = warp_sum(v);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) red[w] = v;
    __syncthreads();
    double s = 0.0;
    if (w == 0) {
        s = lane < (kThreads >> 5) ? red[lane] : 0.0;
        s = warp_sum(s);
    }
    __syncthreads();
    return s;
}

__device__ __forceinline__ double2 block_sum2(double a, double b, double *red) {
    a = warp_sum(a);
    b = warp_sum(b);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) {
        red[w] = a;
        red[32 + w] = b;
    }
    __syncthreads();
    double sa = 0.0, sb = 0.0;
    if (w == 0) {
        sa = lane < (kThreads >> 5) ? red[lane] : 0.0;
        sb = lane < (kThreads >> 5) ? red[32 + lane] : 0.0;
        sa = warp_sum(sa);
        sb = warp_sum(sb);
    }
    __syncthreads();
    return make_double2(sa, sb);
}

// Ticket on a per-system counter after thread 0 published this CTA's partial.
// Returns true in every thread of the CTA that took the last ticket.
__device__ __forceinline__ bool take_ticket(uint32_t *counter, uint32_t total, int *s_last) {
    if (threadIdx.x == 0) {
        __threadfence();
        const uint32_t t = atomicAdd(counter, 1u);
        *s_last = (t + 1 == total);
    }
    __syncthreads();
    const bool last = *s_last != 0;
    if (last) __threadfence();
    return last;
}

// y(row0 + t) for the t < nrows rows of one CSR tile. The tile's nonzeros
// [row_ptr[row0], row_ptr[row0+nrows]) are streamed in chunks of kCsrCap:
// 16-byte aligned float4/uint4 loads, products val*x[col] stored in shared
// memory, then one thread per row adds its products in index order.
__device__ __forceinline__ float csr_rows(const SysDesc &S, uint32_t row0, uint32_t nrows,
                                          const float *__restrict__ xin, float *prod, uint32_t *rp) {
    const uint32_t tid = threadIdx.x;
    const uint32_t *__restrict__ row_ptr = S.row_ptr;
    const float *__restrict__ val = S.val;
    const uint32_t *__restrict__ col = S.col;
    for (uint32_t i = tid; i <= nrows; i += kThreads) rp[i] = __ldg(row_ptr + row0 + i);
    __syncthreads();
    const uint32_t k0 = rp[0], k1 = rp[nrows];
    uint32_t ms = 0, me = 0;
    if (tid < nrows) {
        ms = rp[tid];
        me = rp[tid + 1];
    }
    float acc = 0.0f;
    for (uint32_t c0 = k0; c0 < k1; c0 += kCsrCap) {
        const uint32_t c1 = min(k1, c0 + (uint32_t)kCsrCap);
        const uint32_t a0 = c0 & ~3u;
        uint32_t q = a0 + 4u * tid;
        for (; q + 4u * kThreads < c1; q += 8u * kThreads) {
            const float4 v0 = __ldcs(reinterpret_cast<const float4 *>(val + q));
            const uint4 i0 = __ldcs(reinterpret_cast<const uint4 *>(col + q));
            const float4 v1 = __ldcs(reinterpret_cast<const float4 *>(val + q + 4u * kThreads));
            const uint4 i1 = __ldcs(reinterpret_cast<const uint4 *>(col + q + 4u * kThreads));
            const float x00 = __ldg(xin + i0.x), x01 = __ldg(xin + i0.y), x02 = __ldg(xin + i0.z),
                        x03 = __ldg(xin + i0.w);
            const float x10 = __ldg(xin + i1.x), x11 = __ldg(xin + i1.y), x12 = __ldg(xin + i1.z),
                        x13 = __ldg(xin + i1.w);
            *reinterpret_cast<float4 *>(prod + (q - a0)) =
                make_float4(__fmul_rn(v0.x, x00), __fmul_rn(v0.y, x01), __fmul_rn(v0.z, x02), __fmul_rn(v0.w, x03));
            *reinterpret_cast<float4 *>(prod + (q + 4u * kThreads - a0)) =
                make_float4(__fmul_rn(v1.x, x10), __fmul_rn(v1.y, x11), __fmul_rn(v1.z, x12), __fmul_rn(v1.w, x13));
        }
        if (q < c1) {
            const float4 v0 = __ldcs(reinterpret_cast<const float4 *>(val + q));
            const uint4 i0 = __ldcs(reinterpret_cast<const uint4 *>(col + q));
            *reinterpret_cast<float4 *>(prod + (q - a0)) =
                make_float4(__fmul_rn(v0.x, __ldg(xin + i0.x)), __fmul_rn(v0.y, __ldg(xin + i0.y)),
                            __fmul_rn(v0.z, __ldg(xin + i0.z)), __fmul_rn(v0.w, __ldg(xin + i0.w)));
        }
        __syncthreads();
        const uint32_t s = max(ms, c0), e = min(me, c1);
        for (uint32_t j = s; j < e; ++j) acc = __fadd_rn(acc, prod[j - a0]);
        __syncthreads();
    }
    return acc;
}

// y for the 6*nbrows rows of one BSR6 tile: 144-byte blocks staged with
// float4 loads; thread t owns row (t/6, t%6) and walks its block row's blocks
// in column order, six products each, added in index order. For a matrix that
// stores complete 6x6 blocks with sorted columns this is exactly the CSR row
// order, so both layouts round identically.
__device__ __forceinline__ float bsr_rows(const SysDesc &S, uint32_t brow0, uint32_t nbrows,
                                          const float *__restrict__ xin, float *sval, uint32_t *rp) {
    const uint32_t tid = threadIdx.x;
    uint32_t *scol = reinterpret_cast<uint32_t *>(sval + kBsrCapBlocks * 36);
    for (uint32_t i = tid; i <= nbrows; i += kThreads) rp[i] = __ldg(S.brow_ptr + brow0 + i);
    __syncthreads();
    const uint32_t k0 = rp[0], k1 = rp[nbrows];
    const uint32_t br = tid / 6u, a = tid - 6u * br;
    uint32_t ms = 0, me = 0;
    if (tid < 6u * nbrows) {
        ms = rp[br];
        me = rp[br + 1];
    }
    float acc = 0.0f;
    for (uint32_t c0 = k0; c0 < k1; c0 += kBsrCapBlocks) {
        const uint32_t c1 = min(k1, c0 + (uint32_t)kBsrCapBlocks);
        const uint32_t nblk = c1 - c0;
        const float4 *__restrict__ src = reinterpret_cast<const float4 *>(S.bval) + (size_t)c0 * 9u;
        float4 *dst = reinterpret_cast<float4 *>(sval);
        for (uint32_t q = tid; q < nblk * 9u; q += kThreads) dst[q] = __ldcs(src + q);
        for (uint32_t q = tid; q < nblk; q += kThreads) scol[q] = __ldcs(S.bcol + c0 + q);
        __syncthreads();
        const uint32_t s = max(ms, c0), e = min(me, c1);
        for (uint32_t blk = s; blk < e; ++blk) {
            const float *B = sval + (blk - c0) * 36u + a * 6u;
            const float2 *xx = reinterpret_cast<const float2 *>(xin + 6u * (size_t)scol[blk - c0]);
            const float2 x01 = __ldg(xx), x23 = __ldg(xx + 1), x45 = __ldg(xx + 2);
            acc = __fadd_rn(acc, __fmul_rn(B[0], x01.x));
            acc = __fadd_rn(acc, __fmul_rn(B[1], x01.y));
            acc = __fadd_rn(acc, __fmul_rn(B[2], x23.x));
            acc = __fadd_rn(acc, __fmul_rn(B[3], x23.y));
            acc = __fadd_rn(acc, __fmul_rn(B[4], x45.x));
            acc = __fadd_rn(acc, __fmul_rn(B[5], x45.y));
        }
        __syncthreads();
    }
    return acc;
}

// Rows [row0, row0+nrows) of A*xin for one SpMV tile of either layout.
struct TileRows {
    float acc;
    uint32_t row0, nrows;
};

__device__ __forceinline__ TileRows tile_spmv(const SysDesc &S, const SpmvTile &T, const float *__restrict__ xin,
                                              float *buf, uint32_t *rp) {
    TileRows out;
    if (S.layout == LAYOUT_BSR6) {
        out.row0 = 6u * T.row0;
        out.nrows = 6u * (T.row1 - T.row0);
        out.acc = bsr_rows(S, T.row0, T.row1 - T.row0, xin, buf, rp);
    } else {
        out.row0 = T.row0;
        out.nrows = T.row1 - T.row0;
        out.acc = csr_rows(S, T.row0, T.row1 - T.row0, xin, buf, rp);
    }
    return out;
}

// z = U^-1 L^-1 r for the blocks that start inside the tile (block_jacobi.wgsl:
// forward solve with unit L, lines 93-101; backward solve dividing by U(i,i),
// lines 103-122; rows i < m = min(6, len) only, lines 79 and 124-126). LU
// factors (144 B per block) are staged through shared memory with coalesced
// float4 loads, kLuStage blocks per pass; one thread solves one block in
// registers. sr: the tile's r; outputs sz and sflag (1 where z was solved).
__device__ __forceinline__ void bj_tile(const SysDesc &S, const UpdTile &T, const float *sr, float *sz,
                                        uint32_t *sflag, float *slu) {
    const uint32_t nblk = T.blk1 - T.blk0;
    for (uint32_t pb = 0; pb < nblk; pb += kLuStage) {
        const uint32_t nbp = min(nblk - pb, (uint32_t)kLuStage);
        const float4 *__restrict__ src = reinterpret_cast<const float4 *>(S.lu) + (size_t)(T.blk0 + pb) * 9u;
        float4 *dst = reinterpret_cast<float4 *>(slu);
        for (uint32_t q = threadIdx.x; q < nbp * 9u; q += kThreads) dst[q] = __ldcs(src + q);
        __syncthreads();
        if (threadIdx.x < nbp) {
            const uint32_t blk = T.blk0 + pb + threadIdx.x;
            const uint32_t off = __ldg(S.bstart + blk), nxt = __ldg(S.bstart + blk + 1);
            const uint32_t m = min(nxt - off, 6u);
            const uint32_t lo = off - T.row0;
            const float *L = slu + threadIdx.x * 36u;
            float y[6], xs[6];
#pragma unroll
            for (int i = 0; i < 6; ++i) {
                y[i] = 0.0f;
                xs[i] = 0.0f;
            }
#pragma unroll
            for (int i = 0; i < 6; ++i) {
                if ((uint32_t)i < m) {
                    float s = sr[lo + i];
#pragma unroll
                    for (int j = 0; j < i; ++j) s = __fsub_rn(s, __fmul_rn(L[i * 6 + j], y[j]));
                    y[i] = s;
                }
            }
#pragma unroll
            for (int i = 5; i >= 0; --i) {
                if ((uint32_t)i < m) {
                    float s = y[i];
#pragma unroll
                    for (int j = i + 1; j < 6; ++j)
                        if ((uint32_t)j < m) s = __fsub_rn(s, __fmul_rn(L[i * 6 + j], xs[j]));
                    xs[i] = __fdiv_rn(s, L[i * 6 + i]);
                }
            }
#pragma unroll
            for (int i = 0; i < 6; ++i)
                if ((uint32_t)i < m) {
                    sz[lo + i] = xs[i];
                    sflag[lo + i] = 1u;
                }
        }
        __syncthreads();
    }
}

}  // namespace

// ---------------------------------------------------------------------------
// kInit = false: Ap = A p over sp->work_a, FP64 p.Ap; the last CTA of each
// system sets pAp and alpha = rz_old / pAp (0 when pAp == 0, as
// pcg_update_scalars.wgsl:59-62).
// kInit = true: Ap = A x (initial residual) over sp->init_a, no reduction.
// ---------------------------------------------------------------------------
template <bool kInit>
__device__ __forceinline__ void spmv_pass(const SysDesc *__restrict__ sys, StepParams *sp, float *smem) {
    float *buf = smem;
    uint32_t *rp = reinterpret_cast<uint32_t *>(smem + kCsrCap + 8);
    __shared__ double red[64];
    __shared__ int s_last;
    const uint32_t nw = kInit ? sp->n_init_a : sp->n_work_a;
    const WorkItem *__restrict__ work = kInit ? sp->init_a : sp->work_a;
    for (uint32_t w = blockIdx.x; w < nw; w += gridDim.x) {
        const WorkItem it = work[w];
        const SysDesc &S = sys[it.sys];
        SysState *st = S.st;
        if (!kInit && !st->active) continue;
        const SpmvTile T = S.stiles[it.tile];
        const float *__restrict__ xin = kInit ? S.x : S.p;
        const TileRows tr = tile_spmv(S, T, xin, buf, rp);
        const float acc = tr.acc;
        double part = 0.0;
        if (threadIdx.x < tr.nrows) {
            const uint32_t i = tr.row0 + threadIdx.x;
            S.ap[i] = acc;
            if (!kInit) part = (double)__ldg(xin + i) * (double)acc;
        }
        if (!kInit) {
            const double tot = block_sum(part, red);
            if (threadIdx.x == 0) S.part_a[it.tile] = tot;
            if (take_ticket(&st->cnt_a, S.n_stiles, &s_last)) {
                double v = 0.0;
                for (uint32_t i = threadIdx.x; i < S.n_stiles; i += kThreads) v += __ldcg(S.part_a + i);
                const double pap = block_sum(v, red);
                if (threadIdx.x == 0) {
                    const double alpha = pap != 0.0 ? st->rz_old / pap : 0.0;
                    st->pap = pap;
                    st->alpha = alpha;
                    st->alpha_f = (float)alpha;
                    st->cnt_a = 0;
                }
            }
        }
        __syncthreads();
    }
}
__global__ void __launch_bounds__(kThreads) k_spmv_loop(const SysDesc *__restrict__ sys, StepParams *sp) {
    extern __shared__ __align__(16) float smem[];
    spmv_pass<false>(sys, sp, smem);
}

__global__ void __launch_bounds__(kThreads) k_spmv_init(const SysDesc *__restrict__ sys, StepParams *sp) {
    extern __shared__ __align__(16) float smem[];
    spmv_pass<true>(sys, sp, smem);
}

// ---------------------------------------------------------------------------
// k_update: x += alpha p; r += (-alpha) Ap; z = M^-1 r; FP64 r.r and r.z.
// The last CTA of a system runs the host-side logic of compute.rs:466-488 on
// the device: breakdown checks (pAp == 0, then rz_old == 0), the stop test
// r.r <= abs^2 or r.r <= rel^2 * b.b, the iteration limit, beta = rz_new /
// rz_old, and the residual history entry.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads) k_update(const SysDesc *__restrict__ sys, StepParams *sp) {
    __shared__ float sr[kTileRows], sz[kTileRows];
    __shared__ uint32_t sflag[kTileRows];
    __shared__ __align__(16) float slu[kLuStage * 36];
    __shared__ double red[64];
    __shared__ int s_last;
    const uint32_t nw = sp->n_work_b;
    const WorkItem *__restrict__ work = sp->work_b;
    const uint32_t t = threadIdx.x;
    for (uint32_t w = blockIdx.x; w < nw; w += gridDim.x) {
        const WorkItem it = work[w];
        const SysDesc &S = sys[it.sys];
        SysState *st = S.st;
        if (!st->active) continue;
        const UpdTile T = S.utiles[it.tile];
        const float a = st->alpha_f, ma = -a;
        const uint32_t rows = T.row1 - T.row0;
        float ri = 0.0f;
        double rr = 0.0;
        sflag[t] = 0u;
        if (t < rows) {
            const uint32_t i = T.row0 + t;
            const float pi = S.p[i], api = S.ap[i];
            float xi = S.x[i];
            ri = S.r[i];
            xi = __fadd_rn(xi, __fmul_rn(a, pi));
            ri = __fadd_rn(ri, __fmul_rn(ma, api));
            S.x[i] = xi;
            S.r[i] = ri;
            sr[t] = ri;
            rr = (double)ri * (double)ri;
        }
        __syncthreads();
        bj_tile(S, T, sr, sz, sflag, slu);
        double rz = 0.0;
        if (t < rows) {
            const uint32_t i = T.row0 + t;
            float zi;
            if (sflag[t]) {
                zi = sz[t];
                S.z[i] = zi;
            } else {
                zi = S.z[i];
            }
            rz = (double)ri * (double)zi;
        }
        const double2 tot = block_sum2(rr, rz, red);
        if (t == 0) S.part_b[it.tile] = tot;
        if (take_ticket(&st->cnt_b, S.n_utiles, &s_last)) {
            double va = 0.0, vb = 0.0;
            for (uint32_t i = t; i < S.n_utiles; i += kThreads) {
                const double2 q = __ldcg(S.part_b + i);
                va += q.x;
                vb += q.y;
            }
            const double2 sum = block_sum2(va, vb, red);
            if (t == 0) {
                const double rr_t = sum.x, rz_new = sum.y;
                const uint32_t k = st->iter;
                const double pap = st->pap, rz_old = st->rz_old;
                if (S.history && k < S.hist_cap) S.history[k] = rr_t;
                st->rr = rr_t;
                st->rz_new = rz_new;
                st->iter = k + 1;
                uint32_t status = ST_RUNNING;
                if (pap == 0.0) {
                    status = ST_BREAKDOWN;
                    st->breakdown = 1;
                } else if (rz_old == 0.0) {
                    status = ST_BREAKDOWN;
                    st->breakdown = 2;
                } else if (rr_t <= st->abs2 || rr_t <= st->rel2 * st->bb) {
                    status = ST_CONVERGED;
                } else if (k + 1 >= st->max_iter) {
                    status = ST_MAXITER;
                }
                const double beta = rz_old != 0.0 ? rz_new / rz_old : 0.0;
                st->beta = beta;
                st->beta_f = (float)beta;
                if (status != ST_RUNNING) {
                    st->status = status;
                    st->active = 0;
                    atomicSub(&sp->num_active, 1u);
                } else {
                    st->rz_old = rz_new;
                }
                st->cnt_b = 0;
            }
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// k_init (after k_spmv<true>): r = b + (-1)(A x0); z = M^-1 r; p = z;
// FP64 b.b and r.z (compute.rs:226-331). The last CTA stores b.b and rz_old;
// b.b == 0 finishes the system with 0 iterations and x untouched
// (compute.rs:252-254); max_iter == 0 finishes it as not converged.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads) k_init(const SysDesc *__restrict__ sys, StepParams *sp) {
    __shared__ float sr[kTileRows], sz[kTileRows];
    __shared__ uint32_t sflag[kTileRows];
    __shared__ __align__(16) float slu[kLuStage * 36];
    __shared__ double red[64];
    __shared__ int s_last;
    const uint32_t nw = sp->n_init_b;
    const WorkItem *__restrict__ work = sp->init_b;
    const uint32_t t = threadIdx.x;
    for (uint32_t w = blockIdx.x; w < nw; w += gridDim.x) {
        const WorkItem it = work[w];
        const SysDesc &S = sys[it.sys];
        SysState *st = S.st;
        const UpdTile T = S.utiles[it.tile];
        const uint32_t rows = T.row1 - T.row0;
        float ri = 0.0f;
        double bb = 0.0;
        sflag[t] = 0u;
        if (t < rows) {
            const uint32_t i = T.row0 + t;
            const float bi = S.b[i];
            ri = __fsub_rn(bi, S.ap[i]);
            S.r[i] = ri;
            sr[t] = ri;
            bb = (double)bi * (double)bi;
        }
        __syncthreads();
        bj_tile(S, T, sr, sz, sflag, slu);
        double rz = 0.0;
        if (t < rows) {
            const uint32_t i = T.row0 + t;
            float zi;
            if (sflag[t]) {
                zi = sz[t];
                S.z[i] = zi;
            } else {
                zi = S.z[i];
            }
            S.p[i] = zi;
            rz = (double)ri * (double)zi;
        }
        const double2 tot = block_sum2(bb, rz, red);
        if (t == 0) S.part_b[it.tile] = tot;
        if (take_ticket(&st->cnt_b, S.n_utiles, &s_last)) {
            double va = 0.0, vb = 0.0;
            for (uint32_t i = t; i < S.n_utiles; i += kThreads) {
                const double2 q = __ldcg(S.part_b + i);
                va += q.x;
                vb += q.y;
            }
            const double2 sum = block_sum2(va, vb, red);
            if (t == 0) {
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
                st->cnt_b = 0;
            }
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// k_pupdate: p = p*beta + z (scale_from_scalar_results.wgsl then axpy.wgsl
// with alpha 1). CTA 0 then ends the graph's while loop when no system is
// active or the step's iteration budget is used.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads) k_pupdate(const SysDesc *__restrict__ sys, StepParams *sp,
                                                      cudaGraphConditionalHandle h) {
    const uint32_t nw = sp->n_work_b;
    const WorkItem *__restrict__ work = sp->work_b;
    for (uint32_t w = blockIdx.x; w < nw; w += gridDim.x) {
        const WorkItem it = work[w];
        const SysDesc &S = sys[it.sys];
        const SysState *st = S.st;
        if (!st->active) continue;
        const UpdTile T = S.utiles[it.tile];
        const float bf = st->beta_f;
        const uint32_t rows = T.row1 - T.row0;
        if (threadIdx.x < rows) {
            const uint32_t i = T.row0 + threadIdx.x;
            S.p[i] = __fadd_rn(__fmul_rn(S.p[i], bf), S.z[i]);
        }
    }
    if (h != 0 && blockIdx.x == 0 && threadIdx.x == 0) {
        const uint32_t c = sp->loop_count + 1;
        sp->loop_count = c;
        if (sp->num_active == 0 || c >= sp->loop_limit) cudaGraphSetConditional(h, 0);
    }
}

// Parent-graph node in front of the while loop: resets the step's iteration
// count and skips the loop when nothing is active.
__global__ void k_loop_gate(StepParams *sp, cudaGraphConditionalHandle h) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        sp->loop_count = 0;
        cudaGraphSetConditional(h, (sp->num_active > 0 && sp->loop_limit > 0) ? 1u : 0u);
    }
}

// ---------------------------------------------------------------------------
// Mixed precision (FP64 outer iterative refinement).
// k_resid64: r64 = b - A x64 with FP32 matrix entries and FP64 accumulation;
// the inner right-hand side becomes (float) r64; FP64 ||r64||^2 and ||b||^2.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads) k_resid64(const SysDesc *__restrict__ sys, StepParams *sp) {
    __shared__ double red[64];
    __shared__ int s_last;
    const uint32_t nw = sp->n_aux_b;
    const WorkItem *__restrict__ work = sp->aux_b;
    const uint32_t t = threadIdx.x;
    for (uint32_t w = blockIdx.x; w < nw; w += gridDim.x) {
        const WorkItem it = work[w];
        const SysDesc &S = sys[it.sys];
        SysState *st = S.st;
        const UpdTile T = S.utiles[it.tile];
        const uint32_t rows = T.row1 - T.row0;
        double rr = 0.0, bb = 0.0;
        if (t < rows) {
            const uint32_t i = T.row0 + t;
            const double *__restrict__ x64 = S.x64;
            double s = 0.0;
            if (S.layout == LAYOUT_BSR6) {
                const uint32_t br = i / 6u, a = i - 6u * br;
                for (uint32_t k = S.brow_ptr[br]; k < S.brow_ptr[br + 1]; ++k) {
                    const float *B = S.bval + (size_t)k * 36u + a * 6u;
                    const double *xc = x64 + 6u * (size_t)S.bcol[k];
#pragma unroll
                    for (int j = 0; j < 6; ++j) s += (double)B[j] * xc[j];
                }
            } else {
                for (uint32_t k = S.row_ptr[i]; k < S.row_ptr[i + 1]; ++k) s += (double)S.val[k] * x64[S.col[k]];
            }
            const double bi = (double)S.b_orig[i];
            const double r64 = bi - s;
            const_cast<float *>(S.b)[i] = (float)r64;
            rr = r64 * r64;
            bb = bi * bi;
        }
        const double2 tot = block_sum2(rr, bb, red);
        if (t == 0) S.part_b[it.tile] = tot;
        if (take_ticket(&st->cnt_c, S.n_utiles, &s_last)) {
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
        __syncthreads();
    }
}

// x64 += d (the inner solution in x), then d = 0 for the next inner solve.
__global__ void __launch_bounds__(kThreads) k_refine(const SysDesc *__restrict__ sys, StepParams *sp) {
    const uint32_t nw = sp->n_aux_b;
    const WorkItem *__restrict__ work = sp->aux_b;
    for (uint32_t w = blockIdx.x; w < nw; w += gridDim.x) {
        const WorkItem it = work[w];
        const SysDesc &S = sys[it.sys];
        const UpdTile T = S.utiles[it.tile];
        if (threadIdx.x < T.row1 - T.row0) {
            const uint32_t i = T.row0 + threadIdx.x;
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
        const SysDesc &S = sys[it.sys];
        const UpdTile T = S.utiles[it.tile];
        if (threadIdx.x < T.row1 - T.row0) {
            const uint32_t i = T.row0 + threadIdx.x;
            S.x[i] = (float)S.x64[i];
        }
    }
}

// y = A x over all SpMV tiles of one system (no reduction).
__global__ void __launch_bounds__(kThreads) k_spmv_plain(const SysDesc *__restrict__ sys, const float *__restrict__ x,
                                                         float *__restrict__ y) {
    extern __shared__ __align__(16) float smem[];
    float *buf = smem;
    uint32_t *rp = reinterpret_cast<uint32_t *>(smem + kCsrCap + 8);
    const SysDesc &S = sys[0];
    for (uint32_t w = blockIdx.x; w < S.n_stiles; w += gridDim.x) {
        const SpmvTile T = S.stiles[w];
        const TileRows tr = tile_spmv(S, T, x, buf, rp);
        if (threadIdx.x < tr.nrows) y[tr.row0 + threadIdx.x] = tr.acc;
        __syncthreads();
    }
}

}  // namespace wsb
