// Fused PCG kernels for sm_100a (declarations shared with the engine).
//
// One PCG iteration of every active system is three launches:
//   k_spmv     Ap = A p (CSR or BSR6 tiles streamed through shared memory by
//              TMA bulk copies, x gathered by cp.async), FP64 p.Ap per tile,
//              and in the last CTA of each system: pAp, alpha = rz_old / pAp.
//   k_update   x += alpha p, r -= alpha Ap, z = (LU)^-1 r per 6x6 block in
//              registers, FP64 r.r and r.z per tile; the last CTA of each system
//              computes beta, the stop test, the residual history and status.
//   k_pupdate  p = z + beta p; one thread of CTA 0 clears the graph's while
//              condition when no system is left.
// These replace the reference's 17 passes per iteration (compute.rs:336-489):
// spmv.wgsl, dot_partials.wgsl + dot_reduce.wgsl (x3), pcg_update_scalars.wgsl
// (x2), axpy*.wgsl (x3), scale_from_scalar_results.wgsl, block_jacobi.wgsl.
#pragma once
#include "wsb_internal.h"

namespace wsb {

// Shared-memory stages (floats) of the two TMA-pipelined kernels. The SpMV
// runs a ring of kSpmvStages stages, the update kernel kUpdStages.
// SpMV stage: CSR values [0, kCsrCap+8) and columns [kCsrCap+8, 2(kCsrCap+8)),
// or BSR6 block values [0, 36 cap), block columns, then the gathered x (6 per
// block); the row pointers at kSpmvRpOff.
constexpr int kSpmvBcolOff = 36 * kBsrCapBlocks;
constexpr int kSpmvXgOff = kSpmvBcolOff + kBsrCapBlocks + 8;
constexpr int kSpmvBsrEnd = kSpmvXgOff + 6 * kBsrCapBlocks;
constexpr int kSpmvCsrEnd = 2 * (kCsrCap + 8);
constexpr int kSpmvRpOff = (((kSpmvCsrEnd > kSpmvBsrEnd) ? kSpmvCsrEnd : kSpmvBsrEnd) + 3) & ~3;
constexpr int kSpmvStageFloats = ((kSpmvRpOff + kSpmvTileRows + 8) + 31) & ~31;
constexpr int kUpdStageFloats = ((4 * (kUpdTileRows + 8) + kUpdBlocks * 36 + kUpdBlocks + 8) + 31) & ~31;
// The single-reduction update kernel stages six vector slices.
constexpr int kUpdStageFloatsSr = ((6 * (kUpdTileRows + 8) + kUpdBlocks * 36 + kUpdBlocks + 8) + 31) & ~31;
// Threads per CTA of the TMA-pipelined kernels: consumers (kUpdConsumers in
// the update kernels, kSpmvConsumers in the SpMV) plus one producer warp,
// plus the gather warps in the SpMV.
#ifndef WSB_GATHER_WARPS
#define WSB_GATHER_WARPS 2
#endif
constexpr int kGatherWarps = WSB_GATHER_WARPS;
// 1: the gather warps read row pointers and BSR6 block columns with an L2
// evict-last hint.
#ifndef WSB_GATHER_KEEP_L2
#define WSB_GATHER_KEEP_L2 0
#endif
// The SpMV producer prefetches the index data of the tile this many tiles
// ahead of the one it issues into the L2 (0: no prefetch).
#ifndef WSB_SPMV_PREFETCH_AHEAD
#define WSB_SPMV_PREFETCH_AHEAD 2
#endif
constexpr uint32_t kSpmvPrefetchAhead = WSB_SPMV_PREFETCH_AHEAD;
// 16-byte column loads each gather lane keeps in flight for a CSR tile.
#ifndef WSB_CSR_GATHER_BATCH
#define WSB_CSR_GATHER_BATCH 8
#endif
constexpr int kUpdThreads = kUpdConsumers + 32;
#ifndef WSB_UPD_MIN_CTAS
#define WSB_UPD_MIN_CTAS 3
#endif
constexpr int kUpdMinCtas = WSB_UPD_MIN_CTAS;
constexpr int kSpmvThreads = kSpmvConsumers + 32 + 32 * kGatherWarps;
// CTAs per SM the SpMV kernels are compiled for (register budget).
#ifndef WSB_SPMV_MIN_CTAS
#define WSB_SPMV_MIN_CTAS 3
#endif
constexpr int kSpmvMinCtas = WSB_SPMV_MIN_CTAS;
constexpr size_t kSpmvSmem = (size_t)kSpmvStages * kSpmvStageFloats * sizeof(float);
constexpr size_t kUpdSmem = (size_t)kUpdStages * kUpdStageFloats * sizeof(float);
constexpr size_t kUpdSmemSr = (size_t)kUpdStages * kUpdStageFloatsSr * sizeof(float);

// k_spmv_loop: Ap = A p with p.Ap and alpha; k_spmv_init: Ap = A x.
__global__ void k_spmv_loop(const SysDesc *__restrict__ sys, StepParams *sp);
__global__ void k_spmv_init(const SysDesc *__restrict__ sys, StepParams *sp);
__global__ void k_update(const SysDesc *__restrict__ sys, StepParams *sp);
// Single-reduction recurrence: the update kernel ends the loop body itself.
__global__ void k_update_sr(const SysDesc *__restrict__ sys, StepParams *sp, cudaGraphConditionalHandle h);
__global__ void k_init(const SysDesc *__restrict__ sys, StepParams *sp);
__global__ void k_pupdate(const SysDesc *__restrict__ sys, StepParams *sp, cudaGraphConditionalHandle h);
__global__ void k_loop_gate(StepParams *sp, cudaGraphConditionalHandle h);

// Mixed precision.
__global__ void k_resid64(const SysDesc *__restrict__ sys, StepParams *sp);
__global__ void k_refine(const SysDesc *__restrict__ sys, StepParams *sp);
__global__ void k_x64_to_x32(const SysDesc *__restrict__ sys, StepParams *sp);

// Plain y = A x of one system (sys[0]) over its own tiles (no reduction);
// sp receives the error code of a timed-out wait.
__global__ void k_spmv_plain(const SysDesc *__restrict__ sys, StepParams *sp, const float *__restrict__ x,
                             float *__restrict__ y);

}  // namespace wsb
