// Reference-arithmetic kernels (one per WGSL pass of the reference).
#pragma once
#include "wsb_internal.h"

namespace wsb {

// Device-resident state of a reference-arithmetic solve (the host variables
// of compute.rs:189-495: b_norm2, rz_old, tolerances, iteration counter).
struct RefState {
    float b_norm2, rel2, abs2, rz_old;
    float rel_tol, abs_tol, last_rr, pad;
    uint32_t iter, max_iter, status, active;
    uint32_t breakdown, pad2[3];
};

__global__ void k_ref_spmv(uint32_t n, const uint32_t *__restrict__ row_ptr, const uint32_t *__restrict__ col,
                           const float *__restrict__ val, const float *__restrict__ x, float *__restrict__ y);
__global__ void k_ref_dot_partials(uint32_t n, const float *__restrict__ a, const float *__restrict__ b,
                                   float *__restrict__ partial);
__global__ void k_ref_dot_reduce(uint32_t n, const float *__restrict__ in, float *__restrict__ out);
__global__ void k_ref_store_scalar(const float *src, float *dst);
__global__ void k_ref_axpy(uint32_t n, float alpha, const float *__restrict__ x, float *__restrict__ y);
__global__ void k_ref_axpy_s(uint32_t n, const float *__restrict__ x, float *__restrict__ y,
                             const float *__restrict__ s, uint32_t k);
__global__ void k_ref_scale_s(uint32_t n, float *__restrict__ x, const float *__restrict__ s, uint32_t k);
__global__ void k_ref_block_jacobi(uint32_t n, uint32_t nb, const float *__restrict__ lu,
                                   const uint32_t *__restrict__ bs, const float *__restrict__ r, float *__restrict__ z);
__global__ void k_ref_update_scalars(float *s, uint32_t p_ap, uint32_t rz_new, uint32_t rz_old, uint32_t alpha,
                                     uint32_t minus_alpha, uint32_t beta);
__global__ void k_ref_after_bnorm(RefState *st, const float *s);
__global__ void k_ref_after_init(RefState *st, const float *s);
__global__ void k_ref_write_rz_old(const RefState *st, float *s);
__global__ void k_ref_check(RefState *st, const float *s, double *history, uint64_t hist_cap,
                            cudaGraphConditionalHandle h);
__global__ void k_ref_gate(const RefState *st, cudaGraphConditionalHandle h);

// Host-side launch helpers (stream-ordered).
// Dot product with the reference's pass structure into s_out (a device float);
// scratch needs ceil(n/256) + ceil(n/65536) + 2 floats.
cudaError_t ref_dot(cudaStream_t st, uint32_t n, const float *a, const float *b, float *scratch, float *s_out);
size_t ref_dot_scratch_floats(uint64_t n);

}  // namespace wsb
