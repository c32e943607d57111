// The reference's individual passes on the GPU with the reference's
// arithmetic (separately rounded FP32 multiply/add/divide, 256-wide shared
// memory tree for dot products). They back the executor entry points and the
// WSB_PREC_REFERENCE_F32 solve, whose iterates are bit-identical to the CPU
// restatement of compute.rs:189-495.
#include "kernels_ref.cuh"

namespace wsb {

// spmv.wgsl:43-64 - one row per thread, sequential sum in index order.
__global__ void k_ref_spmv(uint32_t n, const uint32_t *__restrict__ row_ptr, const uint32_t *__restrict__ col,
                           const float *__restrict__ val, const float *__restrict__ x, float *__restrict__ y) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float sum = 0.0f;
    for (uint32_t k = row_ptr[i]; k < row_ptr[i + 1]; ++k) sum = __fadd_rn(sum, __fmul_rn(val[k], __ldg(x + col[k])));
    y[i] = sum;
}

// 256-lane tree with offsets 128..1 (dot_partials.wgsl:57-69).
__device__ __forceinline__ float tree256(float *s) {
    const uint32_t t = threadIdx.x;
    for (uint32_t off = 128; off >= 1; off >>= 1) {
        if (t < off) s[t] = __fadd_rn(s[t], s[t + off]);
        __syncthreads();
    }
    return s[0];
}

// dot_partials.wgsl:37-75: partial[wg] = tree sum of a[i]*b[i] over 256 lanes.
__global__ void __launch_bounds__(256) k_ref_dot_partials(uint32_t n, const float *__restrict__ a,
                                                          const float *__restrict__ b, float *__restrict__ partial) {
    __shared__ float s[256];
    const uint32_t i = blockIdx.x * 256u + threadIdx.x;
    s[threadIdx.x] = i < n ? __fmul_rn(a[i], b[i]) : 0.0f;
    __syncthreads();
    const float v = tree256(s);
    if (threadIdx.x == 0) partial[blockIdx.x] = v;
}

// dot_reduce.wgsl:36-74: output[wg] = tree sum of input[wg*256 .. +255].
__global__ void __launch_bounds__(256) k_ref_dot_reduce(uint32_t n, const float *__restrict__ in, float *__restrict__ out) {
    __shared__ float s[256];
    const uint32_t i = blockIdx.x * 256u + threadIdx.x;
    s[threadIdx.x] = i < n ? in[i] : 0.0f;
    __syncthreads();
    const float v = tree256(s);
    if (threadIdx.x == 0) out[blockIdx.x] = v;
}

// copy_buffer_to_buffer of the final scalar (dot_scalar_exec.rs:239-246), or
// the n == 0 case that writes 0 (dot_scalar_exec.rs:165-174) when src is null.
__global__ void k_ref_store_scalar(const float *src, float *dst) {
    if (threadIdx.x == 0 && blockIdx.x == 0) *dst = src ? *src : 0.0f;
}

// axpy.wgsl:32-42: y = y + alpha * x
__global__ void k_ref_axpy(uint32_t n, float alpha, const float *__restrict__ x, float *__restrict__ y) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) y[i] = __fadd_rn(y[i], __fmul_rn(alpha, x[i]));
}

// axpy_from_scalar_results.wgsl:28-42: y = y + s[k] * x
__global__ void k_ref_axpy_s(uint32_t n, const float *__restrict__ x, float *__restrict__ y,
                             const float *__restrict__ s, uint32_t k) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) y[i] = __fadd_rn(y[i], __fmul_rn(s[k], x[i]));
}

// scale_from_scalar_results.wgsl:26-38: x = x * s[k]
__global__ void k_ref_scale_s(uint32_t n, float *__restrict__ x, const float *__restrict__ s, uint32_t k) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) x[i] = __fmul_rn(x[i], s[k]);
}

// block_jacobi.wgsl:63-127, one thread per block (the WGSL runs one
// single-invocation workgroup per block).
__global__ void k_ref_block_jacobi(uint32_t n, uint32_t nb, const float *__restrict__ lu,
                                   const uint32_t *__restrict__ bs, const float *__restrict__ r, float *__restrict__ z) {
    const uint32_t blk = blockIdx.x * blockDim.x + threadIdx.x;
    if (blk >= nb) return;
    const uint32_t offset = bs[blk], next = bs[blk + 1];
    if (offset >= n || next <= offset) return;
    const uint32_t m = min(6u, next - offset);
    const float *L = lu + (size_t)blk * 36u;
    float y[6] = {0, 0, 0, 0, 0, 0}, x[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        if ((uint32_t)i < m) {
            float sum = r[offset + i];
#pragma unroll
            for (int j = 0; j < i; ++j) sum = __fsub_rn(sum, __fmul_rn(L[i * 6 + j], y[j]));
            y[i] = sum;
        }
    }
#pragma unroll
    for (int i = 5; i >= 0; --i) {
        if ((uint32_t)i < m) {
            float sum = y[i];
#pragma unroll
            for (int j = i + 1; j < 6; ++j)
                if ((uint32_t)j < m) sum = __fsub_rn(sum, __fmul_rn(L[i * 6 + j], x[j]));
            x[i] = __fdiv_rn(sum, L[i * 6 + i]);
        }
    }
#pragma unroll
    for (int i = 0; i < 6; ++i)
        if ((uint32_t)i < m) z[offset + i] = x[i];
}

// pcg_update_scalars.wgsl:47-73 (one thread).
__global__ void k_ref_update_scalars(float *s, uint32_t p_ap, uint32_t rz_new, uint32_t rz_old, uint32_t alpha,
                                     uint32_t minus_alpha, uint32_t beta) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const float pap = s[p_ap], rzn = s[rz_new], rzo = s[rz_old];
    float a = 0.0f, b = 0.0f;
    if (pap != 0.0f) a = __fdiv_rn(rzo, pap);
    if (rzo != 0.0f) b = __fdiv_rn(rzn, rzo);
    s[alpha] = a;
    s[minus_alpha] = -a;
    s[beta] = b;
}

// After the ||b||^2 dot (compute.rs:228-257): store it, stop with Ok(0) when
// it is zero, otherwise open the iteration.
__global__ void k_ref_after_bnorm(RefState *st, const float *s) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    st->b_norm2 = s[0];
    st->rel2 = __fmul_rn(st->rel_tol, st->rel_tol);
    st->abs2 = __fmul_rn(st->abs_tol, st->abs_tol);
    st->iter = 0;
    st->breakdown = 0;
    if (st->b_norm2 == 0.0f) {
        st->status = ST_CONVERGED;
        st->active = 0;
    } else {
        st->status = ST_RUNNING;
        st->active = 1;
    }
}

// End of init (compute.rs:330): rz_old = scalar_results[3].
__global__ void k_ref_after_init(RefState *st, const float *s) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    st->rz_old = s[3];
    if (st->active && st->max_iter == 0) {
        st->status = ST_MAXITER;
        st->active = 0;
    }
}

// Step C (compute.rs:362-370): scalar_results[rz_old] = host rz_old.
__global__ void k_ref_write_rz_old(const RefState *st, float *s) {
    if (threadIdx.x == 0 && blockIdx.x == 0) s[3] = st->rz_old;
}

// The host side of one iteration (compute.rs:466-488) done on the device:
// breakdown checks, stop test in f32, rz_old = rz_new; clears the graph's
// while condition when the solve ends.
__global__ void k_ref_check(RefState *st, const float *s, double *history, uint64_t hist_cap,
                            cudaGraphConditionalHandle h) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const float p_ap = s[0], r_norm2 = s[1], rz_new = s[2];
    const uint32_t k = st->iter;
    if (history && k < hist_cap) history[k] = (double)r_norm2;
    st->iter = k + 1;
    st->last_rr = r_norm2;
    uint32_t status = ST_RUNNING;
    if (p_ap == 0.0f) {
        status = ST_BREAKDOWN;
        st->breakdown = 1;
    } else if (st->rz_old == 0.0f) {
        status = ST_BREAKDOWN;
        st->breakdown = 2;
    } else if (r_norm2 <= st->abs2 || r_norm2 <= __fmul_rn(st->rel2, st->b_norm2)) {
        status = ST_CONVERGED;
    } else if (k + 1 >= st->max_iter) {
        status = ST_MAXITER;
    } else {
        st->rz_old = rz_new;
    }
    if (status != ST_RUNNING) {
        st->status = status;
        st->active = 0;
    }
    if (h != 0 && (status != ST_RUNNING)) cudaGraphSetConditional(h, 0);
}

__global__ void k_ref_gate(const RefState *st, cudaGraphConditionalHandle h) {
    if (threadIdx.x == 0 && blockIdx.x == 0) cudaGraphSetConditional(h, st->active ? 1u : 0u);
}

}  // namespace wsb

namespace wsb {

size_t ref_dot_scratch_floats(uint64_t n) {
    const uint64_t l1 = (n + 255) / 256, l2 = (l1 + 255) / 256;
    return (size_t)(l1 + l2 + 2);
}

// The pass structure of encode_dot_scalar_into (dot_scalar_exec.rs:151-247):
// one dot_partials pass, then dot_reduce passes (ping-pong between the two
// halves of scratch) until one value is left, then a copy into s_out.
cudaError_t ref_dot(cudaStream_t st, uint32_t n, const float *a, const float *b, float *scratch, float *s_out) {
    if (n == 0) {
        k_ref_store_scalar<<<1, 32, 0, st>>>(nullptr, s_out);
        return cudaGetLastError();
    }
    const uint32_t l1 = (n + 255) / 256;
    float *in = scratch, *out = scratch + l1 + 1;
    k_ref_dot_partials<<<l1, 256, 0, st>>>(n, a, b, in);
    uint32_t len = l1;
    while (len > 1) {
        const uint32_t ol = (len + 255) / 256;
        k_ref_dot_reduce<<<ol, 256, 0, st>>>(len, in, out);
        len = ol;
        float *t = in;
        in = out;
        out = t;
    }
    k_ref_store_scalar<<<1, 32, 0, st>>>(in, s_out);
    return cudaGetLastError();
}

}  // namespace wsb
