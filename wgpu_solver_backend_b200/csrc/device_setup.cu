// Device-side preparation of a system: the O(nnz) parts of the set-up that
// the host would otherwise do before a solve can start.
//
//  - column range check (loaders.rs:83-113: every column < n);
//  - the BSR6 eligibility test and the CSR -> BSR6 conversion (the same rule
//    and layout as the host conversion in host_setup.cpp);
//  - the block-Jacobi LU build, build_lu_blocks_from_csr_block_starts_6 /
//    lu_factor_inplace_6 (compute.rs:37-181): identity-padded extraction of
//    the leading m = min(6, len) rows and columns of each diagonal block
//    (later duplicates overwrite earlier ones), then the no-pivot LU with
//    every division, multiply and subtract rounded separately, in the
//    reference's loop order, so the factors are bit-identical to the host
//    builder's.
//
// Only the O(n) checks of row pointers and block starts stay on the host, so
// admitting a request costs little more than copying its arrays.
#include <algorithm>
#include <cstring>

#include "engine.h"

namespace wsb {

namespace {

constexpr uint32_t kNoBlock = 0xffffffffu;

struct PrepResult {
    uint32_t max_col;     // largest column index (atomicMax)
    uint32_t bsr_ok;      // 1 while every block row passes the BSR6 test
    uint32_t first_bad;   // smallest block index with a zero pivot, or kNoBlock
    uint32_t pad;
};

__global__ void k_prep_max_col(const uint32_t *__restrict__ col, uint64_t nnz, PrepResult *res) {
    uint32_t m = 0;
    for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < nnz; k += (uint64_t)gridDim.x * blockDim.x)
        m = max(m, col[k]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_down_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31u) == 0) atomicMax(&res->max_col, m);
}

// One thread per block row: rows 6br..6br+5 must store complete, aligned
// 6-column groups with strictly increasing columns, the same groups in all
// six rows (then the BSR6 sum order equals the CSR sequential order).
__global__ void k_prep_bsr6_check(uint32_t nbr, const uint32_t *__restrict__ row_ptr,
                                  const uint32_t *__restrict__ col, PrepResult *res) {
    for (uint32_t br = blockIdx.x * blockDim.x + threadIdx.x; br < nbr; br += gridDim.x * blockDim.x) {
        const uint32_t r0 = 6u * br;
        const uint32_t base = row_ptr[r0];
        const uint32_t len0 = row_ptr[r0 + 1] - base;
        bool ok = (len0 % 6u) == 0;
        for (uint32_t a = 0; ok && a < 6; ++a) {
            const uint32_t s = row_ptr[r0 + a], e = row_ptr[r0 + a + 1];
            if (e - s != len0) {
                ok = false;
                break;
            }
            for (uint32_t k = s; ok && k < e; k += 6) {
                const uint32_t c0 = col[k];
                if (c0 % 6u) ok = false;
                else if (k > s && c0 <= col[k - 1]) ok = false;
                else if (col[k] != col[base + (k - s)]) ok = false;
                for (uint32_t j = 1; ok && j < 6; ++j)
                    if (col[k + j] != c0 + j) ok = false;
            }
        }
        if (!ok) atomicAnd(&res->bsr_ok, 0u);
    }
}

// One thread per (block row, row in block): the row's values into the 6x6
// blocks (row-major), and the block columns (row 0 only). For an eligible
// matrix every block row holds 36 values per block, so its first block is
// brow_ptr[br] = row_ptr[6 br] / 36.
__global__ void k_prep_bsr6_fill(uint32_t nbr, const uint32_t *__restrict__ row_ptr, const uint32_t *__restrict__ col,
                                 const float *__restrict__ val, uint32_t *__restrict__ bcol, float *__restrict__ bval) {
    const uint64_t total = 6ull * nbr;
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < total; t += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t br = (uint32_t)(t / 6u), a = (uint32_t)(t - 6ull * br);
        const uint32_t r = 6u * br + a;
        const uint32_t s = row_ptr[r], e = row_ptr[r + 1];
        const uint64_t b0 = row_ptr[6u * br] / 36u;
        for (uint32_t q = 0; s + 6u * q < e; ++q) {
            const uint32_t k = s + 6u * q;
            float *dst = bval + (b0 + q) * 36u + a * 6u;
#pragma unroll
            for (int j = 0; j < 6; ++j) dst[j] = val[k + j];
            if (a == 0) bcol[b0 + q] = col[k] / 6u;
        }
    }
}

// One thread per diagonal block: identity-padded extraction and the no-pivot
// LU (host_setup.cpp's lu_factor_inplace_6, operation by operation).
__global__ void k_prep_lu_blocks(uint32_t n, const uint32_t *__restrict__ row_ptr, const uint32_t *__restrict__ col,
                                 const float *__restrict__ val, const uint32_t *__restrict__ bs, uint32_t nb,
                                 float *__restrict__ out, PrepResult *res) {
    for (uint32_t blk = blockIdx.x * blockDim.x + threadIdx.x; blk < nb; blk += gridDim.x * blockDim.x) {
        float mat[36];
#pragma unroll
        for (int i = 0; i < 36; ++i) mat[i] = 0.0f;
        const uint32_t offset = bs[blk], end = bs[blk + 1];
        bool bad = false;
        if (end <= n && offset < end) {
            const uint32_t m = min(end - offset, 6u);
#pragma unroll
            for (int i = 0; i < 6; ++i) mat[i * 6 + i] = 1.0f;
            for (uint32_t il = 0; il < m; ++il) {
                const uint32_t i = offset + il;
                for (uint32_t k = row_ptr[i]; k < row_ptr[i + 1]; ++k) {
                    const uint32_t j = col[k];
                    if (j >= offset && j < offset + m) mat[il * 6 + (j - offset)] = val[k];
                }
            }
            for (uint32_t kk = 0; kk < m && !bad; ++kk) {
                const float a_kk = mat[kk * 6 + kk];
                if (a_kk == 0.0f) {
                    bad = true;
                    break;
                }
                for (uint32_t i = kk + 1; i < m; ++i) mat[i * 6 + kk] = __fdiv_rn(mat[i * 6 + kk], a_kk);
                for (uint32_t i = kk + 1; i < m; ++i) {
                    const float l_ik = mat[i * 6 + kk];
                    if (l_ik != 0.0f)
                        for (uint32_t j = kk + 1; j < m; ++j)
                            mat[i * 6 + j] = __fsub_rn(mat[i * 6 + j], __fmul_rn(l_ik, mat[kk * 6 + j]));
                }
            }
        }
        if (bad) atomicMin(&res->first_bad, blk);
        float4 *dst = reinterpret_cast<float4 *>(out + (size_t)blk * 36u);
#pragma unroll
        for (int q = 0; q < 9; ++q) dst[q] = make_float4(mat[4 * q], mat[4 * q + 1], mat[4 * q + 2], mat[4 * q + 3]);
    }
}

// Stream-ordered allocation and upload (cudaMallocAsync): freeing it later with
// cudaFreeAsync does not wait for the whole device, so preparing one request
// never stalls behind the solves running on other streams.
template <class T>
int dev_upload_async(Context *ctx, T **dst, const T *src, size_t count, size_t pad, cudaStream_t st) {
    void *p = nullptr;
    const size_t nbytes = std::max<size_t>(16, (count + pad) * sizeof(T));
    cudaError_t e = cudaMallocAsync(&p, nbytes, st);
    if (e != cudaSuccess)
        return fail(ctx, e == cudaErrorMemoryAllocation ? WSB_ERR_OUT_OF_MEMORY : WSB_ERR_CUDA,
                    "cudaMallocAsync(%zu) failed: %s", nbytes, cudaGetErrorString(e));
    *dst = static_cast<T *>(p);
    if (pad) WSB_CUDA_TRY(ctx, cudaMemsetAsync(p, 0, nbytes, st));
    if (count) WSB_CUDA_TRY(ctx, cudaMemcpyAsync(p, src, count * sizeof(T), cudaMemcpyHostToDevice, st));
    return WSB_OK;
}

template <class T>
int dev_upload(Context *ctx, T **dst, const T *src, size_t count, size_t pad, cudaStream_t st, uint64_t *bytes) {
    void *p = nullptr;
    const size_t nbytes = (count + pad) * sizeof(T);
    int rc = dev_alloc(ctx, &p, nbytes, pad > 0, st);
    if (rc) return rc;
    *dst = static_cast<T *>(p);
    if (count) WSB_CUDA_TRY(ctx, cudaMemcpyAsync(p, src, count * sizeof(T), cudaMemcpyHostToDevice, st));
    *bytes += nbytes;
    return WSB_OK;
}

unsigned grid_of(uint64_t work, unsigned block, int sm_count) {
    const uint64_t g = (work + block - 1) / block;
    return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(g, (uint64_t)std::max(1, sm_count) * 16));
}

}  // namespace

int prepare_system_device(Context *ctx, uint32_t n, const uint32_t *row_ptr, const uint32_t *col, const float *val,
                          uint64_t nnz, const uint32_t *bs, uint64_t bs_len, int layout_req, cudaStream_t st,
                          MatA *A, Precond *M) {
    std::string err;
    int rc = validate_system(n, row_ptr, col, nnz, bs, bs_len, &err, /*check_cols=*/false);
    if (rc) return fail(ctx, rc, "%s", err.c_str());
    const uint32_t nb = bs_len >= 1 ? (uint32_t)(bs_len - 1) : 0;
    A->ctx = ctx;
    A->n = n;
    A->nnz = nnz;
    M->ctx = ctx;
    M->n = n;
    M->nb = nb;
    // The BSR6 test needs blocks of exactly 6 rows (checked here in O(nb)).
    bool bsr_possible = layout_req != WSB_LAYOUT_CSR && n > 0 && n % 6 == 0 && bs_len == (uint64_t)n / 6 + 1;
    for (uint64_t i = 0; bsr_possible && i < bs_len; ++i)
        if (bs[i] != 6 * i) bsr_possible = false;
    if (layout_req == WSB_LAYOUT_BSR6 && !bsr_possible)
        return fail(ctx, WSB_ERR_BAD_INPUT,
                    "BSR6 layout needs blocks of exactly 6 rows whose rows store complete 6x6 blocks with "
                    "strictly increasing columns");
    // The CSR arrays are stream-ordered temporaries: a BSR6 matrix drops them
    // after the conversion, a CSR matrix gets persistent copies.
    uint32_t *d_rp = nullptr, *d_col = nullptr;
    float *d_val = nullptr;
    auto free_csr = [&] {
        if (d_rp) cudaFreeAsync(d_rp, st);
        if (d_col) cudaFreeAsync(d_col, st);
        if (d_val) cudaFreeAsync(d_val, st);
        d_rp = d_col = nullptr;
        d_val = nullptr;
    };
    if ((rc = dev_upload_async(ctx, &d_rp, row_ptr, (size_t)n + 1, 8, st)) ||
        (rc = dev_upload_async(ctx, &d_col, col, nnz, kPadElems, st)) ||
        (rc = dev_upload_async(ctx, &d_val, val, nnz, kPadElems, st))) {
        free_csr();
        return rc;
    }
    if ((rc = dev_upload(ctx, &M->bs, bs, (size_t)bs_len, 8, st, &M->bytes))) {
        free_csr();
        return rc;
    }
    void *p = nullptr;
    if ((rc = dev_alloc(ctx, &p, sizeof(float) * ((size_t)nb * 36 + 4), false, st))) {
        free_csr();
        return rc;
    }
    M->lu = static_cast<float *>(p);
    M->bytes += sizeof(float) * ((size_t)nb * 36 + 4);
    PrepResult *d_res = nullptr;
    PrepResult h_res{0u, bsr_possible ? 1u : 0u, kNoBlock, 0u};
    if ((rc = dev_upload_async(ctx, &d_res, &h_res, 1, 0, st))) {
        free_csr();
        return rc;
    }
    struct ResFree {
        PrepResult *p;
        cudaStream_t st;
        ~ResFree() { cudaFreeAsync(p, st); }
    } res_guard{d_res, st};
    const int sms = ctx->sm_count;
    if (nnz) k_prep_max_col<<<grid_of(nnz, 256, sms), 256, 0, st>>>(d_col, nnz, d_res);
    if (bsr_possible) k_prep_bsr6_check<<<grid_of(n / 6, 128, sms), 128, 0, st>>>(n / 6, d_rp, d_col, d_res);
    if (nb) k_prep_lu_blocks<<<grid_of(nb, 128, sms), 128, 0, st>>>(n, d_rp, d_col, d_val, M->bs, nb, M->lu, d_res);
    WSB_CUDA_TRY(ctx, cudaGetLastError());
    WSB_CUDA_TRY(ctx, cudaMemcpyAsync(&h_res, d_res, sizeof h_res, cudaMemcpyDeviceToHost, st));
    WSB_CUDA_TRY(ctx, cudaStreamSynchronize(st));
    if (nnz && h_res.max_col >= n) {
        free_csr();
        return fail(ctx, WSB_ERR_BAD_INPUT, "CSR col_idx contains out-of-range column %u for n_cols=%u",
                    h_res.max_col, n);
    }
    if (h_res.first_bad != kNoBlock) {
        // The pivot index of the first failing block in block order, as the
        // sequential reference loop reports it (compute.rs:136-178).
        const uint32_t blk = h_res.first_bad, offset = bs[blk], end = bs[blk + 1];
        const uint32_t m = std::min<uint32_t>(end - offset, 6);
        float mat[36];
        std::memset(mat, 0, sizeof mat);
        for (int i = 0; i < 6; ++i) mat[i * 6 + i] = 1.0f;
        for (uint32_t il = 0; il < m; ++il)
            for (uint32_t k = row_ptr[offset + il]; k < row_ptr[offset + il + 1]; ++k)
                if (col[k] >= offset && col[k] < offset + m) mat[il * 6 + (col[k] - offset)] = val[k];
        uint32_t pk = 0;
        lu_factor_inplace_6(mat, m, &pk);
        free_csr();
        return fail(ctx, WSB_ERR_ZERO_PIVOT, "LU zero pivot at k = %u", pk);
    }
    const bool bsr = bsr_possible && h_res.bsr_ok;
    if (layout_req == WSB_LAYOUT_BSR6 && !bsr) {
        free_csr();
        return fail(ctx, WSB_ERR_BAD_INPUT,
                    "BSR6 layout needs blocks of exactly 6 rows whose rows store complete 6x6 blocks with "
                    "strictly increasing columns");
    }
    const TileCaps caps = tile_caps_for(bsr ? LAYOUT_BSR6 : LAYOUT_CSR, n, nnz);
    M->h_bs.assign(bs, bs + bs_len);
    M->tile_rows = caps.upd_rows;
    M->tile_blocks = caps.upd_blocks;
    std::vector<UpdTile> utiles;
    build_upd_tiles(n, bs, nb, &utiles, caps.upd_rows, caps.upd_blocks);
    M->n_utiles = (uint32_t)utiles.size();
    if ((rc = dev_upload(ctx, &M->utiles, utiles.data(), utiles.size(), 1, st, &M->bytes))) {
        free_csr();
        return rc;
    }
    std::vector<SpmvTile> stiles;
    if (bsr) {
        const uint32_t nbr = n / 6;
        std::vector<uint32_t> brow_ptr(nbr + 1);
        for (uint32_t br = 0; br <= nbr; ++br) brow_ptr[br] = row_ptr[6 * br] / 36;
        A->layout = LAYOUT_BSR6;
        A->nbsr = brow_ptr[nbr];
        if ((rc = dev_upload(ctx, &A->brow_ptr, brow_ptr.data(), brow_ptr.size(), 8, st, &A->bytes)) ||
            (rc = dev_alloc(ctx, &p, sizeof(uint32_t) * (A->nbsr + kPadElems), true, st))) {
            free_csr();
            return rc;
        }
        A->bcol = static_cast<uint32_t *>(p);
        A->bytes += sizeof(uint32_t) * (A->nbsr + kPadElems);
        if ((rc = dev_alloc(ctx, &p, sizeof(float) * (A->nbsr * 36 + kPadElems), true, st))) {
            free_csr();
            return rc;
        }
        A->bval = static_cast<float *>(p);
        A->bytes += sizeof(float) * (A->nbsr * 36 + kPadElems);
        k_prep_bsr6_fill<<<grid_of(6ull * nbr, 128, sms), 128, 0, st>>>(nbr, d_rp, d_col, d_val, A->bcol, A->bval);
        WSB_CUDA_TRY(ctx, cudaGetLastError());
        build_spmv_tiles_bsr(nbr, brow_ptr.data(), &stiles, caps.spmv_rows / 6, caps.spmv_cap);
        A->h_rows = std::move(brow_ptr);
        free_csr();
    } else {
        A->layout = LAYOUT_CSR;
        const size_t rp_bytes = sizeof(uint32_t) * ((size_t)n + 1 + 8);
        const size_t nz_bytes = sizeof(uint32_t) * (nnz + kPadElems);
        if ((rc = dev_alloc(ctx, &p, rp_bytes, false, st))) {
            free_csr();
            return rc;
        }
        A->row_ptr = static_cast<uint32_t *>(p);
        if ((rc = dev_alloc(ctx, &p, nz_bytes, false, st))) {
            free_csr();
            return rc;
        }
        A->col = static_cast<uint32_t *>(p);
        if ((rc = dev_alloc(ctx, &p, nz_bytes, false, st))) {
            free_csr();
            return rc;
        }
        A->val = static_cast<float *>(p);
        A->bytes += rp_bytes + 2 * nz_bytes;
        WSB_CUDA_TRY(ctx, cudaMemcpyAsync(A->row_ptr, d_rp, rp_bytes, cudaMemcpyDeviceToDevice, st));
        WSB_CUDA_TRY(ctx, cudaMemcpyAsync(A->col, d_col, nz_bytes, cudaMemcpyDeviceToDevice, st));
        WSB_CUDA_TRY(ctx, cudaMemcpyAsync(A->val, d_val, nz_bytes, cudaMemcpyDeviceToDevice, st));
        free_csr();
        build_spmv_tiles_csr(n, row_ptr, &stiles, caps.spmv_rows, caps.spmv_cap);
        A->h_rows.assign(row_ptr, row_ptr + (size_t)n + 1);
    }
    A->tile_rows = caps.spmv_rows;
    A->tile_cap = caps.spmv_cap;
    A->n_stiles = (uint32_t)stiles.size();
    if ((rc = dev_upload(ctx, &A->stiles, stiles.data(), stiles.size(), 1, st, &A->bytes))) return rc;
    WSB_CUDA_TRY(ctx, cudaStreamSynchronize(st));
    return WSB_OK;
}

}  // namespace wsb
