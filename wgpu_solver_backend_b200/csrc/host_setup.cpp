// Host-side setup: block-Jacobi LU builder, input validation, tile lists,
// CSR -> BSR6 conversion and a small thread pool. Compiled with
// -ffp-contract=off so the LU arithmetic rounds every multiply and subtract
// separately, as the reference's Rust code does.
#include <algorithm>
#include <cstring>
#include <thread>

#include "wsb_internal.h"

namespace wsb {

static std::string fmt(const char *f, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, f);
    vsnprintf(buf, sizeof buf, f, ap);
    va_end(ap);
    return buf;
}

// In-place no-pivot LU of the leading n x n of a row-major 6x6 buffer.
// Follows lu_factor_inplace_6, compute.rs:37-71: strict lower = L (unit
// diagonal implied), diagonal + upper = U; exact-zero pivot is an error; the
// trailing update is skipped when L(i,k) == 0.
int lu_factor_inplace_6(float *mat, uint32_t n, uint32_t *pivot_k) {
    const uint32_t stride = 6;
    for (uint32_t k = 0; k < n; ++k) {
        const float a_kk = mat[k * stride + k];
        if (a_kk == 0.0f) {
            if (pivot_k) *pivot_k = k;
            return WSB_ERR_ZERO_PIVOT;
        }
        for (uint32_t i = k + 1; i < n; ++i) mat[i * stride + k] /= a_kk;
        for (uint32_t i = k + 1; i < n; ++i) {
            const float l_ik = mat[i * stride + k];
            if (l_ik != 0.0f)
                for (uint32_t j = k + 1; j < n; ++j) mat[i * stride + j] -= l_ik * mat[k * stride + j];
        }
    }
    return WSB_OK;
}

// build_lu_blocks_from_csr_block_starts_6, compute.rs:84-181: identity-padded
// 6x6 extraction of each diagonal block (leading m = min(6, len) rows/cols,
// later duplicates overwrite earlier ones), then lu_factor_inplace_6(m).
int build_lu_blocks_6(uint32_t n, const uint32_t *row_ptr, uint64_t row_ptr_len, const uint32_t *col,
                      uint64_t col_len, const float *val, uint64_t val_len, const uint32_t *bs,
                      uint64_t bs_len, float *out, std::string *err) {
    const char *fn = "build_lu_blocks_from_csr_block_starts_6";
    if (row_ptr_len != (uint64_t)n + 1) {
        *err = fmt("%s: row_ptr len must be n+1 (%llu), got %llu", fn, (unsigned long long)n + 1,
                   (unsigned long long)row_ptr_len);
        return WSB_ERR_BAD_INPUT;
    }
    const uint64_t nnz = row_ptr[n];
    if (col_len != nnz || val_len != nnz) {
        *err = fmt("%s: nnz mismatch: row_ptr says %llu, col_idx %llu, values %llu", fn,
                   (unsigned long long)nnz, (unsigned long long)col_len, (unsigned long long)val_len);
        return WSB_ERR_BAD_INPUT;
    }
    if (bs_len < 2) return WSB_OK;
    if (bs[0] != 0) {
        *err = fmt("%s: block_starts must start at 0", fn);
        return WSB_ERR_BAD_INPUT;
    }
    if (bs[bs_len - 1] != n) {
        *err = fmt("%s: block_starts last must equal n (%u), got %u", fn, n, bs[bs_len - 1]);
        return WSB_ERR_BAD_INPUT;
    }
    for (uint64_t i = 0; i + 1 < bs_len; ++i)
        if (bs[i + 1] <= bs[i]) {
            *err = fmt("%s: block_starts must be strictly increasing", fn);
            return WSB_ERR_BAD_INPUT;
        }
    for (uint32_t i = 0; i < n; ++i)
        if (row_ptr[i + 1] < row_ptr[i] || row_ptr[i + 1] > nnz) {
            *err = fmt("%s: row_ptr must be non-decreasing and end at nnz", fn);
            return WSB_ERR_BAD_INPUT;
        }
    const uint64_t nb = bs_len - 1;
    std::atomic<int64_t> first_bad{-1};
    std::atomic<uint32_t> bad_k{0};
    parallel_for((int64_t)nb, 4096, [&](int64_t lo, int64_t hi) {
        for (int64_t blk = lo; blk < hi; ++blk) {
            const uint32_t offset = bs[blk], end = bs[blk + 1];
            float *mat = out + (uint64_t)blk * 36;
            std::memset(mat, 0, 36 * sizeof(float));
            if (end > n || offset >= end) continue;
            const uint32_t m = std::min<uint32_t>(end - offset, 6);
            for (int i = 0; i < 6; ++i) mat[i * 6 + i] = 1.0f;
            for (uint32_t il = 0; il < m; ++il) {
                const uint32_t i = offset + il;
                for (uint32_t k = row_ptr[i]; k < row_ptr[i + 1]; ++k) {
                    const uint32_t j = col[k];
                    if (j >= offset && j < offset + m) mat[il * 6 + (j - offset)] = val[k];
                }
            }
            uint32_t pk = 0;
            if (lu_factor_inplace_6(mat, m, &pk) != WSB_OK) {
                int64_t cur = first_bad.load();
                while ((cur < 0 || blk < cur) && !first_bad.compare_exchange_weak(cur, blk)) {
                }
                if (first_bad.load() == blk) bad_k.store(pk);
            }
        }
    });
    if (first_bad.load() >= 0) {
        // Report the first failing block in block order, as the sequential
        // reference loop would (compute.rs:136-178).
        const int64_t blk = first_bad.load();
        float mat[36];
        const uint32_t offset = bs[blk], end = bs[blk + 1];
        const uint32_t m = std::min<uint32_t>(end - offset, 6);
        std::memset(mat, 0, sizeof mat);
        for (int i = 0; i < 6; ++i) mat[i * 6 + i] = 1.0f;
        for (uint32_t il = 0; il < m; ++il)
            for (uint32_t k = row_ptr[offset + il]; k < row_ptr[offset + il + 1]; ++k)
                if (col[k] >= offset && col[k] < offset + m) mat[il * 6 + (col[k] - offset)] = val[k];
        uint32_t pk = 0;
        lu_factor_inplace_6(mat, m, &pk);
        *err = fmt("LU zero pivot at k = %u", pk);
        return WSB_ERR_ZERO_PIVOT;
    }
    return WSB_OK;
}

// Matrix and partition checks of loaders.rs:83-113 and loaders.rs:164-184,
// plus the bounds every kernel relies on.
int validate_system(uint32_t n, const uint32_t *row_ptr, const uint32_t *col, uint64_t nnz,
                    const uint32_t *bs, uint64_t bs_len, std::string *err, bool check_cols) {
    if (!row_ptr) {
        *err = "row_ptr is null";
        return WSB_ERR_BAD_INPUT;
    }
    if (row_ptr[0] != 0) {
        *err = "CSR row_ptr must start with 0";
        return WSB_ERR_BAD_INPUT;
    }
    if ((uint64_t)row_ptr[n] != nnz) {
        *err = fmt("CSR row_ptr must end with nnz (%llu), got %u", (unsigned long long)nnz, row_ptr[n]);
        return WSB_ERR_BAD_INPUT;
    }
    for (uint32_t i = 0; i < n; ++i)
        if (row_ptr[i + 1] < row_ptr[i]) {
            *err = "CSR row_ptr must be non-decreasing";
            return WSB_ERR_BAD_INPUT;
        }
    if (nnz && !col) {
        *err = "col_idx is null";
        return WSB_ERR_BAD_INPUT;
    }
    uint32_t max_col = 0;
    if (check_cols)
        for (uint64_t k = 0; k < nnz; ++k) max_col = std::max(max_col, col[k]);
    if (check_cols && nnz && max_col >= n) {
        *err = fmt("CSR col_idx contains out-of-range column %u for n_cols=%u", max_col, n);
        return WSB_ERR_BAD_INPUT;
    }
    if (bs_len == 0 || !bs) {
        *err = "block_starts must not be empty";
        return WSB_ERR_BAD_INPUT;
    }
    if (bs[0] != 0) {
        *err = fmt("block_starts must start with 0, got %u", bs[0]);
        return WSB_ERR_BAD_INPUT;
    }
    if (bs[bs_len - 1] != n) {
        *err = fmt("block_starts must end with n (%u), got %u", n, bs[bs_len - 1]);
        return WSB_ERR_BAD_INPUT;
    }
    for (uint64_t i = 0; i + 1 < bs_len; ++i)
        if (bs[i + 1] <= bs[i]) {
            *err = "block_starts must be strictly increasing";
            return WSB_ERR_BAD_INPUT;
        }
    return WSB_OK;
}

// Greedy CSR row tiles: <= max_rows rows and <= max_nnz nonzeros (bounded
// by kSpmvTileRows and kCsrCap, one stage), except a single longer row,
// which gets a tile of its own (beyond kCsrCap the kernel streams it in
// chunks).
void build_spmv_tiles_csr(uint32_t n, const uint32_t *row_ptr, std::vector<SpmvTile> *out, uint32_t max_rows,
                          uint32_t max_nnz) {
    out->clear();
    max_rows = std::max<uint32_t>(1, std::min<uint32_t>(max_rows, kSpmvTileRows));
    max_nnz = std::max<uint32_t>(1, std::min<uint32_t>(max_nnz, kCsrCap));
    uint32_t r0 = 0;
    while (r0 < n) {
        uint32_t r1 = r0;
        while (r1 < n && r1 - r0 < max_rows) {
            const uint64_t tile_nnz = (uint64_t)row_ptr[r1 + 1] - row_ptr[r0];
            if (r1 > r0 && tile_nnz > (uint64_t)max_nnz) break;
            ++r1;
            if (tile_nnz > (uint64_t)max_nnz) break;  // long single row
        }
        out->push_back({r0, r1, row_ptr[r0], row_ptr[r1]});
        r0 = r1;
    }
}

// BSR6 tiles over block rows: <= max_brows block rows and <= max_blocks
// blocks (bounded by kSpmvTileRows / 6 and kBsrCapBlocks; a block row longer
// than kBsrCapBlocks is chunked by the kernel).
void build_spmv_tiles_bsr(uint32_t nbrows, const uint32_t *brow_ptr, std::vector<SpmvTile> *out,
                          uint32_t max_brows, uint32_t max_blocks) {
    out->clear();
    max_brows = std::max<uint32_t>(1, std::min<uint32_t>(max_brows, kSpmvTileRows / 6));
    max_blocks = std::max<uint32_t>(1, std::min<uint32_t>(max_blocks, kBsrCapBlocks));
    uint32_t r0 = 0;
    while (r0 < nbrows) {
        uint32_t r1 = r0;
        while (r1 < nbrows && r1 - r0 < max_brows) {
            const uint64_t blocks = (uint64_t)brow_ptr[r1 + 1] - brow_ptr[r0];
            if (r1 > r0 && blocks > (uint64_t)max_blocks) break;
            ++r1;
            if (blocks > (uint64_t)max_blocks) break;
        }
        out->push_back({r0, r1, brow_ptr[r0], brow_ptr[r1]});
        r0 = r1;
    }
}

// Update tiles of <= max_rows rows holding <= max_blocks block starts
// (bounded by kUpdTileRows and kUpdBlocks). A cut is allowed at a block
// start or at a row whose position inside its block is >= 6 (the reference
// never touches z there, block_jacobi.wgsl:79,124-126), so the solved rows of
// a block are always inside one tile.
void build_upd_tiles(uint32_t n, const uint32_t *bs, uint32_t nb, std::vector<UpdTile> *out, uint32_t max_rows,
                     uint32_t max_blocks) {
    out->clear();
    if (n == 0) return;
    max_rows = std::max<uint32_t>(6, std::min<uint32_t>(max_rows, kUpdTileRows));
    max_blocks = std::max<uint32_t>(1, std::min<uint32_t>(max_blocks, kUpdBlocks));
    std::vector<uint8_t> cut_ok(n + 1, 0);
    std::vector<uint32_t> starts_before(n + 1, 0);  // block starts in [0, r)
    cut_ok[n] = 1;
    for (uint32_t b = 0; b < nb; ++b) {
        cut_ok[bs[b]] = 1;
        for (uint32_t r = bs[b] + 6; r < bs[b + 1]; ++r) cut_ok[r] = 1;
    }
    {
        uint32_t b = 0;
        for (uint32_t r = 0; r <= n; ++r) {
            while (b < nb && bs[b] < r) ++b;
            starts_before[r] = b;
        }
    }
    uint32_t r0 = 0;
    while (r0 < n) {
        uint32_t r1 = std::min<uint32_t>(n, r0 + max_rows);
        while (r1 > r0 + 1 && (!cut_ok[r1] || starts_before[r1] - starts_before[r0] > max_blocks)) --r1;
        // r0 + 1 is always a cut when the block at r0 has one row or r0 is a
        // passive row; otherwise the loop stops at the next block start.
        while (!cut_ok[r1]) ++r1;
        UpdTile t;
        t.row0 = r0;
        t.row1 = r1;
        t.blk0 = starts_before[r0];
        t.blk1 = starts_before[r1];
        out->push_back(t);
        r0 = r1;
    }
}

// BSR6 applies when every block has exactly 6 rows and each row's columns are
// strictly increasing and made of complete aligned 6-column groups, the same
// groups for the 6 rows of a block row. Then the BSR sum order equals the CSR
// sequential order and both SpMVs round identically.
bool bsr6_convertible(uint32_t n, const uint32_t *row_ptr, const uint32_t *col, const uint32_t *bs,
                      uint64_t bs_len) {
    if (n == 0 || n % 6 != 0 || bs_len != (uint64_t)n / 6 + 1) return false;
    for (uint64_t i = 0; i < bs_len; ++i)
        if (bs[i] != 6 * i) return false;
    std::atomic<bool> ok{true};
    parallel_for(n / 6, 8192, [&](int64_t lo, int64_t hi) {
        for (int64_t br = lo; br < hi && ok.load(std::memory_order_relaxed); ++br) {
            const uint32_t r0 = 6 * (uint32_t)br;
            const uint32_t len0 = row_ptr[r0 + 1] - row_ptr[r0];
            if (len0 % 6) { ok = false; return; }
            for (uint32_t a = 0; a < 6; ++a) {
                const uint32_t s = row_ptr[r0 + a], e = row_ptr[r0 + a + 1];
                if (e - s != len0) { ok = false; return; }
                for (uint32_t k = s; k < e; k += 6) {
                    const uint32_t c0 = col[k];
                    if (c0 % 6) { ok = false; return; }
                    if (k > s && c0 <= col[k - 1]) { ok = false; return; }
                    for (uint32_t j = 1; j < 6; ++j)
                        if (col[k + j] != c0 + j) { ok = false; return; }
                    if (col[k] != col[row_ptr[r0] + (k - s)]) { ok = false; return; }
                }
            }
        }
    });
    return ok.load();
}

uint64_t csr_to_bsr6(uint32_t n, const uint32_t *row_ptr, const uint32_t *col, const float *val,
                     std::vector<uint32_t> *brow_ptr, std::vector<uint32_t> *bcol, std::vector<float> *bval) {
    const uint32_t nbr = n / 6;
    brow_ptr->assign(nbr + 1, 0);
    for (uint32_t br = 0; br < nbr; ++br) (*brow_ptr)[br + 1] = (*brow_ptr)[br] + (row_ptr[6 * br + 1] - row_ptr[6 * br]) / 6;
    const uint64_t nblk = (*brow_ptr)[nbr];
    bcol->assign(nblk, 0);
    bval->assign(nblk * 36 + kPadElems, 0.0f);
    parallel_for(nbr, 4096, [&](int64_t lo, int64_t hi) {
        for (int64_t br = lo; br < hi; ++br) {
            const uint32_t b0 = (*brow_ptr)[br];
            const uint32_t nbk = (*brow_ptr)[br + 1] - b0;
            for (uint32_t q = 0; q < nbk; ++q) (*bcol)[b0 + q] = col[row_ptr[6 * br] + 6 * q] / 6;
            for (uint32_t a = 0; a < 6; ++a) {
                const uint32_t s = row_ptr[6 * br + a];
                for (uint32_t q = 0; q < nbk; ++q)
                    for (uint32_t j = 0; j < 6; ++j) (*bval)[(uint64_t)(b0 + q) * 36 + a * 6 + j] = val[s + 6 * q + j];
            }
        }
    });
    return nblk;
}

void parallel_for(int64_t n, int64_t grain, const std::function<void(int64_t, int64_t)> &fn) {
    if (n <= 0) return;
    unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    int64_t nt = std::min<int64_t>(std::min<int64_t>(hw, 64), (n + grain - 1) / grain);
    if (nt <= 1) {
        fn(0, n);
        return;
    }
    std::vector<std::thread> th;
    th.reserve(nt);
    for (int64_t t = 0; t < nt; ++t) {
        const int64_t lo = n * t / nt, hi = n * (t + 1) / nt;
        th.emplace_back([&fn, lo, hi] { fn(lo, hi); });
    }
    for (auto &x : th) x.join();
}

}  // namespace wsb
