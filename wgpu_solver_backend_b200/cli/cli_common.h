// Host-side helpers shared by the two command-line tools: the case-directory
// binary formats (crates/wgpu_solver_backend/src/io/loaders.rs:8-237 and the
// writers of crates/wgpu_solver_backend_cli/src/main.rs:445-475 and
// crates/wgpu_solver_backend_convert_cli/src/main.rs:407-511), and number
// formatting that prints what the Rust tools print (`{}`, `{:?}`, `{:.Ne}` and
// serde_json's float output), so that logs and metrics files compare equal.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace wsbcli {

// ---- formats ---------------------------------------------------------------
constexpr uint32_t kMagicCsr1 = 0x43535231u;  // "CSR1"

struct CsrMatrixBin {
    uint32_t n_rows = 0, n_cols = 0, nnz = 0;
    std::vector<uint32_t> row_ptr, col_idx;
    std::vector<float> values;
};

struct CaseInputBin {
    CsrMatrixBin a;
    std::vector<float> b, x0;
    std::vector<uint32_t> block_starts;
};

// Each loader returns an empty string on success, else the reference's
// error message for the same condition.
std::string load_csr_matrix_bin(const std::string &path, CsrMatrixBin *out);
std::string load_vector_bin(const std::string &path, std::vector<float> *out);
std::string load_block_starts_bin(const std::string &path, std::vector<uint32_t> *out);
std::string load_case_dir(const std::string &case_dir, CaseInputBin *out);
// read_f32_vec_bin of the CLI (main.rs:560-580): u32 length + f32[length].
std::string read_f32_vec_bin(const std::string &path, std::vector<float> *out);

// Creates the parent directory of `path` when it has one, then writes.
std::string write_x_bin(const std::string &path, const std::vector<float> &x);
std::string write_text_file(const std::string &path, const std::string &text);

// Path::join: inserts a separator unless `dir` already ends with one.
std::string path_join(const std::string &dir, const std::string &name);
// io::Error's Display for an errno value: "<strerror> (os error N)".
std::string os_error(int err);

// ---- number formatting -----------------------------------------------------
// Shortest decimal digits that round-trip the float: digits and the decimal
// exponent e such that value = 0.d1d2... * 10^e ... expressed as digits
// string `d` and `point` = position of the decimal point (value = d * 10^(point-len)).
void shortest_digits_f32(float v, std::string *digits, int *point);
void shortest_digits_f64(double v, std::string *digits, int *point);
// Rust `{}` of f32/f64: shortest round-trip digits, never an exponent.
std::string rust_display_f32(float v);
// Rust `{:?}` of f32: as `{}` but an integral value keeps ".0".
std::string rust_debug_f32(float v);
// Rust `{:.Ne}`: N digits after the point, exponent without '+' or padding.
std::string rust_exp(double v, int prec);
// serde_json's output for a finite f32 / f64 (ryu's notation); non-finite -> null.
std::string json_f32(float v);
std::string json_f64(double v);
// A JSON string literal with serde_json's escaping.
std::string json_str(const std::string &s);

// RFC 3339 UTC timestamp as the `time` crate prints it (sub-second digits
// without trailing zeros, 'Z' suffix).
std::string now_utc_rfc3339();

// ---- solve metrics ---------------------------------------------------------
// True relative residual ||b - A x|| / ||b|| in FP64 (matrix and vectors
// widened from f32, rows summed in index order); 0 when b == 0. The caller
// guarantees sizes that match the matrix (a loaded, validated case).
double true_relres_f64(const CsrMatrixBin &a, const std::vector<float> &b, const std::vector<float> &x);
// Algorithmic HBM bytes of one PCG iteration on a CSR matrix, as the
// library's wsb_matrix_info counts them: the SpMV (8 nnz + 4 (n + 1) + 8 n:
// values, columns, row pointers, x read, y written), the update (x, p, r, Ap
// read, x, r, z written: 28 n), p = z + beta p (12 n) and the 6x6 LU factors
// (144 bytes per block; 24 n for blocks of 6 rows).
uint64_t pcg_iteration_bytes_csr(uint64_t n, uint64_t nnz, uint64_t num_blocks);

}  // namespace wsbcli
