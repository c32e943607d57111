// Case-directory I/O and Rust-compatible number formatting for the CLI tools.
#include "cli_common.h"

#include <cerrno>
#include <cstdarg>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <filesystem>
#include <fstream>

namespace wsbcli {
namespace fs = std::filesystem;

std::string os_error(int err) {
    char buf[64];
    snprintf(buf, sizeof buf, " (os error %d)", err);
    return std::string(strerror(err)) + buf;
}

std::string path_join(const std::string &dir, const std::string &name) {
    if (dir.empty()) return name;
    if (!name.empty() && name[0] == '/') return name;
    return dir.back() == '/' ? dir + name : dir + "/" + name;
}

static std::string fmt(const char *f, ...) __attribute__((format(printf, 1, 2)));
static std::string fmt(const char *f, ...) {
    va_list ap;
    va_start(ap, f);
    char buf[1024];
    vsnprintf(buf, sizeof buf, f, ap);
    va_end(ap);
    return buf;
}

static std::string read_all(const std::string &path, std::vector<unsigned char> *out) {
    FILE *fp = fopen(path.c_str(), "rb");
    if (!fp) return "Failed to read " + path + ": " + os_error(errno);
    out->clear();
    unsigned char buf[1 << 16];
    size_t k;
    while ((k = fread(buf, 1, sizeof buf, fp)) > 0) out->insert(out->end(), buf, buf + k);
    const int err = ferror(fp) ? errno : 0;
    fclose(fp);
    if (err) return "Failed to read " + path + ": " + os_error(err);
    return "";
}

// Little-endian cursor with the reference's EOF message (loaders.rs:198-237).
struct Cursor {
    const std::vector<unsigned char> &b;
    size_t pos = 0;
    explicit Cursor(const std::vector<unsigned char> &bytes) : b(bytes) {}
    size_t remaining() const { return pos < b.size() ? b.size() - pos : 0; }
    std::string u32(const std::string &label, uint32_t *v) {
        if (remaining() < 4)
            return fmt("Unexpected EOF while reading %s: need 4 bytes, have %zu", label.c_str(), remaining());
        std::memcpy(v, &b[pos], 4);
        pos += 4;
        return "";
    }
    // Reads `len` 4-byte items; on a short payload names the first missing one.
    template <class T>
    std::string slice(size_t len, const char *label, std::vector<T> *out) {
        const size_t have = remaining() / 4;
        if (have < len)
            return fmt("Unexpected EOF while reading %s[%zu]: need 4 bytes, have %zu", label, have,
                       remaining() - 4 * have);
        out->resize(len);
        if (len) std::memcpy(out->data(), &b[pos], 4 * len);
        pos += 4 * len;
        return "";
    }
};

std::string load_csr_matrix_bin(const std::string &path, CsrMatrixBin *m) {
    std::vector<unsigned char> bytes;
    std::string e = read_all(path, &bytes);
    if (!e.empty()) return e;
    Cursor c(bytes);
    uint32_t magic = 0, version = 0, r0, r1, r2;
    if (!(e = c.u32("magic", &magic)).empty()) return e;
    if (magic != kMagicCsr1)
        return fmt("Bad matrix magic in %s: expected 0x%08x, got 0x%08x", path.c_str(), kMagicCsr1, magic);
    if (!(e = c.u32("version", &version)).empty()) return e;
    if (version != 1) return fmt("Unsupported matrix version in %s: expected 1, got %u", path.c_str(), version);
    if (!(e = c.u32("n_rows", &m->n_rows)).empty()) return e;
    if (!(e = c.u32("n_cols", &m->n_cols)).empty()) return e;
    if (!(e = c.u32("nnz", &m->nnz)).empty()) return e;
    if (!(e = c.u32("reserved0", &r0)).empty()) return e;
    if (!(e = c.u32("reserved1", &r1)).empty()) return e;
    if (!(e = c.u32("reserved2", &r2)).empty()) return e;
    if (!(e = c.slice((size_t)m->n_rows + 1, "row_ptr", &m->row_ptr)).empty()) return e;
    if (!(e = c.slice(m->nnz, "col_idx", &m->col_idx)).empty()) return e;
    if (!(e = c.slice(m->nnz, "values", &m->values)).empty()) return e;
    if (m->row_ptr.front() != 0) return "CSR row_ptr must start with 0";
    if (m->row_ptr.back() != m->nnz)
        return fmt("CSR row_ptr must end with nnz (%u), got Some(%u)", m->nnz, m->row_ptr.back());
    for (size_t i = 1; i < m->row_ptr.size(); ++i)
        if (m->row_ptr[i] < m->row_ptr[i - 1]) return "CSR row_ptr must be non-decreasing";
    uint32_t max_col = 0;
    for (uint32_t c2 : m->col_idx) max_col = c2 > max_col ? c2 : max_col;
    if (m->n_cols > 0 && max_col >= m->n_cols)
        return fmt("CSR col_idx contains out-of-range column %u for n_cols=%u", max_col, m->n_cols);
    if (c.remaining() != 0) return fmt("matrix.csr.bin has %zu trailing bytes after expected payload", c.remaining());
    return "";
}

std::string load_vector_bin(const std::string &path, std::vector<float> *out) {
    std::vector<unsigned char> bytes;
    std::string e = read_all(path, &bytes);
    if (!e.empty()) return e;
    Cursor c(bytes);
    uint32_t n = 0;
    if (!(e = c.u32("n", &n)).empty()) return e;
    if (!(e = c.slice(n, "values", out)).empty()) return e;
    if (c.remaining() != 0)
        return fmt("%s has %zu trailing bytes after expected payload", path.c_str(), c.remaining());
    return "";
}

std::string load_block_starts_bin(const std::string &path, std::vector<uint32_t> *out) {
    std::vector<unsigned char> bytes;
    std::string e = read_all(path, &bytes);
    if (!e.empty()) return e;
    Cursor c(bytes);
    uint32_t len = 0;
    if (!(e = c.u32("len", &len)).empty()) return e;
    if (!(e = c.slice(len, "block_starts", out)).empty()) return e;
    if (c.remaining() != 0)
        return fmt("%s has %zu trailing bytes after expected payload", path.c_str(), c.remaining());
    return "";
}

// validate_block_starts, loaders.rs:160-183.
static std::string validate_block_starts(const std::vector<uint32_t> &s, uint32_t n) {
    if (s.empty()) return "block_starts must not be empty";
    if (s[0] != 0) return fmt("block_starts must start with 0, got %u", s[0]);
    if (s.back() != n) return fmt("block_starts must end with n (%u), got %u", n, s.back());
    for (size_t i = 1; i < s.size(); ++i)
        if (s[i] <= s[i - 1]) return "block_starts must be strictly increasing";
    return "";
}

std::string load_case_dir(const std::string &dir, CaseInputBin *c) {
    std::string e;
    if (!(e = load_csr_matrix_bin(path_join(dir, "matrix.csr.bin"), &c->a)).empty()) return e;
    if (!(e = load_vector_bin(path_join(dir, "rhs.bin"), &c->b)).empty()) return e;
    if (!(e = load_vector_bin(path_join(dir, "x0.bin"), &c->x0)).empty()) return e;
    if (!(e = load_block_starts_bin(path_join(dir, "block_starts.bin"), &c->block_starts)).empty()) return e;
    if (c->a.n_rows != c->a.n_cols)
        return fmt("matrix must be square for PCG: got %ux%u", c->a.n_rows, c->a.n_cols);
    if (c->b.size() != c->a.n_rows)
        return fmt("rhs length mismatch: b.n=%zu but matrix n_rows=%u", c->b.size(), c->a.n_rows);
    if (c->x0.size() != c->a.n_rows)
        return fmt("x0 length mismatch: x0.n=%zu but matrix n_rows=%u", c->x0.size(), c->a.n_rows);
    return validate_block_starts(c->block_starts, c->a.n_rows);
}

std::string read_f32_vec_bin(const std::string &path, std::vector<float> *out) {
    FILE *fp = fopen(path.c_str(), "rb");
    if (!fp) return "open " + path + ": " + os_error(errno);
    uint32_t n = 0;
    if (fread(&n, 4, 1, fp) != 1) {
        fclose(fp);
        return "read len header " + path + ": failed to fill whole buffer";
    }
    out->resize(n);
    const size_t got = n ? fread(out->data(), 4, n, fp) : 0;
    fclose(fp);
    if (got != n) return fmt("read f32[%zu] %s: failed to fill whole buffer", got, path.c_str());
    return "";
}

static std::string make_parent(const std::string &path) {
    const fs::path p(path);
    const fs::path parent = p.parent_path();
    if (!parent.empty()) {
        std::error_code ec;
        fs::create_directories(parent, ec);
        if (ec) return "create_dir_all " + parent.string() + ": " + os_error(ec.value());
    }
    return "";
}

std::string write_x_bin(const std::string &path, const std::vector<float> &x) {
    std::string e = make_parent(path);
    if (!e.empty()) return e;
    FILE *fp = fopen(path.c_str(), "wb");
    if (!fp) return "create " + path + ": " + os_error(errno);
    const uint32_t n = (uint32_t)x.size();
    bool ok = fwrite(&n, 4, 1, fp) == 1;
    if (ok && n) ok = fwrite(x.data(), 4, n, fp) == n;
    const int err = errno;
    ok = (fclose(fp) == 0) && ok;
    if (!ok) return os_error(err);
    return "";
}

std::string write_text_file(const std::string &path, const std::string &text) {
    std::string e = make_parent(path);
    if (!e.empty()) return e;
    FILE *fp = fopen(path.c_str(), "wb");
    if (!fp) return "write " + path + ": " + os_error(errno);
    bool ok = fwrite(text.data(), 1, text.size(), fp) == text.size();
    const int err = errno;
    ok = (fclose(fp) == 0) && ok;
    if (!ok) return "write " + path + ": " + os_error(err);
    return "";
}

// ---------------------------------------------------------------------------
// Number formatting
// ---------------------------------------------------------------------------
// The shortest digit string that reads back to the same value: printf's
// %.*e rounds correctly, so the first precision that round-trips gives the
// shortest correctly rounded digits.
template <class T>
static void shortest_digits(T v, int max_prec, std::string *digits, int *point) {
    char buf[64];
    for (int p = 0; p <= max_prec; ++p) {
        snprintf(buf, sizeof buf, "%.*e", p, (double)v);
        const T back = sizeof(T) == 4 ? (T)strtof(buf, nullptr) : (T)strtod(buf, nullptr);
        if (back == v) break;
    }
    // buf = [-]d[.ddd]e[+-]XX
    const char *s = buf[0] == '-' ? buf + 1 : buf;
    std::string d;
    const char *q = s;
    for (; *q && *q != 'e'; ++q)
        if (*q != '.') d += *q;
    const int e10 = atoi(q + 1);
    while (d.size() > 1 && d.back() == '0') d.pop_back();
    *digits = d;
    *point = e10 + 1;  // value = 0.d1d2... * 10^point
}

void shortest_digits_f32(float v, std::string *d, int *p) { shortest_digits<float>(std::fabs(v), 9, d, p); }
void shortest_digits_f64(double v, std::string *d, int *p) { shortest_digits<double>(std::fabs(v), 17, d, p); }

// Plain positional notation from digits and point.
static std::string positional(const std::string &d, int point) {
    std::string out;
    const int len = (int)d.size();
    if (point <= 0) {
        out = "0." + std::string(-point, '0') + d;
    } else if (point >= len) {
        out = d + std::string(point - len, '0');
    } else {
        out = d.substr(0, point) + "." + d.substr(point);
    }
    return out;
}

std::string rust_display_f32(float v) {
    if (std::isnan(v)) return "NaN";
    if (std::isinf(v)) return v < 0 ? "-inf" : "inf";
    const std::string sign = std::signbit(v) ? "-" : "";
    if (v == 0.f) return sign + "0";
    std::string d;
    int p;
    shortest_digits_f32(v, &d, &p);
    return sign + positional(d, p);
}

std::string rust_debug_f32(float v) {
    if (std::isnan(v) || std::isinf(v)) return rust_display_f32(v);
    const std::string sign = std::signbit(v) ? "-" : "";
    if (v == 0.f) return sign + "0.0";
    const float a = std::fabs(v);
    std::string d;
    int p;
    shortest_digits_f32(v, &d, &p);
    if (a >= 1e-4f && a < 1e16f) {
        std::string s = positional(d, p);
        if (s.find('.') == std::string::npos) s += ".0";
        return sign + s;
    }
    std::string m = d.substr(0, 1);
    if (d.size() > 1) m += "." + d.substr(1);
    return sign + m + "e" + std::to_string(p - 1);
}

std::string rust_exp(double v, int prec) {
    if (std::isnan(v)) return "NaN";
    if (std::isinf(v)) return v < 0 ? "-inf" : "inf";
    char buf[64];
    snprintf(buf, sizeof buf, "%.*e", prec, v);
    std::string s(buf);
    const size_t e = s.find('e');
    const int x = atoi(s.c_str() + e + 1);
    return s.substr(0, e + 1) + std::to_string(x);
}

// ryu's notation (serde_json): decimal when the point falls in a window,
// else d.ddde<exp>. `hi` is 13 for f32 and 16 for f64, `lo` -6 / -5.
static std::string ryu_like(const std::string &d, int point, int hi, int lo) {
    const int len = (int)d.size();
    const int k = point - len;  // value = d * 10^k
    if (k >= 0 && point <= hi) return d + std::string(k, '0') + ".0";
    if (point > 0 && point <= hi) return d.substr(0, point) + "." + d.substr(point);
    if (point > lo && point <= 0) return "0." + std::string(-point, '0') + d;
    std::string m = d.substr(0, 1);
    if (len > 1) m += "." + d.substr(1);
    return m + "e" + std::to_string(point - 1);
}

std::string json_f32(float v) {
    if (!std::isfinite(v)) return "null";
    const std::string sign = std::signbit(v) ? "-" : "";
    if (v == 0.f) return sign + "0.0";
    std::string d;
    int p;
    shortest_digits_f32(v, &d, &p);
    return sign + ryu_like(d, p, 13, -6);
}

std::string json_f64(double v) {
    if (!std::isfinite(v)) return "null";
    const std::string sign = std::signbit(v) ? "-" : "";
    if (v == 0.0) return sign + "0.0";
    std::string d;
    int p;
    shortest_digits_f64(v, &d, &p);
    return sign + ryu_like(d, p, 16, -5);
}

std::string json_str(const std::string &s) {
    std::string out = "\"";
    for (unsigned char c : s) {
        switch (c) {
            case '"': out += "\\\""; break;
            case '\\': out += "\\\\"; break;
            case '\n': out += "\\n"; break;
            case '\r': out += "\\r"; break;
            case '\t': out += "\\t"; break;
            case '\b': out += "\\b"; break;
            case '\f': out += "\\f"; break;
            default:
                if (c < 0x20) {
                    char b[8];
                    snprintf(b, sizeof b, "\\u%04x", c);
                    out += b;
                } else {
                    out += (char)c;
                }
        }
    }
    return out + "\"";
}

std::string now_utc_rfc3339() {
    timespec ts{};
    clock_gettime(CLOCK_REALTIME, &ts);
    tm t{};
    gmtime_r(&ts.tv_sec, &t);
    char buf[64];
    strftime(buf, sizeof buf, "%Y-%m-%dT%H:%M:%S", &t);
    std::string s(buf);
    if (ts.tv_nsec) {
        char ns[16];
        snprintf(ns, sizeof ns, "%09ld", ts.tv_nsec);
        std::string f(ns);
        while (!f.empty() && f.back() == '0') f.pop_back();
        s += "." + f;
    }
    return s + "Z";
}

double true_relres_f64(const CsrMatrixBin &a, const std::vector<float> &b, const std::vector<float> &x) {
    double rr = 0.0, bb = 0.0;
    for (uint32_t i = 0; i < a.n_rows; ++i) {
        double ax = 0.0;
        for (uint32_t k = a.row_ptr[i]; k < a.row_ptr[i + 1]; ++k)
            ax += (double)a.values[k] * (double)x[a.col_idx[k]];
        const double r = (double)b[i] - ax;
        rr += r * r;
        bb += (double)b[i] * (double)b[i];
    }
    return bb > 0.0 ? std::sqrt(rr / bb) : 0.0;
}

uint64_t pcg_iteration_bytes_csr(uint64_t n, uint64_t nnz, uint64_t num_blocks) {
    return 8 * nnz + 4 * (n + 1) + 8 * n + 28 * n + 12 * n + 144 * num_blocks;
}

}  // namespace wsbcli
