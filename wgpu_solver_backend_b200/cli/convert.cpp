// wgpu_solver_backend_convert_cli: `text-to-bin` converts a dataset text
// bundle (sections n, nnz, row_ptr_u32, col_idx_u32, values_f32, b_f32,
// x0_f32, block_starts_u32, optional x_ref_f32) into a case directory with
// matrix.csr.bin, rhs.bin, x0.bin, block_starts.bin, x_ref.bin and meta.json.
// Parsing rules, validation messages and output bytes follow
// crates/wgpu_solver_backend_convert_cli/src/main.rs (104-401 parse,
// 407-494 write). A failure prints `Error: "<message>"` and exits 1, as a
// Rust main returning Err(String) does.
#include <cerrno>
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <optional>
#include <string>
#include <vector>

#include "cli_common.h"

using namespace wsbcli;
namespace fs = std::filesystem;

namespace {

struct Fail {
    std::string msg;
};

std::string trim(const std::string &s) {
    size_t a = 0, b = s.size();
    while (a < b && isspace((unsigned char)s[a])) ++a;
    while (b > a && isspace((unsigned char)s[b - 1])) --b;
    return s.substr(a, b - a);
}

bool ends_with(const std::string &s, const char *suf) {
    const size_t k = strlen(suf);
    return s.size() >= k && s.compare(s.size() - k, k, suf) == 0;
}

struct Reader {
    std::ifstream in;
    // Next non-empty, non-comment line (trimmed); false at EOF.
    bool next_data_line(std::string *out) {
        std::string line;
        while (std::getline(in, line)) {
            line = trim(line);
            if (line.empty() || line[0] == '#') continue;
            *out = line;
            return true;
        }
        return false;
    }
    bool raw_line(std::string *out) {
        std::string line;
        if (!std::getline(in, line)) return false;
        *out = trim(line);
        return true;
    }
};

bool header_like(const std::string &l) {
    return l.rfind("n ", 0) == 0 || l.rfind("nnz ", 0) == 0 || ends_with(l, "_u32") || ends_with(l, "_f32");
}

// Rust's usize / u32 / f32 `parse`: the whole token must be a number.
bool parse_usize(const std::string &t, uint64_t *v) {
    if (t.empty()) return false;
    size_t i = t[0] == '+' ? 1 : 0;
    if (i == t.size()) return false;
    uint64_t x = 0;
    for (; i < t.size(); ++i) {
        if (t[i] < '0' || t[i] > '9') return false;
        const uint64_t d = (uint64_t)(t[i] - '0');
        if (x > (UINT64_MAX - d) / 10) return false;
        x = x * 10 + d;
    }
    *v = x;
    return true;
}

bool parse_u32(const std::string &t, uint32_t *v) {
    uint64_t x;
    if (!parse_usize(t, &x) || x > 0xffffffffull) return false;
    *v = (uint32_t)x;
    return true;
}

bool parse_f32(const std::string &t, float *v) {
    if (t.empty()) return false;
    // Rust accepts decimal and exponent forms, "inf"/"infinity"/"nan" (any
    // case) with an optional sign, but no hexadecimal floats.
    for (char c : t)
        if (c == 'x' || c == 'X' || c == 'p' || c == 'P') return false;
    char *end = nullptr;
    errno = 0;
    const float f = strtof(t.c_str(), &end);
    if (end != t.c_str() + t.size()) return false;
    *v = f;
    return true;
}

uint64_t parse_len_line(const std::string &line, const std::string &section) {
    if (line.rfind("len ", 0) != 0) throw Fail{"Section " + section + ": expected 'len N', got '" + line + "'"};
    const std::string rest = line.substr(4);
    uint64_t v;
    if (!parse_usize(rest, &v)) throw Fail{"Section " + section + ": bad len '" + rest + "': invalid digit found in string"};
    return v;
}

template <class T, class P>
std::vector<T> read_tokens(Reader &r, const std::string &section, uint64_t need, P parse_tok, const char *ty) {
    std::vector<T> out;
    out.reserve(need);
    std::string line;
    while (out.size() < need) {
        if (!r.raw_line(&line))
            throw Fail{"Section " + section + ": EOF while reading values (got " + std::to_string(out.size()) +
                       ", need " + std::to_string(need) + ")"};
        if (line.empty() || line[0] == '#') continue;
        if (header_like(line))
            throw Fail{"Section " + section + ": hit unexpected header '" + line + "' before collecting len=" +
                       std::to_string(need) + " values"};
        size_t p = 0;
        while (p < line.size() && out.size() < need) {
            while (p < line.size() && isspace((unsigned char)line[p])) ++p;
            if (p >= line.size()) break;
            size_t q = p;
            while (q < line.size() && !isspace((unsigned char)line[q])) ++q;
            const std::string tok = line.substr(p, q - p);
            T v;
            if (!parse_tok(tok, &v))
                throw Fail{"Section " + section + ": failed to parse " + ty + " token '" + tok + "': " +
                           (ty[0] == 'f' ? "invalid float literal" : "invalid digit found in string")};
            out.push_back(v);
            p = q;
        }
    }
    return out;
}

struct Dataset {
    uint64_t n = 0, nnz = 0;
    std::vector<uint32_t> row_ptr, col_idx, block_starts;
    std::vector<float> values, b, x0, x_ref;
    bool has_x_ref = false;
};

Dataset parse_dataset(const std::string &path) {
    Reader r;
    r.in.open(path);
    if (!r.in) throw Fail{"Failed to open " + path + ": " + os_error(errno)};
    std::optional<uint64_t> n, nnz;
    std::optional<std::vector<uint32_t>> row_ptr, col_idx, block_starts;
    std::optional<std::vector<float>> values, b, x0, x_ref;
    std::string line;
    auto u32s = [&](const std::string &sec, uint64_t len) {
        return read_tokens<uint32_t>(r, sec, len, parse_u32, "u32");
    };
    auto f32s = [&](const std::string &sec, uint64_t len) {
        return read_tokens<float>(r, sec, len, parse_f32, "f32");
    };
    while (r.next_data_line(&line)) {
        if (line.rfind("n ", 0) == 0) {
            uint64_t v;
            if (!parse_usize(line.substr(2), &v)) throw Fail{"Bad n: invalid digit found in string"};
            n = v;
            continue;
        }
        if (line.rfind("nnz ", 0) == 0) {
            uint64_t v;
            if (!parse_usize(line.substr(4), &v)) throw Fail{"Bad nnz: invalid digit found in string"};
            nnz = v;
            continue;
        }
        const std::string section = line;
        std::string len_line;
        if (!r.next_data_line(&len_line)) throw Fail{"Section " + section + ": missing len line (EOF)"};
        const uint64_t len = parse_len_line(len_line, section);
        if (section == "row_ptr_u32") row_ptr = u32s(section, len);
        else if (section == "col_idx_u32") col_idx = u32s(section, len);
        else if (section == "values_f32") values = f32s(section, len);
        else if (section == "b_f32") b = f32s(section, len);
        else if (section == "x0_f32") x0 = f32s(section, len);
        else if (section == "block_starts_u32") block_starts = u32s(section, len);
        else if (section == "x_ref_f32") x_ref = f32s(section, len);
        else {
            fprintf(stderr, "Warning: skipping unknown section: %s (len %llu)\n", section.c_str(),
                    (unsigned long long)len);
            uint64_t skipped = 0;
            std::string l;
            while (skipped < len) {
                if (!r.raw_line(&l))
                    throw Fail{"Section " + section + ": EOF while skipping values (skipped " +
                               std::to_string(skipped) + ", need " + std::to_string(len) + ")"};
                if (l.empty() || l[0] == '#') continue;
                if (header_like(l))
                    throw Fail{"Section " + section + ": hit unexpected header '" + l + "' before skipping len=" +
                               std::to_string(len) + " tokens"};
                size_t p = 0;
                while (p < l.size()) {
                    while (p < l.size() && isspace((unsigned char)l[p])) ++p;
                    if (p >= l.size()) break;
                    ++skipped;
                    while (p < l.size() && !isspace((unsigned char)l[p])) ++p;
                }
            }
        }
    }
    if (!n) throw Fail{"Missing 'n'"};
    if (!nnz) throw Fail{"Missing 'nnz'"};
    if (!row_ptr) throw Fail{"Missing row_ptr_u32"};
    if (!col_idx) throw Fail{"Missing col_idx_u32"};
    if (!values) throw Fail{"Missing values_f32"};
    if (!b) throw Fail{"Missing b_f32"};
    if (!x0) throw Fail{"Missing x0_f32"};
    if (!block_starts) throw Fail{"Missing block_starts_u32"};
    Dataset d;
    d.n = *n;
    d.nnz = *nnz;
    d.row_ptr = std::move(*row_ptr);
    d.col_idx = std::move(*col_idx);
    d.values = std::move(*values);
    d.b = std::move(*b);
    d.x0 = std::move(*x0);
    d.block_starts = std::move(*block_starts);
    if (x_ref) {
        d.x_ref = std::move(*x_ref);
        d.has_x_ref = true;
    }
    const auto S = [](uint64_t v) { return std::to_string(v); };
    if (d.row_ptr.size() != d.n + 1)
        throw Fail{"row_ptr_u32 len must be n+1 (" + S(d.n + 1) + "), got " + S(d.row_ptr.size())};
    if (d.col_idx.size() != d.nnz || d.values.size() != d.nnz)
        throw Fail{"col_idx/values len must be nnz (" + S(d.nnz) + "), got col_idx=" + S(d.col_idx.size()) +
                   ", values=" + S(d.values.size())};
    if (d.b.size() != d.n || d.x0.size() != d.n)
        throw Fail{"b/x0 len must be n (" + S(d.n) + "), got b=" + S(d.b.size()) + ", x0=" + S(d.x0.size())};
    if (d.has_x_ref && d.x_ref.size() != d.n)
        throw Fail{"x_ref_f32 len must be n (" + S(d.n) + "), got " + S(d.x_ref.size())};
    if (d.block_starts.empty()) throw Fail{"block_starts_u32 must not be empty"};
    if (d.block_starts[0] != 0) throw Fail{"block_starts_u32 must start with 0, got " + S(d.block_starts[0])};
    if (d.block_starts.back() != (uint32_t)d.n)
        throw Fail{"block_starts_u32 must end with n (" + S(d.n) + "), got " + S(d.block_starts.back())};
    for (size_t i = 1; i < d.block_starts.size(); ++i)
        if (d.block_starts[i] <= d.block_starts[i - 1]) throw Fail{"block_starts_u32 must be strictly increasing"};
    return d;
}

void put_u32(std::string &s, uint32_t v) { s.append(reinterpret_cast<const char *>(&v), 4); }
template <class T>
void put_all(std::string &s, const std::vector<T> &v) {
    if (!v.empty()) s.append(reinterpret_cast<const char *>(v.data()), 4 * v.size());
}

void write_file(const fs::path &p, const std::string &bytes, const char *name) {
    FILE *fp = fopen(p.c_str(), "wb");
    if (!fp) throw Fail{std::string("Failed to create ") + name + ": " + os_error(errno)};
    const bool ok = fwrite(bytes.data(), 1, bytes.size(), fp) == bytes.size();
    const int err = errno;
    if (fclose(fp) != 0 || !ok) throw Fail{std::string("Failed to write ") + name + ": " + os_error(err)};
}

void write_bins(const Dataset &d, const fs::path &out, bool force) {
    std::error_code ec;
    if (fs::exists(out)) {
        if (!force) throw Fail{"Output dir " + out.string() + " already exists. Use --force to overwrite."};
        fs::remove_all(out, ec);
        if (ec) throw Fail{"Failed to remove " + out.string() + ": " + os_error(ec.value())};
    }
    fs::create_directories(out, ec);
    if (ec) throw Fail{"Failed to create " + out.string() + ": " + os_error(ec.value())};
    std::string m;
    put_u32(m, kMagicCsr1);
    put_u32(m, 1);
    put_u32(m, (uint32_t)d.n);
    put_u32(m, (uint32_t)d.n);
    put_u32(m, (uint32_t)d.nnz);
    put_u32(m, 0);
    put_u32(m, 0);
    put_u32(m, 0);
    put_all(m, d.row_ptr);
    put_all(m, d.col_idx);
    put_all(m, d.values);
    write_file(out / "matrix.csr.bin", m, "matrix.csr.bin");
    auto vec_file = [&](const char *name, const std::vector<float> &v) {
        std::string s;
        put_u32(s, (uint32_t)d.n);
        put_all(s, v);
        write_file(out / name, s, name);
    };
    vec_file("rhs.bin", d.b);
    vec_file("x0.bin", d.x0);
    std::string bs;
    put_u32(bs, (uint32_t)d.block_starts.size());
    put_all(bs, d.block_starts);
    write_file(out / "block_starts.bin", bs, "block_starts.bin");
    if (d.has_x_ref) vec_file("x_ref.bin", d.x_ref);
    const auto S = [](uint64_t v) { return std::to_string(v); };
    std::string meta = "{\n";
    meta += "  \"format\": \"wgpu-solver-backend-text-v0\",\n";
    meta += "  \"n\": " + S(d.n) + ",\n";
    meta += "  \"nnz\": " + S(d.nnz) + ",\n";
    meta += "  \"row_ptr_len\": " + S(d.row_ptr.size()) + ",\n";
    meta += "  \"col_idx_len\": " + S(d.col_idx.size()) + ",\n";
    meta += "  \"values_len\": " + S(d.values.size()) + ",\n";
    meta += "  \"rhs_len\": " + S(d.b.size()) + ",\n";
    meta += "  \"x0_len\": " + S(d.x0.size()) + ",\n";
    meta += "  \"block_starts_len\": " + S(d.block_starts.size()) + ",\n";
    meta += std::string("  \"x_ref_present\": ") + (d.has_x_ref ? "true" : "false") + "\n}";
    write_file(out / "meta.json", meta, "meta.json");
}

std::string debug_str(const std::string &s) {
    // Rust's Debug of a String: quoted, with \" \\ \n \t \r escaped.
    std::string o = "\"";
    for (char c : s) {
        if (c == '"') o += "\\\"";
        else if (c == '\\') o += "\\\\";
        else if (c == '\n') o += "\\n";
        else if (c == '\t') o += "\\t";
        else if (c == '\r') o += "\\r";
        else o += c;
    }
    return o + "\"";
}

}  // namespace

int main(int argc, char **argv) {
    std::string cmd, input, out_dir;
    bool force = false, have_in = false, have_out = false;
    for (int i = 1; i < argc; ++i) {
        std::string s = argv[i];
        if (s == "-h" || s == "--help") {
            printf("Converters for wgpu-solver-backend datasets (text -> bin)\n\n"
                   "Usage: wgpu_solver_backend_convert_cli text-to-bin --input <INPUT> --out-dir <OUT_DIR> [--force]\n");
            return 0;
        }
        if (s == "--force") {
            force = true;
            continue;
        }
        if (s.rfind("--input", 0) == 0 || s.rfind("--out-dir", 0) == 0) {
            const size_t eq = s.find('=');
            std::string v;
            if (eq != std::string::npos) v = s.substr(eq + 1);
            else if (i + 1 < argc) v = argv[++i];
            else {
                fprintf(stderr, "error: a value is required for '%s <VALUE>' but none was supplied\n", s.c_str());
                return 2;
            }
            if (s.rfind("--input", 0) == 0) input = v, have_in = true;
            else out_dir = v, have_out = true;
            continue;
        }
        if (cmd.empty() && s.rfind("-", 0) != 0) {
            cmd = s;
            continue;
        }
        fprintf(stderr, "error: unexpected argument '%s' found\n", s.c_str());
        return 2;
    }
    if (cmd != "text-to-bin") {
        fprintf(stderr, cmd.empty() ? "error: a subcommand is required\n" : "error: unrecognized subcommand '%s'\n",
                cmd.c_str());
        return 2;
    }
    if (!have_in || !have_out) {
        fprintf(stderr, "error: the following required arguments were not provided:%s%s\n",
                have_in ? "" : "\n  --input <INPUT>", have_out ? "" : "\n  --out-dir <OUT_DIR>");
        return 2;
    }
    try {
        const Dataset d = parse_dataset(input);
        write_bins(d, fs::path(out_dir), force);
        printf("Wrote binaries into %s\n", out_dir.c_str());
    } catch (const Fail &f) {
        fprintf(stderr, "Error: %s\n", debug_str(f.msg).c_str());
        return 1;
    }
    return 0;
}
