// wgpu_solver_backend_cli: the command-line front end of the solver, with the
// subcommands, flags, output text, metrics JSON and exit codes of the
// reference CLI (crates/wgpu_solver_backend_cli/src/main.rs), running on the
// CUDA library through its C ABI (include/wsb.h).
//
//   [--backend auto|vulkan|dx12|metal] [--device N] <command> [flags]
//   info | vec-test | dot-test | spmv-test | block-jacobi-test |
//   pcg-update-scalars-test | run-pcg-case ... | compare-x ...
//
// --backend is accepted for compatibility (main.rs:31-32, 151-162); every
// value runs on the CUDA device. Exit codes: 2 for a failed context, a
// failed write or a failed compare-x (main.rs:735-890) and for usage errors;
// 101 when a sanity check's assertion fails (a Rust panic). run-pcg-case
// exits 0 after a failed solve and reports it in the metrics (main.rs:807-877).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "../../include/wsb.h"
#include "cli_common.h"

using namespace wsbcli;

namespace {

const char *kVersion = "0.1.0";

struct Args {
    std::string backend = "auto";
    int device = 0;
    std::string cmd;
    std::map<std::string, std::string> kv;
};

[[noreturn]] void usage_error(const std::string &msg) {
    fprintf(stderr, "error: %s\n\nFor more information, try '--help'.\n", msg.c_str());
    exit(2);
}

void print_help() {
    printf(
        "Compute-first solver backend for iterative solvers (CUDA sm_100a)\n\n"
        "Usage: wgpu_solver_backend_cli [OPTIONS] <COMMAND>\n\n"
        "Commands:\n"
        "  info                     Print GPU adapter info and emit a metrics JSON blob (stdout)\n"
        "  vec-test                 Sanity test for vec ops (AXPY): y = y + alpha * x\n"
        "  dot-test\n"
        "  spmv-test\n"
        "  block-jacobi-test\n"
        "  pcg-update-scalars-test\n"
        "  run-pcg-case             Run PCG(Block-Jacobi) on a case directory\n"
        "  compare-x                Compare two solution vectors stored in .bin format (u32 len + f32[len])\n\n"
        "Options:\n"
        "      --backend <BACKEND>  [default: auto] (accepted; the solver runs on CUDA)\n"
        "      --device <N>         CUDA device ordinal [default: 0]\n"
        "  -h, --help               Print help\n"
        "  -V, --version            Print version\n\n"
        "run-pcg-case: --case-dir DIR --out-x PATH --out-metrics PATH [--max-iters 2000]\n"
        "              [--rel-tol 1e-8] [--abs-tol 0] [--precision f32-f64dot|reference-f32|mixed]\n"
        "              [--target-relres 1e-10] [--layout executors|auto|csr|bsr6] [--out-history PATH]\n"
        "              [--algorithm classic|single-reduction]\n"
        "              [--hbm-peak-gbs 7700]\n"
        "compare-x:    --x-ref PATH --x PATH [--rel-tol 1e-3] [--abs-tol 1e-4] [--top-k 10]\n");
}

Args parse(int argc, char **argv) {
    Args a;
    auto take = [&](int &i, const std::string &flag) -> std::string {
        const std::string s = argv[i];
        const size_t eq = s.find('=');
        if (eq != std::string::npos) return s.substr(eq + 1);
        if (i + 1 >= argc) usage_error("a value is required for '" + flag + " <VALUE>' but none was supplied");
        return argv[++i];
    };
    for (int i = 1; i < argc; ++i) {
        std::string s = argv[i];
        if (s == "-h" || s == "--help") {
            print_help();
            exit(0);
        }
        if (s == "-V" || s == "--version") {
            printf("wgpu-solver-backend %s\n", kVersion);
            exit(0);
        }
        if (s.rfind("--", 0) == 0) {
            std::string flag = s.substr(0, s.find('='));
            const std::string v = take(i, flag);
            flag = flag.substr(2);
            if (flag == "backend") a.backend = v;
            else if (flag == "device") a.device = atoi(v.c_str());
            else if (a.cmd.empty()) usage_error("unexpected argument '" + s + "' found");
            else a.kv[flag] = v;
            continue;
        }
        if (!a.cmd.empty()) usage_error("unexpected argument '" + s + "' found");
        a.cmd = s;
    }
    if (a.cmd.empty()) {
        print_help();
        exit(2);
    }
    return a;
}

// parse_backend, main.rs:151-162: unknown names warn and fall back to auto.
void check_backend(const std::string &b) {
    std::string l = b;
    for (auto &c : l) c = (char)tolower(c);
    if (l != "auto" && l != "vulkan" && l != "dx12" && l != "metal" && l != "cuda")
        fprintf(stderr, "Unknown backend '%s', using auto\n", l.c_str());
}

wsb_context *context_or_exit(int device) {
    wsb_context *ctx = nullptr;
    if (wsb_context_create(device, &ctx) != WSB_OK) {
        fprintf(stderr, "Failed to init GPU context: %s\n", wsb_last_error(nullptr));
        exit(2);
    }
    return ctx;
}

[[noreturn]] void panic(const std::string &msg) {
    fprintf(stderr, "thread 'main' panicked:\n%s\n", msg.c_str());
    exit(101);
}

void check(wsb_context *ctx, int rc, const char *what) {
    if (rc != WSB_OK) panic(std::string(what) + ": " + wsb_last_error(ctx));
}

struct Buf {
    wsb_buffer *b = nullptr;
    ~Buf() { wsb_buffer_destroy(b); }
};

std::vector<float> read_floats(wsb_context *ctx, const wsb_buffer *b, size_t n) {
    std::vector<float> out(n);
    check(ctx, wsb_buffer_read(ctx, b, 0, out.data(), n * sizeof(float)), "readback");
    return out;
}

// ---- sanity subcommands (main.rs:171-443) -----------------------------------
void run_vec_test(wsb_context *ctx) {
    const uint32_t n = 1024;
    const float alpha = 3.0f;
    std::vector<float> xh(n, 2.0f), yh(n, 1.0f);
    Buf x, y;
    check(ctx, wsb_buffer_create(ctx, xh.data(), n * 4, &x.b), "x");
    check(ctx, wsb_buffer_create(ctx, yh.data(), n * 4, &y.b), "y");
    check(ctx, wsb_vec_axpy_inplace(ctx, x.b, y.b, n, alpha), "axpy");
    const std::vector<float> out = read_floats(ctx, y.b, n);
    const float expected = 1.0f + alpha * 2.0f;
    for (uint32_t i = 0; i < n; ++i)
        if (!(std::fabs(out[i] - expected) < 1e-6f))
            panic("vec-test failed at i=" + std::to_string(i) + ": got " + rust_display_f32(out[i]) + ", expected " +
                  rust_display_f32(expected));
    printf("VecTest OK: all y[i] == %s\n", rust_display_f32(expected).c_str());
}

void run_dot_test(wsb_context *ctx) {
    const float a[3] = {1, 2, 3}, b[3] = {4, 5, 6};
    Buf ab, bb;
    check(ctx, wsb_buffer_create(ctx, a, sizeof a, &ab.b), "a");
    check(ctx, wsb_buffer_create(ctx, b, sizeof b, &bb.b), "b");
    wsb_dot_scalar_executor *ex = nullptr;
    check(ctx, wsb_dot_scalar_executor_create(ctx, 3, 4, &ex), "DotScalarExecutor::create");
    check(ctx, wsb_dot_scalar_executor_dot_into(ex, ab.b, bb.b, 3, 0), "dot");
    float s[4];
    check(ctx, wsb_dot_scalar_executor_readback(ex, s, 4), "readback");
    wsb_dot_scalar_executor_destroy(ex);
    const float got = s[0], expected = 32.0f;
    if (!(std::fabs(got - expected) < 1e-5f))
        panic("dot-test failed: got " + rust_display_f32(got) + ", expected " + rust_display_f32(expected));
    printf("DotTest OK: got %s\n", rust_display_f32(got).c_str());
}

void run_spmv_test(wsb_context *ctx) {
    const uint32_t n = 3;
    const uint32_t row_ptr[4] = {0, 2, 4, 6}, col[6] = {0, 2, 0, 1, 1, 2};
    const float val[6] = {10, 2, 3, 9, 7, 8}, xh[3] = {1, 2, 3}, expected[3] = {16, 21, 38};
    Buf x, y;
    check(ctx, wsb_buffer_create(ctx, xh, sizeof xh, &x.b), "x");
    check(ctx, wsb_buffer_create(ctx, nullptr, sizeof xh, &y.b), "y");
    wsb_spmv_executor *ex = nullptr;
    check(ctx, wsb_spmv_executor_create(ctx, n, row_ptr, col, val, 6, &ex), "SpmvExecutor::create");
    check(ctx, wsb_spmv_executor_spmv(ex, x.b, y.b), "spmv");
    const std::vector<float> out = read_floats(ctx, y.b, n);
    wsb_spmv_executor_destroy(ex);
    for (uint32_t i = 0; i < n; ++i)
        if (!(std::fabs(out[i] - expected[i]) < 1e-6f))
            panic("spmv-test failed at i=" + std::to_string(i) + ": got " + rust_display_f32(out[i]) + ", expected " +
                  rust_display_f32(expected[i]));
    std::string list = "[";
    for (uint32_t i = 0; i < n; ++i) list += (i ? ", " : "") + rust_debug_f32(out[i]);
    printf("SpmvTest OK: y == %s]\n", list.c_str());
}

void run_block_jacobi_test(wsb_context *ctx) {
    const uint32_t n = 12;
    const uint32_t bs[3] = {0, 6, 12};
    std::vector<float> lu(72, 0.0f);
    for (int b = 0; b < 2; ++b)
        for (int i = 0; i < 6; ++i) lu[b * 36 + i * 6 + i] = 1.0f;
    std::vector<float> r(n);
    for (uint32_t i = 0; i < n; ++i) r[i] = (float)(i + 1);
    Buf rb, zb;
    check(ctx, wsb_buffer_create(ctx, r.data(), n * 4, &rb.b), "r");
    check(ctx, wsb_buffer_create(ctx, nullptr, n * 4, &zb.b), "z");
    wsb_block_jacobi_executor *bj = nullptr;
    check(ctx, wsb_block_jacobi_executor_create(ctx, n, lu.data(), lu.size(), bs, 3, &bj),
          "BlockJacobiExecutor::create");
    check(ctx, wsb_block_jacobi_executor_apply(bj, rb.b, zb.b), "apply");
    const std::vector<float> z = read_floats(ctx, zb.b, n);
    wsb_block_jacobi_executor_destroy(bj);
    for (uint32_t i = 0; i < n; ++i)
        if (!(std::fabs(z[i] - r[i]) < 1e-6f))
            panic("block-jacobi-test failed at i=" + std::to_string(i) + ": got " + rust_display_f32(z[i]) +
                  ", expected " + rust_display_f32(r[i]));
    printf("BlockJacobiTest OK: z == r (identity blocks)\n");
}

void run_pcg_update_scalars_test(wsb_context *ctx) {
    // Mailbox layout of main.rs:378-383.
    const uint32_t PAP = 0, RZ_NEW = 1, RZ_OLD = 2, ALPHA = 3, MINUS_ALPHA = 4, BETA = 5;
    std::vector<float> host(8, 0.0f);
    host[PAP] = 2.0f;
    host[RZ_OLD] = 10.0f;
    host[RZ_NEW] = 5.0f;
    Buf s;
    check(ctx, wsb_buffer_create(ctx, host.data(), host.size() * 4, &s.b), "scalars");
    check(ctx, wsb_pcg_update_scalars(ctx, s.b, PAP, RZ_NEW, RZ_OLD, ALPHA, MINUS_ALPHA, BETA), "update_scalars");
    const std::vector<float> out = read_floats(ctx, s.b, 8);
    const float alpha = out[ALPHA], minus_alpha = out[MINUS_ALPHA], beta = out[BETA];
    const float ea = 10.0f / 2.0f, ema = -ea, eb = 5.0f / 10.0f, eps = 1e-6f;
    if (!(std::fabs(alpha - ea) < eps)) panic("alpha got " + rust_display_f32(alpha) + ", expected " + rust_display_f32(ea));
    if (!(std::fabs(minus_alpha - ema) < eps))
        panic("minus_alpha got " + rust_display_f32(minus_alpha) + ", expected " + rust_display_f32(ema));
    if (!(std::fabs(beta - eb) < eps)) panic("beta got " + rust_display_f32(beta) + ", expected " + rust_display_f32(eb));
    printf("PcgUpdateScalarsTest OK: alpha=%s, minus_alpha=%s, beta=%s\n", rust_display_f32(alpha).c_str(),
           rust_display_f32(minus_alpha).c_str(), rust_display_f32(beta).c_str());
}

// ---- metrics JSON (main.rs:95-149), pretty-printed as serde_json does -------
struct Json {
    std::string s;
    int depth = 0;
    bool first = true;
    void open() {
        s += "{";
        ++depth;
        first = true;
    }
    void close() {
        --depth;
        s += "\n" + std::string(2 * depth, ' ') + "}";
        first = false;
    }
    void key(const char *k) {
        s += (first ? "\n" : ",\n") + std::string(2 * depth, ' ') + json_str(k) + ": ";
        first = false;
    }
    void raw(const char *k, const std::string &v) {
        key(k);
        s += v;
    }
    void obj(const char *k) {
        key(k);
        open();
    }
};

void gpu_metrics(Json &j, const wsb_adapter_info &ai) {
    j.obj("gpu");
    j.raw("adapter_name", json_str(ai.name));
    j.raw("backend", json_str(ai.backend));
    j.raw("device_type", json_str(ai.device_type));
    j.raw("vendor", std::to_string(ai.vendor));
    j.raw("device", std::to_string(ai.device));
    j.close();
}

void build_metrics(Json &j) {
    j.obj("build");
    j.raw("crate_version", json_str(kVersion));
#ifdef WSB_GIT_REV
    j.raw("git_rev", json_str(WSB_GIT_REV));
#else
    j.raw("git_rev", "null");
#endif
    j.close();
}

int cmd_info(const Args &a) {
    wsb_context *ctx = context_or_exit(a.device);
    char desc[512];
    wsb_context_describe(ctx, desc, sizeof desc);
    printf("%s\n", desc);
    wsb_adapter_info ai;
    wsb_context_adapter_info(ctx, &ai);
    Json j;
    j.open();
    j.raw("run_id", json_str(now_utc_rfc3339()));
    j.raw("command", json_str("info"));
    gpu_metrics(j, ai);
    build_metrics(j);
    j.close();
    printf("%s\n", j.s.c_str());
    wsb_context_destroy(ctx);
    return 0;
}

// ---- run-pcg-case (main.rs:477-558, 794-878) --------------------------------
using Clock = std::chrono::steady_clock;
long long ms_since(Clock::time_point t) {
    return std::chrono::duration_cast<std::chrono::milliseconds>(Clock::now() - t).count();
}

std::string get(const Args &a, const char *k, const char *def, bool required = false) {
    auto it = a.kv.find(k);
    if (it != a.kv.end()) return it->second;
    if (required) usage_error(std::string("the following required arguments were not provided:\n  --") + k + " <" + k + ">");
    return def;
}

int parse_precision(const Args &a) {
    const std::string p = get(a, "precision", "f32-f64dot");
    if (p == "f32-f64dot") return WSB_PREC_F32_F64DOT;
    if (p == "reference-f32") return WSB_PREC_REFERENCE_F32;
    if (p == "mixed") return WSB_PREC_MIXED_F64_IR;
    usage_error("invalid value '" + p + "' for '--precision' [possible values: f32-f64dot, reference-f32, mixed]");
}

int parse_algorithm(const Args &a) {
    const std::string p = get(a, "algorithm", "classic");
    if (p == "classic") return WSB_ALG_CLASSIC;
    if (p == "single-reduction") return WSB_ALG_SINGLE_REDUCTION;
    usage_error("invalid value '" + p + "' for '--algorithm' [possible values: classic, single-reduction]");
}

struct SolveOut {
    uint64_t iterations = 0;
    std::vector<float> x;
    uint32_t n = 0, nnz = 0;
    wsb_solve_result res{};
    std::vector<double> history;
    long long load_ms = 0, setup_ms = 0;
    CaseInputBin input;           // the loaded case (kept for the residual check)
    uint64_t iteration_bytes = 0; // algorithmic HBM bytes of one PCG iteration
};

// Loads the case, builds the executors and LU (as run_pcg_case does) and
// solves; returns the error string of the failing step, or "".
std::string run_pcg_case(wsb_context *ctx, const Args &a, uint64_t max_iters, float rel, float abs_tol,
                         SolveOut *o) {
    const auto t_load = Clock::now();
    CaseInputBin &c = o->input;
    std::string e = load_case_dir(get(a, "case-dir", ""), &c);
    o->load_ms = ms_since(t_load);
    if (!e.empty()) return e;
    const uint32_t n = c.a.n_rows;
    const auto t_setup = Clock::now();
    wsb_solve_opts opts;
    wsb_solve_opts_default(&opts);
    opts.precision = parse_precision(a);
    opts.algorithm = parse_algorithm(a);
    opts.target_relres = atof(get(a, "target-relres", "1e-10").c_str());
    const bool want_hist = a.kv.count("out-history");
    if (want_hist) {
        o->history.resize(max_iters + 1);
        opts.history_out = o->history.data();
        opts.history_capacity = o->history.size();
    }
    const std::string layout = get(a, "layout", "executors");
    o->x = c.x0;
    int rc;
    if (layout == "executors") {
        // SpmvExecutor + LU + BlockJacobiExecutor, then the driver (main.rs:490-552).
        wsb_spmv_executor *spmv = nullptr;
        wsb_block_jacobi_executor *bj = nullptr;
        if ((rc = wsb_spmv_executor_create(ctx, n, c.a.row_ptr.data(), c.a.col_idx.data(), c.a.values.data(), c.a.nnz,
                                           &spmv)))
            return wsb_last_error(ctx);
        std::vector<float> lu((c.block_starts.size() - 1) * 36);
        if ((rc = wsb_build_lu_blocks_from_csr_block_starts_6(n, c.a.row_ptr.data(), c.a.row_ptr.size(),
                                                              c.a.col_idx.data(), c.a.col_idx.size(),
                                                              c.a.values.data(), c.a.values.size(),
                                                              c.block_starts.data(), c.block_starts.size(), lu.data()))) {
            wsb_spmv_executor_destroy(spmv);
            return wsb_last_error(nullptr);
        }
        if ((rc = wsb_block_jacobi_executor_create(ctx, n, lu.data(), lu.size(), c.block_starts.data(),
                                                   c.block_starts.size(), &bj))) {
            wsb_spmv_executor_destroy(spmv);
            return wsb_last_error(ctx);
        }
        o->setup_ms = ms_since(t_setup);
        o->iteration_bytes = pcg_iteration_bytes_csr(n, c.a.nnz, c.block_starts.size() - 1);
        rc = wsb_pcg_block_jacobi_csr(ctx, n, c.b.data(), n, o->x.data(), n, max_iters, rel, abs_tol, spmv, bj, &opts,
                                      &o->iterations, &o->res);
        e = rc ? wsb_last_error(ctx) : "";
        wsb_block_jacobi_executor_destroy(bj);
        wsb_spmv_executor_destroy(spmv);
    } else {
        int32_t lay = WSB_LAYOUT_AUTO;
        if (layout == "csr") lay = WSB_LAYOUT_CSR;
        else if (layout == "bsr6") lay = WSB_LAYOUT_BSR6;
        else if (layout != "auto") usage_error("invalid value '" + layout + "' for '--layout'");
        wsb_matrix *m = nullptr;
        if ((rc = wsb_matrix_create(ctx, n, c.a.row_ptr.data(), c.a.col_idx.data(), c.a.values.data(), c.a.nnz,
                                    c.block_starts.data(), c.block_starts.size(), lay, &m)))
            return wsb_last_error(ctx);
        o->setup_ms = ms_since(t_setup);
        wsb_matrix_info info;
        if (wsb_matrix_info_get(m, &info) == WSB_OK) o->iteration_bytes = info.iteration_bytes;
        rc = wsb_solve(ctx, m, c.b.data(), o->x.data(), max_iters, rel, abs_tol, &opts, &o->res);
        e = rc ? wsb_last_error(ctx) : "";
        o->iterations = o->res.iterations;
        wsb_matrix_destroy(m);
    }
    if (!e.empty()) return e;
    // The single-reduction iteration also reads and writes s = A p.
    if (opts.algorithm == WSB_ALG_SINGLE_REDUCTION) o->iteration_bytes += 4ull * n;
    o->n = n;
    o->nnz = c.a.nnz;
    if (want_hist) o->history.resize(o->res.history_len);
    return "";
}

const char *precision_name(int p) {
    return p == WSB_PREC_REFERENCE_F32 ? "reference-f32" : p == WSB_PREC_MIXED_F64_IR ? "mixed" : "f32-f64dot";
}

int cmd_run_pcg_case(const Args &a) {
    const std::string case_dir = get(a, "case-dir", "", true);
    const std::string out_x = get(a, "out-x", "", true);
    const std::string out_metrics = get(a, "out-metrics", "", true);
    const uint64_t max_iters = strtoull(get(a, "max-iters", "2000").c_str(), nullptr, 10);
    const float rel = strtof(get(a, "rel-tol", "1e-8").c_str(), nullptr);
    const float abs_tol = strtof(get(a, "abs-tol", "0").c_str(), nullptr);
    parse_precision(a);  // usage errors before any work
    parse_algorithm(a);
    const auto t0 = Clock::now();
    const auto t_gpu0 = Clock::now();
    wsb_context *ctx = context_or_exit(a.device);
    const long long gpu_init = ms_since(t_gpu0);
    const auto t_solve0 = Clock::now();
    SolveOut o;
    std::string err = run_pcg_case(ctx, a, max_iters, rel, abs_tol, &o);
    const long long solve_total = ms_since(t_solve0);
    const bool converged = err.empty();
    if (!converged) fprintf(stderr, "Solve failed: %s\n", err.c_str());
    const auto t_write0 = Clock::now();
    if (converged) {
        const std::string we = write_x_bin(out_x, o.x);
        if (!we.empty()) {
            fprintf(stderr, "Failed to write x.bin: %s\n", we.c_str());
            exit(2);
        }
        if (a.kv.count("out-history")) {
            std::string h = "{\"r_norm2\": [";
            for (size_t i = 0; i < o.history.size(); ++i) h += (i ? ", " : "") + json_f64(o.history[i]);
            h += "]}\n";
            const std::string he = write_text_file(a.kv.at("out-history"), h);
            if (!he.empty()) {
                fprintf(stderr, "Failed to write history: %s\n", he.c_str());
                exit(2);
            }
        }
    }
    const long long write_ms = ms_since(t_write0);
    // Host-side checks of the result, outside the timed phases: the true FP64
    // relative residual of x, and the PCG iterations' achieved HBM bandwidth
    // (algorithmic bytes x iterations / device time) against --hbm-peak-gbs.
    const double true_relres = converged ? true_relres_f64(o.input.a, o.input.b, o.x) : NAN;
    const double peak_gbs = atof(get(a, "hbm-peak-gbs", "7700").c_str());
    const double gbps = converged && o.res.device_ms > 0.0
                            ? (double)o.iteration_bytes * (double)o.iterations / (o.res.device_ms * 1e6)
                            : NAN;
    wsb_adapter_info ai;
    wsb_context_adapter_info(ctx, &ai);
    Json j;
    j.open();
    j.raw("run_id", json_str(now_utc_rfc3339()));
    j.raw("command", json_str("run_pcg_case"));
    j.raw("case_dir", json_str(case_dir));
    j.raw("n", std::to_string(o.n));
    j.raw("nnz", std::to_string(o.nnz));
    j.raw("max_iters", std::to_string(max_iters));
    j.raw("rel_tol", json_f32(rel));
    j.raw("abs_tol", json_f32(abs_tol));
    j.raw("iterations", converged ? std::to_string(o.iterations) : "null");
    j.raw("converged", converged ? "true" : "false");
    j.raw("error", converged ? "null" : json_str(err));
    j.obj("timings_ms");
    j.raw("total", std::to_string(ms_since(t0)));
    j.raw("load_io", std::to_string(o.load_ms));
    j.raw("gpu_init", std::to_string(gpu_init));
    j.raw("gpu_setup", std::to_string(o.setup_ms));
    j.raw("solve", std::to_string(solve_total - o.load_ms - o.setup_ms));
    j.raw("write_out", std::to_string(write_ms));
    j.close();
    gpu_metrics(j, ai);
    build_metrics(j);
    // Fields of this implementation only; the reference's keys come first.
    j.obj("solver");
    j.raw("precision", json_str(precision_name(parse_precision(a))));
    j.raw("algorithm", json_str(get(a, "algorithm", "classic")));
    j.raw("path", json_str(get(a, "layout", "executors")));
    j.raw("device_ms", json_f64(o.res.device_ms));
    j.raw("final_r_norm2", json_f64(o.res.final_r_norm2));
    j.raw("final_relres", json_f64(o.res.final_relres));
    j.raw("refine_sweeps", std::to_string(o.res.refine_sweeps));
    j.raw("final_relres_true_f64", json_f64(true_relres));
    j.raw("iteration_bytes", std::to_string(o.iteration_bytes));
    j.raw("gbps", json_f64(gbps));
    j.raw("roofline_peak_gbs", json_f64(peak_gbs));
    j.raw("roofline_fraction", json_f64(peak_gbs > 0.0 ? gbps / peak_gbs : NAN));
    j.close();
    j.close();
    const std::string we = write_text_file(out_metrics, j.s);
    if (!we.empty()) {
        fprintf(stderr, "Failed to write metrics: %s\n", we.c_str());
        exit(2);
    }
    printf("%s\n", j.s.c_str());
    wsb_context_destroy(ctx);
    return 0;
}

// ---- compare-x (main.rs:582-719) -------------------------------------------
struct Worst {
    size_t i;
    float x_ref, x, abs_err;
};

int cmd_compare_x(const Args &a) {
    const std::string ref_path = get(a, "x-ref", "", true), x_path = get(a, "x", "", true);
    const float rel_tol = strtof(get(a, "rel-tol", "1e-3").c_str(), nullptr);
    const float abs_tol = strtof(get(a, "abs-tol", "1e-4").c_str(), nullptr);
    const size_t top_k = strtoull(get(a, "top-k", "10").c_str(), nullptr, 10);
    std::vector<float> xr, x;
    std::string e = read_f32_vec_bin(ref_path, &xr);
    if (e.empty()) e = read_f32_vec_bin(x_path, &x);
    if (e.empty() && xr.size() != x.size())
        e = "Length mismatch: x_ref len " + std::to_string(xr.size()) + " vs x len " + std::to_string(x.size());
    if (!e.empty()) {
        fprintf(stderr, "%s\n", e.c_str());
        return 2;
    }
    const size_t n = std::min(xr.size(), x.size());
    double sum_sq_err = 0.0, sum_sq_ref = 0.0;
    float max_abs_err = 0.0f;
    std::vector<Worst> worst;
    auto by_err_desc = [](const Worst &p, const Worst &q) { return q.abs_err < p.abs_err; };
    for (size_t i = 0; i < n; ++i) {
        const float ar = xr[i], b = x[i];
        const float abs_err = std::fabs(b - ar);
        max_abs_err = std::fmax(max_abs_err, abs_err);
        sum_sq_err += (double)abs_err * (double)abs_err;
        sum_sq_ref += (double)ar * (double)ar;
        if (top_k > 0) {
            if (worst.size() < top_k) {
                worst.push_back({i, ar, b, abs_err});
                std::stable_sort(worst.begin(), worst.end(), by_err_desc);
            } else if (abs_err > worst.back().abs_err) {
                worst.pop_back();
                worst.push_back({i, ar, b, abs_err});
                std::stable_sort(worst.begin(), worst.end(), by_err_desc);
            }
        }
    }
    const double l2_err = std::sqrt(sum_sq_err), l2_ref = std::sqrt(sum_sq_ref);
    const double rel_l2 = l2_err / std::max(l2_ref, 1e-30);
    const double rmse = std::sqrt(sum_sq_err / (double)std::max<size_t>(n, 1));
    const bool pass_rel = rel_l2 <= (double)rel_tol, pass_rmse = rmse <= (double)abs_tol, pass = pass_rel || pass_rmse;
    printf("CompareX:\n");
    printf("  n                 : %zu\n", n);
    printf("  rtol (rel L2)      : %s\n", rust_exp(rel_tol, 3).c_str());
    printf("  atol (RMSE)        : %s\n", rust_exp(abs_tol, 3).c_str());
    printf("  ||x_ref||_2        : %s\n", rust_exp(l2_ref, 9).c_str());
    printf("  ||x - x_ref||_2    : %s\n", rust_exp(l2_err, 9).c_str());
    printf("  rel_l2             : %s\n", rust_exp(rel_l2, 9).c_str());
    printf("  rmse               : %s\n", rust_exp(rmse, 9).c_str());
    printf("  max_abs_err (diag) : %s\n", rust_exp(max_abs_err, 9).c_str());
    printf("  pass_rel_l2        : %s\n", pass_rel ? "true" : "false");
    printf("  pass_rmse          : %s\n", pass_rmse ? "true" : "false");
    printf("  pass               : %s\n", pass ? "true" : "false");
    if (!worst.empty()) {
        printf("\nTop %zu worst entries (by abs error):\n", worst.size());
        for (const Worst &w : worst)
            printf("  i=%-8zu x_ref=%s  x=%s  abs=%s\n", w.i, rust_exp(w.x_ref, 9).c_str(), rust_exp(w.x, 9).c_str(),
                   rust_exp(w.abs_err, 9).c_str());
    }
    if (pass) return 0;
    fprintf(stderr, "CompareX failed tolerances (rel_l2 and rmse)\n");
    return 2;
}

}  // namespace

int main(int argc, char **argv) {
    const Args a = parse(argc, argv);
    check_backend(a.backend);
    if (a.cmd == "info") return cmd_info(a);
    if (a.cmd == "run-pcg-case") return cmd_run_pcg_case(a);
    if (a.cmd == "compare-x") return cmd_compare_x(a);
    if (a.cmd == "vec-test" || a.cmd == "dot-test" || a.cmd == "spmv-test" || a.cmd == "block-jacobi-test" ||
        a.cmd == "pcg-update-scalars-test") {
        if (!a.kv.empty()) usage_error("unexpected argument '--" + a.kv.begin()->first + "' found");
        wsb_context *ctx = context_or_exit(a.device);
        if (a.cmd == "vec-test") run_vec_test(ctx);
        else if (a.cmd == "dot-test") run_dot_test(ctx);
        else if (a.cmd == "spmv-test") run_spmv_test(ctx);
        else if (a.cmd == "block-jacobi-test") run_block_jacobi_test(ctx);
        else run_pcg_update_scalars_test(ctx);
        wsb_context_destroy(ctx);
        return 0;
    }
    usage_error("unrecognized subcommand '" + a.cmd + "'");
}
