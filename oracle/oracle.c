/*
 * CPU oracle for the block-Jacobi preconditioned CG path.
 *
 * TEST INFRASTRUCTURE ONLY. This file is the checker: tests, the smoke check
 * and the CPU-baseline leg of the benchmark call it; the product library never
 * links, loads or calls it.
 *
 * It restates, in plain C with IEEE single precision and no contraction of
 * multiply-add (build with -ffp-contract=off), the arithmetic of the reference
 * crate `wgpu_solver_backend` (Rust host + WGSL shaders). Every function cites
 * the reference file:line it follows (paths relative to the reference repo).
 *
 * Three solvers live here:
 *   orc_pcg_ref_f32     exact restatement of pcg_block_jacobi_csr_wgpu
 *                       (compute.rs:189-495): FP32 everything, dot products by
 *                       the 256-wide shared-memory tree of dot_partials.wgsl and
 *                       dot_reduce.wgsl, f32 stop test on the host.
 *   orc_pcg_f64dot      the same iteration with FP64 dot accumulation and FP64
 *                       scalars (the semantics of the fused GPU path); vectors
 *                       and the matrix stay FP32.
 *   orc_pcg_f64         a full FP64 PCG (matrix values widened from f32, LU
 *                       factors recomputed in FP64) used for residual claims.
 *
 * Pinning: orc_pcg_ref_f32 is checked against the reference's own golden data
 * (datasets/pcg_block_jacobi_dataset_{1,2,3}.txt with their x_ref sections,
 * judged by the compare-x rule of wgpu_solver_backend_cli/src/main.rs:603-719
 * at the tolerances of commands.txt:56-78) and against the five known-answer
 * sanity tests of wgpu_solver_backend_cli/src/main.rs:171-443.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_OK 0
#define ORC_BAD_INPUT 1
#define ORC_ZERO_PIVOT 2
#define ORC_BREAKDOWN 3
#define ORC_MAXITER 4
#define ORC_NO_MEMORY 6

#define ORC_PAR_MIN 32768 /* below this many rows, loops stay serial */

/* ------------------------------------------------------------------------- */
/* LU of one 6x6-stored block, compute.rs:37-71.                             */
/* Returns ORC_OK or ORC_ZERO_PIVOT (pivot index in *pivot_k).               */
/* ------------------------------------------------------------------------- */
int orc_lu_factor_inplace_6(float *mat, int n, int *pivot_k)
{
    const int stride = 6;
    if (n > 6 || n < 0) return ORC_BAD_INPUT;
    for (int k = 0; k < n; ++k) {
        float a_kk = mat[k * stride + k];
        if (a_kk == 0.0f) {
            if (pivot_k) *pivot_k = k;
            return ORC_ZERO_PIVOT;
        }
        for (int i = k + 1; i < n; ++i) mat[i * stride + k] /= a_kk;
        for (int i = k + 1; i < n; ++i) {
            float l_ik = mat[i * stride + k];
            if (l_ik != 0.0f) {
                for (int j = k + 1; j < n; ++j) mat[i * stride + j] -= l_ik * mat[k * stride + j];
            }
        }
    }
    return ORC_OK;
}

/* ------------------------------------------------------------------------- */
/* Block-Jacobi LU builder, compute.rs:84-181.                               */
/* out: (bs_len-1)*36 floats. Returns ORC_OK, ORC_BAD_INPUT, ORC_ZERO_PIVOT. */
/* ------------------------------------------------------------------------- */
int orc_build_lu_blocks_6(uint32_t n, const uint32_t *row_ptr, uint64_t row_ptr_len,
                          const uint32_t *col_idx, uint64_t col_len, const float *values,
                          uint64_t val_len, const uint32_t *bs, uint64_t bs_len, float *out,
                          int64_t *bad_block, int *pivot_k)
{
    if (row_ptr_len != (uint64_t)n + 1) return ORC_BAD_INPUT;
    uint64_t nnz = row_ptr[n];
    if (col_len != nnz || val_len != nnz) return ORC_BAD_INPUT;
    if (bs_len < 2) return ORC_OK;
    if (bs[0] != 0) return ORC_BAD_INPUT;
    if (bs[bs_len - 1] != n) return ORC_BAD_INPUT;
    for (uint64_t i = 0; i + 1 < bs_len; ++i)
        if (bs[i + 1] <= bs[i]) return ORC_BAD_INPUT;
    uint64_t nb = bs_len - 1;
    memset(out, 0, sizeof(float) * 36 * nb);
    for (uint64_t blk = 0; blk < nb; ++blk) {
        uint32_t offset = bs[blk], end = bs[blk + 1];
        if (end > n || offset >= end) continue;
        uint32_t m = end - offset < 6 ? end - offset : 6;
        float mat[36];
        memset(mat, 0, sizeof(mat));
        for (int i = 0; i < 6; ++i) mat[i * 6 + i] = 1.0f;
        for (uint32_t il = 0; il < m; ++il) {
            uint32_t i = offset + il;
            for (uint32_t idx = row_ptr[i]; idx < row_ptr[i + 1]; ++idx) {
                uint32_t j = col_idx[idx];
                if (j >= offset && j < offset + m) mat[il * 6 + (j - offset)] = values[idx];
            }
        }
        int pk = 0;
        int st = orc_lu_factor_inplace_6(mat, (int)m, &pk);
        if (st != ORC_OK) {
            if (bad_block) *bad_block = (int64_t)blk;
            if (pivot_k) *pivot_k = pk;
            return st;
        }
        memcpy(out + blk * 36, mat, sizeof(mat));
    }
    return ORC_OK;
}

/* ------------------------------------------------------------------------- */
/* CSR SpMV, one sequential sum per row: spmv.wgsl:43-64.                    */
/* ------------------------------------------------------------------------- */
void orc_spmv_csr(uint32_t n, const uint32_t *row_ptr, const uint32_t *col, const float *val,
                  const float *x, float *y)
{
#pragma omp parallel for schedule(static) if (n >= ORC_PAR_MIN)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        float sum = 0.0f;
        for (uint32_t k = row_ptr[i]; k < row_ptr[i + 1]; ++k) sum = sum + val[k] * x[col[k]];
        y[i] = sum;
    }
}

/* One 256-lane shared-memory tree: offsets 128, 64, ..., 1
 * (dot_partials.wgsl:57-69 and dot_reduce.wgsl:56-68). */
static float tree256(float *s)
{
    for (int off = 128; off >= 1; off >>= 1)
        for (int t = 0; t < off; ++t) s[t] = s[t] + s[t + off];
    return s[0];
}

/* ------------------------------------------------------------------------- */
/* FP32 dot product with the reference's reduction order:                    */
/* pass 1 dot_partials.wgsl:46-74, passes 2..k dot_reduce.wgsl:47-73, driven */
/* by dot_scalar_exec.rs:151-247 (n == 0 gives 0, lines 165-174).            */
/* ------------------------------------------------------------------------- */
float orc_dot_tree256(uint32_t n, const float *a, const float *b)
{
    if (n == 0) return 0.0f;
    uint32_t len = (n + 255) / 256;
    float *part = (float *)malloc(sizeof(float) * len);
    float *tmp = (float *)malloc(sizeof(float) * ((len + 255) / 256 + 1));
#pragma omp parallel for schedule(static) if (n >= ORC_PAR_MIN)
    for (int64_t c = 0; c < (int64_t)len; ++c) {
        float s[256];
        for (int t = 0; t < 256; ++t) {
            uint64_t i = (uint64_t)c * 256 + t;
            s[t] = i < n ? a[i] * b[i] : 0.0f;
        }
        part[c] = tree256(s);
    }
    float *in = part, *outb = tmp;
    while (len > 1) {
        uint32_t out_len = (len + 255) / 256;
        for (uint32_t c = 0; c < out_len; ++c) {
            float s[256];
            for (int t = 0; t < 256; ++t) {
                uint64_t i = (uint64_t)c * 256 + t;
                s[t] = i < len ? in[i] : 0.0f;
            }
            outb[c] = tree256(s);
        }
        float *sw = in;
        in = outb;
        outb = sw;
        len = out_len;
    }
    float r = in[0];
    free(part);
    free(tmp);
    return r;
}

/* ------------------------------------------------------------------------- */
/* Block-Jacobi apply z = U^-1 L^-1 r per block: block_jacobi.wgsl:63-127.   */
/* Rows 6.. of a block longer than 6 are left untouched.                      */
/* ------------------------------------------------------------------------- */
void orc_block_jacobi_apply(uint32_t n, uint32_t nb, const float *lu, const uint32_t *bs,
                            const float *r, float *z)
{
#pragma omp parallel for schedule(static) if (nb >= ORC_PAR_MIN / 6)
    for (int64_t blk = 0; blk < (int64_t)nb; ++blk) {
        uint32_t offset = bs[blk], next = bs[blk + 1];
        if (offset >= n || next <= offset) continue;
        uint32_t m = next - offset < 6 ? next - offset : 6;
        const float *L = lu + (uint64_t)blk * 36;
        float y[6] = {0}, x[6] = {0};
        for (uint32_t i = 0; i < m; ++i) {
            float sum = r[offset + i];
            for (uint32_t j = 0; j < i; ++j) sum = sum - L[i * 6 + j] * y[j];
            y[i] = sum;
        }
        for (int ii = (int)m - 1; ii >= 0; --ii) {
            float sum = y[ii];
            for (uint32_t j = (uint32_t)ii + 1; j < m; ++j) sum = sum - L[ii * 6 + j] * x[j];
            x[ii] = sum / L[ii * 6 + ii];
        }
        for (uint32_t i = 0; i < m; ++i) z[offset + i] = x[i];
    }
}

/* y = y + alpha*x : axpy.wgsl:32-42 and axpy_from_scalar_results.wgsl:28-42 */
void orc_axpy(uint32_t n, float alpha, const float *x, float *y)
{
#pragma omp parallel for schedule(static) if (n >= ORC_PAR_MIN)
    for (int64_t i = 0; i < (int64_t)n; ++i) y[i] = y[i] + alpha * x[i];
}

/* x = x*s : scale_from_scalar_results.wgsl:26-38 */
void orc_scale(uint32_t n, float s, float *x)
{
#pragma omp parallel for schedule(static) if (n >= ORC_PAR_MIN)
    for (int64_t i = 0; i < (int64_t)n; ++i) x[i] = x[i] * s;
}

/* alpha, -alpha, beta with zero-denominator guards: pcg_update_scalars.wgsl:47-73 */
void orc_update_scalars(float *s, uint32_t p_ap, uint32_t rz_new, uint32_t rz_old, uint32_t alpha,
                        uint32_t minus_alpha, uint32_t beta)
{
    float pap = s[p_ap], rzn = s[rz_new], rzo = s[rz_old];
    float a = 0.0f, bt = 0.0f;
    if (pap != 0.0f) a = rzo / pap;
    if (rzo != 0.0f) bt = rzn / rzo;
    s[alpha] = a;
    s[minus_alpha] = -a;
    s[beta] = bt;
}

/* ------------------------------------------------------------------------- */
/* Exact restatement of pcg_block_jacobi_csr_wgpu, compute.rs:189-495.       */
/* x: in x0, out solution (written only on ORC_OK, compute.rs:482-484).      */
/* history (optional, length >= max_iter): r.r after each iteration.         */
/* Returns ORC_OK / ORC_BREAKDOWN (*breakdown_kind 1 = pAp, 2 = rz_old) /    */
/* ORC_MAXITER. *iters_out = iterations (k+1) on success.                    */
/* ------------------------------------------------------------------------- */
int orc_pcg_ref_f32(uint32_t n, const uint32_t *row_ptr, const uint32_t *col, const float *val,
                    uint32_t nb, const float *lu, const uint32_t *bs, const float *b, float *x,
                    uint64_t max_iter, float rel_tol, float abs_tol, uint64_t *iters_out,
                    float *history, int *breakdown_kind)
{
    enum { S_PAP = 0, S_RR = 1, S_RZN = 2, S_RZO = 3, S_A = 4, S_MA = 5, S_B = 6 };
    float sr[7] = {0};
    if (iters_out) *iters_out = 0;
    /* 1) ||b||^2 once (compute.rs:228-250) */
    float b_norm2 = orc_dot_tree256(n, b, b);
    if (b_norm2 == 0.0f) return ORC_OK; /* compute.rs:252-254 */
    float rel2 = rel_tol * rel_tol, abs2 = abs_tol * abs_tol;
    size_t nbytes = sizeof(float) * (size_t)(n ? n : 1);
    float *xg = (float *)malloc(nbytes), *r = (float *)malloc(nbytes), *p = (float *)malloc(nbytes),
          *z = (float *)calloc(n ? n : 1, sizeof(float)), *ap = (float *)malloc(nbytes);
    if (!xg || !r || !p || !z || !ap) {
        free(xg); free(r); free(p); free(z); free(ap);
        return ORC_NO_MEMORY;
    }
    memcpy(xg, x, sizeof(float) * n);
    /* 2) init (compute.rs:283-331): r=b; Ap=A x; r += -1*Ap; z=M^-1 r; p=z; rz */
    memcpy(r, b, sizeof(float) * n);
    orc_spmv_csr(n, row_ptr, col, val, xg, ap);
    orc_axpy(n, -1.0f, ap, r);
    orc_block_jacobi_apply(n, nb, lu, bs, r, z);
    memcpy(p, z, sizeof(float) * n);
    sr[S_RZO] = orc_dot_tree256(n, r, z);
    float rz_old = sr[S_RZO];
    int status = ORC_MAXITER;
    for (uint64_t k = 0; k < max_iter; ++k) {
        orc_spmv_csr(n, row_ptr, col, val, p, ap);                 /* A */
        sr[S_PAP] = orc_dot_tree256(n, p, ap);                     /* B */
        sr[S_RZO] = rz_old;                                        /* C */
        orc_update_scalars(sr, S_PAP, S_RZN, S_RZO, S_A, S_MA, S_B); /* D */
        orc_axpy(n, sr[S_A], p, xg);                               /* E */
        orc_axpy(n, sr[S_MA], ap, r);
        sr[S_RR] = orc_dot_tree256(n, r, r);                       /* F */
        orc_block_jacobi_apply(n, nb, lu, bs, r, z);               /* G */
        sr[S_RZN] = orc_dot_tree256(n, r, z);                      /* H */
        orc_update_scalars(sr, S_PAP, S_RZN, S_RZO, S_A, S_MA, S_B); /* I */
        orc_scale(n, sr[S_B], p);                                  /* J */
        orc_axpy(n, 1.0f, z, p);
        float p_ap = sr[S_PAP], r_norm2 = sr[S_RR], rz_new = sr[S_RZN];
        if (history) history[k] = r_norm2;
        if (iters_out) *iters_out = k + 1;
        if (p_ap == 0.0f) { if (breakdown_kind) *breakdown_kind = 1; status = ORC_BREAKDOWN; break; }
        if (rz_old == 0.0f) { if (breakdown_kind) *breakdown_kind = 2; status = ORC_BREAKDOWN; break; }
        if (r_norm2 <= abs2 || r_norm2 <= rel2 * b_norm2) {
            memcpy(x, xg, sizeof(float) * n);
            status = ORC_OK;
            break;
        }
        rz_old = rz_new;
    }
    free(xg); free(r); free(p); free(z); free(ap);
    return status;
}

/* Sequential FP64 dot of FP32 vectors (products are exact in FP64). */
static double dot_f64(uint32_t n, const float *a, const float *b)
{
    double s = 0.0;
#pragma omp parallel for reduction(+ : s) schedule(static) if (n >= ORC_PAR_MIN)
    for (int64_t i = 0; i < (int64_t)n; ++i) s += (double)a[i] * (double)b[i];
    return s;
}

/* ------------------------------------------------------------------------- */
/* The reference iteration (compute.rs:336-489) with FP64 dot products and   */
/* FP64 scalars; alpha/beta are rounded to f32 where they scale f32 vectors. */
/* Stop test in FP64: rr <= abs^2 or rr <= rel^2 * bb.                       */
/* ------------------------------------------------------------------------- */
int orc_pcg_f64dot(uint32_t n, const uint32_t *row_ptr, const uint32_t *col, const float *val,
                   uint32_t nb, const float *lu, const uint32_t *bs, const float *b, float *x,
                   uint64_t max_iter, float rel_tol, float abs_tol, uint64_t *iters_out,
                   double *history, int *breakdown_kind)
{
    if (iters_out) *iters_out = 0;
    double bb = dot_f64(n, b, b);
    if (bb == 0.0) return ORC_OK;
    double rel2 = (double)rel_tol * (double)rel_tol, abs2 = (double)abs_tol * (double)abs_tol;
    size_t nbytes = sizeof(float) * (size_t)(n ? n : 1);
    float *xg = (float *)malloc(nbytes), *r = (float *)malloc(nbytes), *p = (float *)malloc(nbytes),
          *z = (float *)calloc(n ? n : 1, sizeof(float)), *ap = (float *)malloc(nbytes);
    if (!xg || !r || !p || !z || !ap) {
        free(xg); free(r); free(p); free(z); free(ap);
        return ORC_NO_MEMORY;
    }
    memcpy(xg, x, sizeof(float) * n);
    memcpy(r, b, sizeof(float) * n);
    orc_spmv_csr(n, row_ptr, col, val, xg, ap);
    orc_axpy(n, -1.0f, ap, r);
    orc_block_jacobi_apply(n, nb, lu, bs, r, z);
    memcpy(p, z, sizeof(float) * n);
    double rz_old = dot_f64(n, r, z);
    int status = ORC_MAXITER;
    for (uint64_t k = 0; k < max_iter; ++k) {
        orc_spmv_csr(n, row_ptr, col, val, p, ap);
        double pap = dot_f64(n, p, ap);
        double alpha = pap != 0.0 ? rz_old / pap : 0.0;
        float af = (float)alpha, maf = -af;
        orc_axpy(n, af, p, xg);
        orc_axpy(n, maf, ap, r);
        double rr = dot_f64(n, r, r);
        orc_block_jacobi_apply(n, nb, lu, bs, r, z);
        double rz_new = dot_f64(n, r, z);
        double beta = rz_old != 0.0 ? rz_new / rz_old : 0.0;
        orc_scale(n, (float)beta, p);
        orc_axpy(n, 1.0f, z, p);
        if (history) history[k] = rr;
        if (iters_out) *iters_out = k + 1;
        if (pap == 0.0) { if (breakdown_kind) *breakdown_kind = 1; status = ORC_BREAKDOWN; break; }
        if (rz_old == 0.0) { if (breakdown_kind) *breakdown_kind = 2; status = ORC_BREAKDOWN; break; }
        if (rr <= abs2 || rr <= rel2 * bb) {
            memcpy(x, xg, sizeof(float) * n);
            status = ORC_OK;
            break;
        }
        rz_old = rz_new;
    }
    free(xg); free(r); free(p); free(z); free(ap);
    return status;
}

/* M applied with rows >= 6 of a longer block set to 0 (the values the
 * reference's apply leaves in its zero-initialised z for those rows). */
static void orc_bj_zero_tail(uint32_t n, uint32_t nb, const float *lu, const uint32_t *bs, const float *in,
                             float *out)
{
    memset(out, 0, sizeof(float) * n);
    orc_block_jacobi_apply(n, nb, lu, bs, in, out);
}

/* ------------------------------------------------------------------------- */
/* Single-reduction PCG of Chronopoulos & Gear (J. Comput. Appl. Math. 25     */
/* (1989)): u = M r and w = A u are formed explicitly every iteration, s = A p */
/* by recurrence, and both dots of an iteration, (r, u) and (w, u), come      */
/* from the same pass. Arithmetic as orc_pcg_f64dot (FP32 vectors, FP64 dots */
/* and scalars, alpha/beta rounded to f32 where they scale f32 vectors), M as */
/* orc_block_jacobi_apply with rows >= 6 of a longer block set to 0.         */
/* ------------------------------------------------------------------------- */
int orc_pcg_single_reduction_f64dot(uint32_t n, const uint32_t *row_ptr, const uint32_t *col, const float *val,
                                    uint32_t nb, const float *lu, const uint32_t *bs, const float *b, float *x,
                                    uint64_t max_iter, float rel_tol, float abs_tol, uint64_t *iters_out,
                                    double *history)
{
    if (iters_out) *iters_out = 0;
    double bb = dot_f64(n, b, b);
    if (bb == 0.0) return ORC_OK;
    double rel2 = (double)rel_tol * (double)rel_tol, abs2 = (double)abs_tol * (double)abs_tol;
    size_t nn = n ? n : 1;
    float *v[7];
    for (int k = 0; k < 7; ++k) {
        v[k] = (float *)calloc(nn, sizeof(float));
        if (!v[k]) {
            for (int j = 0; j < k; ++j) free(v[j]);
            return ORC_NO_MEMORY;
        }
    }
    float *xg = v[0], *r = v[1], *u = v[2], *w = v[3], *p = v[4], *s = v[5], *tmp = v[6];
    memcpy(xg, x, sizeof(float) * n);
    orc_spmv_csr(n, row_ptr, col, val, xg, tmp);
    for (uint32_t i = 0; i < n; ++i) r[i] = b[i] + (-1.0f) * tmp[i];
    orc_bj_zero_tail(n, nb, lu, bs, r, u);
    orc_spmv_csr(n, row_ptr, col, val, u, w);
    double gamma = dot_f64(n, r, u), delta = dot_f64(n, w, u);
    int status = ORC_MAXITER;
    if (max_iter == 0) goto done;
    if (delta == 0.0) { status = ORC_BREAKDOWN; goto done; }
    double alpha = gamma / delta, beta = 0.0;
    for (uint64_t k = 0; k < max_iter; ++k) {
        float af = (float)alpha, bf = (float)beta, maf = -af;
#pragma omp parallel for schedule(static) if (n >= ORC_PAR_MIN)
        for (int64_t i = 0; i < (int64_t)n; ++i) {
            float pi = u[i] + bf * p[i], si = w[i] + bf * s[i];
            p[i] = pi;
            s[i] = si;
            xg[i] = xg[i] + af * pi;
            r[i] = r[i] + maf * si;
        }
        double rr = dot_f64(n, r, r);
        if (history) history[k] = rr;
        if (iters_out) *iters_out = k + 1;
        if (rr <= abs2 || rr <= rel2 * bb) {
            memcpy(x, xg, sizeof(float) * n);
            status = ORC_OK;
            break;
        }
        orc_bj_zero_tail(n, nb, lu, bs, r, u);
        orc_spmv_csr(n, row_ptr, col, val, u, w);
        double g2 = dot_f64(n, r, u), d2 = dot_f64(n, w, u);
        if (gamma == 0.0) { status = ORC_BREAKDOWN; break; }
        beta = g2 / gamma;
        double den = d2 - beta * g2 / alpha;
        if (den == 0.0) { status = ORC_BREAKDOWN; break; }
        alpha = g2 / den;
        gamma = g2;
    }
done:
    for (int k = 0; k < 7; ++k) free(v[k]);
    return status;
}

/* ------------------------------------------------------------------------- */
/* Full FP64 block-Jacobi PCG: FP32 matrix entries widened to FP64, block    */
/* LU recomputed in FP64 with the same no-pivot algorithm (compute.rs:37-71, */
/* identity padding as compute.rs:148-171), FP64 vectors. Stops on the       */
/* recursive residual ||r||/||b|| <= rel_tol. x in/out (double).             */
/* ------------------------------------------------------------------------- */
int orc_pcg_f64(uint32_t n, const uint32_t *row_ptr, const uint32_t *col, const float *val,
                uint32_t nb, const uint32_t *bs, const double *b, double *x, uint64_t max_iter,
                double rel_tol, uint64_t *iters_out)
{
    if (iters_out) *iters_out = 0;
    double *lu = (double *)calloc((size_t)nb * 36 + 1, sizeof(double));
    double *r = (double *)malloc(sizeof(double) * (n + 1)), *p = (double *)malloc(sizeof(double) * (n + 1));
    double *z = (double *)calloc(n + 1, sizeof(double)), *ap = (double *)malloc(sizeof(double) * (n + 1));
    if (!lu || !r || !p || !z || !ap) {
        free(lu); free(r); free(p); free(z); free(ap);
        return ORC_NO_MEMORY;
    }
    int status = ORC_OK;
    for (uint32_t blk = 0; blk < nb && status == ORC_OK; ++blk) {
        uint32_t off = bs[blk], end = bs[blk + 1];
        uint32_t m = end - off < 6 ? end - off : 6;
        double *M = lu + (size_t)blk * 36;
        for (int i = 0; i < 6; ++i) M[i * 6 + i] = 1.0;
        for (uint32_t il = 0; il < m; ++il)
            for (uint32_t k = row_ptr[off + il]; k < row_ptr[off + il + 1]; ++k)
                if (col[k] >= off && col[k] < off + m) M[il * 6 + (col[k] - off)] = (double)val[k];
        for (uint32_t k = 0; k < m; ++k) {
            if (M[k * 6 + k] == 0.0) { status = ORC_ZERO_PIVOT; break; }
            for (uint32_t i = k + 1; i < m; ++i) M[i * 6 + k] /= M[k * 6 + k];
            for (uint32_t i = k + 1; i < m; ++i)
                for (uint32_t j = k + 1; j < m; ++j) M[i * 6 + j] -= M[i * 6 + k] * M[k * 6 + j];
        }
    }
    if (status != ORC_OK) {
        free(lu); free(r); free(p); free(z); free(ap);
        return status;
    }
#define SPMV64(in, out)                                                                   \
    _Pragma("omp parallel for schedule(static) if (n >= ORC_PAR_MIN)") for (int64_t i = 0; \
                                                                           i < (int64_t)n; \
                                                                           ++i)            \
    {                                                                                     \
        double s = 0.0;                                                                   \
        for (uint32_t k = row_ptr[i]; k < row_ptr[i + 1]; ++k) s += (double)val[k] * in[col[k]]; \
        out[i] = s;                                                                       \
    }
#define PREC64(in, out)                                                                   \
    _Pragma("omp parallel for schedule(static) if (nb >= ORC_PAR_MIN / 6)") for (int64_t blk = 0; \
                                                                             blk < (int64_t)nb; \
                                                                             ++blk)      \
    {                                                                                     \
        uint32_t off = bs[blk], end = bs[blk + 1];                                        \
        uint32_t m = end - off < 6 ? end - off : 6;                                       \
        const double *M = lu + (size_t)blk * 36;                                          \
        double y[6];                                                                      \
        for (uint32_t i = 0; i < m; ++i) {                                                \
            double s = in[off + i];                                                       \
            for (uint32_t j = 0; j < i; ++j) s -= M[i * 6 + j] * y[j];                    \
            y[i] = s;                                                                     \
        }                                                                                 \
        for (int i = (int)m - 1; i >= 0; --i) {                                           \
            double s = y[i];                                                              \
            for (uint32_t j = i + 1; j < m; ++j) s -= M[i * 6 + j] * out[off + j];        \
            out[off + i] = s / M[i * 6 + i];                                              \
        }                                                                                 \
    }
    double bb = 0.0;
    for (uint32_t i = 0; i < n; ++i) bb += b[i] * b[i];
    if (bb == 0.0) {
        free(lu); free(r); free(p); free(z); free(ap);
        return ORC_OK;
    }
    SPMV64(x, ap);
    for (uint32_t i = 0; i < n; ++i) r[i] = b[i] - ap[i];
    PREC64(r, z);
    for (uint32_t i = 0; i < n; ++i) p[i] = z[i];
    double rz = 0.0;
    for (uint32_t i = 0; i < n; ++i) rz += r[i] * z[i];
    double tol2 = rel_tol * rel_tol * bb;
    status = ORC_MAXITER;
    for (uint64_t k = 0; k < max_iter; ++k) {
        SPMV64(p, ap);
        double pap = 0.0;
#pragma omp parallel for reduction(+ : pap) schedule(static) if (n >= ORC_PAR_MIN)
        for (int64_t i = 0; i < (int64_t)n; ++i) pap += p[i] * ap[i];
        if (pap == 0.0 || rz == 0.0) { status = ORC_BREAKDOWN; if (iters_out) *iters_out = k; break; }
        double alpha = rz / pap, rr = 0.0;
#pragma omp parallel for reduction(+ : rr) schedule(static) if (n >= ORC_PAR_MIN)
        for (int64_t i = 0; i < (int64_t)n; ++i) {
            x[i] += alpha * p[i];
            r[i] -= alpha * ap[i];
            rr += r[i] * r[i];
        }
        if (iters_out) *iters_out = k + 1;
        if (rr <= tol2) { status = ORC_OK; break; }
        PREC64(r, z);
        double rzn = 0.0;
#pragma omp parallel for reduction(+ : rzn) schedule(static) if (n >= ORC_PAR_MIN)
        for (int64_t i = 0; i < (int64_t)n; ++i) rzn += r[i] * z[i];
        double beta = rzn / rz;
        rz = rzn;
#pragma omp parallel for schedule(static) if (n >= ORC_PAR_MIN)
        for (int64_t i = 0; i < (int64_t)n; ++i) p[i] = z[i] + beta * p[i];
    }
#undef SPMV64
#undef PREC64
    free(lu); free(r); free(p); free(z); free(ap);
    return status;
}

/* ||b - A x|| / ||b|| in FP64 with the FP32 matrix entries; x given in FP32 or FP64. */
double orc_true_relres_f64(uint32_t n, const uint32_t *row_ptr, const uint32_t *col, const float *val,
                           const float *b, const float *x32, const double *x64)
{
    double rr = 0.0, bb = 0.0;
#pragma omp parallel for reduction(+ : rr, bb) schedule(static) if (n >= ORC_PAR_MIN)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        double s = 0.0;
        for (uint32_t k = row_ptr[i]; k < row_ptr[i + 1]; ++k)
            s += (double)val[k] * (x64 ? x64[col[k]] : (double)x32[col[k]]);
        double ri = (double)b[i] - s;
        rr += ri * ri;
        bb += (double)b[i] * (double)b[i];
    }
    return bb > 0.0 ? sqrt(rr / bb) : sqrt(rr);
}

/* compare-x statistics, wgpu_solver_backend_cli/src/main.rs:603-662:
 * out[0]=l2_ref, out[1]=l2_err, out[2]=rel_l2, out[3]=rmse, out[4]=max_abs_err */
void orc_compare_x(uint64_t n, const float *x_ref, const float *x, double *out)
{
    double se = 0.0, sr = 0.0;
    float mx = 0.0f;
    for (uint64_t i = 0; i < n; ++i) {
        float a = x_ref[i], b = x[i];
        float e = fabsf(b - a);
        mx = fmaxf(mx, e);
        se += (double)e * (double)e;
        sr += (double)a * (double)a;
    }
    out[0] = sqrt(sr);
    out[1] = sqrt(se);
    out[2] = out[1] / (out[0] > 1e-30 ? out[0] : 1e-30);
    out[3] = sqrt(se / (double)(n > 0 ? n : 1));
    out[4] = mx;
}

/* ------------------------------------------------------------------------- */
/* Synthetic 6-DOF lattice systems (the measured workloads; not a reference   */
/* algorithm). An independent C statement of the generator the product ships */
/* (wsb_lattice_generate), so that the CPU baseline and the reference arm of  */
/* the benchmark build their inputs without loading the product library. The */
/* test suite checks the two for bit identity.                               */
/* Node u = x + L y + L^2 z owns rows 6u..6u+5; every axis-neighbour edge     */
/* (keyed by its lower node and axis) gets S = (R R^T / 6 + 0.1 I) 10^U(-a,a) */
/* with R ~ N(0,1) by Box-Muller, assembled as [[S,-S],[-S,S]]; 1e-3 is added */
/* on the diagonal; b_i ~ U[-1,1). FP64 accumulation, one rounding to f32.     */
/* ------------------------------------------------------------------------- */
#define ORC_GOLDEN 0x9E3779B97F4A7C15ull

static uint64_t orc_fin64(uint64_t z)
{
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

/* Counter-based stream keyed by (seed, key). */
static uint64_t orc_stream_init(uint64_t seed, uint64_t key)
{
    return orc_fin64((seed ^ orc_fin64(key * 0xD1B54A32D192ED03ull + 1 + ORC_GOLDEN)) + ORC_GOLDEN);
}

static double orc_stream_uniform(uint64_t *state) /* [0, 1) */
{
    *state += ORC_GOLDEN;
    return (double)(orc_fin64(*state) >> 11) * 0x1.0p-53;
}

static void orc_edge_stiffness(uint64_t seed, uint64_t key, double aniso, double S[36])
{
    uint64_t st = orc_stream_init(seed, key);
    double R[36];
    for (int k = 0; k < 36; k += 2) {
        double u1 = 1.0 - orc_stream_uniform(&st);
        double u2 = orc_stream_uniform(&st);
        double rad = sqrt(-2.0 * log(u1));
        R[k] = rad * cos(6.283185307179586 * u2);
        R[k + 1] = rad * sin(6.283185307179586 * u2);
    }
    double scale = 1.0;
    if (aniso > 0.0) scale = pow(10.0, (2.0 * orc_stream_uniform(&st) - 1.0) * aniso);
    for (int i = 0; i < 6; ++i)
        for (int j = 0; j < 6; ++j) {
            double dotp = 0.0;
            for (int k = 0; k < 6; ++k) dotp += R[i * 6 + k] * R[j * 6 + k];
            S[i * 6 + j] = (dotp / 6.0 + (i == j ? 0.1 : 0.0)) * scale;
        }
}

/* Axis neighbours of node u including itself, ascending index order
 * (-z, -y, -x, self, +x, +y, +z). axis -1 marks the node itself; lower = 1
 * when the neighbour is the edge's lower node. Returns the count. */
static int orc_lattice_nbrs(int64_t u, int64_t L, int64_t *w, int *axis, int *lower)
{
    const int64_t LL = L * L, x = u % L, y = (u / L) % L, z = u / LL;
    int c = 0;
#define ORC_NB(cond, node, ax, lo) if (cond) { w[c] = (node); axis[c] = (ax); lower[c] = (lo); ++c; }
    ORC_NB(z > 0, u - LL, 2, 1)
    ORC_NB(y > 0, u - L, 1, 1)
    ORC_NB(x > 0, u - 1, 0, 1)
    ORC_NB(1, u, -1, 0)
    ORC_NB(x + 1 < L, u + 1, 0, 0)
    ORC_NB(y + 1 < L, u + L, 1, 0)
    ORC_NB(z + 1 < L, u + LL, 2, 0)
#undef ORC_NB
    return c;
}

/* Sizes of the side-L lattice system: out[0] = n, out[1] = nnz, out[2] = nodes. */
int orc_lattice_sizes(uint32_t L, uint64_t *out)
{
    uint64_t l = L, nodes = l * l * l, edges = l >= 1 ? 3 * l * l * (l - 1) : 0;
    out[0] = 6 * nodes;
    out[1] = 36 * (nodes + 2 * edges);
    out[2] = nodes;
    return (out[0] > 0xffffffffull || out[1] > 0xffffffffull) ? ORC_BAD_INPUT : ORC_OK;
}

int orc_lattice_generate(uint32_t L, uint64_t seed, double aniso, uint32_t *row_ptr, uint32_t *col,
                         float *val, uint32_t *bs, float *b)
{
    uint64_t sz[3];
    if (orc_lattice_sizes(L, sz) != ORC_OK) return ORC_BAD_INPUT;
    const int64_t nodes = (int64_t)sz[2];
    /* First entry of each node's rows: 36 per neighbour (self included). */
    uint64_t *node_off = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)(nodes + 1));
    if (!node_off) return ORC_NO_MEMORY;
    node_off[0] = 0;
    for (int64_t u = 0; u < nodes; ++u) {
        int64_t w[7];
        int ax[7], lo[7];
        node_off[u + 1] = node_off[u] + 36ull * (uint64_t)orc_lattice_nbrs(u, L, w, ax, lo);
    }
#pragma omp parallel for schedule(dynamic, 1024)
    for (int64_t u = 0; u < nodes; ++u) {
        int64_t w[7];
        int ax[7], lo[7];
        const int c = orc_lattice_nbrs(u, L, w, ax, lo);
        double blk[7][36], diag[36];
        memset(diag, 0, sizeof diag);
        int self = 0;
        for (int k = 0; k < c; ++k) {
            if (ax[k] < 0) {
                self = k;
                continue;
            }
            const int64_t low = lo[k] ? w[k] : u;
            double S[36];
            orc_edge_stiffness(seed, (uint64_t)low * 3 + (uint64_t)ax[k] + 1, aniso, S);
            for (int q = 0; q < 36; ++q) {
                blk[k][q] = -S[q];
                diag[q] += S[q];
            }
        }
        for (int i = 0; i < 6; ++i) diag[i * 6 + i] += 1e-3;
        memcpy(blk[self], diag, sizeof diag);
        for (int a = 0; a < 6; ++a) {
            const uint64_t row = 6 * (uint64_t)u + (uint64_t)a;
            uint64_t k0 = node_off[u] + (uint64_t)a * 6 * (uint64_t)c;
            row_ptr[row] = (uint32_t)k0;
            for (int k = 0; k < c; ++k)
                for (int j = 0; j < 6; ++j, ++k0) {
                    col[k0] = (uint32_t)(6 * w[k] + j);
                    val[k0] = (float)blk[k][a * 6 + j];
                }
            uint64_t sb = orc_stream_init(seed, 0x4000000000000000ull + row);
            b[row] = (float)(2.0 * orc_stream_uniform(&sb) - 1.0);
        }
        bs[u] = (uint32_t)(6 * u);
    }
    row_ptr[sz[0]] = (uint32_t)node_off[nodes];
    bs[nodes] = (uint32_t)sz[0];
    free(node_off);
    return ORC_OK;
}

/* ------------------------------------------------------------------------- */
/* Many independent FP32 reference solves (orc_pcg_ref_f32 each), for the    */
/* timed CPU baseline: systems with n >= par_min_n run one after another with */
/* every host thread inside each solve; the smaller ones run concurrently,   */
/* one thread each (the inner loops stay serial below ORC_PAR_MIN rows, and  */
/* nested parallel regions are off; callers list the systems largest first */
/* so that the dynamic schedule balances). Per-system status and iteration   */
/* counts out; x[i] receives the solution of system i.                       */
/* ------------------------------------------------------------------------- */
int orc_pcg_ref_f32_many(uint32_t count, const uint32_t *n, const uint32_t *const *row_ptr,
                         const uint32_t *const *col, const float *const *val, const uint32_t *nb,
                         const float *const *lu, const uint32_t *const *bs, const float *const *b,
                         float *const *x, uint64_t max_iter, float rel_tol, float abs_tol, uint32_t par_min_n,
                         int *status, uint64_t *iters)
{
    for (uint32_t i = 0; i < count; ++i)
        if (n[i] >= par_min_n)
            status[i] = orc_pcg_ref_f32(n[i], row_ptr[i], col[i], val[i], nb[i], lu[i], bs[i], b[i], x[i],
                                        max_iter, rel_tol, abs_tol, &iters[i], NULL, NULL);
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t j = 0; j < (int64_t)count; ++j) {
        const uint32_t i = (uint32_t)j;
        if (n[i] < par_min_n)
            status[i] = orc_pcg_ref_f32(n[i], row_ptr[i], col[i], val[i], nb[i], lu[i], bs[i], b[i], x[i],
                                        max_iter, rel_tol, abs_tol, &iters[i], NULL, NULL);
    }
    return ORC_OK;
}

int orc_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
