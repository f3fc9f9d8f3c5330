/* TEST INFRASTRUCTURE (oracle). Plain-C restatement of the apxchol reference's
 * CPU solve phase; see apxoracle.h for the contract and the parity pin. Only
 * the tests, smoke() and bench.py's CPU-baseline leg load this library. */
#include "apxoracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ---------------------------------------------------------------- host prep */

/* factor_drop.h:90-96: max |off-diagonal| of a column whose first entry is the
 * diagonal, in double, stored fp32; 1.0f when there is none. */
static float column_scale(const float* v, uint32_t first, uint32_t last) {
    double mx = 0.0;
    for (uint32_t p = first + 1; p < last; ++p) {
        const double a = fabs((double)v[p]);
        if (a > mx) mx = a;
    }
    return mx > 0.0 ? (float)mx : 1.0f;
}

/* omp.h:476-481 on the fp32 storage: keep iff |v| >= rel*s and v != 0. */
static int keep_offdiag(float v, float s, double rel) {
    return fabs((double)v) >= rel * (double)s && v != 0.0f;
}

int64_t ora_prepare(uint32_t n, uint32_t m, const uint32_t* colptr, const uint32_t* rowidx,
                    const float* vals, double rel,
                    uint32_t* csr_ptr, uint32_t* csr_idx, float* csr_val,
                    uint32_t* csc_ptr, uint32_t* csc_idx, float* csc_val) {
    if (m != n && m + 1 != n) return -1;
    /* L11 = leading m x m block: drop entries of row n-1 (omp.h:543-581). */
    uint32_t* lo = (uint32_t*)malloc(sizeof(uint32_t) * ((size_t)m + 1));
    uint32_t* li = (uint32_t*)malloc(sizeof(uint32_t) * (colptr[n] ? colptr[n] : 1));
    float* lv = (float*)malloc(sizeof(float) * (colptr[n] ? colptr[n] : 1));
    uint32_t w = 0;
    lo[0] = 0;
    for (uint32_t j = 0; j < m; ++j) {
        if (colptr[j] >= colptr[j + 1] || rowidx[colptr[j]] != j) { free(lo); free(li); free(lv); return -1; }
        for (uint32_t p = colptr[j]; p < colptr[j + 1]; ++p) {
            if (m != n && rowidx[p] == n - 1) continue;
            li[w] = rowidx[p]; lv[w] = vals[p]; ++w;
        }
        lo[j + 1] = w;
    }
    /* Compacting drop with column-sum compensation (factor_drop.h:131-211);
     * the scale is taken before the drop (omp.h:627-650). */
    uint32_t nnz = w;
    if (rel > 0.0) {
        uint32_t q = 0;
        uint32_t first_out = 0;
        for (uint32_t j = 0; j < m; ++j) {
            const float s = column_scale(lv, lo[j], lo[j + 1]);
            double dropped_sum = 0.0, kept_abs = 0.0;
            const uint32_t first = q;
            for (uint32_t p = lo[j]; p < lo[j + 1]; ++p) {
                const float v = lv[p];
                if (li[p] != j) {
                    if (!keep_offdiag(v, s, rel)) { dropped_sum += (double)v; continue; }
                    kept_abs += fabs((double)v);
                }
                /* in place: q <= p always */
                li[q] = li[p]; lv[q] = v; ++q;
            }
            if (dropped_sum != 0.0 && kept_abs > 0.0) {
                const double per_abs = dropped_sum / kept_abs;
                for (uint32_t t = first; t < q; ++t) {
                    if (li[t] == j) continue;
                    const double v = (double)lv[t];
                    lv[t] = (float)(v + per_abs * fabs(v));
                }
            }
            lo[j] = first_out;          /* rewrite column start after compaction */
            first_out = q;
        }
        lo[m] = q;
        nnz = q;
    }
    /* CSC copy (omp.h:752-760) */
    memcpy(csc_ptr, lo, sizeof(uint32_t) * ((size_t)m + 1));
    memcpy(csc_idx, li, sizeof(uint32_t) * nnz);
    memcpy(csc_val, lv, sizeof(float) * nnz);
    /* CSR by the serial column-order scatter (transpose.h:116-246): rows get
     * their columns ascending. */
    memset(csr_ptr, 0, sizeof(uint32_t) * ((size_t)m + 1));
    for (uint32_t p = 0; p < nnz; ++p) csr_ptr[li[p] + 1]++;
    for (uint32_t i = 0; i < m; ++i) csr_ptr[i + 1] += csr_ptr[i];
    uint32_t* cur = (uint32_t*)malloc(sizeof(uint32_t) * ((size_t)m + 1));
    memcpy(cur, csr_ptr, sizeof(uint32_t) * ((size_t)m + 1));
    for (uint32_t j = 0; j < m; ++j)
        for (uint32_t p = lo[j]; p < lo[j + 1]; ++p) {
            const uint32_t slot = cur[li[p]]++;
            csr_idx[slot] = j;
            csr_val[slot] = lv[p];
        }
    free(cur); free(lo); free(li); free(lv);
    return (int64_t)nnz;
}

int32_t ora_levels(uint32_t m, const uint32_t* csr_ptr, const uint32_t* csr_idx,
                   const uint32_t* csc_ptr, const uint32_t* csc_idx,
                   const uint64_t* rounds, uint32_t n_rounds,
                   int32_t* fwd_level, int32_t* bck_level, int32_t* n_bck) {
    /* Round bounds as apx_cholesky::install_factor builds them
     * (preconditioner.h:247-258): cumulative IS sizes clamped to m. */
    if (n_rounds > 0) {
        uint64_t* b = (uint64_t*)malloc(sizeof(uint64_t) * ((size_t)n_rounds + 1));
        uint64_t acc = 0;
        b[0] = 0;
        for (uint32_t r = 0; r < n_rounds; ++r) {
            acc += rounds[r];
            if (acc > m) acc = m;
            b[r + 1] = acc;
        }
        /* omp.h:893-932: level = round index; columns past the last bound get
         * their own sequential levels; backward levels reversed. */
        if (b[n_rounds] <= m) {
            const uint64_t last = b[n_rounds];
            int32_t maxd = 0;
            uint32_t r = 0;
            for (uint32_t c = 0; c < m; ++c) {
                int32_t d;
                if (c >= last) d = (int32_t)(n_rounds + (c - last));
                else {
                    while (r + 1 < n_rounds + 1 && c >= b[r + 1]) ++r;
                    d = (int32_t)r;
                }
                fwd_level[c] = d;
                if (d > maxd) maxd = d;
            }
            for (uint32_t c = 0; c < m; ++c) bck_level[c] = maxd - fwd_level[c];
            free(b);
            *n_bck = maxd + 1;
            return maxd + 1;
        }
        free(b);
    }
    /* Topological depths (omp.h:933-975). */
    int32_t maxf = 0, maxb = 0;
    for (uint32_t i = 0; i < m; ++i) {
        int32_t d = 0;
        for (uint32_t p = csr_ptr[i]; p + 1 < csr_ptr[i + 1]; ++p) {
            const int32_t e = fwd_level[csr_idx[p]] + 1;
            if (e > d) d = e;
        }
        fwd_level[i] = d;
        if (d > maxf) maxf = d;
    }
    for (uint32_t j = m; j-- > 0;) {
        int32_t d = 0;
        for (uint32_t p = csc_ptr[j]; p < csc_ptr[j + 1]; ++p) {
            const uint32_t k = csc_idx[p];
            if (k > j) { const int32_t e = bck_level[k] + 1; if (e > d) d = e; }
        }
        bck_level[j] = d;
        if (d > maxb) maxb = d;
    }
    *n_bck = maxb + 1;
    return maxf + 1;
}

void ora_thin_flags(uint32_t m, const int32_t* level, int32_t n_levels, uint32_t threshold,
                    uint8_t* thin) {
    uint32_t* cnt = (uint32_t*)calloc((size_t)n_levels + 1, sizeof(uint32_t));
    for (uint32_t i = 0; i < m; ++i) cnt[level[i]]++;
    for (uint32_t i = 0; i < m; ++i) thin[i] = cnt[level[i]] <= threshold ? 1 : 0;
    free(cnt);
}

/* ---------------------------------------------------------------- sweeps */

/* dot_thin (omp.h:1343-1357): four interleaved partial sums, then the tail. */
static double dot_thin(const float* v, const uint32_t* idx, uint32_t p, uint32_t end, const double* y) {
    double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
    for (; p + 4 <= end; p += 4) {
        s0 += (double)v[p + 0] * y[idx[p + 0]];
        s1 += (double)v[p + 1] * y[idx[p + 1]];
        s2 += (double)v[p + 2] * y[idx[p + 2]];
        s3 += (double)v[p + 3] * y[idx[p + 3]];
    }
    double sum = (s0 + s1) + (s2 + s3);
    for (; p < end; ++p) sum += (double)v[p] * y[idx[p]];
    return sum;
}

/* The fat-level loop (omp.h:1434-1439): one serial sum. */
static double dot_fat(const float* v, const uint32_t* idx, uint32_t p, uint32_t end, const double* y) {
    double sum = 0.0;
    for (; p < end; ++p) sum += (double)v[p] * y[idx[p]];
    return sum;
}

void ora_sweep(int dir, uint32_t m, const uint32_t* ptr, const uint32_t* idx, const float* val,
               const uint8_t* thin, const double* in, double* out) {
    if (dir == 0) {
        for (uint32_t i = 0; i < m; ++i) {
            const uint32_t p0 = ptr[i], p1 = ptr[i + 1] - 1;     /* diagonal last */
            const double sum = thin[i] ? dot_thin(val, idx, p0, p1, out) : dot_fat(val, idx, p0, p1, out);
            out[i] = (in[i] - sum) / (double)val[p1];
        }
    } else {
        for (uint32_t j = m; j-- > 0;) {
            const uint32_t p0 = ptr[j] + 1, p1 = ptr[j + 1];     /* diagonal first */
            const double sum = thin[j] ? dot_thin(val, idx, p0, p1, out) : dot_fat(val, idx, p0, p1, out);
            out[j] = (in[j] - sum) / (double)val[ptr[j]];
        }
    }
}

/* The value of an IEEE binary16 bit pattern (exact in double). */
static double half_value(uint16_t h) {
    const int e = (h >> 10) & 0x1f, mant = h & 0x3ff;
    const double sgn = (h & 0x8000u) ? -1.0 : 1.0;
    if (e == 0) return sgn * ldexp((double)mant, -24);
    if (e == 31) return mant ? NAN : sgn * INFINITY;
    return sgn * ldexp((double)(mant | 0x400), e - 25);
}

void ora_sweep16(int dir, uint32_t m, const uint32_t* ptr, const uint32_t* idx, const uint16_t* val16,
                 const float* diag, const double* in_scale, const double* rhs, double* out) {
    for (uint32_t k = 0; k < m; ++k) {
        const uint32_t i = dir == 0 ? k : m - 1 - k;
        double sum = 0.0;
        for (uint32_t p = ptr[i]; p < ptr[i + 1]; ++p)
            if (idx[p] != i) sum += half_value(val16[p]) * out[idx[p]];
        const double r = rhs[i] * (in_scale ? in_scale[i] : 1.0);
        out[i] = (r - sum) / (double)diag[i];
    }
}

/* ---------------------------------------------------------------- reductions */

#define FUSED_OMP_MIN 2000  /* preconditioner.h:55 */

static int team(const ora_system* s, uint32_t n) { return n > FUSED_OMP_MIN ? s->nt : 1; }

/* static_chunk (preconditioner.h:69-75) */
static void chunk(uint32_t n, int tid, int nt, uint32_t* lo, uint32_t* hi) {
    const uint32_t base = n / (uint32_t)nt, rem = n % (uint32_t)nt;
    *lo = (uint32_t)tid * base + ((uint32_t)tid < rem ? (uint32_t)tid : rem);
    *hi = *lo + base + ((uint32_t)tid < rem ? 1u : 0u);
}

/* det_sum (preconditioner.h:108-125) */
static double det_sum(const ora_system* s, const double* v, uint32_t n) {
    const int nt = team(s, n);
    double total = 0.0;
    for (int t = 0; t < nt; ++t) {
        uint32_t lo, hi, i;
        chunk(n, t, nt, &lo, &hi);
        double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
        for (i = lo; i + 4 <= hi; i += 4) { s0 += v[i]; s1 += v[i + 1]; s2 += v[i + 2]; s3 += v[i + 3]; }
        double p = (s0 + s1) + (s2 + s3);
        for (; i < hi; ++i) p += v[i];
        total += p;          /* reduce_parts: serial in thread order */
    }
    return total;
}

/* ---------------------------------------------------------------- apply */

/* gather_out (preconditioner.h:423-447): z[v] = src[P[v]] - shift, b.z. */
static double gather_out(const ora_system* s, const double* src, double shift, const double* b, double* z) {
    const uint32_t n = s->n;
    const int nt = team(s, n);
    double total = 0.0;
    for (int t = 0; t < nt; ++t) {
        uint32_t lo, hi, v;
        chunk(n, t, nt, &lo, &hi);
        double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
        for (v = lo; v + 4 <= hi; v += 4) {
            const double z0 = src[s->perm[v + 0]] - shift;
            const double z1 = src[s->perm[v + 1]] - shift;
            const double z2 = src[s->perm[v + 2]] - shift;
            const double z3 = src[s->perm[v + 3]] - shift;
            z[v] = z0; z[v + 1] = z1; z[v + 2] = z2; z[v + 3] = z3;
            s0 += b[v] * z0; s1 += b[v + 1] * z1; s2 += b[v + 2] * z2; s3 += b[v + 3] * z3;
        }
        double p = (s0 + s1) + (s2 + s3);
        for (; v < hi; ++v) {
            const double zv = src[s->perm[v]] - shift;
            z[v] = zv;
            p += b[v] * zv;
        }
        total += p;
    }
    return total;
}

double ora_apply_core(ora_system* s, const double* b, double b_sum, int center, double* z, int want_rz) {
    const uint32_t n = s->n, m = s->m;
    double* zp = (double*)malloc(sizeof(double) * n);
    double* y = (double*)malloc(sizeof(double) * n);
    double* out = (double*)malloc(sizeof(double) * n);
    double rz, shift = 0.0;
    if (s->sddm) {
        for (uint32_t v = 0; v < n; ++v) zp[s->perm[v]] = b[v];
        ora_sweep(0, m, s->csr_ptr, s->csr_idx, s->csr_val, s->fwd_thin, zp, y);
        ora_sweep(1, m, s->csc_ptr, s->csc_idx, s->csc_val, s->bck_thin, y, out);
    } else {
        if (center) {
            const double b_mean = b_sum / (double)n;
            for (uint32_t v = 0; v < n; ++v) zp[s->perm[v]] = b[v] - b_mean;
        } else {
            for (uint32_t v = 0; v < n; ++v) zp[s->perm[v]] = b[v];
        }
        ora_sweep(0, m, s->csr_ptr, s->csr_idx, s->csr_val, s->fwd_thin, zp, y);
        ora_sweep(1, m, s->csc_ptr, s->csc_idx, s->csc_val, s->bck_thin, y, out);
        out[m] = 0.0;
        if (center) shift = det_sum(s, out, n) / (double)n;
    }
    rz = gather_out(s, out, shift, b, z);
    free(zp); free(y); free(out);
    return want_rz ? rz : 0.0;
}

/* take_center_ (preconditioner.h:393-397) under center-k. */
static int take_center(ora_system* s) {
    return (++s->apply_count % (uint64_t)s->center_k) == 0;
}

double ora_apply_fused(ora_system* s, const double* r, double r_sum, double* z) {
    const int center = !s->sddm && take_center(s);
    return ora_apply_core(s, r, r_sum, center, z, 1);
}

void ora_apply(ora_system* s, const double* b, double* z) {
    const int center = !s->sddm && take_center(s);
    const double b_sum = center ? det_sum(s, b, s->n) : 0.0;
    (void)ora_apply_core(s, b, b_sum, center, z, 0);
}

/* ---------------------------------------------------------------- PCG */

/* parallel_spmv_csr (src/solve.cpp:122-161) */
static double spmv(const ora_system* s, const double* x, double* y) {
    const uint32_t n = s->n;
    const int nt = team(s, n);
    double total = 0.0;
    for (int t = 0; t < nt; ++t) {
        uint32_t lo, hi;
        chunk(n, t, nt, &lo, &hi);
        double xy = 0.0;
        for (uint32_t i = lo; i < hi; ++i) {
            double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
            int32_t k = s->a_ptr[i];
            const int32_t e = s->a_ptr[i + 1];
            for (; k + 4 <= e; k += 4) {
                s0 += s->a_val[k + 0] * x[s->a_idx[k + 0]];
                s1 += s->a_val[k + 1] * x[s->a_idx[k + 1]];
                s2 += s->a_val[k + 2] * x[s->a_idx[k + 2]];
                s3 += s->a_val[k + 3] * x[s->a_idx[k + 3]];
            }
            double sum = (s0 + s1) + (s2 + s3);
            for (; k < e; ++k) sum += s->a_val[k] * x[s->a_idx[k]];
            y[i] = sum;
            xy += x[i] * sum;
        }
        total += xy;
    }
    return total;
}

/* update_xr (src/solve.cpp:169-208) and init_residual without x0 (:218-260). */
static void update_xr(const ora_system* s, double* x, const double* p, double* r, const double* Ap,
                      double alpha, int init, double* rr, double* rs) {
    const uint32_t n = s->n;
    const int nt = team(s, n);
    double tq = 0.0, ts = 0.0;
    for (int t = 0; t < nt; ++t) {
        uint32_t lo, hi, i;
        chunk(n, t, nt, &lo, &hi);
        double q0 = 0.0, q1 = 0.0, q2 = 0.0, q3 = 0.0, s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
        for (i = lo; i + 4 <= hi; i += 4) {
            double r0, r1, r2, r3;
            if (init) { r0 = p[i]; r1 = p[i + 1]; r2 = p[i + 2]; r3 = p[i + 3]; }
            else {
                x[i] += alpha * p[i]; x[i + 1] += alpha * p[i + 1];
                x[i + 2] += alpha * p[i + 2]; x[i + 3] += alpha * p[i + 3];
                r0 = r[i] - alpha * Ap[i]; r1 = r[i + 1] - alpha * Ap[i + 1];
                r2 = r[i + 2] - alpha * Ap[i + 2]; r3 = r[i + 3] - alpha * Ap[i + 3];
            }
            r[i] = r0; r[i + 1] = r1; r[i + 2] = r2; r[i + 3] = r3;
            q0 += r0 * r0; q1 += r1 * r1; q2 += r2 * r2; q3 += r3 * r3;
            s0 += r0; s1 += r1; s2 += r2; s3 += r3;
        }
        double q = (q0 + q1) + (q2 + q3);
        double sm = (s0 + s1) + (s2 + s3);
        for (; i < hi; ++i) {
            double ri;
            if (init) ri = p[i];
            else { x[i] += alpha * p[i]; ri = r[i] - alpha * Ap[i]; }
            r[i] = ri;
            q += ri * ri;
            sm += ri;
        }
        tq += q; ts += sm;
    }
    *rr = tq; *rs = ts;
}

int ora_pcg(ora_system* s, const double* b, double tol, int max_iter, double* x,
            int* iters, double* residual) {
    const uint32_t n = s->n;
    double* r = (double*)malloc(sizeof(double) * n);
    double* z = (double*)malloc(sizeof(double) * n);
    double* p = (double*)malloc(sizeof(double) * n);
    double* Ap = (double*)malloc(sizeof(double) * n);
    double rr, rs, bnorm, rz, prev_check = 1.0;
    *iters = 0; *residual = 0.0;
    update_xr(s, NULL, b, r, NULL, 0.0, 1, &rr, &rs);          /* r = b */
    bnorm = sqrt(rr);
    if (bnorm == 0.0) { memset(x, 0, sizeof(double) * n); goto done; }
    memset(x, 0, sizeof(double) * n);
    *residual = 1.0;
    s->apply_count = 0;                                        /* reset_apply_count */
    rz = ora_apply_fused(s, r, rs, z);
    memcpy(p, z, sizeof(double) * n);
    for (int i = 0; i < max_iter; ++i) {
        const double pAp = spmv(s, p, Ap);
        if (pAp <= 0.0) break;
        const double alpha = rz / pAp;
        update_xr(s, x, p, r, Ap, alpha, 0, &rr, &rs);
        const double rnorm = sqrt(rr) / bnorm;
        *iters = i + 1;
        *residual = rnorm;
        if (rnorm < tol) break;
        if ((i + 1) % 50 == 0) {                                /* stagnation_window */
            if (rnorm > prev_check * 0.5) break;
            prev_check = rnorm;
        }
        const double rz_new = ora_apply_fused(s, r, rs, z);
        const double beta = rz_new / rz;
        for (uint32_t k = 0; k < n; ++k) p[k] = z[k] + beta * p[k];
        rz = rz_new;
    }
    if (!s->sddm) {                                            /* center_x (:265-269) */
        const double mean = det_sum(s, x, n) / (double)n;
        for (uint32_t k = 0; k < n; ++k) x[k] -= mean;
    }
done:
    free(r); free(z); free(p); free(Ap);
    return 0;
}
