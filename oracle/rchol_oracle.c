/*
 * rchol_oracle.c -- CPU restatement of the reference's randomized-Cholesky
 * factor + PCG.  TEST INFRASTRUCTURE ONLY (the checker and the CPU-baseline
 * leg of bench.py); nothing in the product links or calls it.
 *
 * Every function cites the reference lines it restates.  Compiled with
 * -ffp-contract=off so that no multiply-add is fused: the CUDA factor uses
 * the same separately rounded double operations, which makes the factor in
 * ORC_MODE_B200 bit-identical to the GPU's.
 */
#include "rchol_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ======================================================================== */
/* random numbers                                                           */
/* ======================================================================== */

void orc_mt_seed(orc_mt19937* g, uint32_t seed) {
    g->mt[0] = seed;
    for (int i = 1; i < 624; ++i)
        g->mt[i] = 1812433253u * (g->mt[i - 1] ^ (g->mt[i - 1] >> 30)) + (uint32_t)i;
    g->idx = 624;
}

static void orc_mt_twist(orc_mt19937* g) {
    for (int i = 0; i < 624; ++i) {
        uint32_t y = (g->mt[i] & 0x80000000u) | (g->mt[(i + 1) % 624] & 0x7fffffffu);
        uint32_t v = g->mt[(i + 397) % 624] ^ (y >> 1);
        if (y & 1u) v ^= 0x9908b0dfu;
        g->mt[i] = v;
    }
    g->idx = 0;
}

uint32_t orc_mt_next(orc_mt19937* g) {
    if (g->idx >= 624) orc_mt_twist(g);
    uint32_t y = g->mt[g->idx++];
    y ^= y >> 11;
    y ^= (y << 7) & 0x9d2c5680u;
    y ^= (y << 15) & 0xefc60000u;
    y ^= y >> 18;
    return y;
}

/* generate_canonical<double,53>: two 32-bit draws, low word first,
 * (g1 + g2 * 2^32) / 2^64, clamped below 1. */
double orc_mt_uniform01(orc_mt19937* g) {
    double sum = (double)orc_mt_next(g);
    sum += (double)orc_mt_next(g) * 4294967296.0;
    double r = sum / 18446744073709551616.0;
    if (r >= 1.0) r = nextafter(1.0, 0.0);
    return r;
}

/* solver.hpp:43-61 / custom_cg.hpp:45-63 */
void orc_zero_sum_vector(double* out, int64_t n, uint32_t seed) {
    orc_mt19937 g;
    orc_mt_seed(&g, seed);
    double sum = 0.0;
    for (int64_t i = 0; i < n; ++i) {
        out[i] = orc_mt_uniform01(&g);
        sum += out[i];
    }
    double mean = sum / (double)n;
    for (int64_t i = 0; i < n; ++i) out[i] -= mean;
}

void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    uint32_t k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; ++r) {
        if (r > 0) {
            k0 += 0x9E3779B9u;
            k1 += 0xBB67AE85u;
        }
        uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ c1 ^ k0;
        uint32_t n2 = hi0 ^ c3 ^ k1;
        c0 = n0;
        c1 = lo1;
        c2 = n2;
        c3 = lo0;
    }
    out[0] = c0;
    out[1] = c1;
    out[2] = c2;
    out[3] = c3;
}

double orc_sample_uniform(uint64_t seed, int32_t vertex, int32_t i) {
    uint32_t ctr[4] = {(uint32_t)vertex, (uint32_t)i >> 1, 0u, 0u};
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    uint32_t o[4];
    orc_philox4x32_10(ctr, key, o);
    uint32_t a = o[2 * (i & 1)], b = o[2 * (i & 1) + 1];
    return ((double)(a >> 5) * 67108864.0 + (double)(b >> 6)) * (1.0 / 9007199254740992.0);
}

/* ======================================================================== */
/* preprocessing                                                            */
/* ======================================================================== */

int orc_has_diagonal(int64_t nnz, const int32_t* rows, const int32_t* cols) {
    for (int64_t i = 0; i < nnz; ++i)
        if (rows[i] == cols[i]) return 1;
    return 0;
}

/* pre_process.hpp:189-306: sort_triplets_append_diagonal + triplet_to_csc.
 * The reference sorts an index vector by (col,row) with std::sort and keeps
 * duplicates; equal (col,row) keys keep input order here (counting sort by
 * row, then stable by col). */
int64_t orc_triplets_to_csc(int32_t n, int64_t nnz, const int32_t* rows, const int32_t* cols,
                            const double* vals, int32_t* colptr, int32_t* rowind, double* val) {
    int add_diag = !orc_has_diagonal(nnz, rows, cols);
    int64_t total = nnz + (add_diag ? n : 0);
    int32_t* r = (int32_t*)malloc(sizeof(int32_t) * (size_t)(total ? total : 1));
    int32_t* c = (int32_t*)malloc(sizeof(int32_t) * (size_t)(total ? total : 1));
    double* v = (double*)malloc(sizeof(double) * (size_t)(total ? total : 1));
    for (int64_t i = 0; i < nnz; ++i) {
        r[i] = rows[i];
        c[i] = cols[i];
        v[i] = (rows[i] != cols[i]) ? -fabs(vals[i]) : fabs(vals[i]);
    }
    if (add_diag) {
        for (int32_t i = 0; i < n; ++i) {
            r[nnz + i] = i;
            c[nnz + i] = i;
            v[nnz + i] = 0.0;
        }
        for (int64_t i = 0; i < nnz; ++i) v[nnz + c[i]] += fabs(v[i]);
    }
    /* two-pass stable counting sort: by row, then by col */
    int32_t* cnt = (int32_t*)calloc((size_t)n + 1, sizeof(int32_t));
    int64_t* tmp_idx = (int64_t*)malloc(sizeof(int64_t) * (size_t)(total ? total : 1));
    int64_t* ord = (int64_t*)malloc(sizeof(int64_t) * (size_t)(total ? total : 1));
    for (int64_t i = 0; i < total; ++i) cnt[r[i] + 1]++;
    for (int32_t i = 0; i < n; ++i) cnt[i + 1] += cnt[i];
    for (int64_t i = 0; i < total; ++i) tmp_idx[cnt[r[i]]++] = i;
    memset(cnt, 0, sizeof(int32_t) * ((size_t)n + 1));
    for (int64_t i = 0; i < total; ++i) cnt[c[i] + 1]++;
    for (int32_t i = 0; i < n; ++i) cnt[i + 1] += cnt[i];
    for (int32_t i = 0; i <= n; ++i) colptr[i] = cnt[i];
    for (int64_t t = 0; t < total; ++t) {
        int64_t i = tmp_idx[t];
        ord[cnt[c[i]]++] = i;
    }
    for (int64_t t = 0; t < total; ++t) {
        rowind[t] = r[ord[t]];
        val[t] = v[ord[t]];
    }
    free(cnt);
    free(tmp_idx);
    free(ord);
    free(r);
    free(c);
    free(v);
    return total;
}

int64_t orc_lower_count(int32_t n, const int32_t* colptr, const int32_t* rowind) {
    int64_t c = 0;
    for (int32_t k = 0; k < n; ++k)
        for (int32_t p = colptr[k]; p < colptr[k + 1]; ++p)
            if (rowind[p] > k) ++c;
    return c;
}

/* cpu_implementation/pre_process.hpp:785-867 (make_lower_triangular) */
void orc_lower_triangle(int32_t n, const int32_t* colptr, const int32_t* rowind, const double* val,
                        int32_t* lcolptr, int32_t* lrow, double* lval) {
    int32_t pos = 0;
    lcolptr[0] = 0;
    for (int32_t k = 0; k < n; ++k) {
        for (int32_t p = colptr[k]; p < colptr[k + 1]; ++p) {
            if (rowind[p] > k) {
                lrow[pos] = rowind[p];
                lval[pos] = fabs(val[p]);
                ++pos;
            }
        }
        lcolptr[k + 1] = pos;
    }
}

/* pre_process.hpp:474-496 (count_minimum_dependencies) */
void orc_dependency_counts(int32_t n, const int32_t* colptr, const int32_t* rowind, int32_t* dep) {
    for (int32_t k = 0; k < n; ++k) {
        int32_t c = 0;
        for (int32_t p = colptr[k]; p < colptr[k + 1]; ++p)
            if (rowind[p] < k) ++c;
        dep[k] = c;
    }
}

/* custom_cg.hpp:10-43 (remove_last_row_and_column) */
int64_t orc_trim_last(int32_t n, const int32_t* colptr, const int32_t* rowind, const double* val,
                      int32_t* ocolptr, int32_t* orowind, double* oval) {
    int32_t m = n - 1;
    int32_t k = 0;
    for (int32_t j = 0; j < m; ++j) {
        ocolptr[j] = k;
        for (int32_t p = colptr[j]; p < colptr[j + 1]; ++p) {
            if (rowind[p] < m) {
                orowind[k] = rowind[p];
                oval[k] = val[p];
                ++k;
            }
        }
    }
    ocolptr[m] = k;
    return k;
}

/* ======================================================================== */
/* factorization                                                            */
/* ======================================================================== */

typedef struct {
    int32_t row;
    int32_t mult;
    int32_t pos;       /* position in the row-ordered merged list */
    int32_t order;     /* input position (stable sorts) */
    double value;
    double cum;
} orc_entry;

typedef struct {
    int32_t* row;
    double* val;
    int32_t cnt, cap;
} orc_bucket;

struct orc_factor {
    int32_t n;
    int64_t* colptr;
    int32_t* rowind;
    double* val;
    double* diag;
    int32_t* fills_received;
    orc_factor_stats stats;
};

static uint64_t dbits(double x) {
    uint64_t u;
    memcpy(&u, &x, 8);
    return u;
}

/* (row, value bits, input order): the merge order of ORC_MODE_B200 */
static int cmp_row_value(const void* a, const void* b) {
    const orc_entry* x = (const orc_entry*)a;
    const orc_entry* y = (const orc_entry*)b;
    if (x->row != y->row) return x->row < y->row ? -1 : 1;
    uint64_t ux = dbits(x->value), uy = dbits(y->value);
    if (ux != uy) return ux < uy ? -1 : 1;
    return (x->order > y->order) - (x->order < y->order);
}

/* (row, input order): a stable row sort (reference replay) */
static int cmp_row_stable(const void* a, const void* b) {
    const orc_entry* x = (const orc_entry*)a;
    const orc_entry* y = (const orc_entry*)b;
    if (x->row != y->row) return x->row < y->row ? -1 : 1;
    return (x->order > y->order) - (x->order < y->order);
}

/* (value, row): the sampling order; rows are distinct after the merge, so
 * this is a total order.  For the replay, the input is row-ordered, so this
 * equals a stable sort by value. */
static int cmp_value_row(const void* a, const void* b) {
    const orc_entry* x = (const orc_entry*)a;
    const orc_entry* y = (const orc_entry*)b;
    if (x->value != y->value) return x->value < y->value ? -1 : 1;
    return (x->row > y->row) - (x->row < y->row);
}

static int bucket_push(orc_bucket* bk, int32_t row, double v) {
    if (bk->cnt == bk->cap) {
        int32_t nc = bk->cap ? bk->cap * 2 : 4;
        int32_t* nr = (int32_t*)realloc(bk->row, sizeof(int32_t) * (size_t)nc);
        double* nv = (double*)realloc(bk->val, sizeof(double) * (size_t)nc);
        if (!nr || !nv) return -1;
        bk->row = nr;
        bk->val = nv;
        bk->cap = nc;
    }
    bk->row[bk->cnt] = row;
    bk->val[bk->cnt] = v;
    bk->cnt++;
    return 0;
}

/* Chunked inclusive scan: Kogge-Stone within each 32-wide chunk (lane l adds
 * lane l-off for off = 1,2,4,8,16), then each element adds the running
 * carry, which is the final value of the previous chunk's last lane. */
static void chunked_scan(orc_entry* e, int32_t m) {
    double carry = 0.0;
    for (int32_t c0 = 0; c0 < m; c0 += 32) {
        double loc[32];
        for (int l = 0; l < 32; ++l) loc[l] = (c0 + l < m) ? e[c0 + l].value : 0.0;
        for (int off = 1; off < 32; off <<= 1) {
            double nxt[32];
            for (int l = 0; l < 32; ++l) nxt[l] = (l >= off) ? loc[l] + loc[l - off] : loc[l];
            memcpy(loc, nxt, sizeof(loc));
        }
        double last = 0.0;
        for (int l = 0; l < 32; ++l) {
            double f = (c0 == 0) ? loc[l] : carry + loc[l];
            if (c0 + l < m) e[c0 + l].cum = f;
            last = f;
        }
        carry = last;
    }
}

/* Per-vertex elimination, shared by both modes:
 * driver_local.cpp:454-639 (CPU) / driver.cu:287-1156 (GPU). */
orc_factor* orc_factor_run(int32_t n, const int32_t* lcolptr, const int32_t* lrow,
                           const double* lval, const int32_t* dep0, int mode, uint64_t seed) {
    orc_factor* F = (orc_factor*)calloc(1, sizeof(orc_factor));
    if (!F) return NULL;
    F->n = n;
    F->colptr = (int64_t*)calloc((size_t)n + 1, sizeof(int64_t));
    F->diag = (double*)calloc((size_t)n ? (size_t)n : 1, sizeof(double));
    F->fills_received = (int32_t*)calloc((size_t)n ? (size_t)n : 1, sizeof(int32_t));
    orc_bucket* bk = (orc_bucket*)calloc((size_t)n ? (size_t)n : 1, sizeof(orc_bucket));
    int32_t* colcnt = (int32_t*)calloc((size_t)n ? (size_t)n : 1, sizeof(int32_t));
    int32_t** colrow = (int32_t**)calloc((size_t)n ? (size_t)n : 1, sizeof(int32_t*));
    double** colval = (double**)calloc((size_t)n ? (size_t)n : 1, sizeof(double*));
    int32_t* dep = (int32_t*)malloc(sizeof(int32_t) * ((size_t)n ? (size_t)n : 1));
    int32_t* queue = (int32_t*)malloc(sizeof(int32_t) * ((size_t)n ? (size_t)n : 1));
    int32_t wcap = 256;
    orc_entry* w = (orc_entry*)malloc(sizeof(orc_entry) * (size_t)wcap);
    orc_entry* rowsorted = (orc_entry*)malloc(sizeof(orc_entry) * (size_t)wcap);
    if (!F->colptr || !F->diag || !F->fills_received || !bk || !colcnt || !colrow || !colval ||
        !dep || !queue || !w || !rowsorted)
        return NULL;

    orc_mt19937 gen;
    orc_mt_seed(&gen, (uint32_t)seed);

    int32_t qhead = 0, qtail = 0;
    if (mode == ORC_MODE_REF_REPLAY) {
        for (int32_t i = 0; i < n; ++i) {
            dep[i] = dep0[i];
            if (dep0[i] == 0) queue[qtail++] = i;
        }
    }

    for (int32_t step = 0; step < n; ++step) {
        int32_t k;
        if (mode == ORC_MODE_REF_REPLAY) {
            if (qhead >= qtail) break; /* cannot happen for a valid input */
            k = queue[qhead++];
        } else {
            k = step; /* any topological order gives the same factor */
        }
        int32_t nf = bk[k].cnt;
        int32_t no = lcolptr[k + 1] - lcolptr[k];
        int32_t total = nf + no;
        F->fills_received[k] = nf;
        if (total > wcap) {
            while (wcap < total) wcap *= 2;
            w = (orc_entry*)realloc(w, sizeof(orc_entry) * (size_t)wcap);
            rowsorted = (orc_entry*)realloc(rowsorted, sizeof(orc_entry) * (size_t)wcap);
        }
        if (total > F->stats.max_gather) F->stats.max_gather = total;
        /* gather: fills (newest first for the replay, as the linked list of
         * driver_local.cpp:615-616 is walked by auxilliary.hpp:142-168),
         * then the original strict-lower column (driver_local.cpp:486-491) */
        int32_t t = 0;
        for (int32_t q = 0; q < nf; ++q) {
            int32_t s = (mode == ORC_MODE_REF_REPLAY) ? nf - 1 - q : q;
            w[t].row = bk[k].row[s];
            w[t].value = bk[k].val[s];
            w[t].mult = 1;
            w[t].order = t;
            ++t;
        }
        for (int32_t p = lcolptr[k]; p < lcolptr[k + 1]; ++p) {
            w[t].row = lrow[p];
            w[t].value = lval[p];
            w[t].mult = 1;
            w[t].order = t;
            ++t;
        }
        free(bk[k].row);
        free(bk[k].val);
        bk[k].row = NULL;
        bk[k].val = NULL;
        bk[k].cnt = bk[k].cap = 0;

        if (total == 0) { /* driver_local.cpp:470-477 */
            F->diag[k] = 0.0;
            colcnt[k] = 0;
            continue;
        }
        /* sort by row, merge equal rows (driver_local.cpp:511-568) */
        qsort(w, (size_t)total, sizeof(orc_entry),
              mode == ORC_MODE_REF_REPLAY ? cmp_row_stable : cmp_row_value);
        int32_t m = 0;
        for (int32_t q = 0; q < total; ++q) {
            if (m > 0 && w[q].row == w[m - 1].row) {
                w[m - 1].value = w[m - 1].value + w[q].value;
                w[m - 1].mult += w[q].mult;
            } else {
                w[m] = w[q];
                ++m;
            }
        }
        F->stats.merged_away += total - m;
        if (m > F->stats.max_degree) F->stats.max_degree = m;
        for (int32_t q = 0; q < m; ++q) {
            w[q].pos = q;
            w[q].order = q;
            rowsorted[q] = w[q];
        }
        /* sort by value (driver_local.cpp:573-575), prefix sums (:582-593) */
        qsort(w, (size_t)m, sizeof(orc_entry), cmp_value_row);
        if (mode == ORC_MODE_REF_REPLAY) {
            double total_sum = 0.0;
            w[0].cum = w[0].value;
            total_sum += w[0].value;
            for (int32_t q = 1; q < m; ++q) {
                w[q].cum = w[q].value + w[q - 1].cum;
                total_sum += w[q].value;
            }
            /* total_sum equals w[m-1].cum: same additions in the same order */
        } else {
            chunked_scan(w, m);
        }
        double S = w[m - 1].cum;
        F->diag[k] = S;
        /* clique sampling (driver_local.cpp:598-631, auxilliary.hpp:543-592) */
        for (int32_t i = 0; i + 1 < m; ++i) {
            double u = (mode == ORC_MODE_REF_REPLAY) ? orc_mt_uniform01(&gen)
                                                     : orc_sample_uniform(seed, k, i);
            double rem = S - w[i].cum;
            double target = u * rem;
            /* lower_bound over (i, m): first j with (C_j - C_i) >= target */
            int32_t lo = i + 1, hi = m;
            while (lo < hi) {
                int32_t mid = lo + (hi - lo) / 2;
                if ((w[mid].cum - w[i].cum) < target) lo = mid + 1;
                else hi = mid;
            }
            int32_t j = lo < m ? lo : m - 1;
            int32_t grow = w[j].row > w[i].row ? w[j].row : w[i].row;
            int32_t gcol = w[j].row < w[i].row ? w[j].row : w[i].row;
            double gval = (w[i].value * rem) / S;
            if (bucket_push(&bk[gcol], grow, gval) != 0) return NULL;
            F->stats.fills++;
            if (mode == ORC_MODE_REF_REPLAY) dep[grow]++;
        }
        /* L column k in row order, normalised and negated
         * (driver_local.cpp:635-639 and assembly :880-956) */
        colcnt[k] = m;
        colrow[k] = (int32_t*)malloc(sizeof(int32_t) * (size_t)m);
        colval[k] = (double*)malloc(sizeof(double) * (size_t)m);
        for (int32_t q = 0; q < m; ++q) {
            int32_t p = w[q].pos;
            colrow[k][p] = w[q].row;
            colval[k][p] = -(w[q].value / S);
        }
        if (mode == ORC_MODE_REF_REPLAY) {
            /* dependency release in value order (driver_local.cpp:653-687) */
            for (int32_t q = 0; q < m; ++q) {
                int32_t r = w[q].row;
                int32_t old = dep[r];
                dep[r] -= w[q].mult;
                if (old == w[q].mult) queue[qtail++] = r;
            }
        }
    }

    /* assemble the strict CSC */
    F->colptr[0] = 0;
    for (int32_t k = 0; k < n; ++k) F->colptr[k + 1] = F->colptr[k] + colcnt[k];
    int64_t nnz = F->colptr[n];
    F->stats.nnz_strict = nnz;
    F->rowind = (int32_t*)malloc(sizeof(int32_t) * (size_t)(nnz ? nnz : 1));
    F->val = (double*)malloc(sizeof(double) * (size_t)(nnz ? nnz : 1));
    for (int32_t k = 0; k < n; ++k) {
        if (colcnt[k]) {
            memcpy(F->rowind + F->colptr[k], colrow[k], sizeof(int32_t) * (size_t)colcnt[k]);
            memcpy(F->val + F->colptr[k], colval[k], sizeof(double) * (size_t)colcnt[k]);
        }
        free(colrow[k]);
        free(colval[k]);
    }
    for (int32_t k = 0; k < n; ++k) {
        free(bk[k].row);
        free(bk[k].val);
    }
    free(bk);
    free(colcnt);
    free(colrow);
    free(colval);
    free(dep);
    free(queue);
    free(w);
    free(rowsorted);
    return F;
}

void orc_factor_stats_get(const orc_factor* f, orc_factor_stats* s) { *s = f->stats; }

void orc_factor_export(const orc_factor* f, int64_t* colptr, int32_t* rowind, double* val,
                       double* diag, int32_t* fills_received) {
    int64_t nnz = f->colptr[f->n];
    if (colptr) memcpy(colptr, f->colptr, sizeof(int64_t) * ((size_t)f->n + 1));
    if (rowind) memcpy(rowind, f->rowind, sizeof(int32_t) * (size_t)nnz);
    if (val) memcpy(val, f->val, sizeof(double) * (size_t)nnz);
    if (diag) memcpy(diag, f->diag, sizeof(double) * (size_t)f->n);
    if (fills_received) memcpy(fills_received, f->fills_received, sizeof(int32_t) * (size_t)f->n);
}

void orc_factor_free(orc_factor* f) {
    if (!f) return;
    free(f->colptr);
    free(f->rowind);
    free(f->val);
    free(f->diag);
    free(f->fills_received);
    free(f);
}

/* ======================================================================== */
/* PCG                                                                      */
/* ======================================================================== */

void orc_spmv(int32_t n, const int32_t* rowptr, const int32_t* colind, const double* val,
              const double* x, double* y, int nthreads) {
#ifdef _OPENMP
#pragma omp parallel for schedule(static) num_threads(nthreads > 0 ? nthreads : 1)
#endif
    for (int32_t i = 0; i < n; ++i) {
        double s = 0.0;
        for (int32_t p = rowptr[i]; p < rowptr[i + 1]; ++p) s += val[p] * x[colind[p]];
        y[i] = s;
    }
}

/* solver.hpp:150-233 / custom_cg.hpp:225-236: forward solve with L (the
 * TRANSPOSE solve of the CSR-upper factor), D^+ (skip D = 0), backward solve
 * with L^T. */
void orc_precond_apply(int32_t n, const int64_t* lcolptr, const int32_t* lrow, const double* lval,
                       const double* diag, const double* r, double* z, double* y) {
    for (int32_t i = 0; i < n; ++i) y[i] = r[i];
    for (int32_t j = 0; j < n; ++j) {
        double yj = y[j];
        for (int64_t p = lcolptr[j]; p < lcolptr[j + 1]; ++p) y[lrow[p]] = y[lrow[p]] - lval[p] * yj;
    }
    for (int32_t j = 0; j < n; ++j)
        if (diag[j] != 0.0) y[j] = y[j] / diag[j];
    for (int32_t j = n - 1; j >= 0; --j) {
        double s = y[j];
        for (int64_t p = lcolptr[j]; p < lcolptr[j + 1]; ++p) s = s - lval[p] * z[lrow[p]];
        z[j] = s;
    }
}

static double dot(int32_t n, const double* a, const double* b, int nthreads) {
    double s = 0.0;
#ifdef _OPENMP
#pragma omp parallel for reduction(+ : s) schedule(static) num_threads(nthreads > 0 ? nthreads : 1)
#endif
    for (int32_t i = 0; i < n; ++i) s += a[i] * b[i];
    return s;
}

static double true_relres(int32_t n, const int32_t* arowptr, const int32_t* acolind,
                          const double* aval, const double* b, const double* x, double* tmp,
                          double bnorm, int nthreads) {
    orc_spmv(n, arowptr, acolind, aval, x, tmp, nthreads);
    for (int32_t i = 0; i < n; ++i) tmp[i] = b[i] - tmp[i];
    return sqrt(dot(n, tmp, tmp, nthreads)) / bnorm;
}

/* solver.hpp:457-569 (recurrence, true-residual report) and
 * custom_cg.hpp:65-265 (trim handled by the caller, x0 = 0). */
int orc_pcg(int32_t n, const int32_t* arowptr, const int32_t* acolind, const double* aval,
            const int64_t* lcolptr, const int32_t* lrow, const double* lval, const double* diag,
            const double* b, double* x, double tol, int32_t max_iter, int stop_rule, int nthreads,
            orc_pcg_info* info) {
    size_t sz = (size_t)(n ? n : 1);
    double* r = (double*)malloc(sizeof(double) * sz);
    double* z = (double*)malloc(sizeof(double) * sz);
    double* p = (double*)malloc(sizeof(double) * sz);
    double* q = (double*)malloc(sizeof(double) * sz);
    double* work = (double*)malloc(sizeof(double) * sz);
    if (!r || !z || !p || !q || !work) return -1;
    memset(info, 0, sizeof(*info));
    for (int32_t i = 0; i < n; ++i) {
        x[i] = 0.0;
        r[i] = b[i];
    }
    double bnorm = sqrt(dot(n, b, b, nthreads));
    if (bnorm == 0.0) {
        info->converged = 1;
        goto done;
    }
    orc_precond_apply(n, lcolptr, lrow, lval, diag, r, z, work);
    for (int32_t i = 0; i < n; ++i) p[i] = z[i];
    double rz = dot(n, r, z, nthreads);
    double rz0 = rz;
    int32_t k = 0;
    int converged = 0;
    if (stop_rule == ORC_STOP_PRECOND && !(rz > tol)) converged = 1;
    while (!converged && k < max_iter) {
        orc_spmv(n, arowptr, acolind, aval, p, q, nthreads);
        double alpha = rz / dot(n, p, q, nthreads);
        for (int32_t i = 0; i < n; ++i) {
            x[i] = x[i] + alpha * p[i];
            r[i] = r[i] - alpha * q[i];
        }
        ++k;
        if (stop_rule == ORC_STOP_RELRES) {
            double rr = dot(n, r, r, nthreads);
            if (sqrt(rr) / bnorm <= tol) {
                double tr = true_relres(n, arowptr, acolind, aval, b, x, work, bnorm, nthreads);
                if (tr <= tol) {
                    converged = 1;
                    break;
                }
                /* residual replacement: continue from the true residual */
                orc_spmv(n, arowptr, acolind, aval, x, work, nthreads);
                for (int32_t i = 0; i < n; ++i) r[i] = b[i] - work[i];
            }
        } else if (stop_rule == ORC_STOP_ABS_R2) {
            if (dot(n, r, r, nthreads) <= tol) {
                converged = 1;
                break;
            }
        }
        if (k >= max_iter) break;
        orc_precond_apply(n, lcolptr, lrow, lval, diag, r, z, work);
        double rz_new = dot(n, r, z, nthreads);
        double beta = rz_new / rz;
        rz = rz_new;
        for (int32_t i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
        if (stop_rule == ORC_STOP_PRECOND && !(sqrt(rz) / sqrt(rz0) > tol)) converged = 1;
    }
    info->iterations = k;
    info->converged = converged;
    info->precond_ratio = rz0 > 0 ? sqrt(rz) / sqrt(rz0) : 0.0;
    info->relres_rec = sqrt(dot(n, r, r, nthreads)) / bnorm;
    info->relres_true = true_relres(n, arowptr, acolind, aval, b, x, work, bnorm, nthreads);
done:
    free(r);
    free(z);
    free(p);
    free(q);
    free(work);
    return 0;
}
