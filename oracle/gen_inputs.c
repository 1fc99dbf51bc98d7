/*
 * gen_inputs.c -- the synthetic benchmark inputs, generated without the
 * product library.  TEST INFRASTRUCTURE ONLY: the CPU legs of bench.py (the
 * reference arm and the CPU baseline) build their .mtx input with this code
 * so that the reference's processes never load librchol_b200.so.
 *
 * It restates the grid part of the library's own generator (rchol_generate)
 * step for step -- the same counter-based splitmix64 streams, the same edge
 * order, the same arithmetic -- so both produce bit-identical triplets; a
 * CPU test compares them.  The conversion of an SDDM to a Laplacian by one
 * ground vertex and the ascending-nnz order with a seeded tie-break follow
 * cpu_implementation/write_graph.jl:112-128 and 153-163.
 */
#include "rchol_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

static uint64_t gen_mix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

static uint64_t gen_hash3(uint64_t seed, uint64_t stream, uint64_t i) {
    return gen_mix64(gen_mix64(gen_mix64(seed) ^ (stream * 0xD1B54A32D192ED03ull)) ^ i);
}

static double gen_unit(uint64_t h) { return (double)(h >> 11) * (1.0 / 9007199254740992.0); }

enum { S_WEIGHT = 1, S_EXCESS_PICK = 2, S_EXCESS_VAL = 3, S_ORDER = 4 };

static double gen_weight(uint64_t seed, double wlo, double whi, int log_weights, uint64_t e) {
    double u = gen_unit(gen_hash3(seed, S_WEIGHT, e));
    if (log_weights) return exp(log(wlo) + u * (log(whi) - log(wlo)));
    return wlo + u * (whi - wlo);
}

typedef struct {
    int64_t deg;
    uint64_t key;
    int64_t id;
} gen_ord;

static int gen_ord_cmp(const void* a, const void* b) {
    const gen_ord* x = (const gen_ord*)a;
    const gen_ord* y = (const gen_ord*)b;
    if (x->deg != y->deg) return x->deg < y->deg ? -1 : 1;
    if (x->key != y->key) return x->key < y->key ? -1 : 1;
    return x->id < y->id ? -1 : (x->id > y->id);
}

int orc_generate_grid(const char* kind, const int64_t* dims, int ndims, double wlo, double whi, int log_weights,
                      double aniso_z, double excess_frac, double excess_lo, double excess_hi, uint64_t seed,
                      int32_t* n_out, int64_t* nnz_out, int32_t** rows_out, int32_t** cols_out,
                      double** vals_out, int32_t* has_ground_out) {
    const int p27 = strcmp(kind, "grid3d27") == 0;
    if (!p27 && strcmp(kind, "grid2d") != 0 && strcmp(kind, "grid3d") != 0) return -1;
    if (ndims < 1) return -1;
    const int is3 = ndims >= 3;
    const int64_t nx = dims[0], ny = ndims > 1 ? dims[1] : dims[0], nz = is3 ? dims[2] : 1;
    const int64_t n = nx * ny * nz;
    /* neighbour offsets whose first nonzero component is positive */
    int offs[3 * 13];
    int no = 0;
    if (p27) {
        for (int dz = -1; dz <= 1; ++dz)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx) {
                    int first = dz != 0 ? dz : (dy != 0 ? dy : dx);
                    if (first > 0) {
                        offs[3 * no] = dx;
                        offs[3 * no + 1] = dy;
                        offs[3 * no + 2] = dz;
                        ++no;
                    }
                }
    } else {
        static const int o[] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
        no = is3 ? 3 : 2;
        memcpy(offs, o, sizeof(int) * 3 * (size_t)no);
    }
    const int64_t emax = n * no;
    int64_t* ea = (int64_t*)malloc(sizeof(int64_t) * (size_t)(emax ? emax : 1));
    int64_t* eb = (int64_t*)malloc(sizeof(int64_t) * (size_t)(emax ? emax : 1));
    double* ew = (double*)malloc(sizeof(double) * (size_t)(emax ? emax : 1));
    if (!ea || !eb || !ew) return -2;
    int64_t ne = 0;
    uint64_t e = 0;
    for (int64_t z = 0; z < nz; ++z)
        for (int64_t y = 0; y < ny; ++y)
            for (int64_t x = 0; x < nx; ++x)
                for (int k = 0; k < no; ++k) {
                    int dx = offs[3 * k], dy = offs[3 * k + 1], dz = offs[3 * k + 2];
                    int64_t X = x + dx, Y = y + dy, Z = z + dz;
                    if (X < 0 || X >= nx || Y < 0 || Y >= ny || Z < 0 || Z >= nz) continue;
                    double base = 1.0;
                    if (aniso_z != 1.0) {
                        double d2 = (double)(dx * dx + dy * dy + dz * dz);
                        base = ((double)(dx * dx) + (double)(dy * dy) + aniso_z * (double)(dz * dz)) / (d2 * d2);
                    } else if (p27) {
                        double d2 = (double)(dx * dx + dy * dy + dz * dz);
                        base = 1.0 / d2;
                    }
                    ea[ne] = x + nx * (y + ny * z);
                    eb[ne] = X + nx * (Y + ny * Z);
                    ew[ne] = base * gen_weight(seed, wlo, whi, log_weights, e);
                    ++ne;
                    ++e;
                }
    double* wdeg = (double*)calloc((size_t)n, sizeof(double));
    double* excess = (double*)calloc((size_t)n, sizeof(double));
    gen_ord* ord = (gen_ord*)malloc(sizeof(gen_ord) * (size_t)n);
    int32_t* pos = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
    if (!wdeg || !excess || !ord || !pos) return -2;
    for (int64_t i = 0; i < n; ++i) {
        ord[i].deg = 0;
        ord[i].key = gen_hash3(seed, S_ORDER, (uint64_t)i);
        ord[i].id = i;
    }
    for (int64_t k = 0; k < ne; ++k) {
        wdeg[ea[k]] += ew[k];
        wdeg[eb[k]] += ew[k];
        ord[ea[k]].deg++;
        ord[eb[k]].deg++;
    }
    int has_ground = 0;
    if (excess_frac > 0.0) {
        for (int64_t i = 0; i < n; ++i) {
            if (gen_unit(gen_hash3(seed, S_EXCESS_PICK, (uint64_t)i)) < excess_frac) {
                double u = gen_unit(gen_hash3(seed, S_EXCESS_VAL, (uint64_t)i));
                excess[i] = (excess_lo + u * (excess_hi - excess_lo)) * wdeg[i];
                if (excess[i] > 0.0) has_ground = 1;
            }
        }
    }
    /* ascending degree, ties by the seeded key (then by index) */
    qsort(ord, (size_t)n, sizeof(gen_ord), gen_ord_cmp);
    for (int64_t i = 0; i < n; ++i) pos[ord[i].id] = (int32_t)i;
    free(ord);
    const int32_t N = (int32_t)(n + (has_ground ? 1 : 0));
    int64_t ng = 0;
    if (has_ground)
        for (int64_t i = 0; i < n; ++i) ng += excess[i] > 0.0;
    const int64_t total = 2 * ne + 2 * ng + N;
    int32_t* rows = (int32_t*)malloc(sizeof(int32_t) * (size_t)total);
    int32_t* cols = (int32_t*)malloc(sizeof(int32_t) * (size_t)total);
    double* vals = (double*)malloc(sizeof(double) * (size_t)total);
    if (!rows || !cols || !vals) return -2;
    int64_t t = 0;
    for (int64_t k = 0; k < ne; ++k) {
        int32_t u = pos[ea[k]], v = pos[eb[k]];
        rows[t] = u;
        cols[t] = v;
        vals[t++] = -ew[k];
        rows[t] = v;
        cols[t] = u;
        vals[t++] = -ew[k];
    }
    double gsum = 0.0;
    if (has_ground) {
        for (int64_t i = 0; i < n; ++i) {
            double x = excess[i];
            if (x <= 0.0) continue;
            int32_t u = pos[i];
            rows[t] = u;
            cols[t] = N - 1;
            vals[t++] = -x;
            rows[t] = N - 1;
            cols[t] = u;
            vals[t++] = -x;
            gsum += x;
        }
    }
    for (int64_t i = 0; i < n; ++i) {
        int32_t u = pos[i];
        rows[t] = u;
        cols[t] = u;
        vals[t++] = wdeg[i] + excess[i];
    }
    if (has_ground) {
        rows[t] = N - 1;
        cols[t] = N - 1;
        vals[t++] = gsum;
    }
    free(ea);
    free(eb);
    free(ew);
    free(wdeg);
    free(excess);
    free(pos);
    *n_out = N;
    *nnz_out = t;
    *rows_out = rows;
    *cols_out = cols;
    *vals_out = vals;
    *has_ground_out = has_ground;
    return 0;
}

void orc_free(void* p) { free(p); }

int orc_write_mtx(const char* path, int32_t n, int64_t nnz, const int32_t* rows, const int32_t* cols,
                  const double* vals) {
    FILE* f = fopen(path, "w");
    if (!f) return -1;
    static char buf[1 << 20];
    setvbuf(f, buf, _IOFBF, sizeof(buf));
    fprintf(f, "%%%%MatrixMarket matrix coordinate real general\n%d %d %lld\n", n, n, (long long)nnz);
    for (int64_t k = 0; k < nnz; ++k) fprintf(f, "%d %d %.17g\n", rows[k] + 1, cols[k] + 1, vals[k]);
    return fclose(f) == 0 ? 0 : -1;
}
