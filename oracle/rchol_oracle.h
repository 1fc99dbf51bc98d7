/*
 * rchol_oracle.h -- CPU restatement of the reference's randomized-Cholesky
 * factor + PCG path.  TEST INFRASTRUCTURE ONLY: it is the checker that the
 * CUDA path is compared against, and the CPU-baseline leg of bench.py.  The
 * product (the C-ABI library and the CLI drivers) never links or calls it.
 *
 * Parity pins (see tests/test_oracle_*.py):
 *   - the factor in ORC_MODE_REF_REPLAY is checked against the reference CPU
 *     factor (cpu_implementation/driver_local.cpp) compiled from its sources
 *     with its std::random_device seed pinned, 1 thread: same sparsity
 *     pattern, values within 1e-12 relative;
 *   - orc_zero_sum_vector is checked bit-exactly against golden vectors made
 *     by the reference's own generate_zero_sum_vector (solver.hpp:43-61);
 *   - the preprocessing is checked against the reference's parsed CSC.
 */
#ifndef RCHOL_ORACLE_H
#define RCHOL_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- random numbers ---------------------------------------------------- */

/* std::mt19937 (Matsumoto-Nishimura 1998) + libstdc++'s
 * generate_canonical<double,53> as used by
 * std::uniform_real_distribution<double>(0,1). */
typedef struct {
    uint32_t mt[624];
    int idx;
} orc_mt19937;

void orc_mt_seed(orc_mt19937* g, uint32_t seed);
uint32_t orc_mt_next(orc_mt19937* g);
double orc_mt_uniform01(orc_mt19937* g);

/* generate_zero_sum_vector(h_vec, n, seed): solver.hpp:43-61,
 * custom_cg.hpp:45-63.  U[0,1) draws minus their mean. */
void orc_zero_sum_vector(double* out, int64_t n, uint32_t seed);

/* Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11). */
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);

/* The clique-sampling uniform of vertex `vertex`, neighbour slot `i`:
 * Philox4x32-10 with key = seed, counter = (vertex, i/2, 0, 0); the two
 * 32-bit words (2*(i%2), 2*(i%2)+1) give a 53-bit value in [0,1). */
double orc_sample_uniform(uint64_t seed, int32_t vertex, int32_t i);

/* ---- preprocessing (gpu_implementation/pre_process.hpp:189-306, 474-496,
 *      cpu_implementation/pre_process.hpp:785-867) ------------------------ */

/* 1 if any triplet lies on the diagonal (pre_process.hpp:338-345). */
int orc_has_diagonal(int64_t nnz, const int32_t* rows, const int32_t* cols);

/* Sign-normalise (off-diagonal -> -|v|, diagonal -> |v|), append the
 * diagonal as the column sum of |off-diagonal| when the input has none, sort
 * by (col,row) and build CSC.  Duplicate (row,col) entries are kept.
 * Output sizes: colptr[n+1], rowind/val[nnz + (has_diag ? 0 : n)].
 * Returns the number of CSC entries. */
int64_t orc_triplets_to_csc(int32_t n, int64_t nnz, const int32_t* rows, const int32_t* cols,
                            const double* vals, int32_t* colptr, int32_t* rowind, double* val);

/* Number of strict-lower entries (row > col) of a CSC matrix. */
int64_t orc_lower_count(int32_t n, const int32_t* colptr, const int32_t* rowind);

/* Strict lower triangle with |values| (make_lower_triangular). */
void orc_lower_triangle(int32_t n, const int32_t* colptr, const int32_t* rowind, const double* val,
                        int32_t* lcolptr, int32_t* lrow, double* lval);

/* dep[k] = number of entries of column k with row < k
 * (count_minimum_dependencies, pre_process.hpp:474-496). */
void orc_dependency_counts(int32_t n, const int32_t* colptr, const int32_t* rowind, int32_t* dep);

/* Drop the last row and column of a CSC matrix (ground-vertex trim,
 * custom_cg.hpp:10-43).  Output arrays sized like the input.  Returns the
 * new nnz. */
int64_t orc_trim_last(int32_t n, const int32_t* colptr, const int32_t* rowind, const double* val,
                      int32_t* ocolptr, int32_t* orowind, double* oval);

/* ---- factorization ------------------------------------------------------ */

enum {
    /* Semantics of the CUDA factor: uniforms from Philox keyed by
     * (seed, vertex, slot); duplicates merged in (row, value) order; samples
     * drawn over the merged neighbours in (value, row) order; prefix sums
     * computed in 32-wide chunks (Kogge-Stone inside a chunk, carried
     * sequentially across chunks).  The result does not depend on the order
     * in which independent vertices are eliminated. */
    ORC_MODE_B200 = 0,
    /* Exact single-thread replay of the reference CPU factor
     * (cpu_implementation/driver_local.cpp:302-707): FIFO ready queue, one
     * std::mt19937(seed) stream consumed in elimination order, fills
     * gathered newest-first then the original column, stable row sort,
     * sequential merge and prefix sums. */
    ORC_MODE_REF_REPLAY = 1
};

typedef struct orc_factor orc_factor;

typedef struct {
    int64_t nnz_strict;     /* off-diagonal entries of L */
    int64_t fills;          /* sampled fill edges emitted */
    int64_t merged_away;    /* duplicate entries combined during merges */
    int32_t max_degree;     /* largest merged neighbour count */
    int32_t max_gather;     /* largest pre-merge neighbour count */
} orc_factor_stats;

/* Factor the strict-lower CSC (values positive, |a_ij|) with initial
 * dependency counts dep0.  Returns NULL on allocation failure. */
orc_factor* orc_factor_run(int32_t n, const int32_t* lcolptr, const int32_t* lrow,
                           const double* lval, const int32_t* dep0, int mode, uint64_t seed);
void orc_factor_stats_get(const orc_factor* f, orc_factor_stats* s);

/* Export the factor: strict CSC of L (rows ascending per column, values
 * -w/sum as in the assembled reference factor), the diagonal D, and the
 * number of fill edges each column received. */
void orc_factor_export(const orc_factor* f, int64_t* colptr, int32_t* rowind, double* val,
                       double* diag, int32_t* fills_received);
void orc_factor_free(orc_factor* f);

/* ---- PCG (solver.hpp:236-593, custom_cg.hpp:65-265) --------------------- */

enum {
    ORC_STOP_RELRES = 0,     /* ||r|| / ||b|| <= tol on the recurrence residual,
                                confirmed on the true residual b - A x */
    ORC_STOP_PRECOND = 1,    /* sqrt(r.z / r0.z0) <= tol (solver.hpp:536), max iters */
    ORC_STOP_ABS_R2 = 2      /* ||r||^2 <= tol (custom_cg.hpp:214-223) */
};

typedef struct {
    int32_t iterations;
    int32_t converged;
    double relres_true;      /* ||b - A x|| / ||b|| at exit */
    double relres_rec;       /* ||r|| / ||b|| of the recurrence at exit */
    double precond_ratio;    /* sqrt(r.z / r0.z0) at exit */
} orc_pcg_info;

/* y = A x for a CSR matrix (a symmetric CSC is its own CSR). */
void orc_spmv(int32_t n, const int32_t* rowptr, const int32_t* colind, const double* val,
              const double* x, double* y, int nthreads);

/* z = L^-T D^+ L^-1 r with L unit lower triangular given by its strict CSC
 * (column-major, as exported) and D^+ dividing only where D != 0
 * (solver.hpp:150-233, custom_cg.hpp:225-236). */
void orc_precond_apply(int32_t n, const int64_t* lcolptr, const int32_t* lrow, const double* lval,
                       const double* diag, const double* r, double* z, double* work);

int orc_pcg(int32_t n, const int32_t* arowptr, const int32_t* acolind, const double* aval,
            const int64_t* lcolptr, const int32_t* lrow, const double* lval, const double* diag,
            const double* b, double* x, double tol, int32_t max_iter, int stop_rule,
            int nthreads, orc_pcg_info* info);

/* ---- synthetic inputs without the product library (gen_inputs.c) ------ */

/* The library's grid generator (rchol_generate with ordering 0) restated:
 * kind "grid2d", "grid3d" or "grid3d27"; ascending-nnz order with a seeded
 * tie-break; a ground vertex appended when any row has diagonal excess.
 * The triplet arrays are malloc'ed (release with orc_free).  Returns 0, or
 * a negative value for a bad kind or a failed allocation. */
int orc_generate_grid(const char* kind, const int64_t* dims, int ndims, double wlo, double whi, int log_weights,
                      double aniso_z, double excess_frac, double excess_lo, double excess_hi, uint64_t seed,
                      int32_t* n_out, int64_t* nnz_out, int32_t** rows_out, int32_t** cols_out,
                      double** vals_out, int32_t* has_ground_out);
void orc_free(void* p);
/* 1-based coordinate/real/general MatrixMarket file, entries in order. */
int orc_write_mtx(const char* path, int32_t n, int64_t nnz, const int32_t* rows, const int32_t* cols,
                  const double* vals);

#ifdef __cplusplus
}
#endif

#endif
