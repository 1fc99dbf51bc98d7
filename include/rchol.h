/*
 * rchol.h -- C ABI of the B200-native randomized-Cholesky PCG solver.
 *
 * Plain C types only (pointers, sizes, status codes).  Every entry point
 * returns an rchol_status; nothing throws across the boundary.  Buffers are
 * owned by the caller unless an entry point says it allocates.  One context
 * per host thread; all device work of a context runs on its own stream.
 *
 * Reference interfaces replaced (Tianyu-Liang/Parallel-Randomized-Cholesky):
 *   factorization_driver<int,double>(processor, num_blocks, check_solve, tol)
 *       gpu_implementation/driver.cu:1551 (driver_physics.cu:1744)
 *   prepare_and_solve<int,double>(spmat_device, csr_rowptr, csr_val, csr_col,
 *       diag, tol, physics, factor_nnz, removal)   gpu_implementation/solver.hpp:236-238
 *   example_pcg_solver(A, M, diag, is_graph)       experiment/custom_cg.hpp:65-66
 *   sparse_matrix_processor<int,double>(path)      gpu_implementation/pre_process.hpp:322
 *   factor write-out (l_sol.mtx + sol_diag.txt)    experiment/driver_local.cpp:958-988
 */
#ifndef RCHOL_H
#define RCHOL_H

#ifdef __cplusplus
extern "C" {
#endif

typedef enum rchol_status {
    RCHOL_OK = 0,
    RCHOL_ERR_INVALID = 1,       /* bad argument or malformed input */
    RCHOL_ERR_IO = 2,            /* file could not be read or written */
    RCHOL_ERR_CUDA = 3,          /* a CUDA runtime call failed */
    RCHOL_ERR_CAPACITY = 4,      /* a device pool stayed too small after retries */
    RCHOL_ERR_TIMEOUT = 5,       /* a bounded device wait gave up */
    RCHOL_ERR_NOT_CONVERGED = 6, /* PCG stopped before reaching the tolerance */
    RCHOL_ERR_NO_DEVICE = 7,     /* no CUDA device (the library has no CPU path) */
    RCHOL_ERR_NUMERIC = 8,       /* NaN/Inf or a negative weight in the input */
    RCHOL_ERR_NO_MATRIX = 9      /* no matrix loaded into the context */
} rchol_status;

enum { RCHOL_PREC_FP64 = 0, RCHOL_PREC_FP32_FACTOR = 1 };

enum {
    RCHOL_STOP_RELRES = 0,  /* ||b - A x|| / ||b|| <= tol (true FP64 residual) */
    RCHOL_STOP_PRECOND = 1, /* sqrt(r.z / r0.z0) <= tol, as solver.hpp:536 */
    RCHOL_STOP_ABS_R2 = 2   /* ||r||^2 <= tol, as custom_cg.hpp:214-223 */
};

enum { RCHOL_SPMV_AUTO = 0, RCHOL_SPMV_CSR = 1 };

typedef struct rchol_ctx rchol_ctx;
typedef struct rchol_factor rchol_factor_t;

typedef struct rchol_opts {
    int precision;            /* RCHOL_PREC_FP64 or RCHOL_PREC_FP32_FACTOR */
    unsigned long long seed;  /* factorization seed (Philox key) */
    int num_blocks;           /* reference <num_blocks>: 32-thread squads for the
                                 factor; 0 = the whole resident grid */
    int warps_per_block;      /* factor CTA size in warps (1..8) */
    int slab_entries;         /* per-warp shared-memory slab (power of two) */
    int bucket_cap;           /* first fill chunk per column (default 64; larger buckets
                                 spare the overflow-chunk walks of big gathers) */
    double pool_mult;         /* factor pool capacity / nnz(strict lower A) */
    int max_iter;             /* PCG iteration cap */
    double tol;               /* PCG tolerance (meaning set by stop_rule) */
    int stop_rule;            /* RCHOL_STOP_* */
    int unroll;               /* PCG iterations per graph launch */
    int use_graph;            /* capture PCG iterations in a CUDA graph */
    int device;               /* CUDA device ordinal */
    double timeout_s;         /* bound on every device-side wait */
    int verbose;              /* print phase timings (the reference's stdout) */
    int poll_ns;              /* back-off (ns) between polls in the triangular solves */
    int sched_epl;            /* triangular-solve schedule: matrix entries per lane (1..64), or 0:
                                 automatic (3 when every row of L has at most 1024 entries, else 2) */
    int exact_bwd_levels;     /* order the backward solve by its true DAG levels (default 1) */
    int spmv_layout;          /* one-RHS PCG SpMV: RCHOL_SPMV_AUTO (sliced-ELL copy of A
                                 when its padding is at most 25%, else CSR) or RCHOL_SPMV_CSR */
    int tail_vertices;        /* the last tail_vertices vertices are eliminated one at a time by a
                                 whole 1024-thread CTA each, after the rest (hubs and dense cores of
                                 power-law graphs); 0 = none; rchol_autotune picks it */
    int rhs_block;            /* multi-RHS PCG: solve k right-hand sides in blocks of this width
                                 (1, 2, 4, 8, 16, 32; 0 = all k at once); rchol_autotune picks it */
    int bwd_head;             /* one-RHS PCG (exact backward levels): solve the narrow first levels
                                 of the backward DAG in one CTA with the values in shared memory
                                 before the persistent kernel (default 1; 0 = off) */
} rchol_opts;

typedef struct rchol_factor_info {
    int n;                    /* dimension of the solve (ground trimmed) */
    int n_factored;           /* dimension that was eliminated */
    long long nnz_strict;     /* off-diagonal entries of L */
    long long nnz_lower_a;    /* strict-lower entries of the input */
    long long fills;          /* sampled fill edges */
    int max_gather;           /* largest pre-merge neighbour list */
    int big_vertices;         /* vertices staged in the global slab */
    int overflow_fills;       /* fills that went to overflow chunks */
    int chunks_used;
    int factor_grid;          /* CTAs of the factor launch */
    float ms_setup;           /* lower triangle + dependency counts + queue */
    float ms_factor;          /* the elimination kernel */
    float ms_assemble;        /* pool -> CSC/CSR, trim, FP32 copies */
    int attempts;             /* capacity retries + 1 */
    int solve_depth;          /* levels of the triangular-solve dependency DAG */
    int kernel_launches;      /* device kernels launched by this factorization */
    /* device pointers (valid while the factor lives) */
    const long long* lc_ptr;  /* strict CSC of L  [n+1] */
    const int* lc_idx;
    const double* lc_val;
    const long long* lr_ptr;  /* strict CSR of L  [n+1] */
    const int* lr_idx;
    const double* lr_val;
    const double* diag;       /* D [n] */
    int tail_vertices;        /* vertices eliminated by the cooperative tail pass */
    int solve_depth_b;        /* levels of the backward-solve DAG (exact levels) */
    int bwd_head_levels;      /* backward levels solved by the one-CTA head kernel (0: none) */
    int bwd_head_rows;        /* rows in those levels */
} rchol_factor_info;

typedef struct rchol_solve_info {
    int iterations;           /* max over right-hand sides */
    int converged;            /* 1 if every right-hand side met the stop rule */
    int device_status;        /* 0, or the device error code */
    double relres_true;       /* max ||b - A x|| / ||b|| (FP64, recomputed) */
    double relres_rec;        /* max recurrence ||r|| / ||b|| */
    double precond_ratio;     /* max sqrt(r.z / r0.z0) */
    float ms_total;           /* device time of the solve */
    float ms_iterations;      /* device time of the iteration loop */
    int kernel_launches;
    int graph_launches;
} rchol_solve_info;

/* ---- context -------------------------------------------------------- */
rchol_status rchol_opts_default(rchol_opts* opts);
rchol_status rchol_create(rchol_ctx** ctx, const rchol_opts* opts);
void rchol_destroy(rchol_ctx* ctx);
rchol_status rchol_set_opts(rchol_ctx* ctx, const rchol_opts* opts);
const char* rchol_status_string(rchol_status s);
const char* rchol_last_error(const rchol_ctx* ctx);

/* ---- input ------------------------------------------------------------
 * rchol_load_mtx replaces sparse_matrix_processor(path) (pre_process.hpp:322):
 * MatrixMarket coordinate file, symmetric files generalised, off-diagonals
 * forced to -|v|, diagonal |v|, diagonal appended as sum|off| when absent.
 * trim_ground = 1 marks an SDDM converted to a Laplacian by appending a ground
 * vertex (the reference's trailing "1" / driver_physics build): the last
 * vertex is eliminated and then removed from the factor and from A. */
rchol_status rchol_load_mtx(rchol_ctx* ctx, const char* path, int trim_ground);
/* Same preprocessing from 0-based host triplets. */
rchol_status rchol_set_triplets(rchol_ctx* ctx, int n, long long nnz, const int* rows, const int* cols,
                                const double* vals, int trim_ground);
/* An SDDM (or a Laplacian) as the reference's physics preprocessing takes
 * it -- physics_produce, cpu_implementation/write_graph.jl:98-183, run there
 * offline in Julia -- converted and ordered on the device:
 *   signs normalised (off-diagonal -|v|, diagonal |v|; a diagonal of
 *   sum |off| per column appended when the input has none);
 *   ordering RCHOL_ORDER_NNZ_SORT: a seeded random permutation, then a
 *   stable sort by column nnz (write_graph.jl:112-128); RCHOL_ORDER_RANDOM:
 *   the seeded permutation alone; RCHOL_ORDER_GIVEN: the input order;
 *   RCHOL_ORDER_RCM / RCHOL_ORDER_ND: computed on the host (see below);
 *   ground vertex (write_graph.jl:153-163): when the entries sum to more
 *   than 1e-9, vertex n is appended with entries -c_j for every column sum
 *   c_j > 0 and diagonal sum c_j, and the context trims it after factoring
 *   (*has_ground = 1); a sum below -1e-9 returns RCHOL_ERR_NUMERIC.
 * rows/cols/vals: nnz 0-based triplets (both triangles), host (on_device =
 * 0) or device (1).  perm (host, n entries, may be NULL) receives the
 * position of each input vertex in the context's matrix: right-hand sides
 * and solutions of the input's numbering map through it. */
enum {
    RCHOL_ORDER_GIVEN = 0,
    RCHOL_ORDER_NNZ_SORT = 1,
    RCHOL_ORDER_RANDOM = 2,
    RCHOL_ORDER_RCM = 3,  /* reverse Cuthill-McKee (host, from the pattern) */
    RCHOL_ORDER_ND = 4    /* nested dissection by level-structure bisection (host); the
                             reference's "amd" / "nd" come from Julia's AMD / Metis
                             (write_graph.jl:61-75), not part of this build */
};
/* Host-only: the RCHOL_ORDER_RCM or RCHOL_ORDER_ND order of a symmetric
 * pattern (0-based triplets; the diagonal is ignored): order[k] = vertex
 * placed at position k.  Reverse Cuthill-McKee runs a breadth-first search
 * per component from a pseudo-peripheral vertex, neighbours by ascending
 * degree, and reverses it; nested dissection cuts each region's
 * breadth-first levels at the median level (the separator, numbered after
 * both halves) down to regions of 64 vertices. */
rchol_status rchol_ordering(int kind, int n, long long nnz, const int* rows, const int* cols, int* order);
rchol_status rchol_set_sddm(rchol_ctx* ctx, int n, long long nnz, const int* rows, const int* cols,
                            const double* vals, int on_device, int ordering, unsigned long long order_seed,
                            int* perm, int* has_ground);
/* A preprocessed matrix in CSC (== CSR, symmetric, diagonal included), host
 * (on_device = 0) or device (on_device = 1) arrays; copied into the context. */
rchol_status rchol_set_csc(rchol_ctx* ctx, int n, const int* colptr, const int* rowind, const double* val,
                           int on_device, int trim_ground);
/* Host-only preprocessing (no device needed): the CSC that rchol_load_mtx /
 * rchol_set_triplets would build.  Call with colptr = NULL to get *nnz_out,
 * then again with colptr[n+1], rowind[*nnz_out], val[*nnz_out]. */
rchol_status rchol_csc_from_triplets(int n, long long nnz, const int* rows, const int* cols, const double* vals,
                                     int* colptr, int* rowind, double* val, long long* nnz_out);
/* Host-only MatrixMarket read (0-based triplets, symmetric files generalised);
 * arrays are malloc'ed, release them with rchol_free_host. */
rchol_status rchol_read_mtx(const char* path, int* n, long long* nnz, int** rows, int** cols, double** vals);
/* Binary matrix cache: a preprocessed CSC with its trim flag, read back with
 * one read per array instead of a text parse (the reference reads text
 * MatrixMarket only, gpu_implementation/pre_process.hpp:322-356).  Layout:
 * "RCHOLCSC", uint32 version 1, int32 trim flag, int64 n, int64 nnz, int32
 * colptr[n+1], int32 rowind[nnz], float64 val[nnz], host byte order.
 * rchol_write_bin / rchol_read_bin are host-only (read_bin's arrays are
 * malloc'ed: release them with rchol_free_host); rchol_save_bin writes the
 * context's matrix and rchol_load_bin installs a file as rchol_set_csc does. */
rchol_status rchol_write_bin(const char* path, int n, const int* colptr, const int* rowind, const double* val,
                             int trim_ground);
rchol_status rchol_read_bin(const char* path, int* n, long long* nnz, int** colptr, int** rowind, double** val,
                            int* trim_ground);
rchol_status rchol_save_bin(const rchol_ctx* ctx, const char* path);
rchol_status rchol_load_bin(rchol_ctx* ctx, const char* path);
/* n and nnz of the loaded matrix (before trimming). */
rchol_status rchol_matrix_info(const rchol_ctx* ctx, int* n, long long* nnz);
/* Copy the preprocessed CSC back to the host (sizes from rchol_matrix_info). */
rchol_status rchol_matrix_copy_to_host(const rchol_ctx* ctx, int* colptr, int* rowind, double* val);

/* ---- factorization (driver.cu:43-1302 kernel + :1309-1548 assembly) ---- */
rchol_status rchol_factor(rchol_ctx* ctx, rchol_factor_t** out);
rchol_status rchol_factor_get_info(const rchol_factor_t* f, rchol_factor_info* info);
/* Strict CSC of L (colptr[n+1], rowind/val[nnz_strict]) and D[n] to the host. */
rchol_status rchol_factor_copy_to_host(const rchol_factor_t* f, long long* colptr, int* rowind, double* val,
                                       double* diag);
/* <prefix>l_sol.mtx and <prefix>sol_diag.txt (experiment/driver_local.cpp:958-988). */
rchol_status rchol_factor_write(const rchol_factor_t* f, const char* prefix);
/* Load a factor written in that format for the loaded matrix. */
rchol_status rchol_factor_read(rchol_ctx* ctx, const char* prefix, rchol_factor_t** out);
/* Adopt a factor in the reference's device format: CSR of L^T with a unit
 * diagonal (int32 rowptr[n+1], colind, val) and D[n] (solver.hpp:236-238).
 * on_device selects host or device pointers. */
rchol_status rchol_factor_from_csr_upper(rchol_ctx* ctx, int n, const int* rowptr, const int* colind,
                                         const double* val, const double* diag, int on_device,
                                         rchol_factor_t** out);
void rchol_factor_free(rchol_factor_t* f);

/* ---- solve ---------------------------------------------------------------
 * PCG for k right-hand sides (k in {1,2,4,8,16,32}) held column-major with
 * leading dimension ldb >= n (B[c*ldb + i]), host (on_device = 0) or device
 * (on_device = 1).  X receives the solutions in the same layout. */
rchol_status rchol_pcg_solve(rchol_ctx* ctx, const rchol_factor_t* f, int k, const double* B, double* X,
                             int ldb, int on_device, rchol_solve_info* info);
/* One preconditioner application Z = L^-T D^+ L^-1 R (same layout rules). */
rchol_status rchol_precond_apply(rchol_ctx* ctx, const rchol_factor_t* f, int k, const double* R, double* Z,
                                 int ldb, int on_device, int fp32);
/* Allocation-free variant of rchol_precond_apply, Z = L^-T D^+ L^-1 R, for
 * callers that must not allocate device memory: code running inside another
 * framework's memory budget (a caching allocator that already holds most of
 * HBM, where a cudaMalloc can fail) and latency-sensitive loops, where
 * cudaMalloc/cudaFree stall because they synchronise with the device.  R and
 * Z are caller-owned DEVICE arrays, row-major n x k (R[i*k + c]), that must
 * not overlap; k in {1,2,4,8,16,32}; stream may be NULL (legacy default
 * stream).  The call returns after the stream has finished the apply.
 * Scratch is one fixed array in the library's device code, limited to
 * n * k <= 4194304 (2^22 doubles, 32 MiB, plus 4 KiB for scalars); larger
 * sizes return RCHOL_ERR_INVALID.  That array belongs to the library's
 * device code, so every device that loads the library holds those 32 MiB
 * until the process exits, whether or not this entry point is called.  Each
 * call looks up the array's address in the current context; the first
 * lookup on a device may load the library's device code, so make the first
 * call before any stream capture.  All calls on a device share the array,
 * and every solve or apply of one factor shares that factor's split-row
 * partial sums: a call that overlaps on the GPU (other threads or streams)
 * with another call, or with rchol_pcg_solve / rchol_precond_apply on the
 * same factor, races with it, so the caller must serialise them.  No
 * counterpart in the reference, which allocates its solver work vectors for
 * each solve. */
rchol_status rchol_precond_apply_noalloc(const rchol_factor_t* f, int k, const double* R, double* Z, int fp32,
                                         void* stream);
/* ---- autotuner ---------------------------------------------------------
 * Picks, for the loaded matrix on this GPU, the options the reference fixes
 * by hand (WARPS_PER_SQUAD, gpu_implementation/auxilliary.hpp:10-19):
 *   tail_vertices  the last vertices eliminated by one whole CTA each (the
 *                  longest suffix in which 3/4 of the vertices gather >= 1024
 *                  entries), kept only when a timed factorization is faster;
 *   bucket_cap     the power of two covering 95% of the vertices' gathers,
 *                  then twice and four times that (at most 128, and only
 *                  while the buckets take at most a quarter of the free
 *                  device memory), each kept only when faster;
 *   rhs_block      the block width (<= max_rhs) of least iteration time per
 *                  right-hand side.
 * One profiling factorization plus at most five timed trials; the choices
 * are written into the context's options and cached per process for the
 * same matrix fingerprint (n, nnz, trim, column-length histogram), GPU,
 * precision and max_rhs (from_cache = 1 on a hit). */
typedef struct rchol_tune_result {
    int tail_vertices;
    int bucket_cap;
    int rhs_block;
    int from_cache;
    int max_gather;          /* largest gathered neighbour list of the profile */
    float ms_factor_default; /* factor time with the options on entry, no tail */
    float ms_factor_tuned;   /* factor time with the chosen options */
    float per_rhs_ms[6];     /* iteration time per right-hand side, k = 1, 2, 4, 8, 16, 32 */
} rchol_tune_result;
rchol_status rchol_autotune(rchol_ctx* ctx, int max_rhs, rchol_tune_result* out);
/* Mean device time (ms) of the three PCG iteration kernels over `reps`
 * iterations on this factor with k right-hand sides: ms_out[0] SpMV +
 * vector update, ms_out[1] forward solve, ms_out[2] backward solve. */
rchol_status rchol_profile_solve(rchol_ctx* ctx, const rchol_factor_t* f, int k, int reps, float* ms_out);
/* The latency floor of the sync-free triangular solves: the mean time (ns)
 * of one producer -> consumer hop, a relaxed store on one SM seen by a
 * polling load on another, measured by two co-resident CTAs passing a
 * counter back and forth `rounds` times (64 .. 2^20) on the context's device.
 * A solve of depth d cannot finish in less than d hops.  sm_pair (may be
 * NULL) receives the two CTAs' SM ids.  No reference counterpart. */
rchol_status rchol_hop_latency(rchol_ctx* ctx, int rounds, double* ns_per_hop, int* sm_pair);
/* Y = A X with the (trimmed) matrix of the context. */
rchol_status rchol_spmv(rchol_ctx* ctx, int k, const double* X, double* Y, int ldb, int on_device);

/* ---- batched independent systems (many uneven Laplacians at once) -------
 * rchol_batch_set stacks nsys preprocessed systems (host CSC, diagonal
 * included, each a Laplacian or SDDM without a ground vertex, at least 32
 * vertices each) into one block-diagonal matrix of the context: system s owns
 * rows offsets[s] .. offsets[s+1]-1 (offsets may be NULL).  rchol_factor then
 * eliminates every system in one persistent launch, and rchol_batch_solve runs
 * one PCG per (system, right-hand side) pair -- own step lengths, own stop
 * test -- with one set of kernel launches per iteration for all of them.  B/X
 * are (n_total x k) column-major with rows grouped by system.  per_system
 * (nsys entries, may be NULL) receives each system's iterations (max over its
 * right-hand sides) and true relative residual; total the whole batch. */
typedef struct rchol_system {
    int n;
    const int* colptr;
    const int* rowind;
    const double* val;
} rchol_system;
rchol_status rchol_batch_set(rchol_ctx* ctx, int nsys, const rchol_system* systems, long long* offsets);
rchol_status rchol_batch_solve(rchol_ctx* ctx, const rchol_factor_t* f, int k, const double* B, double* X, int ldb,
                               int on_device, rchol_solve_info* per_system, rchol_solve_info* total);

/* ---- reference drop-ins ---------------------------------------------------
 * The whole CLI path of driver.cu main (:2148-2160) / driver_physics.cu main:
 * load, factor with num_blocks squads, and when check_solve = 1 run PCG to
 * `tol` on the reference right-hand side generate_zero_sum_vector(seed 0)
 * (solver.hpp:43-61), printing the reference's timing lines. */
rchol_status rchol_factorization_driver(const char* path, int num_blocks, int check_solve, double tol,
                                        int physics);
/* prepare_and_solve (solver.hpp:236-593) on device arrays: the Laplacian in
 * CSR (n = lap_n, int32), the factor as CSR of L^T with unit diagonal
 * (factor_nnz entries) and D.  physics = 1 uses the zero-sum right-hand side
 * (the reference always passes 1); removal = 1 means the factor arrays still
 * hold the ground vertex (n+1 rows) and are trimmed here.  Stops on the
 * reference rule sqrt(r.z/r0.z0) <= tol, at most 300 iterations.  X (device,
 * may be NULL) receives the solution; info (may be NULL) the statistics. */
rchol_status rchol_prepare_and_solve(int lap_n, long long lap_nnz, const int* lap_rowptr, const int* lap_colind,
                                     const double* lap_val, const int* csr_rowptr, const double* csr_val,
                                     const int* csr_colind, const double* diag, double tol, int physics,
                                     long long factor_nnz, int removal, double* X, rchol_solve_info* info);

/* ---- synthetic inputs (the benchmark configurations) -------------------
 * Builds a Laplacian as 0-based triplets (both triangles + diagonal) in the
 * ascending-nnz order with a seeded tie-break (write_graph.jl:112-128), with
 * a ground vertex appended for SDDM inputs (write_graph.jl:148-163).
 *   kind: "grid2d", "grid3d", "grid3d27", "chunglu"
 *   dims: side lengths (grid) or {n_vertices, n_edges, dmin, dmax} (chunglu)
 *   wlo/whi: weight range; log_weights = 1 draws log-uniform
 *   aniso_z: multiplier of the z-direction conductance (27-point)
 *   excess_frac/excess_lo/excess_hi: rows with diagonal excess and its range
 *   as a multiple of the weighted degree (SDDM when excess_frac > 0)
 *   ordering: 0 ascending nnz, 1 random, 2 natural
 * The arrays are malloc'ed; release them with rchol_free_host. */
rchol_status rchol_generate(const char* kind, const long long* dims, int ndims, double wlo, double whi,
                            int log_weights, double aniso_z, double excess_frac, double excess_lo,
                            double excess_hi, int ordering, unsigned long long seed, int* n_out,
                            long long* nnz_out, int** rows, int** cols, double** vals, int* has_ground);
void rchol_free_host(void* p);
/* The reference right-hand side generate_zero_sum_vector(out, n, seed)
 * (gpu_implementation/solver.hpp:43-61, experiment/custom_cg.hpp:45-63):
 * n draws of std::mt19937(seed) through uniform_real_distribution<double>(0,1),
 * minus their mean.  Host only; out[n] is caller-owned. */
rchol_status rchol_zero_sum_vector(int n, unsigned int seed, double* out);
/* Write 0-based triplets as a MatrixMarket coordinate/real/general file. */
rchol_status rchol_write_mtx(const char* path, int n, long long nnz, const int* rows, const int* cols,
                             const double* vals);

#ifdef __cplusplus
}
#endif

#endif
