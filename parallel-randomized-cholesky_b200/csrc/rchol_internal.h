// Internal declarations shared by the CUDA translation units and the host
// C-ABI layer.  Nothing here is part of the public interface (include/rchol.h).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include <vector>

namespace rchol {

// Bump allocator for the temporaries of one assembly (reset per call):
// avoids a cudaMalloc/cudaFree (and the device sync of cudaFree) per
// temporary.  Requests beyond the arena fall back to cudaMalloc and are
// released at the next reset.
struct Scratch {
    char* base = nullptr;
    size_t cap = 0, used = 0;
    std::vector<void*> overflow;
    size_t overflow_bytes = 0;  // requests the arena could not serve since the last reset
    cudaError_t reserve(size_t bytes) {
        if (bytes <= cap) return cudaSuccess;
        cudaFree(base);
        base = nullptr;
        cap = 0;
        cudaError_t e = cudaMalloc((void**)&base, bytes);
        if (e == cudaSuccess) cap = bytes;
        return e;
    }
    // Releases everything; after an overflow the arena grows to the peak use
    // so that the next user of the same sizes allocates nothing.
    void reset() {
        const size_t peak = used + overflow_bytes;
        used = 0;
        for (void* p : overflow) cudaFree(p);
        overflow.clear();
        if (overflow_bytes) {
            overflow_bytes = 0;
            reserve(peak + (peak >> 3));
        }
    }
    template <typename T>
    cudaError_t get(T** p, int64_t n) {
        size_t bytes = (sizeof(T) * (size_t)(n > 0 ? n : 1) + 255) & ~(size_t)255;
        if (used + bytes <= cap) {
            *p = reinterpret_cast<T*>(base + used);
            used += bytes;
            return cudaSuccess;
        }
        cudaError_t e = cudaMalloc((void**)p, bytes);
        if (e == cudaSuccess) {
            overflow.push_back(*p);
            overflow_bytes += bytes;
        }
        return e;
    }
    void release() {
        reset();
        cudaFree(base);
        base = nullptr;
        cap = 0;
    }
};

// Error codes written to the device status word (first writer wins).
enum DeviceError : int {
    kDevOk = 0,
    kDevTimeout = 1,       // a bounded wait gave up
    kDevCapacity = 2,      // a preallocated pool was too small
    kDevBadInput = 3,      // an invariant of the input did not hold
};

// ---------------------------------------------------------------------------
// Matrix in HBM: the full symmetric Laplacian/SDDM in CSC, which is also its
// CSR (A = A^T).  int32 indices, FP64 values.
// ---------------------------------------------------------------------------
struct DevCsc {
    int32_t n = 0;
    int64_t nnz = 0;
    int32_t* colptr = nullptr;  // [n+1]
    int32_t* rowind = nullptr;  // [nnz]
    double* val = nullptr;      // [nnz]
    int64_t cap = 0;            // entries allocated in rowind / val (trim_matrix output)
};

// Rows longer than kLongRow entries (the hubs of power-law graphs) are left
// out of the one-RHS SpMV kernels' tiles and slices: each gets a CTA of its
// own (spmv_long_kernel).
constexpr int kLongRow = 2048;

// Columns of the input longer than kHugeCol entries are counted by the whole
// grid rather than one warp (count_lower, factor.cu); the list that carries
// them holds kHugeColCap ids after its count word.
constexpr int kHugeCol = 4096;
constexpr int kHugeColCap = 1024;

// Sliced-ELL copy of a DevCsc for the one-RHS SpMV (sell.cu): slice s of
// 32 rows owns slots [sptr[s] * 32, sptr[s + 1] * 32), column-major (slot
// (sptr[s] + k) * 32 + lane = entry k of row 32 s + lane; index -1 past the
// row's end).
struct DevSell {
    int32_t n = 0;
    int32_t nslices = 0;
    int64_t slots = 0;          // 0: no copy (the CSR SpMV is used)
    int64_t* sptr = nullptr;    // [nslices + 1], in units of 32 slots
    int32_t* sidx = nullptr;    // [slots]
    double* sval = nullptr;     // [slots]
    int64_t cap_slices = 0, cap_slots = 0;  // allocated sizes, reused by the next build
};

// Working state of one factorization (all device pointers).
struct FactorWork {
    int32_t n = 0;
    // strict lower triangle of A, |a_ij|, CSC
    int32_t* lcolptr = nullptr;
    int32_t* lrow = nullptr;
    double* lval = nullptr;
    int64_t lnnz = 0;
    // dependency counters and ready queue (queue[i] = -1 until written)
    int32_t* dep = nullptr;
    int32_t* queue = nullptr;
    // per-column fill buckets: a first chunk of `c0` slots per column, then
    // 64-slot overflow chunks linked per column
    int32_t c0 = 32;
    int32_t* fcnt = nullptr;      // [n] fills appended to each column
    int32_t* brow = nullptr;      // [n*c0]
    double* bval = nullptr;       // [n*c0]
    int32_t* chead = nullptr;     // [n] first overflow chunk of each column (-1)
    int32_t* cnext = nullptr;     // [nchunks] next chunk (-1), by the chunk's first pool unit
    int32_t* crow = nullptr;      // [nchunks*64]
    double* cval = nullptr;       // [nchunks*64]
    int32_t nchunks = 0;
    // L pool: each eliminated column appends its merged neighbours
    int64_t pool_cap = 0;
    int32_t* prow = nullptr;      // [pool_cap]
    double* pval = nullptr;       // [pool_cap]  (w / sum, positive)
    int64_t* pstart = nullptr;    // [n] column start in the pool
    int32_t* pcnt = nullptr;      // [n] merged neighbour count
    int32_t* hcols = nullptr;     // [kHugeColCap + 1] long input columns (count, ids)
    double* diag = nullptr;       // [n] D
    int32_t* level = nullptr;     // [n] forward level (longest dependency chain) of each row of L
    // per-warp scratch for vertices that do not fit the shared-memory slab
    int64_t gscratch_entries = 0; // entries per warp
    unsigned char* gscratch = nullptr;
    // a few shared slabs for vertices larger than the per-warp scratch,
    // each taken with a lock word (hlock[i] = 1 while held)
    int64_t hscratch_entries = 0; // entries per shared slab
    int32_t nhuge = 0;            // shared slabs (and cooperative-tail CTAs)
    unsigned char* hscratch = nullptr;
    int32_t* hlock = nullptr;
    // counters: [0] queue head, [1] queue tail, [2] chunk cursor, [3] status,
    // [4] abort, [5] big-vertex count, [6] max gather, [7] overflow fills;
    // pool cursor is int64 in counters64[0]
    int32_t* counters = nullptr;
    unsigned long long* counters64 = nullptr;
    void* scan_tmp = nullptr;     // scan_tmp_bytes(n)
};

// The assembled factor, trimmed when the input carried a ground vertex.
//   Lc: strict CSC of L  (column j: rows i > j, values L_ij < 0)
//   Lr: strict CSR of L  (row i: columns j < i), the transpose of Lc
struct DevFactor {
    int32_t n = 0;            // size of the factor used by the solve
    int64_t nnz = 0;          // strict entries
    int64_t* lc_ptr = nullptr;
    int32_t* lc_idx = nullptr;
    double* lc_val = nullptr;
    float* lc_val32 = nullptr;
    int64_t* lr_ptr = nullptr;
    int32_t* lr_idx = nullptr;
    double* lr_val = nullptr;
    float* lr_val32 = nullptr;
    double* diag = nullptr;
    float* diag32 = nullptr;
    // Solve schedules.  order_f lists the rows by (forward level, lane
    // class); order_b by (backward level = depth-1-forward level, class), a
    // topological order of the L^T solve.  A row of length len gets
    // G = pow2 >= ceil(len / epl) lanes (1..32); a task packs
    // 32/G rows of one level and one class into a warp: int2 {first position
    // in the order, row count | log2(G) << 8}.
    int32_t* order_f = nullptr;
    int32_t* order_b = nullptr;
    int2* tasks_f = nullptr;
    int2* tasks_b = nullptr;
    int32_t ntasks_f = 0, ntasks_b = 0;
    // Multi-RHS layouts (built on the first k > 1 use, build_solve_layouts):
    // the rows of Lr (forward) and of L^T = columns of Lc (backward) copied
    // in schedule order, so that position p of order_f owns entries
    // sf_ptr[p]..sf_ptr[p+1] (same for the backward side) and consecutive
    // rows of a schedule are adjacent in memory.  lay_ready is false until
    // they hold this factor's rows (buffers of a released factor are reused).
    bool lay_ready = false;
    int64_t* sf_ptr = nullptr;
    int32_t* sf_idx = nullptr;
    double* sf_val = nullptr;
    float* sf_val32 = nullptr;
    int64_t* sb_ptr = nullptr;
    int32_t* sb_idx = nullptr;
    double* sb_val = nullptr;
    float* sb_val32 = nullptr;
    // Task slabs of the K = 1 solves.  Task t (descriptor int4 {first
    // position, slab offset in 32-slot units, row count | log2(G) << 8,
    // slots per lane m}) owns slots (d.y + k) * 32 + lane, k < m: lane
    // lane/G-th row of the task, entry k * G + lane % G of that row (index
    // -1 and value 0 past the row's end).  All of a lane's entries are thus
    // addressable from the descriptor alone and load in one round trip.
    int4* pack_f = nullptr;
    int4* pack_b = nullptr;
    int32_t* pf_idx = nullptr;
    double* pf_val = nullptr;
    float* pf_val32 = nullptr;
    int32_t* pb_idx = nullptr;
    double* pb_val = nullptr;
    float* pb_val32 = nullptr;
    int64_t slots_f = 0, slots_b = 0;
    // Rows longer than kSplitMin* entries run as several part tasks (flag
    // 1 << 11 in d.z, part index in d.z >> 12, part count in d.w >> 8); part
    // tasks carry {split row id, first partial} in split_*, write partial
    // sums to psum_*, and the last part to finish (pcount_*) publishes the row.
    int32_t npt_f = 0, npt_b = 0;        // task count after the split
    int32_t nsplit_f = 0, nsplit_b = 0;  // split rows
    int2* split_f = nullptr;
    int2* split_b = nullptr;
    double* psum_f = nullptr;
    double* psum_b = nullptr;
    int32_t* pcount_f = nullptr;
    int32_t* pcount_b = nullptr;
    int32_t* srow_f = nullptr;
    int32_t* srow_b = nullptr;
    int64_t cap_sf = 0, cap_sb = 0, cap_qf = 0, cap_qb = 0, cap_cf = 0, cap_cb = 0, cap_rf = 0, cap_rb = 0;
    int64_t cap_pdf = 0, cap_pdb = 0, cap_pif = 0, cap_pib = 0, cap_pvf = 0, cap_pvb = 0, cap_pwf = 0,
            cap_pwb = 0;
    int32_t depth = 0;        // number of levels of the forward solve DAG
    int32_t depth_b = 0;      // levels of the backward schedule
    // Backward head: the first hb_nlev levels of the backward schedule
    // (exact levels only), narrow levels of the vertices eliminated last
    // whose rows depend only on earlier head rows.  One CTA solves them
    // before the persistent kernel, which then starts at task hb_ntask.
    // hb_lv[l] = {first task, first slab unit, first position in order_b, 0}
    // for l <= hb_nlev; hb_idx holds the head's slab slots with every index
    // replaced by its position in order_b (-1 past a row's end).
    int32_t hb_nlev = 0, hb_ntask = 0, hb_rows = 0, hb_stage = 0;
    int4* hb_lv = nullptr;
    int32_t* hb_idx = nullptr;
    int64_t cap_hl = 0, cap_hi = 0;
    // allocated capacities (buffers of a released factor are reused)
    int64_t cap_n = 0, cap_nnz = 0, cap_tf = 0, cap_tb = 0, cap_ln = 0, cap_lz = 0;
};

// Rows longer than kSplitMin* entries run in the K = 1 solves as part tasks
// of kSplitLen* entries (shorter rows are faster in one warp); F for the
// forward solve (rows of L), B for the backward one (columns of L).
#ifndef RCHOL_SPLIT_MIN_B
#define RCHOL_SPLIT_MIN_B 512
#endif
#ifndef RCHOL_SPLIT_LEN_B
#define RCHOL_SPLIT_LEN_B 128
#endif
constexpr int kSplitMinF = 1024;
constexpr int kSplitLenF = 512;
constexpr int kSplitMinB = RCHOL_SPLIT_MIN_B;
constexpr int kSplitLenB = RCHOL_SPLIT_LEN_B;

// Lane classes of the K = 1 solves: a row gets G = 1, 2, 4, ..., 32 lanes,
// the smallest G that leaves at most `epl` entries per lane (rows longer
// than 32*epl still get one warp).
constexpr int kLaneClasses = 6;

// Builds order_f/order_b/tasks_f/tasks_b of `f` (device arrays allocated
// here) from the forward level of every row (device array, n entries).
// With exact_bwd the backward order uses the true longest-path levels of
// the L^T solve (one extra sync-free pass); otherwise the reversed forward
// levels, which are also topological.
// Matrix entries per lane of the k = 1 solve schedule when the option asks
// for the automatic choice (sched_epl = 0): 3 when every row of L is short
// (stencil factors; measured 2-4% faster solves), else 2 (power-law factors,
// whose long rows run slower with fewer lanes).
inline int auto_sched_epl(int64_t max_row_len) { return max_row_len <= 1024 ? 3 : 2; }
// The multi-RHS layouts of a factor (DevFactor::sf_ptr); no-op when built.
cudaError_t build_solve_layouts(DevFactor& f, Scratch& sc, cudaStream_t s);

// Shared-memory plan of the backward-head kernel: the head holds at most
// kHeadMaxLevels levels of at most kHeadMaxRows rows and kHeadMaxTasks
// tasks each; its stages (one level each, kHeadStages in flight) and the
// per-row arrays fit kHeadSmem.
constexpr int kHeadThreads = 512;
constexpr int kHeadStages = 5;
constexpr int kHeadMaxLevels = 16384;
// level-table entries the head kernel keeps in shared memory (a ring filled
// kHeadLvAhead levels ahead)
constexpr int kHeadLvRing = 16;
constexpr int kHeadLvAhead = 9;
constexpr int kHeadMaxRows = 1024;
// one task per warp of the 16-warp CTA: levels with more tasks than warps
// took longer in the head kernel than in the persistent one
constexpr int kHeadMaxTasks = kHeadThreads / 32;
constexpr int kHeadMinLevels = 8;
constexpr int kHeadSmem = 220 * 1024;
// Bytes of one head stage (a level's descriptors, slab slots and row
// scalars) for value size vb, each part 16-byte aligned.
inline int head_stage_bytes(int ntask, int units, int rows, int vb) {
    auto al = [](int x) { return (x + 15) & ~15; };
    return 16 * ntask + 128 * units + 32 * vb * units + 2 * al(8 * rows) + al(vb * rows);
}
// Dynamic shared memory of the head kernel: row ids and z values of every
// head row, the level-table ring and the stages.
inline int head_smem_bytes(int rows, int stage) {
    return ((4 * rows + 15) & ~15) + ((8 * rows + 15) & ~15) + 16 * kHeadLvRing + kHeadStages * stage;
}
// bwd_head (exact levels only): build the backward head (DevFactor::hb_nlev).
cudaError_t build_solve_schedule(DevFactor& f, const int32_t* level, int epl, bool exact_bwd, bool bwd_head,
                                 double timeout_s, Scratch& sc, cudaStream_t s);

struct FactorLaunch {
    int grid = 0;
    int block = 256;
    int smem_slab = 256;      // entries per warp slab in shared memory
    uint64_t seed = 1;
    double timeout_s = 20.0;
    int32_t tail = 0;         // the last `tail` vertices are eliminated by one cooperative CTA (0: none)
    int32_t* gsize = nullptr; // device [n]: gathered entries of each vertex (null: not recorded)
};

// ---- setup / factor / assembly (factor.cu) --------------------------------
cudaError_t launch_lower_and_deps(const DevCsc& A, FactorWork& w, cudaStream_t s);
cudaError_t launch_count_lower(const DevCsc& A, int32_t* lower_cnt, int32_t* huge, cudaStream_t s);
cudaError_t launch_init_factor_state(FactorWork& w, cudaStream_t s);
cudaError_t launch_factor(FactorWork& w, const FactorLaunch& cfg, cudaStream_t s);
int factor_resident_grid(int block, int smem_slab, int device);
size_t factor_smem_bytes(int block, int smem_slab);

// Assemble Lc/Lr (and FP32 copies) from the pool; drop the last vertex when
// trim_ground is set.  The device arrays of `f` are allocated here.
// `f` may hold the buffers of a released factor; they are reused when large
// enough.
cudaError_t assemble_factor(const FactorWork& w, bool trim_ground, bool make_fp32, int epl, bool exact_bwd,
                            bool bwd_head, double timeout_s, Scratch& sc, DevFactor& f, cudaStream_t s);
// Drop the last row/column of A (ground vertex) into `out`, whose buffers
// are reused when large enough (else reallocated).
// flag (device int) = 1 unless colptr[0] = 0, colptr[n] = nnz and colptr
// is monotone.
cudaError_t check_colptr(const int32_t* colptr, int32_t n, int32_t nnz, int32_t* flag, cudaStream_t s);
cudaError_t trim_matrix(const DevCsc& A, DevCsc& out, Scratch& sc, cudaStream_t s);

// Return the CUDA error of `x` from the enclosing function.
#define RCHOL_TRY(x)                        \
    do {                                    \
        cudaError_t e__ = (x);              \
        if (e__ != cudaSuccess) return e__; \
    } while (0)

// Shared large slabs of the elimination kernel: between kHugeSlabsMin and
// kHugeSlabsMax (as many as fit kHugeSlabBudget bytes); the cooperative
// tail runs one CTA per slab.
constexpr int kHugeSlabsMin = 8;
constexpr int kHugeSlabsMax = 32;
constexpr size_t kHugeSlabBudget = size_t(512) << 20;
// Bytes per entry of elimination slabs in global memory (with radix-sort buffers).
constexpr int kGlobalSlabBytes = 56;

// *out = max(v[0..n-1]) (device, *out must start at 0).
cudaError_t max_i32(const int32_t* v, int64_t n, int32_t* out, cudaStream_t s);

// Stable order of 0..n-1 by key (0 <= key < nkeys) into `order`; rows with
// equal keys keep ascending index order (bucket_sort.cu).
cudaError_t stable_key_order(const int32_t* key, int32_t n, int32_t nkeys, int32_t* order, Scratch& sc,
                             cudaStream_t s);
// The same, stably re-sorting the items in the order `in` (a permutation of
// 0..n-1; null = identity) by key: chained calls sort by several keys, the
// last call's key being the most significant.  `order` may alias `in`.
cudaError_t stable_key_order_from(const int32_t* key, const int32_t* in, int32_t n, int32_t nkeys, int32_t* order,
                                  Scratch& sc, cudaStream_t s);
// The same order with the keys moved along with the items in every pass
// (sequential key reads; two extra key buffers of scratch): for large n.
cudaError_t stable_key_order_carried(const int32_t* key, int32_t n, int32_t nkeys, int32_t* order, Scratch& sc,
                                     cudaStream_t s);

// ---- SDDM -> ordered Laplacian (ordering.cu) ------------------------------
constexpr int kOrderGiven = 0, kOrderNnzSort = 1, kOrderRandom = 2, kOrderExternal = -1;
// A converted matrix: CSC (rows ascending per column, duplicates kept) in
// the scratch arena, and the position of each input vertex.
struct SddmResult {
    enum { kOk = 0, kBadIndex = 1, kNotDominant = 2 };
    int status = kOk;
    int32_t n = 0;              // input n, plus one with a ground vertex
    int64_t nnz = 0;
    bool ground = false;
    double total = 0.0;         // sum of every entry (before the ground vertex)
    int32_t* colptr = nullptr;  // device, scratch
    int32_t* rowind = nullptr;
    double* val = nullptr;
    int32_t* perm = nullptr;    // device [input n]: new index of input vertex i
};
// Device triplets (0-based, both triangles) of an SDDM or Laplacian: signs
// normalised, ordered (kOrder*; `seed` keys the random permutation), and a
// ground vertex appended when the entries sum to more than 1e-9
// (write_graph.jl:98-183).  Synchronises `s`.
// kOrderExternal takes the order from `order_in` (device [n]: vertex placed
// at each position).
cudaError_t sddm_to_laplacian(int32_t n, int64_t nnz, const int32_t* rows, const int32_t* cols, const double* vals,
                              int ordering, uint64_t seed, Scratch& sc, cudaStream_t s, SddmResult& res,
                              const int32_t* order_in = nullptr);

// ---- scans (scan.cu) -------------------------------------------------------
// out[0] = 0, out[i+1] = sum(in[0..i]); out has n+1 entries.  Uses `tmp`
// scratch of scan_tmp_bytes(n).
size_t scan_tmp_bytes(int64_t n);
cudaError_t exclusive_scan_i32_to_i64(const int32_t* in, int64_t* out, int64_t n, void* tmp,
                                      cudaStream_t s);
cudaError_t exclusive_scan_i32_to_i32(const int32_t* in, int32_t* out, int64_t n, void* tmp,
                                      cudaStream_t s);

// ---- PCG (solve.cu) --------------------------------------------------------
struct PcgScalars;  // device-resident scalars, defined in solve.cu

struct SolveConfig {
    int k = 1;                 // right-hand sides in the block
    bool fp32_factor = false;  // read L and D as FP32
    double tol = 1e-6;
    int max_iter = 1000;
    int stop_rule = 0;         // 0 relres (true residual), 1 precond ratio, 2 abs r^2
    int unroll = 4;            // iterations per captured graph launch
    bool use_graph = true;
    int poll_ns = 0;           // back-off between polls in the triangular solves
    double timeout_s = 20.0;
};

struct SolveResult {
    int iterations = 0;
    int converged = 0;
    int status = 0;            // device status word
    double relres_true = 0;    // max over RHS
    double relres_rec = 0;
    double precond_ratio = 0;
    float ms_total = 0;
    float ms_iterations = 0;
    int graph_launches = 0;
    int kernel_launches = 0;
};

// Solves A X = B for k columns stored row-major (n x k, ldx = k) in device
// memory; X is overwritten.  `A` and `F` must have the same n.
class PcgSolver;
// `sell` (may be null) is a sliced-ELL copy of A used by the one-RHS SpMV.
PcgSolver* pcg_create(const DevCsc& A, const DevFactor& F, const SolveConfig& cfg, int device,
                      cudaStream_t stream, cudaError_t* err, const DevSell* sell = nullptr);
// Points the solver at another matrix of the same size (with its sliced-ELL
// copy, null for none) and another factor; its vectors, and its captured
// iteration graph when the launch arguments come out equal, are kept.
// Fails (cudaErrorInvalidValue) when the sizes or the SpMV form differ.
// new_matrix: A's contents changed since the solver last saw it (its long
// rows are found again)
cudaError_t pcg_rebind(PcgSolver* s, const DevCsc& A, const DevSell* sell, const DevFactor& F, bool new_matrix);
cudaError_t pcg_solve(PcgSolver* s, const double* dB, double* dX, SolveResult* res);
void pcg_destroy(PcgSolver* s);
// Mean device time of spmv_update / fwd / bwd over `reps` iterations.
cudaError_t pcg_profile(PcgSolver* s, const double* dB, double* dX, int reps, float* ms_out);

// Batched independent systems stacked block-diagonally (rows grouped by
// system, offsets h_off[nsys+1]); one PCG per (system, right-hand side).
struct BatchResult {
    int converged = 0;
    int status = 0;
    float ms_total = 0, ms_iterations = 0;
    int kernel_launches = 0, graph_launches = 0;
    std::vector<int> iterations;      // per system (max over its columns)
    std::vector<double> relres;       // per system, true relative residual
};
class BatchSolver;
BatchSolver* batch_create(const DevCsc& A, const DevFactor& F, const SolveConfig& cfg, int device,
                          cudaStream_t stream, const int64_t* h_off, int nsys, cudaError_t* err);
cudaError_t batch_solve(BatchSolver* s, const double* dB, double* dX, BatchResult* res);
void batch_destroy(BatchSolver* s);

// Builds `out` from A when the padded slot count is at most max_fill * nnz
// (otherwise out.slots = 0).  The buffers of `out` are reused when large
// enough.  Reads one scalar back (synchronizes `s`).
cudaError_t build_sell(const DevCsc& A, double max_fill, DevSell& out, Scratch& sc, cudaStream_t s);
void free_sell(DevSell& m);

// Kernel-level entry points used by tests/bench (one operator application).
cudaError_t spmv_f64(const DevCsc& A, const double* x, double* y, int k, cudaStream_t s);
// Layout changes between column-major (ld >= n) and row-major n x k blocks.
cudaError_t cm_to_rm(const double* cm, int ld, double* rm, int32_t n, int k, cudaStream_t s);
cudaError_t rm_to_cm(const double* rm, double* cm, int ld, int32_t n, int k, cudaStream_t s);
cudaError_t precond_apply(const DevFactor& F, const double* r, double* z, double* ywork, int k,
                          bool fp32, int* status, double timeout_s, cudaStream_t s);
// Largest n * k accepted by precond_apply_noalloc (its y vector lives in a
// fixed module array of this many doubles, 32 MiB, plus a 4 KiB header).
constexpr long long kNoAllocMaxElems = 1LL << 22;
// precond_apply on caller-provided device vectors (row-major n x k) with no
// device allocation: scratch comes from the module array, located once per
// device on first use.  Returns cudaErrorInvalidValue when n * k exceeds
// kNoAllocMaxElems.
cudaError_t precond_apply_noalloc(const DevFactor& F, const double* r, double* z, int k, bool fp32, int* status,
                                  double timeout_s, cudaStream_t s);
// Mean time of one store -> poll hop between two CTAs of the current device
// (rounds round trips, the first few untimed); the CTAs' SM ids in sm_pair.
cudaError_t hop_latency(int rounds, double* ns_per_hop, int* sm_pair);

}  // namespace rchol
