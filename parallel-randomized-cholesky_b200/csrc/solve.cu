// Preconditioned conjugate gradient with the randomized-Cholesky
// preconditioner M = L D L^T on sm_100a (gpu_implementation/solver.hpp:150-593,
// experiment/custom_cg.hpp:65-265), for a block of k independent right-hand
// sides stored row-major (n x k) so that every factor and matrix entry is
// read once per block.
//
// One iteration is three kernels, captured into a CUDA graph:
//   spmv_update  q = A z + beta q,  p = z + beta p,  (p.q) -> alpha
//                (A p computed as A z + beta A p_old: no separate p pass)
//   fwd          x += alpha p, r -= alpha q, (r.r); y = L^-1 r   sync-free
//   bwd          z = L^-T D^+ y, (r.z) -> beta, stop test        sync-free
// The triangular solves are persistent kernels over the resident grid: each
// row group waits for the rows it depends on by polling their values, which
// start as a "pending" NaN bit pattern (no separate ready flags, no level
// sets, no analysis phase).  Every wait is bounded by a wall-clock limit and
// reports kDevTimeout instead of hanging.  Reductions write per-block
// partials and the last block sums them in block order (deterministic).
#include <climits>
#include <cmath>
#include <cstdio>
#include <algorithm>
#include <cstring>
#include <type_traits>
#include <vector>

#include "device_common.cuh"
#include "rchol_internal.h"

namespace rchol {

constexpr int kMaxK = 32;

struct PcgScalars {
    double alpha[kMaxK];
    double beta[kMaxK];
    double rz[kMaxK];
    double rz0[kMaxK];
    double rr[kMaxK];
    double pq[kMaxK];
    double bnorm2[kMaxK];
    double tr2[kMaxK];       // ||b - A x||^2 from the true-residual kernel
    int active[kMaxK];
    int iters[kMaxK];
    int done;                // 1: stop iterating (all converged, max iters, error)
    int iter;                // completed iterations
    int phase;               // 0: the next bwd pass initialises rz (start/restart)
    int status;              // device error code
    unsigned ticket[4];
    double hrz;              // r.z over the backward head's rows
};

namespace {

constexpr int kBlock = 256;

__device__ __forceinline__ double pending_value() { return __longlong_as_double((long long)kPendingBits); }
__device__ __forceinline__ bool is_pending(double v) {
    return (unsigned long long)__double_as_longlong(v) == kPendingBits;
}

template <typename TV>
__device__ __forceinline__ double to_d(TV v) {
    return (double)v;
}

struct SolveArgs {
    int32_t n;
    // A (CSR == CSC, symmetric)
    const int32_t* __restrict__ a_ptr;
    const int32_t* __restrict__ a_idx;
    const double* __restrict__ a_val;
    // sliced-ELL copy of A (null when the CSR SpMV is used)
    const int64_t* __restrict__ s_ptr;
    const int32_t* __restrict__ s_idx;
    const double* __restrict__ s_val;
    // factor for the k > 1 solves: with by_pos, the multi-RHS layouts
    // (position p of order_f / order_b owns entries lr_ptr[p]..lr_ptr[p+1] /
    // lc_ptr[p]..lc_ptr[p+1]); without, the strict CSR and CSC of L by row id
    int32_t by_pos;
    const int64_t* __restrict__ lr_ptr;
    const int32_t* __restrict__ lr_idx;
    const void* __restrict__ lr_val;
    const int64_t* __restrict__ lc_ptr;
    const int32_t* __restrict__ lc_idx;
    const void* __restrict__ lc_val;
    const void* __restrict__ diag;
    const int32_t* __restrict__ order_f;  // forward-solve row order
    const int32_t* __restrict__ order_b;  // backward-solve row order
    // K = 1 task slabs (see DevFactor::pack_f)
    const int4* __restrict__ pack_f;
    const int4* __restrict__ pack_b;
    const int32_t* __restrict__ pf_idx;
    const void* __restrict__ pf_val;
    const int32_t* __restrict__ pb_idx;
    const void* __restrict__ pb_val;
    int32_t ntasks_f, ntasks_b;
    // split rows (part tasks) of the K = 1 solves
    const int2* __restrict__ split_f;
    const int2* __restrict__ split_b;
    double* psum_f;
    double* psum_b;
    int32_t* pcount_f;
    int32_t* pcount_b;
    const int32_t* __restrict__ srow_b;
    int32_t nsplit_b;
    // backward head (see DevFactor::hb_nlev); the persistent backward
    // kernel starts at task hb_ntask (0: no head)
    const int4* __restrict__ hb_lv;
    const int32_t* __restrict__ hb_idx;
    int32_t hb_nlev, hb_ntask, hb_rows, hb_stage;
    // vectors (n x K row-major)
    const double* __restrict__ b;
    double* x;
    double* r;
    double* p;
    double* q;
    double* y;
    double* z;
    // reductions
    double* part;            // [3][grid_max][K]
    int grid_max;
    PcgScalars* sc;
    // control
    double tol;
    int max_iter;
    int stop_rule;
    int update;              // fwd: apply the x/r update
    int reduce;              // compute reductions / scalars
    int poll_ns;             // back-off between polls of a pending value
    unsigned long long timeout_ns;
    // one-RHS CSR SpMV: rows longer than kLongRow entries (ascending), each
    // done by a CTA of spmv_long_kernel; their p.q terms in lr_dot[k]
    const int32_t* __restrict__ lrows;
    double* lr_dot;
    int32_t n_lrows;
    // batched systems: row -> system, per-(system, column) step lengths
    const int32_t* __restrict__ seg;
    const double* __restrict__ seg_alpha;
};

// Block-wide sum of one double per (thread, column) slot: `v` holds the
// thread's partial for column (threadIdx.x % K) when K > 1 layouts are
// column-interleaved; here each thread carries K partials in registers.
template <int K>
__device__ void block_partials(const double (&v)[K], double* out_block /* [K] */) {
    __shared__ double red[kBlock / 32][K];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int c = 0; c < K; ++c) {
        double s = v[c];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(kFull, s, o);
        if (lane == 0) red[w][c] = s;
    }
    __syncthreads();
    if (threadIdx.x < K) {
        double s = 0.0;
        for (int i = 0; i < kBlock / 32; ++i) s += red[i][threadIdx.x];
        out_block[threadIdx.x] = s;
    }
    __syncthreads();
}

// Block-wide sum per column when every thread carries the partial of column
// (lane % K): lanes of the same column in a warp are combined first.
template <int K>
__device__ void block_partials_lane(double v, double* out_block /* [K] */) {
    __shared__ double red[kBlock / 32][K];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o >= K; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
    if (lane < K) red[w][lane] = v;
    __syncthreads();
    if (threadIdx.x < K) {
        double s = 0.0;
        for (int i = 0; i < kBlock / 32; ++i) s += red[i][threadIdx.x];
        out_block[threadIdx.x] = s;
    }
    __syncthreads();
}

// Returns true in exactly one thread of the last block to finish; that block
// then reduces the partials.  `ticket` is reset for the next use.
__device__ __forceinline__ bool last_block(unsigned* ticket) {
    __shared__ bool is_last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned t = atomicAdd(ticket, 1u);
        is_last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (is_last) {
        __threadfence();
        return true;
    }
    return false;
}

template <int K>
__device__ void sum_partials(const double* part, int nblocks, double* out) {
    // threads < K each sum one column in block order
    if (threadIdx.x < K) {
        double s = 0.0;
        for (int b = 0; b < nblocks; ++b) s += part[(size_t)b * K + threadIdx.x];
        out[threadIdx.x] = s;
    }
    __syncthreads();
}

__device__ __forceinline__ bool timed_out(unsigned long long t0, unsigned long long limit) {
    return global_timer_ns() - t0 > limit;
}

// Poll a solution component until it has been produced.
__device__ __forceinline__ double wait_value(const double* p, unsigned long long t0, unsigned long long limit,
                                             int* status, bool& ok, int poll_ns) {
    double v = ld_relaxed_f64(p);
    if (!is_pending(v)) return v;
    // exponential back-off capped at poll_ns: waits that end soon keep
    // polling fast, long waits stop flooding L2 with polls
    unsigned spins = 0;
    unsigned sleep_ns = 16;
    while (true) {
        if (poll_ns > 0 && spins >= 2) {
            __nanosleep(sleep_ns);
            sleep_ns = min(2u * sleep_ns, (unsigned)poll_ns);
        }
        v = ld_relaxed_f64(p);
        if (!is_pending(v)) return v;
        if ((++spins & 63u) == 0 && timed_out(t0, limit)) {
            raise_error(status, kDevTimeout);
            ok = false;
            return 0.0;
        }
    }
}


// Last-block bookkeeping after the x/r update (fwd): iteration count and the
// residual-based stop rules.
__device__ void fwd_convergence(SolveArgs& a, int K = 1) {
    const int it = a.sc->iter + 1;
    a.sc->iter = it;
    int any = 0;
    for (int c = 0; c < K; ++c) {
        if (!a.sc->active[c]) continue;
        bool conv = false;
        if (a.stop_rule == 0) conv = sqrt(a.sc->rr[c]) <= a.tol * sqrt(a.sc->bnorm2[c]);
        else if (a.stop_rule == 2) conv = a.sc->rr[c] <= a.tol;
        a.sc->iters[c] = it;
        if (conv) a.sc->active[c] = 0;
        else any = 1;
    }
    if (!any || it >= a.max_iter) a.sc->done = 1;
}

// Last-block bookkeeping after z = M^-1 r (bwd): the new r.z sits in pq;
// beta, rz and the preconditioned stop rule.  phase 0 (start or restart)
// initialises rz and rz0.
__device__ void bwd_scalars(SolveArgs& a, int K) {
    const bool init = a.sc->phase == 0;
    int any = 0;
    for (int c = 0; c < K; ++c) {
        const double rn = a.sc->pq[c];
        if (init) {
            if (a.sc->active[c]) {
                a.sc->rz[c] = rn;
                a.sc->rz0[c] = rn;
                a.sc->beta[c] = 0.0;
                if (a.stop_rule == 1 && !(rn > a.tol)) a.sc->active[c] = 0;
            }
        } else if (a.sc->active[c]) {
            const double ro = a.sc->rz[c];
            a.sc->beta[c] = ro != 0.0 ? rn / ro : 0.0;
            a.sc->rz[c] = rn;
            if (a.stop_rule == 1 && !(sqrt(rn) / sqrt(a.sc->rz0[c]) > a.tol)) a.sc->active[c] = 0;
        } else {
            a.sc->beta[c] = 0.0;
        }
        any |= a.sc->active[c];
    }
    a.sc->phase = 1;
    if (!any) a.sc->done = 1;
    a.sc->ticket[3] = 0;
}

// sum_p val[p] * vec[idx[p] * K + c] over entries s..e, waiting on pending
// components; entries are fetched four at a time so their gathers overlap.
template <typename TV, int K = 1>
__device__ __forceinline__ double row_dot(const int32_t* __restrict__ idx, const TV* __restrict__ val, int64_t s,
                                          int64_t e, const double* vec, unsigned long long t0,
                                          unsigned long long limit, int* status, bool& ok, int poll_ns, int c = 0) {
    double sum = 0.0;
    int64_t p = s;
    for (; p + 4 <= e; p += 4) {
        const double* q0 = vec + (size_t)idx[p] * K + c;
        const double* q1 = vec + (size_t)idx[p + 1] * K + c;
        const double* q2 = vec + (size_t)idx[p + 2] * K + c;
        const double* q3 = vec + (size_t)idx[p + 3] * K + c;
        const double l0 = to_d(val[p]), l1 = to_d(val[p + 1]), l2 = to_d(val[p + 2]), l3 = to_d(val[p + 3]);
        double v0 = ld_relaxed_f64(q0), v1 = ld_relaxed_f64(q1);
        double v2 = ld_relaxed_f64(q2), v3 = ld_relaxed_f64(q3);
        if (is_pending(v0)) v0 = wait_value(q0, t0, limit, status, ok, poll_ns);
        if (is_pending(v1)) v1 = wait_value(q1, t0, limit, status, ok, poll_ns);
        if (is_pending(v2)) v2 = wait_value(q2, t0, limit, status, ok, poll_ns);
        if (is_pending(v3)) v3 = wait_value(q3, t0, limit, status, ok, poll_ns);
        sum += l0 * v0;
        sum += l1 * v1;
        sum += l2 * v2;
        sum += l3 * v3;
    }
    for (; p < e; ++p) {
        const double* q = vec + (size_t)idx[p] * K + c;
        double v = ld_relaxed_f64(q);
        if (is_pending(v)) v = wait_value(q, t0, limit, status, ok, poll_ns);
        sum += to_d(val[p]) * v;
    }
    return sum;
}

// row_dot over the entries in descending order (e-1 down to s).  A row of
// the L^T solve (column j of L, rows ascending) depends most recently on its
// first entries, the rows eliminated right after j; walking it from the end
// adds every entry that has landed while the last dependencies are still
// being produced, so only the last few entries wait on the critical path.
template <typename TV, int K = 1>
__device__ __forceinline__ double row_dot_desc(const int32_t* __restrict__ idx, const TV* __restrict__ val,
                                               int64_t s, int64_t e, const double* vec, unsigned long long t0,
                                               unsigned long long limit, int* status, bool& ok, int poll_ns,
                                               int c = 0) {
    double sum = 0.0;
    int64_t p = e;
    for (; p - 4 >= s; p -= 4) {
        const double* q0 = vec + (size_t)idx[p - 1] * K + c;
        const double* q1 = vec + (size_t)idx[p - 2] * K + c;
        const double* q2 = vec + (size_t)idx[p - 3] * K + c;
        const double* q3 = vec + (size_t)idx[p - 4] * K + c;
        const double l0 = to_d(val[p - 1]), l1 = to_d(val[p - 2]), l2 = to_d(val[p - 3]), l3 = to_d(val[p - 4]);
        double v0 = ld_relaxed_f64(q0), v1 = ld_relaxed_f64(q1);
        double v2 = ld_relaxed_f64(q2), v3 = ld_relaxed_f64(q3);
        if (is_pending(v0)) v0 = wait_value(q0, t0, limit, status, ok, poll_ns);
        if (is_pending(v1)) v1 = wait_value(q1, t0, limit, status, ok, poll_ns);
        if (is_pending(v2)) v2 = wait_value(q2, t0, limit, status, ok, poll_ns);
        if (is_pending(v3)) v3 = wait_value(q3, t0, limit, status, ok, poll_ns);
        sum += l0 * v0;
        sum += l1 * v1;
        sum += l2 * v2;
        sum += l3 * v3;
    }
    for (; p > s; --p) {
        const double* q = vec + (size_t)idx[p - 1] * K + c;
        double v = ld_relaxed_f64(q);
        if (is_pending(v)) v = wait_value(q, t0, limit, status, ok, poll_ns);
        sum += to_d(val[p - 1]) * v;
    }
    return sum;
}

// sum_p val[p] * vec[idx[p] * K + c] for final (non-pending) vectors
template <int K = 1>
__device__ __forceinline__ double row_dot_plain(const int32_t* __restrict__ idx, const double* __restrict__ val,
                                                int64_t s, int64_t e, const double* __restrict__ vec, int c = 0) {
    double sum = 0.0;
    int64_t p = s;
    for (; p + 4 <= e; p += 4) {
        const double v0 = vec[(size_t)idx[p] * K + c], v1 = vec[(size_t)idx[p + 1] * K + c];
        const double v2 = vec[(size_t)idx[p + 2] * K + c], v3 = vec[(size_t)idx[p + 3] * K + c];
        sum += val[p] * v0;
        sum += val[p + 1] * v1;
        sum += val[p + 2] * v2;
        sum += val[p + 3] * v3;
    }
    for (; p < e; ++p) sum += val[p] * vec[(size_t)idx[p] * K + c];
    return sum;
}

// ---------------------------------------------------------------------------
// init: x = 0, r = b, p = q = 0, y = pending; ||b||^2
// ---------------------------------------------------------------------------
template <int K>
__global__ void __launch_bounds__(kBlock) init_kernel(SolveArgs a) {
    // the grid stride is a multiple of K, so every element a thread touches
    // belongs to column (lane % K)
    double acc = 0.0;
    const int64_t total = (int64_t)a.n * K;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += stride) {
        double bv = a.b[t];
        a.x[t] = 0.0;
        a.r[t] = bv;
        a.p[t] = 0.0;
        a.q[t] = 0.0;
        a.y[t] = pending_value();
        acc += bv * bv;
    }
    block_partials_lane<K>(acc, a.part + (size_t)blockIdx.x * K);
    if (last_block(&a.sc->ticket[0])) {
        sum_partials<K>(a.part, gridDim.x, a.sc->bnorm2);
        if (threadIdx.x < K) {
            int c = threadIdx.x;
            a.sc->alpha[c] = 0.0;
            a.sc->beta[c] = 0.0;
            a.sc->rz[c] = 0.0;
            a.sc->active[c] = a.sc->bnorm2[c] > 0.0 ? 1 : 0;
            a.sc->iters[c] = 0;
        }
        if (threadIdx.x == 0) {
            a.sc->ticket[0] = 0;
            a.sc->iter = 0;
            a.sc->phase = 0;
            a.sc->status = 0;
            int any = 0;
            for (int c = 0; c < K; ++c) any |= a.sc->bnorm2[c] > 0.0;
            a.sc->done = any ? 0 : 1;
        }
    }
}

// ---------------------------------------------------------------------------
// spmv_update: s = A z; q = s + beta q; p = z + beta p; (p.q); y = pending
// ---------------------------------------------------------------------------
// K right-hand sides of the long rows (spmv_long_kernel's multi-RHS form):
// one CTA per row; thread t adds column t % K over every (kBlock / K)-th
// entry from t / K in entry order, then column c's kBlock / K partial sums
// are added in group order.  Terms of column c in lr_dot[k * K + c].
template <int K>
__global__ void __launch_bounds__(kBlock) spmv_long_k_kernel(SolveArgs a) {
    if (ld_relaxed(&a.sc->done)) return;
    constexpr int NG = kBlock / K;
    __shared__ double red[NG][K];
    const int32_t i = a.lrows[blockIdx.x];
    const int s = a.a_ptr[i], e = a.a_ptr[i + 1];
    const int c = threadIdx.x % K, g = threadIdx.x / K;
    double sum = 0.0;
    for (int p = s + g; p < e; p += NG) sum += __dmul_rn(a.a_val[p], a.z[(size_t)a.a_idx[p] * K + c]);
    red[g][c] = sum;
    __syncthreads();
    if (threadIdx.x < K) {
        double t = 0.0;
        for (int q = 0; q < NG; ++q) t += red[q][c];
        const size_t o = (size_t)i * K + c;
        const double qi = t + a.sc->beta[c] * a.q[o];
        const double pi = a.z[o] + a.sc->beta[c] * a.p[o];
        a.q[o] = qi;
        a.p[o] = pi;
        a.y[o] = pending_value();
        a.lr_dot[(size_t)blockIdx.x * K + c] = pi * qi;
    }
}

// 8 CTAs per SM (32 registers): the grid is 8 per SM, and the gathers of z
// rows need every warp in flight
template <int K>
__global__ void __launch_bounds__(kBlock, 8) spmv_update_kernel(SolveArgs a) {
    if (ld_relaxed(&a.sc->done)) return;
    // one RHS: a thread per row; K RHS: K lanes per row, lane c owns column c
    constexpr int G = K;
    const int lane = threadIdx.x & 31;
    const int c = lane % G;
    const int64_t group = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / G;
    const int64_t ngroups = (int64_t)gridDim.x * blockDim.x / G;
    const double beta = a.sc->beta[c];
    double acc = 0.0;
    for (int64_t i = group; i < a.n; i += ngroups) {
        const int s = a.a_ptr[i], e = a.a_ptr[i + 1];
        if (a.n_lrows > 0 && e - s > kLongRow) continue;  // spmv_long_k_kernel's
        const double sum = row_dot_plain<K>(a.a_idx, a.a_val, s, e, a.z, c);
        const size_t o = (size_t)i * K + c;
        const double qi = sum + beta * a.q[o];
        const double pi = a.z[o] + beta * a.p[o];
        a.q[o] = qi;
        a.p[o] = pi;
        a.y[o] = pending_value();
        acc += pi * qi;
    }
    block_partials_lane<K>(acc, a.part + (size_t)blockIdx.x * K);
    if (last_block(&a.sc->ticket[1])) {
        sum_partials<K>(a.part, gridDim.x, a.sc->pq);
        if (threadIdx.x < K && a.n_lrows > 0) {
            // the long rows' terms of column c, in row order
            double t = 0.0;
            for (int k = 0; k < a.n_lrows; ++k) t += a.lr_dot[(size_t)k * K + threadIdx.x];
            a.sc->pq[threadIdx.x] += t;
        }
        if (threadIdx.x < K) {
            int c = threadIdx.x;
            double pq = a.sc->pq[c];
            a.sc->alpha[c] = (a.sc->active[c] && pq != 0.0) ? a.sc->rz[c] / pq : 0.0;
        }
        if (threadIdx.x == 0) a.sc->ticket[1] = 0;
    }
}

// One right-hand side: a warp takes 32 consecutive rows at a time.  Their
// matrix entries form one contiguous range, read coalesced kSpmvChunk at a
// time; the products val * z[idx] go to shared memory, and each lane then
// adds the products of its own row in entry order (round the product, then
// add, as a plain row loop without fused multiply-add does).
#ifndef RCHOL_SPMV_CHUNK
#define RCHOL_SPMV_CHUNK 128
#endif
constexpr int kSpmvChunk = RCHOL_SPMV_CHUNK;  // entries staged per warp and chunk

// Rows longer than kLongRow entries (the hubs of power-law graphs): one
// CTA per row, each thread adding every kBlock-th product of the row in
// entry order, then the threads' sums in a fixed tree; the same q, p, y and
// p.q term as the tile and sliced-ELL kernels, which skip these rows.

// pq += the long rows' p.q terms (spmv_long_kernel ran first): each thread
// every kBlock-th term in order, then the threads in a fixed tree.  Called
// by every thread of the SpMV's last block.
__device__ void add_long_row_terms(SolveArgs& a) {
    if (a.n_lrows == 0) return;
    double lt[1] = {0.0};
    for (int k = threadIdx.x; k < a.n_lrows; k += blockDim.x) lt[0] += a.lr_dot[k];
    block_partials<1>(lt, a.lr_dot + a.n_lrows);
    if (threadIdx.x == 0) a.sc->pq[0] += a.lr_dot[a.n_lrows];
}

__global__ void __launch_bounds__(kBlock) spmv_long_kernel(SolveArgs a) {
    if (ld_relaxed(&a.sc->done)) return;
    __shared__ double red[kBlock / 32];
    const int32_t i = a.lrows[blockIdx.x];
    const int s = a.a_ptr[i], e = a.a_ptr[i + 1];
    double sum = 0.0;
    for (int p = s + (int)threadIdx.x; p < e; p += kBlock) sum += __dmul_rn(a.a_val[p], a.z[a.a_idx[p]]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(kFull, sum, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = sum;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < kBlock / 32; ++w) t += red[w];
        const double beta = a.sc->beta[0];
        const double qi = t + beta * a.q[i];
        const double pi = a.z[i] + beta * a.p[i];
        a.q[i] = qi;
        a.p[i] = pi;
        a.y[i] = pending_value();
        a.lr_dot[blockIdx.x] = pi * qi;
    }
}

__global__ void __launch_bounds__(kBlock) spmv_update_tile_kernel(SolveArgs a) {
    if (ld_relaxed(&a.sc->done)) return;
    __shared__ double stage_all[kBlock / 32][kSpmvChunk];
    const int lane = threadIdx.x & 31;
    double* stage = stage_all[threadIdx.x >> 5];
    const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int64_t ntiles = ((int64_t)a.n + 31) / 32;
    const double beta = a.sc->beta[0];
    double acc = 0.0;
    for (int64_t tile = gw; tile < ntiles; tile += nw) {
        const int64_t r0 = tile * 32;
        const int rows = (int)(((int64_t)a.n - r0) < 32 ? ((int64_t)a.n - r0) : 32);
        const bool row = lane < rows;
        const int64_t i = r0 + lane;
        const int ps = row ? a.a_ptr[i] : 0;
        const int tile_end = a.a_ptr[r0 + rows];
        const int nb = __shfl_down_sync(kFull, ps, 1);
        const int pe = lane + 1 < rows ? nb : tile_end;
        const int tile_begin = __shfl_sync(kFull, ps, 0);
        if (a.n_lrows > 0 && __any_sync(kFull, row && pe - ps > kLongRow)) {
            // a tile holding a long row: the long rows are spmv_long_kernel's,
            // every other row is added by its own lane in entry order
            if (row && pe - ps <= kLongRow) {
                double sum = 0.0;
                for (int p = ps; p < pe; ++p) sum += __dmul_rn(a.a_val[p], a.z[a.a_idx[p]]);
                const double qi = sum + beta * a.q[i];
                const double pi = a.z[i] + beta * a.p[i];
                a.q[i] = qi;
                a.p[i] = pi;
                a.y[i] = pending_value();
                acc += pi * qi;
            }
            continue;
        }
        // row vectors in flight while the products are formed
        double qo = 0.0, po = 0.0, zi = 0.0;
        if (row) {
            qo = a.q[i];
            po = a.p[i];
            zi = a.z[i];
        }
        double sum = 0.0;
        for (int c0 = tile_begin; c0 < tile_end; c0 += kSpmvChunk) {
            const int cn = min(kSpmvChunk, tile_end - c0);
            int32_t idx[kSpmvChunk / 32];
            double val[kSpmvChunk / 32], zv[kSpmvChunk / 32];
#pragma unroll
            for (int k = 0; k < kSpmvChunk / 32; ++k) {
                const int e = k * 32 + lane;
                if (e < cn) {
                    idx[k] = a.a_idx[c0 + e];
                    val[k] = a.a_val[c0 + e];
                }
            }
#pragma unroll
            for (int k = 0; k < kSpmvChunk / 32; ++k)
                if (k * 32 + lane < cn) zv[k] = a.z[idx[k]];
#pragma unroll
            for (int k = 0; k < kSpmvChunk / 32; ++k) {
                const int e = k * 32 + lane;
                if (e < cn) stage[e] = __dmul_rn(val[k], zv[k]);
            }
            __syncwarp();
            const int lo = max(ps, c0), hi = min(pe, c0 + cn);
            if (row)
                for (int p = lo; p < hi; ++p) sum += stage[p - c0];
            __syncwarp();
        }
        if (row) {
            const double qi = sum + beta * qo;
            const double pi = zi + beta * po;
            a.q[i] = qi;
            a.p[i] = pi;
            a.y[i] = pending_value();
            acc += pi * qi;
        }
    }
    block_partials_lane<1>(acc, a.part + (size_t)blockIdx.x);
    if (last_block(&a.sc->ticket[1])) {
        sum_partials<1>(a.part, gridDim.x, a.sc->pq);
        add_long_row_terms(a);
        if (threadIdx.x == 0) {
            const double pq = a.sc->pq[0];
            a.sc->alpha[0] = (a.sc->active[0] && pq != 0.0) ? a.sc->rz[0] / pq : 0.0;
            a.sc->ticket[1] = 0;
        }
    }
}

// One right-hand side on the sliced-ELL copy of A: a warp per slice of 32
// rows, a lane per row.  A slice's columns are read 8 at a time (index and
// value loads all in flight before the z gathers), streamed past L2 so that
// the vectors stay resident.  Each lane adds its row's rounded products in
// entry order, so q and p equal those of spmv_update_tile_kernel bit for
// bit; the launch is one resident wave (the p.q partials follow its grid).
constexpr int kSellCols = 8;

__global__ void __launch_bounds__(kBlock) spmv_update_sell_kernel(SolveArgs a) {
    if (ld_relaxed(&a.sc->done)) return;
    const int lane = threadIdx.x & 31;
    const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int64_t ntiles = ((int64_t)a.n + 31) / 32;
    const double beta = a.sc->beta[0];
    double acc = 0.0;
    int64_t s0 = 0, s1 = 0;
    if (gw < ntiles) {
        s0 = a.s_ptr[gw];
        s1 = a.s_ptr[gw + 1];
    }
    for (int64_t tile = gw; tile < ntiles; tile += nw) {
        const int64_t i = tile * 32 + lane;
        const bool row = i < a.n;
        double qo = 0.0, po = 0.0, zi = 0.0;
        if (row) {
            qo = a.q[i];
            po = a.p[i];
            zi = a.z[i];
        }
        // the next slice's column range is in flight during this one
        int64_t n0 = 0, n1 = 0;
        if (tile + nw < ntiles) {
            n0 = a.s_ptr[tile + nw];
            n1 = a.s_ptr[tile + nw + 1];
        }
        double sum = 0.0;
        for (int64_t k0 = s0; k0 < s1; k0 += kSellCols) {
            const int m = (int)min((int64_t)kSellCols, s1 - k0);
            int32_t idx[kSellCols];
            double val[kSellCols], zv[kSellCols];
#pragma unroll
            for (int k = 0; k < kSellCols; ++k) {
                idx[k] = -1;
                if (k < m) {
                    const int64_t slot = (k0 + k) * 32 + lane;
                    idx[k] = __ldcs(a.s_idx + slot);
                    val[k] = __ldcs(a.s_val + slot);
                }
            }
#pragma unroll
            for (int k = 0; k < kSellCols; ++k)
                if (idx[k] >= 0) zv[k] = a.z[idx[k]];
#pragma unroll
            for (int k = 0; k < kSellCols; ++k)
                if (idx[k] >= 0) sum = __dadd_rn(sum, __dmul_rn(val[k], zv[k]));
        }
        // long rows hold no slots here: spmv_long_kernel did them
        const bool mine = row && (a.n_lrows == 0 || a.a_ptr[i + 1] - a.a_ptr[i] <= kLongRow);
        if (mine) {
            const double qi = sum + beta * qo;
            const double pi = zi + beta * po;
            a.q[i] = qi;
            a.p[i] = pi;
            a.y[i] = pending_value();
            acc += pi * qi;
        }
        s0 = n0;
        s1 = n1;
    }
    block_partials_lane<1>(acc, a.part + (size_t)blockIdx.x);
    if (last_block(&a.sc->ticket[1])) {
        sum_partials<1>(a.part, gridDim.x, a.sc->pq);
        add_long_row_terms(a);
        if (threadIdx.x == 0) {
            const double pq = a.sc->pq[0];
            a.sc->alpha[0] = (a.sc->active[0] && pq != 0.0) ? a.sc->rz[0] / pq : 0.0;
            a.sc->ticket[1] = 0;
        }
    }
}

// The k > 1 solve kernels are compiled for 5 CTAs per SM (48 registers).
// With an FP64 factor copy that spills a few bytes and still gains the fifth
// CTA (k = 32 forward 5.0 -> 4.4 ms, backward 4.3 -> 3.9 ms on a 27-point
// 128^3 factor); the FP32 forms needed 48 registers already.
constexpr int kSolveMinBlocks = 5;

// ---------------------------------------------------------------------------
// fwd: x += alpha p; r -= alpha q; (r.r); y = L^{-1} r  (rows ascending)
// ---------------------------------------------------------------------------
template <int K, typename TV>
__global__ void __launch_bounds__(kBlock, kSolveMinBlocks) fwd_kernel(SolveArgs a) {
    // K >= 2 right-hand sides: K lanes per row, lane c owns column c
    if ((a.reduce || a.seg) && ld_relaxed(&a.sc->done)) return;
    constexpr int G = K;
    const int lane = threadIdx.x & 31;
    const int c = lane % G;
    const int64_t group = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / G;
    const int64_t ngroups = (int64_t)gridDim.x * blockDim.x / G;
    const TV* __restrict__ lv = reinterpret_cast<const TV*>(a.lr_val);
    const double alpha = a.update ? a.sc->alpha[c] : 0.0;
    double acc = 0.0;
    const unsigned long long t0 = global_timer_ns();
    bool ok = true;
    for (int64_t t = group; t < a.n && ok; t += ngroups) {
        const int64_t i = a.order_f[t];
        const int64_t ri_ = a.by_pos ? t : i;
        const int64_t s = a.lr_ptr[ri_], e = a.lr_ptr[ri_ + 1];
        const size_t o = (size_t)i * K + c;
        double ri = a.r[o];
        if (a.update) {
            const double al = a.seg ? a.seg_alpha[(size_t)a.seg[i] * K + c] : alpha;
            a.x[o] = a.x[o] + al * a.p[o];
            ri = ri - al * a.q[o];
            a.r[o] = ri;
            acc += ri * ri;
        }
        const double sum = row_dot<TV, K>(a.lr_idx, lv, s, e, a.y, t0, a.timeout_ns, &a.sc->status, ok,
                                          a.poll_ns, c);
        if (a.z) a.z[o] = pending_value();
        st_relaxed_f64(a.y + o, ri - sum);
    }
    // a timed-out wait abandons the pass (block-uniform decision)
    if (__syncthreads_or(!ok)) {
        if (threadIdx.x == 0) a.sc->done = 1;
        return;
    }
    if (!a.reduce) return;
    block_partials_lane<K>(acc, a.part + (size_t)(a.grid_max + blockIdx.x) * K);
    if (last_block(&a.sc->ticket[2])) {
        if (a.update) {
            sum_partials<K>(a.part + (size_t)a.grid_max * K, gridDim.x, a.sc->rr);
            if (threadIdx.x == 0) fwd_convergence(a, K);
        }
        if (threadIdx.x == 0) a.sc->ticket[2] = 0;
    }
}

// ---------------------------------------------------------------------------
// bwd: z = L^{-T} D^+ y  (rows descending); (r.z) -> rz, beta
// ---------------------------------------------------------------------------
template <int K, typename TV>
__global__ void __launch_bounds__(kBlock, kSolveMinBlocks) bwd_kernel(SolveArgs a) {
    // K >= 2 right-hand sides: K lanes per row, lane c owns column c
    if ((a.reduce || a.seg) && ld_relaxed(&a.sc->done)) return;
    constexpr int G = K;
    const int lane = threadIdx.x & 31;
    const int c = lane % G;
    const int64_t group = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / G;
    const int64_t ngroups = (int64_t)gridDim.x * blockDim.x / G;
    const TV* __restrict__ lv = reinterpret_cast<const TV*>(a.lc_val);
    const TV* __restrict__ dv = reinterpret_cast<const TV*>(a.diag);
    double acc = 0.0;
    const unsigned long long t0 = global_timer_ns();
    bool ok = true;
    for (int64_t g = group; g < a.n && ok; g += ngroups) {
        const int64_t j = a.order_b[g];
        const int64_t rj_ = a.by_pos ? g : j;
        const int64_t s = a.lc_ptr[rj_], e = a.lc_ptr[rj_ + 1];
        const double dj = to_d(dv[j]);
        const size_t o = (size_t)j * K + c;
        double t = a.y[o];
        if (dj != 0.0) t = t / dj;
        const double sum = row_dot_desc<TV, K>(a.lc_idx, lv, s, e, a.z, t0, a.timeout_ns, &a.sc->status, ok,
                                          a.poll_ns, c);
        const double zj = t - sum;
        st_relaxed_f64(a.z + o, zj);
        acc += a.r[o] * zj;
    }
    // a timed-out wait abandons the pass (block-uniform decision)
    if (__syncthreads_or(!ok)) {
        if (threadIdx.x == 0) a.sc->done = 1;
        return;
    }
    if (!a.reduce) return;
    block_partials_lane<K>(acc, a.part + (size_t)(2 * a.grid_max + blockIdx.x) * K);
    if (last_block(&a.sc->ticket[3])) {
        sum_partials<K>(a.part + (size_t)2 * a.grid_max * K, gridDim.x, a.sc->pq);
        if (threadIdx.x == 0) bwd_scalars(a, K);
    }
}


// ---------------------------------------------------------------------------
// K = 1 solves over task slabs.  A task is one row group of G = 2^cls lanes
// per row (up to 32 / G rows of one level and lane class per warp; long
// rows take the whole warp, rows longer than 1024 entries are split into
// part tasks).  A warp takes the tasks warp, warp + nwarps, ... in schedule
// order, so every dependency sits in an earlier task.  While it waits on
// the dependencies of one task, the slab entries and row indices of its
// next task are already in flight, so a task's critical path after its last
// dependency lands is one poll round trip, a short dot product and one store.
// ---------------------------------------------------------------------------

constexpr int kPackM = 4;  // slab slots per lane held in registers
// gate rounds per re-read of the other pending slots (0: none)
#ifndef RCHOL_TRICKLE
#define RCHOL_TRICKLE 2
#endif
constexpr unsigned kTrickle = RCHOL_TRICKLE;
// 3 CTAs of 256 threads per SM (80 registers, no spills in the poll loops)
#ifndef RCHOL_PACK_MINB
#define RCHOL_PACK_MINB 3
#endif

template <typename TV>
struct PackLane {
    int4 d;
    int32_t row;
    int32_t idx[kPackM];
    TV val[kPackM];
};

template <typename TV>
__device__ __forceinline__ void pack_load(PackLane<TV>& L, const int4 d, int lane, const int32_t* __restrict__ order,
                                          const int32_t* __restrict__ pidx, const TV* __restrict__ pval) {
    L.d = d;
    const int cls = (d.z >> 8) & 7, cnt = d.z & 0xff;
    L.row = (lane >> cls) < cnt ? order[d.x + (lane >> cls)] : 0;
    const size_t o = (size_t)d.y * 32 + lane;
#pragma unroll
    for (int k = 0; k < kPackM; ++k) {
        if (k < (d.w & 0xff)) {
            L.idx[k] = pidx[o + 32 * k];
            L.val[k] = pval[o + 32 * k];
        } else {
            L.idx[k] = -1;
            L.val[k] = TV(0);
        }
    }
}

// Re-reads the pending components of v (bit k of pend) together until none
// is pending; false on timeout.
__device__ __forceinline__ bool poll_pending(double (&v)[kPackM], const int32_t (&idx)[kPackM], const double* vec,
                                             unsigned pend, unsigned long long t0, unsigned long long limit,
                                             int* status, int poll_ns) {
    unsigned spins = 0, sleep_ns = 16;
    while (pend) {
        if (poll_ns > 0 && spins >= 2) {
            __nanosleep(sleep_ns);
            sleep_ns = min(2u * sleep_ns, (unsigned)poll_ns);
        }
#pragma unroll
        for (int k = 0; k < kPackM; ++k)
            if ((pend >> k) & 1u) v[k] = ld_relaxed_f64(vec + idx[k]);
        pend = 0;
#pragma unroll
        for (int k = 0; k < kPackM; ++k) pend |= (is_pending(v[k]) ? 1u : 0u) << k;
        if (pend && (++spins & 63u) == 0 && timed_out(t0, limit)) {
            raise_error(status, kDevTimeout);
            return false;
        }
    }
    return true;
}

__device__ __forceinline__ unsigned pending_mask(const double (&v)[kPackM]) {
    unsigned pend = 0;
#pragma unroll
    for (int k = 0; k < kPackM; ++k) pend |= (is_pending(v[k]) ? 1u : 0u) << k;
    return pend;
}

// The lane's share of its row's dot product.  Slot 0 of the row's first
// lane holds the row's gate, its dependency scheduled last.  Every slot is
// read once; rows whose gate is still pending then poll the gate alone
// (every kTrickle-th round also re-reading their other pending slots), so
// the values just produced at the solve front are polled by few rows; once
// the gate has landed the remaining pending slots are polled together.
// Slots beyond the first kPackM of long rows are fetched at the start and
// waited on together with the first ones; rows longer than 2 * kPackM slots
// per lane continue kPackM slots at a time.
template <typename TV>
__device__ __forceinline__ void slab_chunk(const PackLane<TV>& L, int k0, int lane, const int32_t* __restrict__ pidx,
                                           const TV* __restrict__ pval, int32_t (&idx)[kPackM], TV (&val)[kPackM]) {
    const size_t o = ((size_t)L.d.y + k0) * 32 + lane;
#pragma unroll
    for (int k = 0; k < kPackM; ++k) {
        if (k0 + k < (L.d.w & 0xff)) {
            idx[k] = pidx[o + 32 * k];
            val[k] = pval[o + 32 * k];
        } else {
            idx[k] = -1;
            val[k] = TV(0);
        }
    }
}

template <typename TV>
__device__ __forceinline__ double pack_dot(const PackLane<TV>& L, int lane, int G, const int32_t* __restrict__ pidx,
                                           const TV* __restrict__ pval, const double* vec, unsigned long long t0,
                                           unsigned long long limit, int* status, bool& ok, int poll_ns) {
    // slots kPackM..2*kPackM-1 of long rows: fetched now, waited on with the rest
    int32_t idx2[kPackM];
    TV val2[kPackM];
    const int mslots = L.d.w & 0xff;
    const bool two = mslots > kPackM;
    if (two) slab_chunk(L, kPackM, lane, pidx, pval, idx2, val2);
    double v[kPackM], v2[kPackM];
#pragma unroll
    for (int k = 0; k < kPackM; ++k) v[k] = L.idx[k] >= 0 ? ld_relaxed_f64(vec + L.idx[k]) : 0.0;
    if (two) {
#pragma unroll
        for (int k = 0; k < kPackM; ++k) v2[k] = idx2[k] >= 0 ? ld_relaxed_f64(vec + idx2[k]) : 0.0;
    }
    const bool first = (lane & (G - 1)) == 0;
    bool gate = first && is_pending(v[0]);
    unsigned spins = 0;
    while (__any_sync(kFull, gate)) {
        if (gate) {
            v[0] = ld_relaxed_f64(vec + L.idx[0]);
            gate = is_pending(v[0]);
        }
        ++spins;
        if (kTrickle > 0 && spins % kTrickle == 0) {
#pragma unroll
            for (int k = 0; k < kPackM; ++k)
                if ((k > 0 || !first) && is_pending(v[k])) v[k] = ld_relaxed_f64(vec + L.idx[k]);
            if (two) {
#pragma unroll
                for (int k = 0; k < kPackM; ++k)
                    if (is_pending(v2[k])) v2[k] = ld_relaxed_f64(vec + idx2[k]);
            }
        }
        if ((spins & 63u) == 0 && __shfl_sync(kFull, timed_out(t0, limit) ? 1 : 0, 0)) {
            if (gate) raise_error(status, kDevTimeout);
            ok = false;
            return 0.0;
        }
    }
    if (!poll_pending(v, L.idx, vec, pending_mask(v), t0, limit, status, poll_ns) ||
        (two && !poll_pending(v2, idx2, vec, pending_mask(v2), t0, limit, status, poll_ns))) {
        ok = false;
        return 0.0;
    }
    double sum = 0.0;
#pragma unroll
    for (int k = 0; k < kPackM; ++k) sum += to_d(L.val[k]) * v[k];
    if (two) {
#pragma unroll
        for (int k = 0; k < kPackM; ++k) sum += to_d(val2[k]) * v2[k];
    }
    for (int k0 = 2 * kPackM; k0 < mslots && ok; k0 += kPackM) {
        int32_t idx[kPackM];
        TV val[kPackM];
        slab_chunk(L, k0, lane, pidx, pval, idx, val);
#pragma unroll
        for (int k = 0; k < kPackM; ++k) v[k] = idx[k] >= 0 ? ld_relaxed_f64(vec + idx[k]) : 0.0;
        if (!poll_pending(v, idx, vec, pending_mask(v), t0, limit, status, poll_ns)) {
            ok = false;
            break;
        }
#pragma unroll
        for (int k = 0; k < kPackM; ++k) sum += to_d(val[k]) * v[k];
    }
    return sum;
}

// Sum over the G lanes of each row group (all 32 lanes take part).
__device__ __forceinline__ double group_sum(double v, int G) {
    for (int o = 16; o > 0; o >>= 1)
        if (o < G) v += __shfl_xor_sync(kFull, v, o);
    return v;
}

// y = L^-1 r (with update: x += alpha p, r -= alpha q, ||r||^2 first)
template <typename TV>
__global__ void __launch_bounds__(kBlock, RCHOL_PACK_MINB) fwd_pack_kernel(SolveArgs a) {
    if ((a.reduce || a.seg) && ld_relaxed(&a.sc->done)) return;
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const TV* __restrict__ pval = reinterpret_cast<const TV*>(a.pf_val);
    const double alpha = a.update ? a.sc->alpha[0] : 0.0;
    double acc[1] = {0.0};
    const unsigned long long t0 = global_timer_ns();
    bool ok = true;
    PackLane<TV> cur, nxt;
    if (warp < a.ntasks_f) pack_load(cur, a.pack_f[warp], lane, a.order_f, a.pf_idx, pval);
    int4 dn = warp + nwarps < a.ntasks_f ? a.pack_f[warp + nwarps] : make_int4(0, 0, 0, 0);
    for (int64_t t = warp; t < a.ntasks_f && ok; t += nwarps) {
        const int cls = (cur.d.z >> 8) & 7, cnt = cur.d.z & 0xff;
        const int G = 1 << cls;
        const bool lead = (lane >> cls) < cnt && (lane & (G - 1)) == 0;
        const bool part = (cur.d.z >> 11) & 1;
        const int ipart = cur.d.z >> 12;
        const int32_t i = cur.row;
        // row data and the x / r update do not depend on the dot product;
        // a split row's update belongs to its part 0
        double ri = 0.0;
        if (lead && (!part || ipart == 0)) {
            ri = a.r[i];
            if (a.update) {
                const double al = a.seg ? a.seg_alpha[a.seg[i]] : alpha;
                const double xi = a.x[i], pi = a.p[i], qi = a.q[i];
                a.x[i] = xi + al * pi;
                ri = ri - al * qi;
                a.r[i] = ri;
                acc[0] += ri * ri;
            }
            if (a.z) a.z[i] = pending_value();
        }
        if (t + nwarps < a.ntasks_f) pack_load(nxt, dn, lane, a.order_f, a.pf_idx, pval);
        if (t + 2 * nwarps < a.ntasks_f) dn = a.pack_f[t + 2 * nwarps];
        double sum = pack_dot<TV>(cur, lane, G, a.pf_idx, pval, a.y, t0, a.timeout_ns, &a.sc->status, ok, a.poll_ns);
        sum = group_sum(sum, G);
        if (lead && !part) st_relaxed_f64(a.y + i, ri - sum);
        if (lead && part) {
            // partial sum; the last part to finish adds them in part order
            const int2 sp = a.split_f[t];
            const int np = cur.d.w >> 8;
            a.psum_f[sp.y + ipart] = sum;
            if (atom_add_acq_rel(a.pcount_f + sp.x, 1) == np - 1) {
                double tot = 0.0;
                for (int q = 0; q < np; ++q) tot += ld_relaxed_f64(a.psum_f + sp.y + q);
                st_relaxed_f64(a.y + i, ld_relaxed_f64(a.r + i) - tot);
                a.pcount_f[sp.x] = 0;
            }
        }
        ok = __all_sync(kFull, ok);
        cur = nxt;
    }
    if (__syncthreads_or(!ok)) {
        if (threadIdx.x == 0) a.sc->done = 1;
        return;
    }
    if (!a.reduce) return;
    block_partials<1>(acc, a.part + (size_t)(a.grid_max + blockIdx.x));
    if (last_block(&a.sc->ticket[2])) {
        if (a.update) {
            sum_partials<1>(a.part + (size_t)a.grid_max, gridDim.x, a.sc->rr);
            if (threadIdx.x == 0) fwd_convergence(a);
        }
        if (threadIdx.x == 0) a.sc->ticket[2] = 0;
    }
}

// z = L^-T D^+ y (with reduce: r.z -> beta, stop test)
template <typename TV>
__global__ void __launch_bounds__(kBlock, RCHOL_PACK_MINB) bwd_pack_kernel(SolveArgs a) {
    if ((a.reduce || a.seg) && ld_relaxed(&a.sc->done)) return;
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const TV* __restrict__ pval = reinterpret_cast<const TV*>(a.pb_val);
    const TV* __restrict__ dv = reinterpret_cast<const TV*>(a.diag);
    double acc[1] = {0.0};
    const unsigned long long t0 = global_timer_ns();
    bool ok = true;
    PackLane<TV> cur, nxt;
    // the head's tasks were solved by bwd_head_kernel
    const int64_t tb = a.hb_ntask + warp;
    if (tb < a.ntasks_b) pack_load(cur, a.pack_b[tb], lane, a.order_b, a.pb_idx, pval);
    int4 dn = tb + nwarps < a.ntasks_b ? a.pack_b[tb + nwarps] : make_int4(0, 0, 0, 0);
    for (int64_t t = tb; t < a.ntasks_b && ok; t += nwarps) {
        const int cls = (cur.d.z >> 8) & 7, cnt = cur.d.z & 0xff;
        const int G = 1 << cls;
        const bool lead = (lane >> cls) < cnt && (lane & (G - 1)) == 0;
        const int32_t j = cur.row;
        double tj = 0.0, rj = 0.0;
        if (lead) {
            const double dj = to_d(dv[j]);
            tj = a.y[j];
            if (dj != 0.0) tj = tj / dj;
            if (a.reduce) rj = a.r[j];
        }
        if (t + nwarps < a.ntasks_b) pack_load(nxt, dn, lane, a.order_b, a.pb_idx, pval);
        if (t + 2 * nwarps < a.ntasks_b) dn = a.pack_b[t + 2 * nwarps];
        double sum = pack_dot<TV>(cur, lane, G, a.pb_idx, pval, a.z, t0, a.timeout_ns, &a.sc->status, ok, a.poll_ns);
        sum = group_sum(sum, G);
        if (lead && !((cur.d.z >> 11) & 1)) {
            const double zj = tj - sum;
            st_relaxed_f64(a.z + j, zj);
            if (a.reduce) acc[0] += rj * zj;
        } else if (lead) {
            // partial sum; the last part to finish adds them in part order.
            // Split rows' r.z terms are added by the reducing block.
            const int2 sp = a.split_b[t];
            const int np = cur.d.w >> 8;
            const int ipart = cur.d.z >> 12;
            a.psum_b[sp.y + ipart] = sum;
            if (atom_add_acq_rel(a.pcount_b + sp.x, 1) == np - 1) {
                double tot = 0.0;
                for (int q = 0; q < np; ++q) tot += ld_relaxed_f64(a.psum_b + sp.y + q);
                st_relaxed_f64(a.z + j, tj - tot);
                a.pcount_b[sp.x] = 0;
            }
        }
        ok = __all_sync(kFull, ok);
        cur = nxt;
    }
    if (__syncthreads_or(!ok)) {
        if (threadIdx.x == 0) a.sc->done = 1;
        return;
    }
    if (!a.reduce) return;
    block_partials<1>(acc, a.part + (size_t)(2 * a.grid_max + blockIdx.x));
    if (last_block(&a.sc->ticket[3])) {
        sum_partials<1>(a.part + (size_t)2 * a.grid_max, gridDim.x, a.sc->pq);
        if (threadIdx.x == 0) {
            if (a.hb_ntask > 0) a.sc->pq[0] += a.sc->hrz;
            if (a.nsplit_b) {  // split rows in id order
                double extra = a.sc->pq[0];
                for (int q = 0; q < a.nsplit_b; ++q) {
                    const int32_t j = a.srow_b[q];
                    extra += a.r[j] * ld_relaxed_f64(a.z + j);
                }
                a.sc->pq[0] = extra;
            }
            bwd_scalars(a, 1);
        }
    }
}

// ---------------------------------------------------------------------------
// Backward head: z for the rows of the first hb_nlev backward levels, solved
// by one CTA level by level.  These levels are narrow (the vertices
// eliminated last) and every dependency of a head row is an earlier head
// row, so the z values live in shared memory and a level costs one CTA
// barrier instead of a store -> poll hop between SMs.  Each level's task
// descriptors and slab slots (contiguous ranges) and its rows' y, r and D
// (gathers) are staged by cp.async kHeadStages - 1 levels ahead.  A lane's
// products are added in slot order and a row's lanes by the same shuffle
// tree as bwd_pack_kernel, so z is the persistent kernel's bit for bit;
// r.z over the head goes to sc->hrz for the backward kernel's reduction.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async8(void* dst, const void* src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async4(void* dst, const void* src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Byte offsets of one level's stage (head_stage_bytes with the value size of TV).
struct HeadLevel {
    int ntask, units, rows, o_idx, o_val, o_y, o_r, o_d;
};

template <typename TV>
__device__ __forceinline__ HeadLevel head_level(const int4& lo, const int4& hi) {
    HeadLevel L;
    L.ntask = hi.x - lo.x;
    L.units = hi.y - lo.y;
    L.rows = hi.z - lo.z;
    L.o_idx = 16 * L.ntask;
    L.o_val = L.o_idx + 128 * L.units;
    L.o_y = L.o_val + 32 * (int)sizeof(TV) * L.units;
    L.o_r = L.o_y + ((8 * L.rows + 15) & ~15);
    L.o_d = L.o_r + ((8 * L.rows + 15) & ~15);
    return L;
}

// Copies of level l into its stage, spread over threads tid of nthr; lv is
// the shared ring of level-table entries (entry x in slot x % kHeadLvRing).
template <typename TV>
__device__ __forceinline__ void head_issue(const SolveArgs& a, const int4* lv, const int32_t* rows_s, int l,
                                           char* buf, int tid, int nthr) {
    const int4 lo = lv[l & (kHeadLvRing - 1)], hi = lv[(l + 1) & (kHeadLvRing - 1)];
    const HeadLevel L = head_level<TV>(lo, hi);
    for (int i = tid; i < L.ntask; i += nthr) cp_async16(buf + 16 * i, a.pack_b + lo.x + i);
    const char* gi = reinterpret_cast<const char*>(a.hb_idx + (size_t)lo.y * 32);
    for (int i = tid; i < 8 * L.units; i += nthr) cp_async16(buf + L.o_idx + 16 * i, gi + 16 * i);
    const char* gv = reinterpret_cast<const char*>(a.pb_val) + (size_t)lo.y * 32 * sizeof(TV);
    for (int i = tid; i < 2 * (int)sizeof(TV) * L.units; i += nthr) cp_async16(buf + L.o_val + 16 * i, gv + 16 * i);
    const TV* dv = reinterpret_cast<const TV*>(a.diag);
    for (int i = tid; i < L.rows; i += nthr) {
        const int32_t j = rows_s[lo.z + i];
        cp_async8(buf + L.o_y + 8 * i, a.y + j);
        if (a.reduce) cp_async8(buf + L.o_r + 8 * i, a.r + j);
        if (sizeof(TV) == 4) cp_async4(buf + L.o_d + 4 * i, dv + j);
        else cp_async8(buf + L.o_d + 8 * i, dv + j);
    }
}

template <typename TV>
__global__ void __launch_bounds__(kHeadThreads, 1) bwd_head_kernel(SolveArgs a) {
    if ((a.reduce || a.seg) && ld_relaxed(&a.sc->done)) return;
    extern __shared__ __align__(16) char hsm[];
    const int R = a.hb_rows, nlev = a.hb_nlev;
    // layout of head_smem_bytes: row ids | z | level-table ring | stages
    int32_t* rows_s = reinterpret_cast<int32_t*>(hsm);
    double* zs = reinterpret_cast<double*>(hsm + ((4 * R + 15) & ~15));
    int4* lv = reinterpret_cast<int4*>(hsm + ((4 * R + 15) & ~15) + ((8 * R + 15) & ~15));
    char* ring = reinterpret_cast<char*>(lv + kHeadLvRing);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int i = tid; i < R; i += kHeadThreads) rows_s[i] = a.order_b[i];
    // entries 0 .. kHeadLvAhead - 1 now; entry l + kHeadLvAhead rides in the
    // commit group of level l, so it has landed by level l + 4 (whose issue
    // reads entries up to l + kHeadLvAhead)
    for (int i = tid; i < kHeadLvAhead && i <= nlev; i += kHeadThreads) lv[i] = a.hb_lv[i];
    __syncthreads();
    constexpr int NW = kHeadThreads / 32;
    // levels 0 .. kHeadStages - 2 in flight; one commit group per level
    for (int l = 0; l < kHeadStages - 1; ++l) {
        if (l < nlev) head_issue<TV>(a, lv, rows_s, l, ring + (size_t)l * a.hb_stage, tid, kHeadThreads);
        cp_async_commit();
    }
    double acc = 0.0;
    for (int l = 0; l < nlev; ++l) {
        // level l's copies have landed (this thread's, then everyone's), and
        // every warp is done with level l - 1, whose stage is refilled with
        // level l + kHeadStages - 1 by the warps that hold no task of level l
        // (all warps when every warp holds one)
        cp_async_wait<kHeadStages - 2>();
        __syncthreads();
        const char* buf = ring + (size_t)(l % kHeadStages) * a.hb_stage;
        const int4 lo = lv[l & (kHeadLvRing - 1)];
        const HeadLevel L = head_level<TV>(lo, lv[(l + 1) & (kHeadLvRing - 1)]);
        {
            const int lf = l + kHeadStages - 1;
            const int busy = L.ntask < NW ? L.ntask : 0;
            if (lf < nlev && warp >= busy)
                head_issue<TV>(a, lv, rows_s, lf, ring + (size_t)(lf % kHeadStages) * a.hb_stage, tid - 32 * busy,
                               kHeadThreads - 32 * busy);
            const int le = l + kHeadLvAhead;
            if (tid == kHeadThreads - 1 && le <= nlev) cp_async16(lv + (le & (kHeadLvRing - 1)), a.hb_lv + le);
            cp_async_commit();
        }
        const int4* desc = reinterpret_cast<const int4*>(buf);
        const int32_t* idx_s = reinterpret_cast<const int32_t*>(buf + L.o_idx);
        const TV* val_s = reinterpret_cast<const TV*>(buf + L.o_val);
        const double* y_s = reinterpret_cast<const double*>(buf + L.o_y);
        const double* r_s = reinterpret_cast<const double*>(buf + L.o_r);
        const TV* d_s = reinterpret_cast<const TV*>(buf + L.o_d);
        for (int ti = warp; ti < L.ntask; ti += NW) {
            const int4 d = desc[ti];
            const int cls = (d.z >> 8) & 7, cnt = d.z & 0xff, m = d.w & 0xff;
            const int G = 1 << cls;
            const int ub = d.y - lo.y;
            double sum = 0.0;
            int k = 0;
            for (; k + 4 <= m; k += 4) {  // four slots' loads in flight, added in slot order
                const int sl = (ub + k) * 32 + lane;
                const int32_t i0 = idx_s[sl], i1 = idx_s[sl + 32], i2 = idx_s[sl + 64], i3 = idx_s[sl + 96];
                const double w0 = to_d(val_s[sl]), w1 = to_d(val_s[sl + 32]), w2 = to_d(val_s[sl + 64]),
                             w3 = to_d(val_s[sl + 96]);
                const double v0 = i0 >= 0 ? zs[i0] : 0.0, v1 = i1 >= 0 ? zs[i1] : 0.0;
                const double v2 = i2 >= 0 ? zs[i2] : 0.0, v3 = i3 >= 0 ? zs[i3] : 0.0;
                sum += w0 * v0;
                sum += w1 * v1;
                sum += w2 * v2;
                sum += w3 * v3;
            }
            for (; k < m; ++k) {
                const int sl = (ub + k) * 32 + lane;
                const int32_t ix = idx_s[sl];
                const double v = ix >= 0 ? zs[ix] : 0.0;
                sum += to_d(val_s[sl]) * v;
            }
            sum = group_sum(sum, G);
            const int qrow = lane >> cls;
            if (qrow < cnt && (lane & (G - 1)) == 0) {
                const int pos = d.x + qrow;
                const int rl = pos - lo.z;
                const double dj = to_d(d_s[rl]);
                double tj = y_s[rl];
                if (dj != 0.0) tj = tj / dj;
                const double zj = tj - sum;
                zs[pos] = zj;
                a.z[rows_s[pos]] = zj;
                if (a.reduce) acc += r_s[rl] * zj;
            }
        }
    }
    cp_async_wait<0>();
    if (!a.reduce) return;
    // r.z over the head: warps in order, lanes by a fixed tree
    __shared__ double red[kHeadThreads / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(kFull, acc, o);
    if (lane == 0) red[warp] = acc;
    __syncthreads();
    if (tid == 0) {
        double t = 0.0;
        for (int w = 0; w < kHeadThreads / 32; ++w) t += red[w];
        a.sc->hrz = t;
    }
}

// ---------------------------------------------------------------------------
// true residual: t = b - A x (written to r when `replace`), ||t||^2 -> tr2
// ---------------------------------------------------------------------------
template <int K>
__global__ void __launch_bounds__(kBlock) true_residual_kernel(SolveArgs a, int replace, double* t_out) {
    constexpr int G = K;
    const int lane = threadIdx.x & 31;
    const int c = lane % G;
    const int64_t group = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / G;
    const int64_t ngroups = (int64_t)gridDim.x * blockDim.x / G;
    double acc = 0.0;
    for (int64_t i = group; i < a.n; i += ngroups) {
        const double sum = row_dot_plain<K>(a.a_idx, a.a_val, a.a_ptr[i], a.a_ptr[i + 1], a.x, c);
        const size_t o = (size_t)i * K + c;
        const double t = a.b[o] - sum;
        if (t_out) t_out[o] = t;
        if (replace) a.r[o] = t;
        acc += t * t;
    }
    block_partials_lane<K>(acc, a.part + (size_t)blockIdx.x * K);
    if (last_block(&a.sc->ticket[0])) {
        sum_partials<K>(a.part, gridDim.x, a.sc->tr2);
        if (threadIdx.x == 0) a.sc->ticket[0] = 0;
    }
}

// restart of the columns that failed the true-residual test: p = q = 0,
// y = pending, phase = 0 (the next fwd/bwd pair rebuilds z and rz)
template <int K>
__global__ void restart_kernel(SolveArgs a, const int* reactivate) {
    const int64_t total = (int64_t)a.n * K;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += stride) {
        int c = (int)(t % K);
        if (reactivate[c]) {
            a.p[t] = 0.0;
            a.q[t] = 0.0;
        }
        a.y[t] = pending_value();
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        for (int c = 0; c < K; ++c) {
            if (reactivate[c]) a.sc->active[c] = 1;
            a.sc->alpha[c] = 0.0;
        }
        a.sc->phase = 0;
        a.sc->done = 0;
    }
}

__global__ void fill_pending_kernel(double* y, int64_t total) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += stride) y[t] = pending_value();
}

__global__ void spmv_plain_kernel(int32_t n, const int32_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                                  const double* __restrict__ val, const double* __restrict__ x, double* y, int K) {
    const int64_t total = (int64_t)n * K;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += stride) {
        int64_t i = t / K;
        int c = (int)(t % K);
        double s = 0.0;
        for (int p = ptr[i]; p < ptr[i + 1]; ++p) s += val[p] * x[(size_t)idx[p] * K + c];
        y[t] = s;
    }
}

// ---- launch plumbing ------------------------------------------------------

template <int K, typename TV>
struct Kernels {
    static void* fwd() { return (void*)fwd_kernel<K, TV>; }
    static void* bwd() { return (void*)bwd_kernel<K, TV>; }
};

// The part-task counters of split rows (pcount_*) return to zero when a row
// completes.  A pass abandoned on a timeout leaves some of them part-way, so
// every solve and every preconditioner apply clears them first (a memset of
// one int per split row; no allocation).
cudaError_t clear_split_counters(const DevFactor& F, cudaStream_t s) {
    if (F.nsplit_f > 0 && F.pcount_f)
        RCHOL_TRY(cudaMemsetAsync(F.pcount_f, 0, sizeof(int32_t) * (size_t)F.nsplit_f, s));
    if (F.nsplit_b > 0 && F.pcount_b)
        RCHOL_TRY(cudaMemsetAsync(F.pcount_b, 0, sizeof(int32_t) * (size_t)F.nsplit_b, s));
    return cudaSuccess;
}

// The solve kernels deal tasks statically (warp w takes tasks w, w + nwarps,
// ...) and wait on tasks dealt to other warps, so every CTA of the grid must
// be resident at once.  A cooperative launch guarantees that or fails
// (cudaErrorCooperativeLaunchTooLarge); it never starts part of the grid
// while work on another stream holds the SMs that the rest would need.
cudaError_t launch_coresident(const void* fn, int grid, void** params, cudaStream_t s) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(kBlock);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelExC(&cfg, fn, params);
}

template <typename Arg>
cudaError_t launch_coresident(const void* fn, int grid, Arg& a, cudaStream_t s) {
    void* params[] = {&a};
    return launch_coresident(fn, grid, params, s);
}

__global__ void long_flag_kernel(int32_t n, const int32_t* __restrict__ ptr, int32_t* flag) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        flag[i] = ptr[i + 1] - ptr[i] > kLongRow ? 1 : 0;
}

__global__ void long_scatter_kernel(int32_t n, const int32_t* __restrict__ flag, const int32_t* __restrict__ pos,
                                    int32_t* rows) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        if (flag[i]) rows[pos[i]] = (int32_t)i;
}

// The factor arrays of the k > 1 solves: the multi-RHS layouts when built,
// else L's own rows and columns by row id.
void set_factor_rows(SolveArgs& a, const DevFactor& F, bool fp32) {
    a.by_pos = F.lay_ready ? 1 : 0;
    if (F.lay_ready) {
        a.lr_ptr = F.sf_ptr;
        a.lr_idx = F.sf_idx;
        a.lr_val = fp32 ? (const void*)F.sf_val32 : (const void*)F.sf_val;
        a.lc_ptr = F.sb_ptr;
        a.lc_idx = F.sb_idx;
        a.lc_val = fp32 ? (const void*)F.sb_val32 : (const void*)F.sb_val;
    } else {
        a.lr_ptr = F.lr_ptr;
        a.lr_idx = F.lr_idx;
        a.lr_val = fp32 ? (const void*)F.lr_val32 : (const void*)F.lr_val;
        a.lc_ptr = F.lc_ptr;
        a.lc_idx = F.lc_idx;
        a.lc_val = fp32 ? (const void*)F.lc_val32 : (const void*)F.lc_val;
    }
}

int resident_blocks(const void* fn, int device) {
    int per_sm = 0, sms = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kBlock, 0);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    return per_sm * sms;
}

}  // namespace

// ===========================================================================

class PcgSolver {
   public:
    DevCsc A;
    DevFactor F;
    DevSell S;  // sliced-ELL copy of A (empty: CSR SpMV)
    SolveConfig cfg;
    int device = 0;
    cudaStream_t stream = nullptr;
    int K = 1;
    double *r = nullptr, *p = nullptr, *q = nullptr, *y = nullptr, *z = nullptr;
    double* part = nullptr;
    int grid_max = 0;
    int grid_spmv = 0, grid_fwd = 0, grid_bwd = 0, grid_vec = 0;
    PcgScalars* sc = nullptr;
    PcgScalars* sc_host = nullptr;  // pinned
    int* react = nullptr;          // device [kMaxK]
    cudaGraphExec_t graph_exec = nullptr;
    SolveArgs graph_args;  // the arguments the graph was captured with
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, ev2 = nullptr;
    void *k_init = nullptr, *k_spmv = nullptr, *k_fwd = nullptr, *k_bwd = nullptr, *k_true = nullptr,
         *k_restart = nullptr;
    void* k_head = nullptr;  // backward head (K = 1)
    void* k_long = nullptr;  // long rows of the SpMV
    // long rows of the one-RHS CSR SpMV (spmv_long_kernel)
    int32_t* lrows = nullptr;
    double* lr_dot = nullptr;
    int32_t n_lrows = 0;
    int64_t cap_lrows = 0;
    int32_t *lflag = nullptr, *lpos = nullptr;  // [n], [n + 1]
    void* ltmp = nullptr;                       // scan scratch

    bool use_head() const { return k_head && F.hb_nlev > 0; }

    // The rows of A longer than kLongRow, ascending: the SpMV gives each its
    // own CTA (the sliced-ELL copy leaves them out).
    cudaError_t find_long_rows() {
        n_lrows = 0;
        if (A.n == 0) return cudaSuccess;
        const int32_t n = A.n;
        // the solver's matrix order is fixed, so these are allocated once
        cudaError_t e = cudaSuccess;
        if (!lflag) e = cudaMalloc(&lflag, sizeof(int32_t) * (size_t)n);
        if (e == cudaSuccess && !lpos) e = cudaMalloc(&lpos, sizeof(int32_t) * ((size_t)n + 1));
        if (e == cudaSuccess && !ltmp) e = cudaMalloc(&ltmp, scan_tmp_bytes(n));
        int32_t *flag = lflag, *pos = lpos;
        void* tmp = ltmp;
        if (e == cudaSuccess) {
            long_flag_kernel<<<grid_for(n, kBlock), kBlock, 0, stream>>>(n, A.colptr, flag);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = exclusive_scan_i32_to_i32(flag, pos, n, tmp, stream);
        int32_t cnt = 0;
        if (e == cudaSuccess) e = cudaMemcpyAsync(&cnt, pos + n, sizeof(int32_t), cudaMemcpyDeviceToHost, stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
        if (e == cudaSuccess && cnt > 0) {
            if (cap_lrows < cnt) {
                cudaFree(lrows);
                cudaFree(lr_dot);
                lrows = nullptr;
                lr_dot = nullptr;
                cap_lrows = 0;
                e = cudaMalloc(&lrows, sizeof(int32_t) * (size_t)cnt);
                if (e == cudaSuccess) e = cudaMalloc(&lr_dot, sizeof(double) * ((size_t)cnt * K + 1));
                if (e == cudaSuccess) cap_lrows = cnt;
            }
            if (e == cudaSuccess) {
                long_scatter_kernel<<<grid_for(n, kBlock), kBlock, 0, stream>>>(n, flag, pos, lrows);
                e = cudaGetLastError();
            }
            if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
            if (e == cudaSuccess) n_lrows = cnt;
        }
        return e;
    }

    SolveArgs args(const double* b, double* x) const {
        SolveArgs a;
        memset(&a, 0, sizeof(a));
        a.n = A.n;
        a.a_ptr = A.colptr;
        a.a_idx = A.rowind;
        a.a_val = A.val;
        a.s_ptr = S.sptr;
        a.s_idx = S.sidx;
        a.s_val = S.sval;
        set_factor_rows(a, F, cfg.fp32_factor);
        a.diag = cfg.fp32_factor ? (const void*)F.diag32 : (const void*)F.diag;
        a.order_f = F.order_f;
        a.order_b = F.order_b;
        a.pack_f = F.pack_f;
        a.pack_b = F.pack_b;
        a.pf_idx = F.pf_idx;
        a.pf_val = cfg.fp32_factor ? (const void*)F.pf_val32 : (const void*)F.pf_val;
        a.pb_idx = F.pb_idx;
        a.pb_val = cfg.fp32_factor ? (const void*)F.pb_val32 : (const void*)F.pb_val;
        a.ntasks_f = F.npt_f;
        a.ntasks_b = F.npt_b;
        a.split_f = F.split_f;
        a.split_b = F.split_b;
        a.psum_f = F.psum_f;
        a.psum_b = F.psum_b;
        a.pcount_f = F.pcount_f;
        a.pcount_b = F.pcount_b;
        a.srow_b = F.srow_b;
        a.nsplit_b = F.nsplit_b;
        a.lrows = lrows;
        a.lr_dot = lr_dot;
        a.n_lrows = n_lrows;
        if (use_head()) {
            a.hb_lv = F.hb_lv;
            a.hb_idx = F.hb_idx;
            a.hb_nlev = F.hb_nlev;
            a.hb_ntask = F.hb_ntask;
            a.hb_rows = F.hb_rows;
            a.hb_stage = F.hb_stage;
        }
        a.b = b;
        a.x = x;
        a.r = r;
        a.p = p;
        a.q = q;
        a.y = y;
        a.z = z;
        a.part = part;
        a.grid_max = grid_max;
        a.sc = sc;
        a.tol = cfg.tol;
        a.max_iter = cfg.max_iter;
        a.stop_rule = cfg.stop_rule;
        a.update = 1;
        a.reduce = 1;
        a.poll_ns = cfg.poll_ns;
        a.timeout_ns = (unsigned long long)(cfg.timeout_s * 1e9);
        a.seg = nullptr;
        a.seg_alpha = nullptr;
        return a;
    }

    cudaError_t launch(void* fn, int grid, SolveArgs& a) {
        void* params[] = {&a};
        if (fn == k_fwd || fn == k_bwd) return launch_coresident(fn, grid, params, stream);
        return cudaLaunchKernel(fn, dim3(grid), dim3(kBlock), params, 0, stream);
    }

    // z = L^-T D^+ y: the backward head (one CTA) first, then the rest
    cudaError_t launch_bwd(SolveArgs& a) {
        if (a.hb_nlev > 0) {
            void* params[] = {&a};
            const size_t smem = (size_t)head_smem_bytes(a.hb_rows, a.hb_stage);
            cudaError_t e = cudaLaunchKernel(k_head, dim3(1), dim3(kHeadThreads), params, smem, stream);
            if (e != cudaSuccess) return e;
        }
        return launch(k_bwd, grid_bwd, a);
    }

    // q = A z + beta q, p = z + beta p, p.q (the long rows' CTAs first)
    cudaError_t launch_spmv(SolveArgs& a) {
        if (a.n_lrows > 0) {
            void* params[] = {&a};
            cudaError_t e = cudaLaunchKernel(k_long, dim3(a.n_lrows), dim3(kBlock), params, 0, stream);
            if (e != cudaSuccess) return e;
        }
        return launch(k_spmv, grid_spmv, a);
    }

    cudaError_t launch_iteration(const double* b, double* x) {
        SolveArgs a = args(b, x);
        cudaError_t e;
        if ((e = launch_spmv(a)) != cudaSuccess) return e;
        if ((e = launch(k_fwd, grid_fwd, a)) != cudaSuccess) return e;
        return launch_bwd(a);
    }

    // fwd (no update) + bwd with phase 0: z = M r, rz = rz0 = r.z
    cudaError_t launch_start(const double* b, double* x) {
        SolveArgs a = args(b, x);
        a.update = 0;
        a.reduce = 1;
        cudaError_t e;
        // fwd with reduce=1 but update=0: no x/r change, no rr test
        if ((e = launch(k_fwd, grid_fwd, a)) != cudaSuccess) return e;
        return launch_bwd(a);
    }
};

template <int K, typename TV>
static void bind_kernels(PcgSolver* s) {
    s->k_init = (void*)init_kernel<K>;
    s->k_spmv = K == 1 ? (void*)spmv_update_tile_kernel : (void*)spmv_update_kernel<K>;
    s->k_fwd = K == 1 ? (void*)fwd_pack_kernel<TV> : (void*)fwd_kernel<K, TV>;
    s->k_bwd = K == 1 ? (void*)bwd_pack_kernel<TV> : (void*)bwd_kernel<K, TV>;
    s->k_true = (void*)true_residual_kernel<K>;
    s->k_restart = (void*)restart_kernel<K>;
    s->k_head = K == 1 ? (void*)bwd_head_kernel<TV> : nullptr;
    s->k_long = K == 1 ? (void*)spmv_long_kernel : (void*)spmv_long_k_kernel<K>;
}

template <typename TV>
static bool bind_for_k(PcgSolver* s, int K) {
    switch (K) {
        case 1: bind_kernels<1, TV>(s); return true;
        case 2: bind_kernels<2, TV>(s); return true;
        case 4: bind_kernels<4, TV>(s); return true;
        case 8: bind_kernels<8, TV>(s); return true;
        case 16: bind_kernels<16, TV>(s); return true;
        case 32: bind_kernels<32, TV>(s); return true;
        default: return false;
    }
}

PcgSolver* pcg_create(const DevCsc& A, const DevFactor& F, const SolveConfig& cfg, int device, cudaStream_t stream,
                      cudaError_t* err, const DevSell* sell) {
    *err = cudaSuccess;
    if (A.n != F.n) {
        *err = cudaErrorInvalidValue;
        return nullptr;
    }
    PcgSolver* s = new PcgSolver();
    s->A = A;
    s->F = F;
    s->cfg = cfg;
    s->device = device;
    s->stream = stream;
    s->K = cfg.k;
    bool okk = cfg.fp32_factor ? bind_for_k<float>(s, cfg.k) : bind_for_k<double>(s, cfg.k);
    if (!okk || (cfg.fp32_factor && !F.lr_val32)) {
        delete s;
        *err = cudaErrorInvalidValue;
        return nullptr;
    }
    bool sell_spmv = false;
    if (cfg.k == 1 && sell && sell->slots > 0 && sell->n == A.n) {
        s->S = *sell;
        s->k_spmv = (void*)spmv_update_sell_kernel;
        sell_spmv = true;
    }
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    s->grid_fwd = resident_blocks(s->k_fwd, device);
    s->grid_bwd = resident_blocks(s->k_bwd, device);
    s->grid_spmv = sell_spmv ? resident_blocks(s->k_spmv, device) : sms * 8;
    s->grid_vec = sms * 8;
    s->grid_max = std::max(std::max(s->grid_fwd, s->grid_bwd), std::max(s->grid_spmv, s->grid_vec));
    const size_t nv = (size_t)A.n * (size_t)cfg.k;
    cudaError_t e = cudaSuccess;
    if (s->k_head) e = cudaFuncSetAttribute(s->k_head, cudaFuncAttributeMaxDynamicSharedMemorySize, kHeadSmem);
    if (e == cudaSuccess) e = cudaMalloc(&s->r, sizeof(double) * std::max<size_t>(nv, 1));
    if (e == cudaSuccess) e = cudaMalloc(&s->p, sizeof(double) * std::max<size_t>(nv, 1));
    if (e == cudaSuccess) e = cudaMalloc(&s->q, sizeof(double) * std::max<size_t>(nv, 1));
    if (e == cudaSuccess) e = cudaMalloc(&s->y, sizeof(double) * std::max<size_t>(nv, 1));
    if (e == cudaSuccess) e = cudaMalloc(&s->z, sizeof(double) * std::max<size_t>(nv, 1));
    if (e == cudaSuccess) e = cudaMalloc(&s->part, sizeof(double) * (size_t)3 * s->grid_max * cfg.k);
    if (e == cudaSuccess) e = cudaMalloc(&s->sc, sizeof(PcgScalars));
    if (e == cudaSuccess) e = cudaMemset(s->sc, 0, sizeof(PcgScalars));
    if (e == cudaSuccess) e = cudaMallocHost(&s->sc_host, sizeof(PcgScalars));
    if (e == cudaSuccess) e = cudaMalloc(&s->react, sizeof(int) * kMaxK);
    if (e == cudaSuccess) e = cudaEventCreate(&s->ev0);
    if (e == cudaSuccess) e = cudaEventCreate(&s->ev1);
    if (e == cudaSuccess) e = cudaEventCreate(&s->ev2);
    if (e == cudaSuccess) e = s->find_long_rows();
    if (e != cudaSuccess || s->grid_fwd <= 0 || s->grid_bwd <= 0) {
        *err = e != cudaSuccess ? e : cudaErrorLaunchOutOfResources;
        pcg_destroy(s);
        return nullptr;
    }
    return s;
}

cudaError_t pcg_rebind(PcgSolver* s, const DevCsc& A, const DevSell* sell, const DevFactor& F, bool new_matrix) {
    const bool want_sell = s->K == 1 && sell && sell->slots > 0 && sell->n == A.n;
    const bool has_sell = s->k_spmv == (void*)spmv_update_sell_kernel;
    if (A.n != s->A.n || F.n != A.n || want_sell != has_sell || (s->cfg.fp32_factor && !F.lr_val32))
        return cudaErrorInvalidValue;
    s->A = A;
    s->S = want_sell ? *sell : DevSell();
    s->F = F;
    return new_matrix ? s->find_long_rows() : cudaSuccess;
}

void pcg_destroy(PcgSolver* s) {
    if (!s) return;
    if (s->graph_exec) cudaGraphExecDestroy(s->graph_exec);
    cudaFree(s->r);
    cudaFree(s->p);
    cudaFree(s->q);
    cudaFree(s->y);
    cudaFree(s->z);
    cudaFree(s->part);
    cudaFree(s->sc);
    cudaFree(s->react);
    cudaFree(s->lrows);
    cudaFree(s->lr_dot);
    cudaFree(s->lflag);
    cudaFree(s->lpos);
    cudaFree(s->ltmp);
    if (s->sc_host) cudaFreeHost(s->sc_host);
    if (s->ev0) cudaEventDestroy(s->ev0);
    if (s->ev1) cudaEventDestroy(s->ev1);
    if (s->ev2) cudaEventDestroy(s->ev2);
    delete s;
}

static cudaError_t build_graph(PcgSolver* s, const double* b, double* x) {
    const SolveArgs want = s->args(b, x);  // zero-filled, so padding compares equal
    if (s->graph_exec && memcmp(&want, &s->graph_args, sizeof(want)) == 0) return cudaSuccess;
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return e;
    for (int u = 0; u < s->cfg.unroll; ++u) {
        e = s->launch_iteration(b, x);
        if (e != cudaSuccess) break;
    }
    cudaError_t e2 = cudaStreamEndCapture(s->stream, &g);
    if (e != cudaSuccess || e2 != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        return e != cudaSuccess ? e : e2;
    }
    // same launch sequence with new arguments (another factor or vectors):
    // update the instantiated graph in place, else instantiate anew
    if (s->graph_exec) {
        cudaGraphExecUpdateResultInfo info;
        if (cudaGraphExecUpdate(s->graph_exec, g, &info) != cudaSuccess) {
            cudaGetLastError();
            cudaGraphExecDestroy(s->graph_exec);
            s->graph_exec = nullptr;
        }
    }
    if (!s->graph_exec) e = cudaGraphInstantiate(&s->graph_exec, g, 0);
    cudaGraphDestroy(g);
    if (e == cudaSuccess) memcpy(&s->graph_args, &want, sizeof(want));
    return e;
}

cudaError_t pcg_solve(PcgSolver* s, const double* dB, double* dX, SolveResult* res) {
    *res = SolveResult();
    const int K = s->K;
    cudaError_t e;
    if (s->cfg.use_graph && (e = build_graph(s, dB, dX)) != cudaSuccess) return e;
    e = cudaEventRecord(s->ev0, s->stream);
    if (e != cudaSuccess) return e;
    if ((e = clear_split_counters(s->F, s->stream)) != cudaSuccess) return e;
    SolveArgs a = s->args(dB, dX);
    if ((e = s->launch(s->k_init, s->grid_vec, a)) != cudaSuccess) return e;
    if ((e = s->launch_start(dB, dX)) != cudaSuccess) return e;
    // per iteration: SpMV, forward, backward (+ the backward head)
    const int per_it = 3 + (s->use_head() ? 1 : 0) + (s->n_lrows > 0 ? 1 : 0);
    res->kernel_launches += per_it;
    if ((e = cudaEventRecord(s->ev1, s->stream)) != cudaSuccess) return e;
    int restarts = 0;
    while (true) {
        // iterate until the device says stop
        while (true) {
            if (s->cfg.use_graph) {
                if ((e = cudaGraphLaunch(s->graph_exec, s->stream)) != cudaSuccess) return e;
                res->graph_launches++;
                res->kernel_launches += per_it * s->cfg.unroll;
            } else {
                for (int u = 0; u < s->cfg.unroll; ++u)
                    if ((e = s->launch_iteration(dB, dX)) != cudaSuccess) return e;
                res->kernel_launches += per_it * s->cfg.unroll;
            }
            if ((e = cudaMemcpyAsync(s->sc_host, s->sc, sizeof(PcgScalars), cudaMemcpyDeviceToHost, s->stream)) !=
                cudaSuccess)
                return e;
            if ((e = cudaStreamSynchronize(s->stream)) != cudaSuccess) return e;
            if (s->sc_host->done) break;
        }
        // confirm on the true residual b - A x
        SolveArgs t = s->args(dB, dX);
        void* params[] = {&t, nullptr, nullptr};
        int replace = 0;
        double* tout = nullptr;
        params[1] = &replace;
        params[2] = &tout;
        if ((e = cudaLaunchKernel(s->k_true, dim3(s->grid_vec), dim3(kBlock), params, 0, s->stream)) != cudaSuccess)
            return e;
        res->kernel_launches++;
        if ((e = cudaMemcpyAsync(s->sc_host, s->sc, sizeof(PcgScalars), cudaMemcpyDeviceToHost, s->stream)) !=
            cudaSuccess)
            return e;
        if ((e = cudaStreamSynchronize(s->stream)) != cudaSuccess) return e;
        const PcgScalars& h = *s->sc_host;
        if (h.status != 0 || s->cfg.stop_rule != 0 || h.iter >= s->cfg.max_iter || restarts >= 3) break;
        int react[kMaxK] = {0};
        int any = 0;
        for (int c = 0; c < K; ++c) {
            double bn = std::sqrt(h.bnorm2[c]);
            if (bn > 0 && std::sqrt(h.tr2[c]) > s->cfg.tol * bn) {
                react[c] = 1;
                any = 1;
            }
        }
        if (!any) break;
        // residual replacement and restart for the failing columns
        ++restarts;
        replace = 1;
        if ((e = cudaMemcpyAsync(s->react, react, sizeof(react), cudaMemcpyHostToDevice, s->stream)) != cudaSuccess)
            return e;
        if ((e = cudaLaunchKernel(s->k_true, dim3(s->grid_vec), dim3(kBlock), params, 0, s->stream)) != cudaSuccess)
            return e;
        SolveArgs ra = s->args(dB, dX);
        void* rparams[] = {&ra, &s->react};
        if ((e = cudaLaunchKernel(s->k_restart, dim3(s->grid_vec), dim3(kBlock), rparams, 0, s->stream)) !=
            cudaSuccess)
            return e;
        if ((e = s->launch_start(dB, dX)) != cudaSuccess) return e;
        res->kernel_launches += per_it + 1;
    }
    if ((e = cudaEventRecord(s->ev2, s->stream)) != cudaSuccess) return e;
    if ((e = cudaEventSynchronize(s->ev2)) != cudaSuccess) return e;
    cudaEventElapsedTime(&res->ms_total, s->ev0, s->ev2);
    cudaEventElapsedTime(&res->ms_iterations, s->ev1, s->ev2);
    const PcgScalars& h = *s->sc_host;
    res->status = h.status;
    res->iterations = 0;
    res->converged = 1;
    for (int c = 0; c < K; ++c) {
        res->iterations = std::max(res->iterations, h.iters[c]);
        double bn = std::sqrt(h.bnorm2[c]);
        double tr = bn > 0 ? std::sqrt(h.tr2[c]) / bn : 0.0;
        double rr = bn > 0 ? std::sqrt(h.rr[c]) / bn : 0.0;
        res->relres_true = std::max(res->relres_true, tr);
        res->relres_rec = std::max(res->relres_rec, rr);
        double pr = h.rz0[c] > 0 ? std::sqrt(h.rz[c] / h.rz0[c]) : 0.0;
        res->precond_ratio = std::max(res->precond_ratio, pr);
        bool conv;
        if (s->cfg.stop_rule == 0) conv = tr <= s->cfg.tol;
        else conv = !h.active[c];
        if (!conv) res->converged = 0;
    }
    if (h.status != 0) res->converged = 0;
    return cudaSuccess;
}

// Per-kernel device time of the iteration kernels: starts a solve of dB
// (tolerance 0, so nothing converges), then times `reps` iterations with an
// event between every launch.  ms_out[0..2] = mean spmv_update, fwd, bwd.
cudaError_t pcg_profile(PcgSolver* s, const double* dB, double* dX, int reps, float* ms_out) {
    SolveConfig keep = s->cfg;
    s->cfg.tol = 0.0;
    s->cfg.max_iter = 1 << 30;
    SolveArgs a = s->args(dB, dX);
    cudaError_t e;
    if ((e = clear_split_counters(s->F, s->stream)) != cudaSuccess) return e;
    if ((e = s->launch(s->k_init, s->grid_vec, a)) != cudaSuccess) return e;
    if ((e = s->launch_start(dB, dX)) != cudaSuccess) return e;
    cudaEvent_t ev[4];
    for (auto& x : ev) cudaEventCreate(&x);
    double acc[3] = {0, 0, 0};
    for (int r = 0; r < reps && e == cudaSuccess; ++r) {
        SolveArgs it = s->args(dB, dX);
        cudaEventRecord(ev[0], s->stream);
        e = s->launch_spmv(it);
        cudaEventRecord(ev[1], s->stream);
        if (e == cudaSuccess) e = s->launch(s->k_fwd, s->grid_fwd, it);
        cudaEventRecord(ev[2], s->stream);
        if (e == cudaSuccess) e = s->launch_bwd(it);
        cudaEventRecord(ev[3], s->stream);
        cudaEventSynchronize(ev[3]);
        float m;
        for (int q = 0; q < 3; ++q) {
            cudaEventElapsedTime(&m, ev[q], ev[q + 1]);
            acc[q] += m;
        }
    }
    for (auto& x : ev) cudaEventDestroy(x);
    for (int q = 0; q < 3; ++q) ms_out[q] = (float)(acc[q] / std::max(reps, 1));
    s->cfg = keep;
    return e;
}


// ===========================================================================
// Batched independent systems (block-diagonal matrix, one PCG per system and
// right-hand side).  Rows are grouped by system; the dot products reduce
// over fixed row chunks (a chunk spans at most two systems) and then over
// the chunks of each system in order, so the sums are deterministic.
// One iteration: batch_spmv (q, p, p.q -> alpha per pair), fwd (x, r, y),
// bwd (z), batch_dots (r.r, r.z -> convergence, beta per pair).
// ===========================================================================

struct BatchScalarsDev {
    double *alpha, *beta, *rz, *rz0, *rr, *pq, *bnorm2, *tr2, *rzn;
    int *active, *iters;
};

struct BatchArgs {
    int32_t n;
    int32_t nsys;
    int32_t chunk;           // rows per reduction chunk
    int32_t nchunks;
    const int32_t* __restrict__ seg;          // row -> system
    const int64_t* __restrict__ sys_off;      // [nsys+1]
    const int32_t* __restrict__ a_ptr;
    const int32_t* __restrict__ a_idx;
    const double* __restrict__ a_val;
    const double* __restrict__ b;
    double *x, *r, *p, *q, *y, *z;
    double* part;            // [nchunks][2 slots][K]
    BatchScalarsDev s;
    PcgScalars* sc;          // global flags: done, iter, phase, status, tickets
    double tol;
    int max_iter;
    int stop_rule;
};

// Per-chunk, per-column sums of (va for the chunk's first system, vb for
// the second); thread column = lane % K.  Deterministic block reduction.
template <int K>
__device__ void chunk_store(double va, double vb, double* out /* [2][K] */) {
    __shared__ double red[2][kBlock / 32][K];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o >= K; o >>= 1) {
        va += __shfl_xor_sync(kFull, va, o);
        vb += __shfl_xor_sync(kFull, vb, o);
    }
    if (lane < K) {
        red[0][w][lane] = va;
        red[1][w][lane] = vb;
    }
    __syncthreads();
    if (threadIdx.x < 2 * K) {
        const int slot = threadIdx.x / K, c = threadIdx.x % K;
        double t = 0.0;
        for (int i = 0; i < kBlock / 32; ++i) t += red[slot][i][c];
        out[slot * K + c] = t;
    }
    __syncthreads();
}

// Sum of the chunk partials of every (system, column) pair into out[pair]:
// one warp per pair, lanes over the system's chunks, fixed tree.
template <int K>
__device__ void reduce_pairs(const BatchArgs& a, const double* part, double* out) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int pairs = a.nsys * K;
    for (int pr = w; pr < pairs; pr += kBlock / 32) {
        const int sys = pr / K, c = pr % K;
        const int64_t r0 = a.sys_off[sys], r1 = a.sys_off[sys + 1];
        double t = 0.0;
        if (r1 > r0) {
            const int64_t c0 = r0 / a.chunk, c1 = (r1 - 1) / a.chunk;
            for (int64_t ch = c0 + lane; ch <= c1; ch += 32) {
                const int slot = a.seg[ch * a.chunk] == sys ? 0 : 1;
                t += part[(size_t)ch * 2 * K + slot * K + c];
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(kFull, t, o);
        if (lane == 0) out[pr] = t;
    }
    __syncthreads();
}

// Row loop of one chunk: fn(row, column) returns the row's contribution.
template <int K, typename F>
__device__ void chunk_rows(const BatchArgs& a, int64_t ch, F fn, double& va, double& vb) {
    const int64_t r0 = ch * a.chunk;
    const int64_t r1 = min((int64_t)a.n, r0 + a.chunk);
    const int first = a.seg[r0];
    const int c = threadIdx.x % K;
    for (int64_t i = r0 + threadIdx.x / K; i < r1; i += kBlock / K) {
        const double v = fn(i, c);
        if (a.seg[i] == first) va += v;
        else vb += v;
    }
}

template <int K>
__global__ void __launch_bounds__(kBlock) batch_init_kernel(BatchArgs a) {
    for (int64_t ch = blockIdx.x; ch < a.nchunks; ch += gridDim.x) {
        double va = 0.0, vb = 0.0;
        chunk_rows<K>(a, ch, [&](int64_t i, int c) {
            const size_t o = (size_t)i * K + c;
            const double bv = a.b[o];
            a.x[o] = 0.0;
            a.r[o] = bv;
            a.p[o] = 0.0;
            a.q[o] = 0.0;
            a.y[o] = pending_value();
            return bv * bv;
        }, va, vb);
        chunk_store<K>(va, vb, a.part + (size_t)ch * 2 * K);
    }
    if (last_block(&a.sc->ticket[0])) {
        reduce_pairs<K>(a, a.part, a.s.bnorm2);
        for (int pr = threadIdx.x; pr < a.nsys * K; pr += kBlock) {
            a.s.alpha[pr] = 0.0;
            a.s.beta[pr] = 0.0;
            a.s.rz[pr] = 0.0;
            a.s.active[pr] = a.s.bnorm2[pr] > 0.0 ? 1 : 0;
            a.s.iters[pr] = 0;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            int any = 0;
            for (int pr = 0; pr < a.nsys * K; ++pr) any |= a.s.active[pr];
            a.sc->done = any ? 0 : 1;
            a.sc->iter = 0;
            a.sc->phase = 0;
            a.sc->status = 0;
            a.sc->ticket[0] = 0;
        }
    }
}

template <int K>
__global__ void __launch_bounds__(kBlock) batch_spmv_kernel(BatchArgs a) {
    if (ld_relaxed(&a.sc->done)) return;
    for (int64_t ch = blockIdx.x; ch < a.nchunks; ch += gridDim.x) {
        double va = 0.0, vb = 0.0;
        chunk_rows<K>(a, ch, [&](int64_t i, int c) {
            const double beta = a.s.beta[(size_t)a.seg[i] * K + c];
            const double sum = row_dot_plain<K>(a.a_idx, a.a_val, a.a_ptr[i], a.a_ptr[i + 1], a.z, c);
            const size_t o = (size_t)i * K + c;
            const double qi = sum + beta * a.q[o];
            const double pi = a.z[o] + beta * a.p[o];
            a.q[o] = qi;
            a.p[o] = pi;
            a.y[o] = pending_value();
            return pi * qi;
        }, va, vb);
        chunk_store<K>(va, vb, a.part + (size_t)ch * 2 * K);
    }
    if (last_block(&a.sc->ticket[1])) {
        reduce_pairs<K>(a, a.part, a.s.pq);
        for (int pr = threadIdx.x; pr < a.nsys * K; pr += kBlock) {
            const double pq = a.s.pq[pr];
            a.s.alpha[pr] = (a.s.active[pr] && pq != 0.0) ? a.s.rz[pr] / pq : 0.0;
        }
        if (threadIdx.x == 0) a.sc->ticket[1] = 0;
    }
}

// r.r and r.z per pair; phase 0 initialises rz, otherwise beta, the stop
// test and the iteration count.
template <int K>
__global__ void __launch_bounds__(kBlock) batch_dots_kernel(BatchArgs a) {
    if (ld_relaxed(&a.sc->done)) return;
    double* part_rr = a.part;
    double* part_rz = a.part + (size_t)a.nchunks * 2 * K;
    for (int64_t ch = blockIdx.x; ch < a.nchunks; ch += gridDim.x) {
        double va = 0.0, vb = 0.0, wa = 0.0, wb = 0.0;
        const int64_t r0 = ch * a.chunk;
        const int64_t r1 = min((int64_t)a.n, r0 + a.chunk);
        const int first = a.seg[r0];
        const int c = threadIdx.x % K;
        for (int64_t i = r0 + threadIdx.x / K; i < r1; i += kBlock / K) {
            const size_t o = (size_t)i * K + c;
            const double ri = a.r[o], zi = a.z[o];
            if (a.seg[i] == first) {
                va += ri * ri;
                wa += ri * zi;
            } else {
                vb += ri * ri;
                wb += ri * zi;
            }
        }
        chunk_store<K>(va, vb, part_rr + (size_t)ch * 2 * K);
        chunk_store<K>(wa, wb, part_rz + (size_t)ch * 2 * K);
    }
    if (last_block(&a.sc->ticket[3])) {
        reduce_pairs<K>(a, part_rr, a.s.rr);
        reduce_pairs<K>(a, part_rz, a.s.rzn);
        const bool init = a.sc->phase == 0;
        const int it = init ? a.sc->iter : a.sc->iter + 1;
        for (int pr = threadIdx.x; pr < a.nsys * K; pr += kBlock) {
            if (!a.s.active[pr]) {
                a.s.beta[pr] = 0.0;
                continue;
            }
            const double rn = a.s.rzn[pr];
            if (init) {
                a.s.rz[pr] = rn;
                a.s.rz0[pr] = rn;
                a.s.beta[pr] = 0.0;
                continue;
            }
            a.s.iters[pr] = it;
            bool conv = false;
            if (a.stop_rule == 0) conv = sqrt(a.s.rr[pr]) <= a.tol * sqrt(a.s.bnorm2[pr]);
            else if (a.stop_rule == 2) conv = a.s.rr[pr] <= a.tol;
            else conv = !(sqrt(rn) / sqrt(a.s.rz0[pr]) > a.tol);
            const double ro = a.s.rz[pr];
            a.s.beta[pr] = ro != 0.0 ? rn / ro : 0.0;
            a.s.rz[pr] = rn;
            if (conv) a.s.active[pr] = 0;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            int any = 0;
            for (int pr = 0; pr < a.nsys * K; ++pr) any |= a.s.active[pr];
            a.sc->iter = it;
            a.sc->phase = 1;
            if (!any || it >= a.max_iter) a.sc->done = 1;
            a.sc->ticket[3] = 0;
        }
    }
}

template <int K>
__global__ void __launch_bounds__(kBlock) batch_true_kernel(BatchArgs a) {
    for (int64_t ch = blockIdx.x; ch < a.nchunks; ch += gridDim.x) {
        double va = 0.0, vb = 0.0;
        chunk_rows<K>(a, ch, [&](int64_t i, int c) {
            const double sum = row_dot_plain<K>(a.a_idx, a.a_val, a.a_ptr[i], a.a_ptr[i + 1], a.x, c);
            const double t = a.b[(size_t)i * K + c] - sum;
            return t * t;
        }, va, vb);
        chunk_store<K>(va, vb, a.part + (size_t)ch * 2 * K);
    }
    if (last_block(&a.sc->ticket[0])) {
        reduce_pairs<K>(a, a.part, a.s.tr2);
        if (threadIdx.x == 0) a.sc->ticket[0] = 0;
    }
}

class BatchSolver {
   public:
    PcgSolver* base = nullptr;       // vectors, factor kernels, scalars struct
    BatchArgs ba;
    int32_t* seg = nullptr;
    int64_t* off = nullptr;
    double* pool = nullptr;          // per-pair scalars
    int* ipool = nullptr;
    double* part = nullptr;
    int grid = 0;
    void *k_init = nullptr, *k_spmv = nullptr, *k_dots = nullptr, *k_true = nullptr;
    cudaGraphExec_t graph = nullptr;
    const double* gb = nullptr;
    double* gx = nullptr;
    std::vector<double> h_tr2, h_b2;
    std::vector<int> h_iters;

    BatchArgs args(const double* b, double* x) {
        BatchArgs a = ba;
        a.b = b;
        a.x = x;
        return a;
    }
    SolveArgs solve_args(const double* b, double* x) {
        SolveArgs a = base->args(b, x);
        // the batched iteration launches no backward head: every task runs
        // in the persistent kernel
        a.hb_lv = nullptr;
        a.hb_idx = nullptr;
        a.hb_nlev = a.hb_ntask = a.hb_rows = a.hb_stage = 0;
        a.lrows = nullptr;
        a.lr_dot = nullptr;
        a.n_lrows = 0;
        a.reduce = 0;
        a.update = 1;
        a.seg = seg;
        a.seg_alpha = ba.s.alpha;
        return a;
    }
    cudaError_t launch(void* fn, int g, void* arg) {
        void* params[] = {arg};
        if (fn == base->k_fwd || fn == base->k_bwd) return launch_coresident(fn, g, params, base->stream);
        return cudaLaunchKernel(fn, dim3(g), dim3(kBlock), params, 0, base->stream);
    }
    cudaError_t iteration(const double* b, double* x) {
        BatchArgs a = args(b, x);
        SolveArgs sa = solve_args(b, x);
        cudaError_t e;
        if ((e = launch(k_spmv, grid, &a)) != cudaSuccess) return e;
        if ((e = launch(base->k_fwd, base->grid_fwd, &sa)) != cudaSuccess) return e;
        if ((e = launch(base->k_bwd, base->grid_bwd, &sa)) != cudaSuccess) return e;
        return launch(k_dots, grid, &a);
    }
};

template <int K>
static void bind_batch(BatchSolver* s) {
    s->k_init = (void*)batch_init_kernel<K>;
    s->k_spmv = (void*)batch_spmv_kernel<K>;
    s->k_dots = (void*)batch_dots_kernel<K>;
    s->k_true = (void*)batch_true_kernel<K>;
}

BatchSolver* batch_create(const DevCsc& A, const DevFactor& F, const SolveConfig& cfg, int device,
                          cudaStream_t stream, const int64_t* h_off, int nsys, cudaError_t* err) {
    *err = cudaSuccess;
    // the smallest system bounds the chunk (a chunk must span <= 2 systems)
    int64_t minsys = INT64_MAX;
    for (int i = 0; i < nsys; ++i) minsys = std::min(minsys, h_off[i + 1] - h_off[i]);
    if (nsys < 1 || minsys < 32 || h_off[nsys] != A.n) {
        *err = cudaErrorInvalidValue;
        return nullptr;
    }
    PcgSolver* base = pcg_create(A, F, cfg, device, stream, err);
    if (!base) return nullptr;
    BatchSolver* s = new BatchSolver();
    s->base = base;
    switch (cfg.k) {
        case 1: bind_batch<1>(s); break;
        case 2: bind_batch<2>(s); break;
        case 4: bind_batch<4>(s); break;
        case 8: bind_batch<8>(s); break;
        case 16: bind_batch<16>(s); break;
        case 32: bind_batch<32>(s); break;
        default: *err = cudaErrorInvalidValue; batch_destroy(s); return nullptr;
    }
    int64_t chunk = 32;
    while (chunk * 2 <= std::min<int64_t>(minsys, 4096)) chunk *= 2;
    const int K = cfg.k;
    const int64_t pairs = (int64_t)nsys * K;
    BatchArgs& a = s->ba;
    a.n = A.n;
    a.nsys = nsys;
    a.chunk = (int32_t)chunk;
    a.nchunks = (int32_t)ceil_div(A.n, chunk);
    a.a_ptr = A.colptr;
    a.a_idx = A.rowind;
    a.a_val = A.val;
    a.r = base->r;
    a.p = base->p;
    a.q = base->q;
    a.y = base->y;
    a.z = base->z;
    a.sc = base->sc;
    a.tol = cfg.tol;
    a.max_iter = cfg.max_iter;
    a.stop_rule = cfg.stop_rule;
    std::vector<int32_t> hseg((size_t)A.n);
    for (int i = 0; i < nsys; ++i)
        for (int64_t r = h_off[i]; r < h_off[i + 1]; ++r) hseg[(size_t)r] = i;
    cudaError_t e = cudaMalloc(&s->seg, sizeof(int32_t) * hseg.size());
    if (e == cudaSuccess) e = cudaMemcpy(s->seg, hseg.data(), sizeof(int32_t) * hseg.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMalloc(&s->off, sizeof(int64_t) * (size_t)(nsys + 1));
    if (e == cudaSuccess)
        e = cudaMemcpy(s->off, h_off, sizeof(int64_t) * (size_t)(nsys + 1), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMalloc(&s->pool, sizeof(double) * (size_t)pairs * 9);
    if (e == cudaSuccess) e = cudaMalloc(&s->ipool, sizeof(int) * (size_t)pairs * 2);
    if (e == cudaSuccess) e = cudaMalloc(&s->part, sizeof(double) * (size_t)a.nchunks * 2 * K * 2);
    if (e != cudaSuccess) {
        *err = e;
        batch_destroy(s);
        return nullptr;
    }
    a.seg = s->seg;
    a.sys_off = s->off;
    a.part = s->part;
    double* P = s->pool;
    a.s.alpha = P;
    a.s.beta = P + pairs;
    a.s.rz = P + 2 * pairs;
    a.s.rz0 = P + 3 * pairs;
    a.s.rr = P + 4 * pairs;
    a.s.pq = P + 5 * pairs;
    a.s.bnorm2 = P + 6 * pairs;
    a.s.tr2 = P + 7 * pairs;
    a.s.rzn = P + 8 * pairs;
    a.s.active = s->ipool;
    a.s.iters = s->ipool + pairs;
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    s->grid = (int)std::min<int64_t>(a.nchunks, (int64_t)sms * 8);
    return s;
}

void batch_destroy(BatchSolver* s) {
    if (!s) return;
    if (s->graph) cudaGraphExecDestroy(s->graph);
    cudaFree(s->seg);
    cudaFree(s->off);
    cudaFree(s->pool);
    cudaFree(s->ipool);
    cudaFree(s->part);
    pcg_destroy(s->base);
    delete s;
}

cudaError_t batch_solve(BatchSolver* s, const double* dB, double* dX, BatchResult* res) {
    PcgSolver* b = s->base;
    const int K = b->K;
    const int nsys = s->ba.nsys;
    const int64_t pairs = (int64_t)nsys * K;
    cudaError_t e;
    if (b->cfg.use_graph && !(s->graph && s->gb == dB && s->gx == dX)) {
        if (s->graph) cudaGraphExecDestroy(s->graph);
        s->graph = nullptr;
        cudaGraph_t g = nullptr;
        if ((e = cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal)) != cudaSuccess) return e;
        cudaError_t ce = cudaSuccess;
        for (int u = 0; u < b->cfg.unroll && ce == cudaSuccess; ++u) ce = s->iteration(dB, dX);
        e = cudaStreamEndCapture(b->stream, &g);
        if (ce != cudaSuccess) return ce;
        if (e != cudaSuccess) return e;
        e = cudaGraphInstantiate(&s->graph, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return e;
        s->gb = dB;
        s->gx = dX;
    }
    cudaEventRecord(b->ev0, b->stream);
    if ((e = clear_split_counters(b->F, b->stream)) != cudaSuccess) return e;
    BatchArgs a = s->args(dB, dX);
    if ((e = s->launch(s->k_init, s->grid, &a)) != cudaSuccess) return e;
    {  // start: z = M r, rz per pair
        SolveArgs sa = s->solve_args(dB, dX);
        sa.update = 0;
        if ((e = s->launch(b->k_fwd, b->grid_fwd, &sa)) != cudaSuccess) return e;
        if ((e = s->launch(b->k_bwd, b->grid_bwd, &sa)) != cudaSuccess) return e;
        if ((e = s->launch(s->k_dots, s->grid, &a)) != cudaSuccess) return e;
    }
    cudaEventRecord(b->ev1, b->stream);
    res->kernel_launches = 4;
    res->graph_launches = 0;
    while (true) {
        if (b->cfg.use_graph) {
            if ((e = cudaGraphLaunch(s->graph, b->stream)) != cudaSuccess) return e;
            res->graph_launches++;
        } else {
            for (int u = 0; u < b->cfg.unroll; ++u)
                if ((e = s->iteration(dB, dX)) != cudaSuccess) return e;
        }
        res->kernel_launches += 4 * b->cfg.unroll;
        if ((e = cudaMemcpyAsync(b->sc_host, b->sc, sizeof(PcgScalars), cudaMemcpyDeviceToHost, b->stream)) !=
            cudaSuccess)
            return e;
        if ((e = cudaStreamSynchronize(b->stream)) != cudaSuccess) return e;
        if (b->sc_host->done) break;
    }
    if ((e = s->launch(s->k_true, s->grid, &a)) != cudaSuccess) return e;
    res->kernel_launches++;
    cudaEventRecord(b->ev2, b->stream);
    s->h_tr2.resize((size_t)pairs);
    s->h_b2.resize((size_t)pairs);
    s->h_iters.resize((size_t)pairs);
    cudaMemcpyAsync(s->h_tr2.data(), s->ba.s.tr2, sizeof(double) * pairs, cudaMemcpyDeviceToHost, b->stream);
    cudaMemcpyAsync(s->h_b2.data(), s->ba.s.bnorm2, sizeof(double) * pairs, cudaMemcpyDeviceToHost, b->stream);
    cudaMemcpyAsync(s->h_iters.data(), s->ba.s.iters, sizeof(int) * pairs, cudaMemcpyDeviceToHost, b->stream);
    cudaMemcpyAsync(b->sc_host, b->sc, sizeof(PcgScalars), cudaMemcpyDeviceToHost, b->stream);
    if ((e = cudaStreamSynchronize(b->stream)) != cudaSuccess) return e;
    cudaEventElapsedTime(&res->ms_total, b->ev0, b->ev2);
    cudaEventElapsedTime(&res->ms_iterations, b->ev1, b->ev2);
    res->status = b->sc_host->status;
    res->iterations.assign((size_t)nsys, 0);
    res->relres.assign((size_t)nsys, 0.0);
    res->converged = 1;
    for (int sys = 0; sys < nsys; ++sys) {
        for (int c = 0; c < K; ++c) {
            const size_t pr = (size_t)sys * K + c;
            const double bn = std::sqrt(s->h_b2[pr]);
            const double rel = bn > 0 ? std::sqrt(s->h_tr2[pr]) / bn : 0.0;
            res->iterations[(size_t)sys] = std::max(res->iterations[(size_t)sys], s->h_iters[pr]);
            res->relres[(size_t)sys] = std::max(res->relres[(size_t)sys], rel);
            if (b->cfg.stop_rule == 0 && rel > b->cfg.tol) res->converged = 0;
        }
    }
    if (res->status != 0) res->converged = 0;
    return cudaSuccess;
}

// ---- single operator applications ----------------------------------------

namespace {
__global__ void cm_to_rm_kernel(const double* __restrict__ cm, int ld, double* rm, int32_t n, int k) {
    const int64_t total = (int64_t)n * k;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += stride) {
        int64_t i = t / k;
        int c = (int)(t % k);
        rm[t] = cm[(size_t)c * ld + i];
    }
}
__global__ void rm_to_cm_kernel(const double* __restrict__ rm, double* cm, int ld, int32_t n, int k) {
    const int64_t total = (int64_t)n * k;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += stride) {
        int64_t i = t / k;
        int c = (int)(t % k);
        cm[(size_t)c * ld + i] = rm[t];
    }
}
}  // namespace

cudaError_t cm_to_rm(const double* cm, int ld, double* rm, int32_t n, int k, cudaStream_t s) {
    int64_t total = (int64_t)n * k;
    int grid = grid_for(total, kBlock, 16);
    cm_to_rm_kernel<<<grid, kBlock, 0, s>>>(cm, ld, rm, n, k);
    return cudaGetLastError();
}

cudaError_t rm_to_cm(const double* rm, double* cm, int ld, int32_t n, int k, cudaStream_t s) {
    int64_t total = (int64_t)n * k;
    int grid = grid_for(total, kBlock, 16);
    rm_to_cm_kernel<<<grid, kBlock, 0, s>>>(rm, cm, ld, n, k);
    return cudaGetLastError();
}

cudaError_t spmv_f64(const DevCsc& A, const double* x, double* y, int k, cudaStream_t s) {
    int64_t total = (int64_t)A.n * k;
    int grid = grid_for(total, kBlock, 16);
    spmv_plain_kernel<<<grid, kBlock, 0, s>>>(A.n, A.colptr, A.rowind, A.val, x, y, k);
    return cudaGetLastError();
}

template <int K, typename TV>
static cudaError_t precond_apply_t(const DevFactor& F, const double* r, double* z, double* y, int* status,
                                   double timeout_s, cudaStream_t s, int device) {
    PcgScalars* sc = nullptr;
    cudaError_t e = cudaMalloc(&sc, sizeof(PcgScalars));
    if (e != cudaSuccess) return e;
    e = cudaMemsetAsync(sc, 0, sizeof(PcgScalars), s);
    if (e == cudaSuccess) e = clear_split_counters(F, s);
    if (e != cudaSuccess) {
        cudaFree(sc);
        return e;
    }
    SolveArgs a;
    memset(&a, 0, sizeof(a));
    a.n = F.n;
    set_factor_rows(a, F, std::is_same<TV, float>::value);
    a.diag = std::is_same<TV, float>::value ? (const void*)F.diag32 : (const void*)F.diag;
    a.order_f = F.order_f;
    a.order_b = F.order_b;
    a.pack_f = F.pack_f;
    a.pack_b = F.pack_b;
    a.pf_idx = F.pf_idx;
    a.pf_val = std::is_same<TV, float>::value ? (const void*)F.pf_val32 : (const void*)F.pf_val;
    a.pb_idx = F.pb_idx;
    a.pb_val = std::is_same<TV, float>::value ? (const void*)F.pb_val32 : (const void*)F.pb_val;
    a.ntasks_f = F.npt_f;
    a.ntasks_b = F.npt_b;
    a.split_f = F.split_f;
    a.split_b = F.split_b;
    a.psum_f = F.psum_f;
    a.psum_b = F.psum_b;
    a.pcount_f = F.pcount_f;
    a.pcount_b = F.pcount_b;
    a.srow_b = F.srow_b;
    a.nsplit_b = F.nsplit_b;
    a.r = const_cast<double*>(r);
    a.y = y;
    a.z = z;
    a.sc = sc;
    a.update = 0;
    a.reduce = 0;
    a.timeout_ns = (unsigned long long)(timeout_s * 1e9);
    const int64_t total = (int64_t)F.n * K;
    fill_pending_kernel<<<grid_for(total, kBlock, 8), kBlock, 0, s>>>(y, total);
    e = cudaGetLastError();
    const void* kf = K == 1 ? (const void*)fwd_pack_kernel<TV> : (const void*)fwd_kernel<K, TV>;
    const void* kb = K == 1 ? (const void*)bwd_pack_kernel<TV> : (const void*)bwd_kernel<K, TV>;
    if (e == cudaSuccess) e = launch_coresident(kf, resident_blocks(kf, device), a, s);
    if (e == cudaSuccess) e = launch_coresident(kb, resident_blocks(kb, device), a, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(status, &sc->status, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaFree(sc);
    return e;
}

cudaError_t precond_apply(const DevFactor& F, const double* r, double* z, double* ywork, int k, bool fp32,
                          int* status, double timeout_s, cudaStream_t s) {
    int device = 0;
    cudaGetDevice(&device);
#define RCHOL_PA(KK)                                                                                     \
    case KK:                                                                                             \
        return fp32 ? precond_apply_t<KK, float>(F, r, z, ywork, status, timeout_s, s, device)           \
                    : precond_apply_t<KK, double>(F, r, z, ywork, status, timeout_s, s, device);
    switch (k) {
        RCHOL_PA(1)
        RCHOL_PA(2)
        RCHOL_PA(4)
        RCHOL_PA(8)
        RCHOL_PA(16)
        RCHOL_PA(32)
        default:
            return cudaErrorInvalidValue;
    }
#undef RCHOL_PA
}

// ---- allocation-free preconditioner apply --------------------------------
// The same forward and backward sweeps as precond_apply, with every piece of
// device scratch (the PCG scalar block that carries the wait status, and the
// n x k forward-solve vector y) taken from one statically sized module
// array instead of cudaMalloc.  All calls on a device share that array and
// leave their contents in it; two calls whose kernels overlap on the GPU
// race on it.  They also share the factor's split-row partial sums and
// counters (psum_*, pcount_*) with every other solve or apply of the same
// factor, so calls must be serialised against those as well.  The array is
// part of this module's device code: every device that loads the library
// holds its 32 MiB + 4 KiB until the process exits, whether or not this
// entry point is ever called.

constexpr int kNoAllocHeadDoubles = 512;  // 4 KiB: the PcgScalars block
static_assert(sizeof(PcgScalars) <= kNoAllocHeadDoubles * sizeof(double), "scalar block does not fit");
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocHeadDoubles + kNoAllocMaxElems];

namespace {

// Device address of g_noalloc_scratch in the current context.  It is looked
// up on every call (cheap once the module is loaded), so a context that was
// torn down and recreated, e.g. after cudaDeviceReset, gets its new address;
// the first lookup in a context may load this module onto the device.
cudaError_t noalloc_scratch(double** out) {
    double* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress((void**)&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    *out = p;
    return cudaSuccess;
}

template <int K, typename TV>
cudaError_t precond_apply_noalloc_t(const DevFactor& F, const double* r, double* z, double* scratch, int* status,
                                    double timeout_s, cudaStream_t s, int device) {
    PcgScalars* sc = reinterpret_cast<PcgScalars*>(scratch);
    double* y = scratch + kNoAllocHeadDoubles;
    // the status word and counters must start at zero; y starts "pending"
    cudaError_t e = cudaMemsetAsync(sc, 0, sizeof(PcgScalars), s);
    if (e == cudaSuccess) e = clear_split_counters(F, s);
    if (e != cudaSuccess) return e;
    SolveArgs a;
    memset(&a, 0, sizeof(a));
    a.n = F.n;
    set_factor_rows(a, F, std::is_same<TV, float>::value);
    a.diag = std::is_same<TV, float>::value ? (const void*)F.diag32 : (const void*)F.diag;
    a.order_f = F.order_f;
    a.order_b = F.order_b;
    a.pack_f = F.pack_f;
    a.pack_b = F.pack_b;
    a.pf_idx = F.pf_idx;
    a.pf_val = std::is_same<TV, float>::value ? (const void*)F.pf_val32 : (const void*)F.pf_val;
    a.pb_idx = F.pb_idx;
    a.pb_val = std::is_same<TV, float>::value ? (const void*)F.pb_val32 : (const void*)F.pb_val;
    a.ntasks_f = F.npt_f;
    a.ntasks_b = F.npt_b;
    a.split_f = F.split_f;
    a.split_b = F.split_b;
    a.psum_f = F.psum_f;
    a.psum_b = F.psum_b;
    a.pcount_f = F.pcount_f;
    a.pcount_b = F.pcount_b;
    a.srow_b = F.srow_b;
    a.nsplit_b = F.nsplit_b;
    a.r = const_cast<double*>(r);
    a.y = y;
    a.z = z;
    a.sc = sc;
    a.update = 0;
    a.reduce = 0;
    a.timeout_ns = (unsigned long long)(timeout_s * 1e9);
    fill_pending_kernel<<<grid_for((int64_t)F.n * K, kBlock, 8), kBlock, 0, s>>>(y, (int64_t)F.n * K);
    e = cudaGetLastError();
    const void* kf = K == 1 ? (const void*)fwd_pack_kernel<TV> : (const void*)fwd_kernel<K, TV>;
    const void* kb = K == 1 ? (const void*)bwd_pack_kernel<TV> : (const void*)bwd_kernel<K, TV>;
    if (e == cudaSuccess) e = launch_coresident(kf, resident_blocks(kf, device), a, s);
    if (e == cudaSuccess) e = launch_coresident(kb, resident_blocks(kb, device), a, s);
    int st = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&st, &sc->status, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    *status = st;
    return e;
}

}  // namespace

cudaError_t precond_apply_noalloc(const DevFactor& F, const double* r, double* z, int k, bool fp32, int* status,
                                  double timeout_s, cudaStream_t s) {
    if ((long long)F.n * k > kNoAllocMaxElems) return cudaErrorInvalidValue;
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) return e;
    double* scratch = nullptr;
    e = noalloc_scratch(&scratch);
    if (e != cudaSuccess) return e;
#define RCHOL_PAN(KK)                                                                                        \
    case KK:                                                                                                 \
        return fp32 ? precond_apply_noalloc_t<KK, float>(F, r, z, scratch, status, timeout_s, s, device)     \
                    : precond_apply_noalloc_t<KK, double>(F, r, z, scratch, status, timeout_s, s, device);
    switch (k) {
        RCHOL_PAN(1)
        RCHOL_PAN(2)
        RCHOL_PAN(4)
        RCHOL_PAN(8)
        RCHOL_PAN(16)
        RCHOL_PAN(32)
        default:
            return cudaErrorInvalidValue;
    }
#undef RCHOL_PAN
}


// ---------------------------------------------------------------------------
// The hop floor of the sync-free solves: two CTAs pass a counter back and
// forth through one global word with the solves' own relaxed store and poll
// (no back-off), so one hop is a store on one SM seen by a poll on another.
// The first kHopWarm round trips are not timed (launch skew).  Every wait is
// bounded by limit_ns; on expiry out[1] = 1 and the CTA returns.
// out: [0] ns for 2 * (rounds - kHopWarm) hops, [1] error, [2..3] SM ids.
// ---------------------------------------------------------------------------
constexpr int kHopWarm = 16;

__global__ void hop_probe_kernel(double* cell, int rounds, unsigned long long limit_ns, long long* out) {
    if (threadIdx.x != 0) return;
    const int me = blockIdx.x;
    unsigned smid;
    asm volatile("mov.u32 %0, %%smid;" : "=r"(smid));
    out[2 + me] = smid;
    const unsigned long long t0 = global_timer_ns();
    unsigned long long ts = t0;
    for (int i = 0; i <= rounds; ++i) {
        if (me == 1 && i == rounds) break;
        const double want = (double)(2 * i + me);
        unsigned spins = 0;
        while (ld_relaxed_f64(cell) != want) {
            if ((++spins & 63u) == 0 && global_timer_ns() - t0 > limit_ns) {
                out[1] = 1;
                return;
            }
        }
        if (me == 0 && i == kHopWarm) ts = global_timer_ns();
        if (i < rounds) st_relaxed_f64(cell, want + 1.0);
    }
    if (me == 0) out[0] = (long long)(global_timer_ns() - ts);
}

cudaError_t hop_latency(int rounds, double* ns_per_hop, int* sm_pair) {
    if (rounds <= kHopWarm) return cudaErrorInvalidValue;
    char* buf = nullptr;
    cudaError_t e = cudaMalloc((void**)&buf, 256);
    if (e != cudaSuccess) return e;
    double* cell = reinterpret_cast<double*>(buf);
    long long* out = reinterpret_cast<long long*>(buf + 128);
    long long h[4] = {0, 0, 0, 0};
    e = cudaMemset(buf, 0, 256);
    if (e == cudaSuccess) {
        unsigned long long limit = 2000000000ull;  // 2 s
        void* params[] = {&cell, &rounds, &limit, &out};
        // cooperative: both CTAs are resident together or the launch fails
        e = cudaLaunchCooperativeKernel((const void*)hop_probe_kernel, dim3(2), dim3(32), params, 0, 0);
    }
    if (e == cudaSuccess) e = cudaMemcpy(h, out, sizeof(h), cudaMemcpyDeviceToHost);
    cudaFree(buf);
    if (e != cudaSuccess) return e;
    if (h[1] != 0) return cudaErrorTimeout;
    *ns_per_hop = (double)h[0] / (2.0 * (rounds - kHopWarm));
    if (sm_pair) {
        sm_pair[0] = (int)h[2];
        sm_pair[1] = (int)h[3];
    }
    return cudaSuccess;
}

}  // namespace rchol
