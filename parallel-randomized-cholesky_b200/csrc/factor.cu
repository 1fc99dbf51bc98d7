// Randomized-Cholesky elimination of a graph Laplacian on sm_100a.
//
// Restates the algorithm of gpu_implementation/driver.cu:43-1302 and
// cpu_implementation/driver_local.cpp:302-707 with a B200-first design:
//   * one persistent launch sized to the resident capacity; every warp pulls
//     ready vertices from a global FIFO (driver.cu:142-234) and releases its
//     neighbours through per-vertex dependency counters with acquire/release
//     atomics (driver.cu:1179-1202 used relaxed atomics and never re-read);
//   * the neighbour merge is a warp bitonic sort + segmented sum staged in a
//     shared-memory slab (a per-warp global slab for large vertices);
//   * sampling uniforms come from Philox4x32-10 keyed by (seed, vertex,
//     slot), so the factor does not depend on which warp took which vertex;
//   * fill edges are appended to per-column buckets by atomics (driver.cu
//     used an open-addressing hash over 4*nnz slots, :1068-1150): a fixed
//     first chunk per column plus 64-entry overflow chunks linked lock-free.
// FP64 arithmetic uses explicitly rounded intrinsics (no contraction), which
// makes the factor bit-identical to the CPU oracle's ORC_MODE_B200.
#include <climits>
#include <cstdio>

#include "device_common.cuh"
#include "rchol_internal.h"

namespace rchol {

namespace {

constexpr int kChunk = 64;                 // overflow pool unit (entries); chunk lvl spans 2^lvl units
constexpr int kPoolGrab = 1024;            // L-pool entries grabbed per warp at once
constexpr unsigned long long kInfBits = 0x7ff0000000000000ull;
constexpr int kSlabBytesPerEntry = 32;     // 8 (a_val) + 8 (b_val) + 8 (b_aux) + 4 + 4

enum Counter { kQHead = 0, kQTail = 1, kChunkCursor = 2, kStatus = 3, kAbort = 4, kBigCount = 5,
               kMaxGather = 6, kOverflowFills = 7, kDone = 8, kTailTicket = 9 };

__device__ __forceinline__ int pow2_at_least(int x) {
    int p = 1;
    while (p < x) p <<= 1;
    return p;
}

// One warp's staging area: a_* hold the gathered entries and, after the
// value sort, the prefix sums; b_* hold the merged neighbours.  Slabs in
// global memory add t_* as the second buffer of their radix sorts.
struct Slab {
    double* a_val;
    int32_t* a_row;
    double* b_val;
    int32_t* b_row;
    long long* b_aux;  // (multiplicity << 32) | row-order position
    double* t_val;
    int32_t* t_row;
    long long* t_aux;
};

__device__ __forceinline__ Slab make_slab(unsigned char* base, int cap) {
    Slab s;
    s.a_val = reinterpret_cast<double*>(base);
    s.b_val = s.a_val + cap;
    s.b_aux = reinterpret_cast<long long*>(s.b_val + cap);
    s.a_row = reinterpret_cast<int32_t*>(s.b_aux + cap);
    s.b_row = s.a_row + cap;
    s.t_val = nullptr;
    s.t_row = nullptr;
    s.t_aux = nullptr;
    return s;
}

// kGlobalSlabBytes per entry: the shared-memory layout plus t_val, t_aux, t_row.
__device__ __forceinline__ Slab make_global_slab(unsigned char* base, int cap) {
    Slab s = make_slab(base, cap);
    s.t_val = reinterpret_cast<double*>(s.b_row + cap);
    s.t_aux = reinterpret_cast<long long*>(s.t_val + cap);
    s.t_row = reinterpret_cast<int32_t*>(s.t_aux + cap);
    return s;
}

// ---- bitonic sorts over slab arrays (P a power of two) -------------------

// ascending by (row, value bits)
__device__ void sort_row_value(int32_t* row, double* val, int P, int lane) {
    for (int k = 2; k <= P; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = lane; i < P; i += kWarp) {
                int l = i ^ j;
                if (l > i) {
                    int32_t ri = row[i], rl = row[l];
                    unsigned long long vi = (unsigned long long)__double_as_longlong(val[i]);
                    unsigned long long vl = (unsigned long long)__double_as_longlong(val[l]);
                    bool gt = (ri > rl) || (ri == rl && vi > vl);
                    bool asc = (i & k) == 0;
                    if (gt == asc) {
                        row[i] = rl;
                        row[l] = ri;
                        val[i] = __longlong_as_double((long long)vl);
                        val[l] = __longlong_as_double((long long)vi);
                    }
                }
            }
            __syncwarp();
        }
    }
}

// ascending by (value, row) carrying aux
__device__ void sort_value_row(double* val, int32_t* row, long long* aux, int P, int lane) {
    for (int k = 2; k <= P; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = lane; i < P; i += kWarp) {
                int l = i ^ j;
                if (l > i) {
                    double vi = val[i], vl = val[l];
                    int32_t ri = row[i], rl = row[l];
                    bool gt = (vi > vl) || (vi == vl && ri > rl);
                    bool asc = (i & k) == 0;
                    if (gt == asc) {
                        val[i] = vl;
                        val[l] = vi;
                        row[i] = rl;
                        row[l] = ri;
                        long long ai = aux[i];
                        aux[i] = aux[l];
                        aux[l] = ai;
                    }
                }
            }
            __syncwarp();
        }
    }
}

// ---- warp radix sorts for slabs in global memory ------------------------
// Stable LSD passes over 8-bit digits.  In a scatter pass each 32-entry
// round ranks equal digits with a match mask, so equal digits keep their
// order, and the next digit is counted on the way; a digit shared by every
// entry moves nothing.  `hist` is 2 x 256 ints of the warp's shared memory.
// The result is the unique order of the keys, the same as the bitonic sorts
// give.

// digit d of (row, value bits): bytes 0-7 of the value bits, then bytes 0-3 of the row
__device__ __forceinline__ int rv_digit(int32_t r, double v, int d) {
    return d < 8 ? (int)(((unsigned long long)__double_as_longlong(v) >> (8 * d)) & 255ull)
                 : (int)(((unsigned)r >> (8 * (d - 8))) & 255u);
}
// digit d of (value bits, row): bytes 0-3 of the row, then bytes 0-7 of the value bits
__device__ __forceinline__ int vr_digit(int32_t r, double v, int d) { return rv_digit(r, v, (d + 8) % 12); }

// Rounds of 32 entries whose loads a pass issues together (one memory
// round trip per kRadixRounds * 32 entries).
#ifndef RCHOL_RADIX_ROUNDS
#define RCHOL_RADIX_ROUNDS 4
#endif
constexpr int kRadixRounds = RCHOL_RADIX_ROUNDS;

// Counts of digit d over n entries into hist (256 ints, zeroed here).
template <bool VR>
__device__ void radix_count(const int32_t* row, const double* val, int n, int d, int* hist, int lane) {
    for (int i = lane; i < 256; i += kWarp) hist[i] = 0;
    __syncwarp();
    for (int base = 0; base < n; base += kRadixRounds * kWarp) {
        int dig[kRadixRounds];
#pragma unroll
        for (int q = 0; q < kRadixRounds; ++q) {
            const int i = base + q * kWarp + lane;
            dig[q] = i < n ? (VR ? vr_digit(row[i], val[i], d) : rv_digit(row[i], val[i], d)) : -1;
        }
#pragma unroll
        for (int q = 0; q < kRadixRounds; ++q)
            if (dig[q] >= 0) atomicAdd(&hist[dig[q]], 1);
    }
    __syncwarp();
}

// Turns the counts in hist into exclusive offsets; true when one digit holds
// all n entries (the pass would move nothing).
__device__ bool radix_offsets(int* hist, int n, int lane) {
    int c[8], tot = 0;
    bool one = false;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        c[q] = hist[8 * lane + q];
        tot += c[q];
        one |= c[q] == n;
    }
    const bool all = __any_sync(kFull, one);
    int incl = tot;
#pragma unroll
    for (int o = 1; o < kWarp; o <<= 1) {
        const int t = __shfl_up_sync(kFull, incl, o);
        if (lane >= o) incl += t;
    }
    int run = incl - tot;
    __syncwarp();
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        hist[8 * lane + q] = run;
        run += c[q];
    }
    __syncwarp();
    return all;
}

// One stable scatter pass of (row, val[, aux]) by digit d (hist holds the
// offsets), counting digit dnext (< 0: none) of the moved entries into hnext
// (zeroed here).
template <bool VR, bool AUX>
__device__ void radix_scatter(const int32_t* row, const double* val, const long long* aux, int32_t* orow, double* oval,
                              long long* oaux, int n, int d, int dnext, int* hist, int* hnext, int lane) {
    const unsigned lt = (1u << lane) - 1u;
    for (int i = lane; i < 256; i += kWarp) hnext[i] = 0;
    __syncwarp();
    for (int base = 0; base < n; base += kRadixRounds * kWarp) {
        // the loads of kRadixRounds rounds first, then the rounds in order
        int32_t r[kRadixRounds];
        double v[kRadixRounds];
        long long x[kRadixRounds];
#pragma unroll
        for (int q = 0; q < kRadixRounds; ++q) {
            const int i = base + q * kWarp + lane;
            r[q] = 0;
            v[q] = 0.0;
            x[q] = 0;
            if (i < n) {
                r[q] = row[i];
                v[q] = val[i];
                if (AUX) x[q] = aux[i];
            }
        }
#pragma unroll
        for (int q = 0; q < kRadixRounds; ++q) {
            const bool valid = base + q * kWarp + lane < n;
            const int dig = valid ? (VR ? vr_digit(r[q], v[q], d) : rv_digit(r[q], v[q], d)) : 256;
            const unsigned peers = __match_any_sync(kFull, dig);
            const int rank = __popc(peers & lt);
            const int at = valid ? hist[dig] + rank : 0;
            __syncwarp();
            if (valid && rank == 0) hist[dig] += __popc(peers);
            if (valid && dnext >= 0) atomicAdd(&hnext[VR ? vr_digit(r[q], v[q], dnext) : rv_digit(r[q], v[q], dnext)], 1);
            __syncwarp();
            if (valid) {
                orow[at] = r[q];
                oval[at] = v[q];
                if (AUX) oaux[at] = x[q];
            }
        }
    }
    __syncwarp();
}

// LSD radix sort of n entries by digits dlo..dhi-1 through the ping-pong
// buffers; the result is copied back into (r_out, v_out[, x_out]) when it
// ends in the other buffer.
template <bool VR, bool AUX>
__device__ void radix_sort(int32_t* r_out, double* v_out, long long* x_out, int32_t* r_tmp, double* v_tmp,
                           long long* x_tmp, int n, int* hist, int* hnext, int lane, int dlo, int dhi) {
    int32_t *r0 = r_out, *r1 = r_tmp;
    double *v0 = v_out, *v1 = v_tmp;
    long long *x0 = x_out, *x1 = x_tmp;
    radix_count<VR>(r0, v0, n, dlo, hist, lane);
    for (int d = dlo; d < dhi; ++d) {
        if (radix_offsets(hist, n, lane)) {
            // nothing moves: count the next digit from the current buffer
            if (d + 1 < dhi) radix_count<VR>(r0, v0, n, d + 1, hist, lane);
            continue;
        }
        radix_scatter<VR, AUX>(r0, v0, x0, r1, v1, x1, n, d, d + 1 < dhi ? d + 1 : -1, hist, hnext, lane);
        int* th = hist; hist = hnext; hnext = th;
        int32_t* tr = r0; r0 = r1; r1 = tr;
        double* tv = v0; v0 = v1; v1 = tv;
        long long* tx = x0; x0 = x1; x1 = tx;
    }
    if (r0 != r_out) {
        for (int i = lane; i < n; i += kWarp) {
            r_out[i] = r0[i];
            v_out[i] = v0[i];
            if (AUX) x_out[i] = x0[i];
        }
        __syncwarp();
    }
}

// (a_row, a_val) ascending by (row, value bits), result in a_*.
__device__ __forceinline__ void radix_sort_rv(const Slab& s, int n, int* hist, int lane) {
    radix_sort<false, false>(s.a_row, s.a_val, nullptr, s.t_row, s.t_val, nullptr, n, hist, hist + 256, lane, 0, 12);
}

// (b_val, b_row, b_aux) ascending by (value, row), result in b_*.  The input
// is in ascending row order, so a stable sort on the value bytes alone gives
// (value, row) order.
__device__ __forceinline__ void radix_sort_vr(const Slab& s, int n, int* hist, int lane) {
    radix_sort<true, true>(s.b_row, s.b_val, s.b_aux, s.t_row, s.t_val, s.t_aux, n, hist, hist + 256, lane, 4, 12);
}

struct FactorArgs {
    int32_t n;
    const int32_t* __restrict__ lcolptr;
    const int32_t* __restrict__ lrow;
    const double* __restrict__ lval;
    int32_t* dep;
    int32_t* queue;
    int32_t c0;
    int32_t* fcnt;
    int32_t* brow;
    double* bval;
    int32_t* chead;
    int32_t* cnext;
    int32_t* crow;
    double* cval;
    int32_t nchunks;
    int64_t pool_cap;
    int32_t* prow;
    double* pval;
    int64_t* pstart;
    int32_t* pcnt;
    double* diag;
    int32_t* level;  // forward level of each row of L (depth in the L-solve DAG)
    unsigned char* gscratch;
    int64_t gscratch_entries;
    unsigned char* hscratch;
    int64_t hscratch_entries;
    int32_t nhuge;
    int32_t* hlock;
    int32_t* counters;
    unsigned long long* pool_cursor;
    uint64_t seed;
    int smem_slab;
    int smem_region;  // bytes of shared memory per warp (slab, or radix histogram + CDF index)
    unsigned long long timeout_ns;
    int32_t tail;     // vertices >= tail are left to factor_tail_kernel (n: none)
    int32_t* gsize;   // gathered entries of each vertex (null: not recorded)
    int32_t tail_cdf_cap;  // prefix sums the tail kernel keeps in shared memory
};

__device__ __forceinline__ bool aborted(const FactorArgs& a) { return ld_relaxed(a.counters + kAbort) != 0; }

__device__ __forceinline__ void fail(const FactorArgs& a, int code) {
    raise_error(a.counters + kStatus, code);
    atomicExch(a.counters + kAbort, 1);
}

// Append one fill edge (row > col) to column col's bucket.  Returns false on
// pool exhaustion.  Chunks are linked with CAS, so no thread ever waits.
__device__ bool append_fill(const FactorArgs& a, int32_t col, int32_t row, double v) {
    int s = atomicAdd(a.fcnt + col, 1);
    if (s < a.c0) {
        size_t o = (size_t)col * (size_t)a.c0 + (size_t)s;
        a.brow[o] = row;
        a.bval[o] = v;
        return true;
    }
    atomicAdd(a.counters + kOverflowFills, 1);
    // overflow chunk number lvl of a column spans kChunk << lvl slots (2^lvl
    // pool units), so slot t is at most log2(t / kChunk + 1) links away
    const int t = s - a.c0;
    const int ci = 31 - __clz(t / kChunk + 1);
    const int off = t - kChunk * ((1 << ci) - 1);
    int32_t* link = a.chead + col;
    int cur = -1;
    for (int lvl = 0;; ++lvl) {
        cur = ld_relaxed(link);
        if (cur < 0) {
            const int units = 1 << lvl;
            const int nc = atomicAdd(a.counters + kChunkCursor, units);
            if (nc > a.nchunks - units) return false;
            const int old = atomicCAS(link, -1, nc);
            cur = (old == -1) ? nc : old;
        }
        if (lvl == ci) break;
        link = a.cnext + cur;
    }
    size_t o = (size_t)cur * kChunk + (size_t)off;
    a.crow[o] = row;
    a.cval[o] = v;
    return true;
}

// Release one chunk of merged neighbours after the elimination of a column:
// raise their forward level, decrement their dependency counters (acq_rel),
// keep the first neighbour that becomes ready in `next` and push the others
// with one queue reservation for the warp.
__device__ __forceinline__ void release_chunk(const FactorArgs& a, int lk, int lane, bool valid, int32_t r, int mult,
                                              int32_t& next) {
    bool ready = false;
    if (valid) {
        atomicMax(a.level + r, lk);
        ready = atom_add_acq_rel(a.dep + r, -mult) == mult;
    }
    unsigned bal = __ballot_sync(kFull, ready);
    if (bal && next < 0) {
        const int leader = __ffs(bal) - 1;
        next = __shfl_sync(kFull, r, leader);
        if (lane == leader) ready = false;
        bal &= bal - 1u;
    }
    if (bal) {
        int slot = 0;
        if (lane == 0) slot = atomicAdd(a.counters + kQTail, __popc(bal));
        slot = __shfl_sync(kFull, slot, 0) + __popc(bal & ((1u << lane) - 1u));
        if (ready) {
            if (slot < a.n) st_release(a.queue + slot, r);
            else fail(a, kDevBadInput);
        }
    }
}

// Reserve m entries of the L pool for this warp (grabbing kPoolGrab at a time).
__device__ __forceinline__ bool pool_take(const FactorArgs& a, int m, int lane, int64_t& pool_cur, int64_t& pool_end,
                                          int64_t& base) {
    if (pool_end - pool_cur < m) {
        const int64_t grab = m > kPoolGrab ? (int64_t)m : (int64_t)kPoolGrab;
        unsigned long long got = 0;
        if (lane == 0) got = atomicAdd(a.pool_cursor, (unsigned long long)grab);
        got = __shfl_sync(kFull, got, 0);
        if ((int64_t)got + grab > a.pool_cap) return false;
        pool_cur = (int64_t)got;
        pool_end = (int64_t)got + grab;
    }
    base = pool_cur;
    pool_cur += m;
    return true;
}

__device__ __forceinline__ bool row_value_gt(int32_t r1, unsigned long long v1, int32_t r2, unsigned long long v2) {
    return (r1 > r2) || (r1 == r2 && v1 > v2);
}

// Elimination of a vertex whose gathered list fits one warp (at most 32
// entries, all fills in the first bucket chunk): one entry per lane; sorts,
// merge, compaction, scan and CDF search as warp shuffles.  Same arithmetic
// in the same order as the slab path (and the oracle), so the bits agree.
__device__ bool eliminate_small(const FactorArgs& a, int32_t k, int total, int32_t brow_l, double bval_l, int lvl,
                                int lane, int64_t& pool_cur, int64_t& pool_end, long long& fills, int32_t& next) {
    // all `total` entries sit in the bucket, entry `lane` in this lane
    int32_t row = INT_MAX;
    unsigned long long vb = kInfBits;
    if (lane < total) {
        row = brow_l;
        vb = (unsigned long long)__double_as_longlong(bval_l);
    }
    // bitonic sort of the 32 lanes by (row, value bits); padding sorts last
#pragma unroll
    for (int kk = 2; kk <= 32; kk <<= 1) {
#pragma unroll
        for (int j = kk >> 1; j > 0; j >>= 1) {
            const int32_t r2 = __shfl_xor_sync(kFull, row, j);
            const unsigned long long v2 = __shfl_xor_sync(kFull, vb, j);
            const bool keep_min = ((lane & j) == 0) == ((lane & kk) == 0);
            const bool take = keep_min ? row_value_gt(row, vb, r2, v2) : row_value_gt(r2, v2, row, vb);
            if (take) {
                row = r2;
                vb = v2;
            }
        }
    }
    // merge equal rows: the head of each run sums its run left to right
    const double v = __longlong_as_double((long long)vb);
    const int32_t rprev = __shfl_up_sync(kFull, row, 1);
    const bool head = lane < total && (lane == 0 || rprev != row);
    double acc = v;
    int cnt = 1;
    bool going = head;
    for (int d = 1; d < 32; ++d) {
        if (!__any_sync(kFull, going)) break;
        const double vd = __shfl_down_sync(kFull, v, d);
        const int32_t rd = __shfl_down_sync(kFull, row, d);
        if (going) {
            if (lane + d < total && rd == row) {
                acc = __dadd_rn(acc, vd);
                ++cnt;
            } else {
                going = false;
            }
        }
    }
    const unsigned hb = __ballot_sync(kFull, head);
    const int m = __popc(hb);
    const int src = lane < m ? (int)__fns(hb, 0, lane + 1) : 0;
    // merged entries in row order, entry `lane` in this lane
    int32_t orow = __shfl_sync(kFull, row, src);
    int ocnt = __shfl_sync(kFull, cnt, src);
    double mval = __shfl_sync(kFull, acc, src);
    if (lane >= m) {
        orow = INT_MAX;
        ocnt = 0;
        mval = __longlong_as_double((long long)kInfBits);
    }
    int pos = lane;  // position in row order
    // sort by (value, row) carrying the row-order position.  Rows are unique
    // and ascend with the position, so ties in value break on the position
    // exactly as on the row (padding, all +inf, sorts last in any order);
    // the row and multiplicity are fetched by position afterwards, which
    // keeps two shuffles per stage off the shared-memory/shuffle pipe.
#pragma unroll
    for (int kk = 2; kk <= 32; kk <<= 1) {
#pragma unroll
        for (int j = kk >> 1; j > 0; j >>= 1) {
            const double v2 = __shfl_xor_sync(kFull, mval, j);
            const int p2 = __shfl_xor_sync(kFull, pos, j);
            const bool keep_min = ((lane & j) == 0) == ((lane & kk) == 0);
            const bool self_gt = (mval > v2) || (mval == v2 && pos > p2);
            const bool other_gt = (v2 > mval) || (v2 == mval && p2 > pos);
            if (keep_min ? self_gt : other_gt) {
                mval = v2;
                pos = p2;
            }
        }
    }
    const int32_t mrow = __shfl_sync(kFull, orow, pos);
    const int mcnt = __shfl_sync(kFull, ocnt, pos);
    // inclusive prefix sum (one 32-wide Kogge-Stone chunk)
    double cum = lane < m ? mval : 0.0;
#pragma unroll
    for (int off = 1; off < kWarp; off <<= 1) {
        const double t = __shfl_up_sync(kFull, cum, off);
        if (lane >= off) cum = __dadd_rn(cum, t);
    }
    const double S = __shfl_sync(kFull, cum, m - 1);
    int64_t pbase = 0;
    if (!pool_take(a, m, lane, pool_cur, pool_end, pbase)) {
        if (lane == 0) fail(a, kDevCapacity);
        return false;
    }
    fills += m - 1;
    if (lane == 0) {
        a.diag[k] = S;
        a.pstart[k] = pbase;
        a.pcnt[k] = m;
    }
    if (lane < m) {
        a.prow[pbase + pos] = mrow;
        a.pval[pbase + pos] = __ddiv_rn(mval, S);
    }
    // clique sampling: first j > lane with (C_j - C_lane) >= u * (S - C_lane)
    const double rem = __dsub_rn(S, cum);
    const double target = __dmul_rn(sample_uniform(a.seed, k, lane), rem);
    int lo = lane + 1, hi = m;
#pragma unroll
    for (int step = 0; step < 6; ++step) {
        const int mid = lo < hi ? lo + ((hi - lo) >> 1) : 0;
        const double cm = __shfl_sync(kFull, cum, mid);
        if (lo < hi) {
            if (__dsub_rn(cm, cum) < target) lo = mid + 1;
            else hi = mid;
        }
    }
    const int jj = lo < m ? lo : m - 1;
    const int32_t rj = __shfl_sync(kFull, mrow, jj);
    bool ok = true;
    if (lane < m - 1) {
        const int32_t grow = mrow > rj ? mrow : rj;
        const int32_t gcol = mrow > rj ? rj : mrow;
        const double gval = __ddiv_rn(__dmul_rn(mval, rem), S);
        if (!append_fill(a, gcol, grow, gval)) ok = false;
        atomicAdd(a.dep + grow, 1);
    }
    if (__any_sync(kFull, !ok)) {
        if (lane == 0) fail(a, kDevCapacity);
        return false;
    }
    const int lk = lvl + 1;
    __threadfence();
    __syncwarp();
    release_chunk(a, lk, lane, lane < m, mrow, mcnt, next);
    __syncwarp();
    return true;
}

template <bool GLOBAL>
__device__ __forceinline__ bool eliminate_slab(const FactorArgs& a, int32_t k, int nf, int o0, int no, int lvl,
                                               Slab s, unsigned char* wsm, int lane, int64_t& pool_cur,
                                               int64_t& pool_end, long long& fills, int32_t& next);

// The global-slab elimination (radix sorts, indexed CDF search).
__device__ __forceinline__ bool eliminate_global(const FactorArgs& a, int32_t k, int nf, int o0, int no, int lvl,
                                              Slab s, unsigned char* wsm, int lane, int64_t& pool_cur,
                                              int64_t& pool_end, long long& fills, int32_t& next) {
    return eliminate_slab<true>(a, k, nf, o0, no, lvl, s, wsm, lane, pool_cur, pool_end, fills, next);
}

// Takes one of the shared large slabs (lane 0 tries the lock words; the
// wait is bounded).  Holders never wait on other vertices, so a slab is
// always released.  Returns the slab index, or -1 when the kernel stops.
__device__ int acquire_huge(const FactorArgs& a, int lane) {
    int got = -1;
    if (lane == 0) {
        const unsigned long long t0 = global_timer_ns();
        unsigned spins = 0;
        while (got < 0) {
            for (int i = 0; i < a.nhuge && got < 0; ++i)
                if (atomicCAS(a.hlock + i, 0, 1) == 0) got = i;
            if (got >= 0 || aborted(a)) break;
            if ((++spins & 63u) == 0 && global_timer_ns() - t0 > a.timeout_ns) {
                fail(a, kDevTimeout);
                break;
            }
            __nanosleep(200);
        }
        __threadfence();
    }
    return __shfl_sync(kFull, got, 0);
}

__device__ void release_huge(const FactorArgs& a, int lane, int h) {
    __syncwarp();
    if (lane == 0) {
        __threadfence();
        atomicExch(a.hlock + h, 0);
    }
}

// Eliminate vertex k with one warp.  Returns false if the kernel must stop.
// `next` receives one neighbour this elimination released (or stays -1);
// the other released neighbours go to the global queue.
__device__ bool eliminate(const FactorArgs& a, int32_t k, Slab sm, unsigned char* wsm, int warp_global, int lane,
                          int64_t& pool_cur, int64_t& pool_end, long long& fills, int32_t& next, int& max_gather) {
    // One round trip: the bucket count (original entries pre-filled at set-up
    // plus fills), the bucket's first 32 slots, the original column range
    // (entries beyond the bucket stay there) and the vertex's level.
    const int nf = ld_relaxed(a.fcnt + k);
    const int oc0 = a.lcolptr[k];
    const int ocnt = a.lcolptr[k + 1] - oc0;
    int32_t brow_l = INT_MAX;
    double bval_l = 0.0;
    if (lane < a.c0) {
        const size_t o = (size_t)k * (size_t)a.c0 + (size_t)lane;
        brow_l = __ldcg(a.brow + o);
        bval_l = __ldcg(a.bval + o);
    }
    const int lvl = ld_relaxed(a.level + k);
    const int o0 = oc0 + min(ocnt, a.c0);  // originals not in the bucket
    const int no = ocnt - min(ocnt, a.c0);
    const int total = nf + no;
    if (total == 0) {  // driver_local.cpp:470-477: empty column, D = 0
        if (lane == 0) {
            a.diag[k] = 0.0;
            a.pcnt[k] = 0;
            a.pstart[k] = 0;
        }
        return true;
    }
    if (total > max_gather) max_gather = total;
    if (a.gsize && lane == 0) a.gsize[k] = total;
    if (no == 0 && nf <= a.c0 && total <= kWarp)  // every entry is in the bucket
        return eliminate_small(a, k, total, brow_l, bval_l, lvl, lane, pool_cur, pool_end, fills, next);
    if (total <= a.smem_slab)
        return eliminate_slab<false>(a, k, nf, o0, no, lvl, sm, wsm, lane, pool_cur, pool_end, fills, next);
    if (lane == 0) atomicAdd(a.counters + kBigCount, 1);
    if ((int64_t)total <= a.gscratch_entries) {
        Slab s = make_global_slab(a.gscratch + (size_t)warp_global * (size_t)a.gscratch_entries * kGlobalSlabBytes,
                                  (int)a.gscratch_entries);
        return eliminate_global(a, k, nf, o0, no, lvl, s, wsm, lane, pool_cur, pool_end, fills, next);
    }
    if ((int64_t)total > a.hscratch_entries) {
        if (lane == 0) fail(a, kDevCapacity);
        return false;
    }
    const int h = acquire_huge(a, lane);
    if (h < 0) return false;
    Slab s = make_global_slab(a.hscratch + (size_t)h * (size_t)a.hscratch_entries * kGlobalSlabBytes,
                              (int)a.hscratch_entries);
    const bool ok = eliminate_global(a, k, nf, o0, no, lvl, s, wsm, lane, pool_cur, pool_end, fills, next);
    release_huge(a, lane, h);
    return ok;
}

// Elimination of vertex k in slab s: nf bucket entries (slots, then
// overflow chunks) and no original entries from lrow[o0..], level lvl.
template <bool GLOBAL>
__device__ __forceinline__ bool eliminate_slab(const FactorArgs& a, int32_t k, int nf, int o0, int no, int lvl,
                                               Slab s, unsigned char* wsm, int lane, int64_t& pool_cur,
                                               int64_t& pool_end, long long& fills, int32_t& next) {
    // slabs in global memory sort with radix passes (one round trip per 32
    // entries and pass) instead of bitonic stages (one per entry pair)
    constexpr bool global = GLOBAL;
    int* hist = reinterpret_cast<int*>(wsm);
    const int total = nf + no;
    const int P = pow2_at_least(total);

    // ---- gather: fills (first chunk, then overflow chunks), original column
    const int n0 = min(nf, a.c0);
    for (int t = lane; t < n0; t += kWarp) {
        size_t o = (size_t)k * (size_t)a.c0 + (size_t)t;
        s.a_row[t] = __ldcg(a.brow + o);
        s.a_val[t] = __ldcg(a.bval + o);
    }
    int rem = nf - n0, pos = n0;
    int chunk = rem > 0 ? ld_relaxed(a.chead + k) : -1;
    for (int lvl = 0; rem > 0; ++lvl) {
        if (chunk < 0 || chunk > a.nchunks - (1 << lvl)) {
            if (lane == 0) fail(a, kDevBadInput);
            return false;
        }
        const int cnt = min(rem, kChunk << lvl);
        for (int t = lane; t < cnt; t += kWarp) {
            s.a_row[pos + t] = __ldcg(a.crow + (size_t)chunk * kChunk + t);
            s.a_val[pos + t] = __ldcg(a.cval + (size_t)chunk * kChunk + t);
        }
        pos += cnt;
        rem -= cnt;
        if (rem > 0) chunk = ld_relaxed(a.cnext + chunk);
    }
    for (int t = lane; t < no; t += kWarp) {
        s.a_row[nf + t] = a.lrow[o0 + t];
        s.a_val[nf + t] = a.lval[o0 + t];
    }
    if (!global) {
        for (int t = total + lane; t < P; t += kWarp) {
            s.a_row[t] = INT_MAX;
            s.a_val[t] = __longlong_as_double((long long)kInfBits);
        }
    }
    __syncwarp();

    // ---- sort by row and merge duplicates (driver_local.cpp:511-568)
    if (global) radix_sort_rv(s, total, hist, lane);
    else sort_row_value(s.a_row, s.a_val, P, lane);
    int m = 0;
    const unsigned lt_mask = (1u << lane) - 1u;
    for (int base = 0; base < total; base += kWarp) {
        int i = base + lane;
        bool valid = i < total;
        int32_t ri = valid ? s.a_row[i] : INT_MAX;
        bool head = valid && (i == 0 || s.a_row[i - 1] != ri);
        unsigned bal = __ballot_sync(kFull, head);
        if (head) {
            int rank = m + __popc(bal & lt_mask);
            double acc = s.a_val[i];
            int cnt = 1;
            if (global) {
                // runs in global slabs: read 8 entries per round trip, add in order
                bool more = true;
                for (int j0 = i + 1; more && j0 < total; j0 += 8) {
                    int32_t rr[8];
                    double vv[8];
#pragma unroll
                    for (int q = 0; q < 8; ++q) {
                        rr[q] = j0 + q < total ? s.a_row[j0 + q] : -1;
                        vv[q] = j0 + q < total ? s.a_val[j0 + q] : 0.0;
                    }
#pragma unroll
                    for (int q = 0; q < 8; ++q) {
                        if (more && rr[q] == ri) {
                            acc = __dadd_rn(acc, vv[q]);
                            ++cnt;
                        } else {
                            more = false;
                        }
                    }
                }
            } else {
                for (int j = i + 1; j < total && s.a_row[j] == ri; ++j) {
                    acc = __dadd_rn(acc, s.a_val[j]);
                    ++cnt;
                }
            }
            s.b_val[rank] = acc;
            s.b_row[rank] = ri;
            s.b_aux[rank] = ((long long)cnt << 32) | (long long)rank;
        }
        m += __popc(bal);
    }
    const int P2 = pow2_at_least(m);
    if (!global) {
        for (int t = m + lane; t < P2; t += kWarp) {
            s.b_val[t] = __longlong_as_double((long long)kInfBits);
            s.b_row[t] = INT_MAX;
            s.b_aux[t] = 0;
        }
    }
    __syncwarp();

    // ---- sort by value, chunked prefix sum (driver_local.cpp:573-593)
    if (global) radix_sort_vr(s, m, hist, lane);
    else sort_value_row(s.b_val, s.b_row, s.b_aux, P2, lane);
    double carry = 0.0;
    for (int c0 = 0; c0 < m; c0 += kWarp) {
        double v = (c0 + lane < m) ? s.b_val[c0 + lane] : 0.0;
#pragma unroll
        for (int off = 1; off < kWarp; off <<= 1) {
            double t = __shfl_up_sync(kFull, v, off);
            if (lane >= off) v = __dadd_rn(v, t);
        }
        double f = (c0 == 0) ? v : __dadd_rn(carry, v);
        if (c0 + lane < m) s.a_val[c0 + lane] = f;
        carry = __shfl_sync(kFull, f, kWarp - 1);
    }
    __syncwarp();
    const double S = s.a_val[m - 1];

    // ---- L column k into the pool (row order), D_k
    int64_t pbase = 0;
    if (!pool_take(a, m, lane, pool_cur, pool_end, pbase)) {
        if (lane == 0) fail(a, kDevCapacity);
        return false;
    }
    fills += m - 1;
    if (lane == 0) {
        a.diag[k] = S;
        a.pstart[k] = pbase;
        a.pcnt[k] = m;
    }
    for (int i = lane; i < m; i += kWarp) {
        int p = (int)(s.b_aux[i] & 0xffffffffll);
        a.prow[pbase + p] = s.b_row[i];
        a.pval[pbase + p] = __ddiv_rn(s.b_val[i], S);
    }

    // ---- clique sampling (driver_local.cpp:598-631, auxilliary.hpp:543-592)
    // Global slabs first search a shared-memory copy of every q-th prefix
    // sum (all of them when they fit), then the at most q entries between
    // two copies; the predicate is monotone in j, so the first j found is
    // the same as a plain binary search's.
    const double* C = s.a_val;
    const double* cidx = reinterpret_cast<const double*>(wsm + 1024);
    int q = 1, nidx = 0;
    if (global) {
        double* ci_w = reinterpret_cast<double*>(wsm + 1024);
        const int cap = (a.smem_region - 1024) / 8;
        while ((m + q - 1) / q > cap) q <<= 1;
        nidx = (m + q - 1) / q;
        for (int t = lane; t < nidx; t += kWarp) ci_w[t] = s.a_val[t * q];
        __syncwarp();
        if (q == 1) C = cidx;
    }
    bool ok = true;
    for (int i = lane; i < m - 1; i += kWarp) {
        const double ci = C[i];
        const double rem_i = __dsub_rn(S, ci);
        const double target = __dmul_rn(sample_uniform(a.seed, k, i), rem_i);
        int lo = i + 1, hi = m;
        if (q > 1) {
            int tl = (lo + q - 1) / q, th = nidx;
            const int tfirst = tl;
            while (tl < th) {
                const int mid = (tl + th) >> 1;
                if (__dsub_rn(cidx[mid], ci) < target) tl = mid + 1;
                else th = mid;
            }
            if (tl < nidx) hi = tl * q + 1;
            if (tl > tfirst) lo = max(lo, (tl - 1) * q + 1);
        }
        while (lo < hi) {
            int mid = lo + ((hi - lo) >> 1);
            if (__dsub_rn(C[mid], ci) < target) lo = mid + 1;
            else hi = mid;
        }
        const int j = lo < m ? lo : m - 1;
        const int32_t r_i = s.b_row[i], r_j = s.b_row[j];
        const int32_t grow = r_i > r_j ? r_i : r_j;
        const int32_t gcol = r_i > r_j ? r_j : r_i;
        const double gval = __ddiv_rn(__dmul_rn(s.b_val[i], rem_i), S);
        if (!append_fill(a, gcol, grow, gval)) ok = false;
        atomicAdd(a.dep + grow, 1);
    }
    if (__any_sync(kFull, !ok)) {
        if (lane == 0) fail(a, kDevCapacity);
        return false;
    }
    // row r of L depends on column k: level[r] >= level[k] + 1.  level[k]
    // is final here: every column with an entry in row k was eliminated
    // before k was released.
    const int lk = lvl + 1;
    // fills, pool writes and levels must be visible before any neighbour is
    // released
    __threadfence();
    __syncwarp();
    for (int base = 0; base < m; base += kWarp) {
        const int i = base + lane;
        const bool valid = i < m;
        release_chunk(a, lk, lane, valid, valid ? s.b_row[i] : -1, valid ? (int)(s.b_aux[i] >> 32) : 0, next);
    }
    __syncwarp();
    return true;
}

// at most 85 registers (3 CTAs per SM): the rare large-vertex paths spill
// rather than costing the common path its occupancy
__global__ void __launch_bounds__(256, 3) factor_kernel(FactorArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = threadIdx.x & (kWarp - 1);
    const int wib = threadIdx.x >> 5;
    const int warp_global = blockIdx.x * (blockDim.x >> 5) + wib;
    unsigned char* wsm = smem + (size_t)wib * (size_t)a.smem_region;
    Slab sm = make_slab(wsm, a.smem_slab);
    const unsigned long long t0 = global_timer_ns();
    int64_t pool_cur = 0, pool_end = 0;
    long long fills = 0;
    int32_t next = -1;
    int max_gather = 0;
    int done_local = 0;  // eliminations not yet added to the global count
    while (true) {
        int k = next;
        next = -1;
        if (k < 0) {
            // publish finished work before waiting: other warps end their
            // waits once the global count reaches n
            if (lane == 0 && done_local) atomicAdd(a.counters + kDone, done_local);
            done_local = 0;
            // pop: reserve the next queue slot and wait for its vertex.  A
            // slot may never be filled (vertices released to the warp that
            // freed them skip the queue), so the wait also ends once every
            // vertex has been eliminated.
            int idx = 0;
            if (lane == 0) idx = atomicAdd(a.counters + kQHead, 1);
            idx = __shfl_sync(kFull, idx, 0);
            if (idx >= a.n) break;
            if (lane == 0) {
                // the limit bounds a wait without progress: it restarts
                // whenever the count of eliminated vertices moves
                unsigned spins = 0;
                int seen = -1;
                unsigned long long since = t0;
                while ((k = ld_acquire(a.queue + idx)) < 0) {
                    if ((++spins & 63u) == 0) {
                        const int done = ld_relaxed(a.counters + kDone);
                        if (done >= a.tail || aborted(a)) break;
                        const unsigned long long now = global_timer_ns();
                        if (done != seen) {
                            seen = done;
                            since = now;
                        } else if (now - since > a.timeout_ns) {
                            fail(a, kDevTimeout);
                            break;
                        }
                    }
                }
            }
            k = __shfl_sync(kFull, k, 0);
            if (k < 0) break;
        }
        if (k >= a.tail) continue;  // left to the cooperative tail pass
        __threadfence();
        if (!eliminate(a, k, sm, wsm, warp_global, lane, pool_cur, pool_end, fills, next, max_gather)) break;
        ++done_local;
        if (aborted(a)) break;
    }
    if (lane == 0 && done_local) atomicAdd(a.counters + kDone, done_local);
    if (lane == 0 && max_gather) atomicMax(a.counters + kMaxGather, max_gather);
    if (lane == 0 && fills) atomicAdd(a.pool_cursor + 1, (unsigned long long)fills);
}

// ---- cooperative elimination of the tail -----------------------------------
// The last vertices of a power-law graph (hubs and the dense core) depend
// on one another in long chains and gather thousands of entries each; a
// warp per vertex leaves the rest of the GPU idle while it sorts.  Vertices
// >= tail are therefore eliminated after factor_kernel by nhuge CTAs of
// kTailThreads threads, a whole CTA per vertex.  A CTA claims the next
// vertex in index order and waits on its dependency counter (every
// dependency has a smaller index, hence was claimed earlier by a running
// CTA), then keeps the counters as factor_kernel does: +1 per fill row,
// -multiplicity per neighbour once the column is written.  The steps
// and their rounding are those of eliminate_slab<true> -- the same radix
// orders, duplicate runs added in sorted order, 32-wide Kogge-Stone chunks
// with the carry chained in chunk order, the same sampling search -- so the
// factor is bit-identical to the warp path's (and the oracle's).

constexpr int kTailThreads = 1024;
constexpr int kTailWarps = kTailThreads / kWarp;
// shared memory of the tail kernel: per-warp digit histograms, 256 totals
// (+ a flag), warp offsets, padded to an even word count; then a copy of up
// to kTailCdfCap prefix sums for the sampling searches
constexpr int kTailIntWords = kTailWarps * 256 + 260 + 36;
constexpr int kTailCdfCap = 20480;
static_assert(kTailIntWords % 2 == 0, "the prefix-sum copy must be 8-byte aligned");

// One stable CTA pass of (row, val[, aux]) by digit d: warp w takes a
// contiguous tile (a multiple of 32 entries), counts, and scatters it in
// order through digit-major, warp-minor offsets.  Returns false when one
// digit holds all n entries (nothing would move; nothing is written).
template <bool VR, bool AUX>
__device__ bool tail_radix_pass(const int32_t* row, const double* val, const long long* aux, int32_t* orow,
                                double* oval, long long* oaux, int n, int d, int* hist, int* tot) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int tile = ((n + kTailWarps - 1) / kTailWarps + 31) & ~31;
    const int t0 = min(n, w * tile), t1 = min(n, t0 + tile);
    int* h = hist + w * 256;
    for (int i = lane; i < 256; i += kWarp) h[i] = 0;
    __syncwarp();
    for (int base = t0; base < t1; base += kRadixRounds * kWarp) {
        int dig[kRadixRounds];
#pragma unroll
        for (int q = 0; q < kRadixRounds; ++q) {
            const int i = base + q * kWarp + lane;
            dig[q] = i < t1 ? (VR ? vr_digit(row[i], val[i], d) : rv_digit(row[i], val[i], d)) : -1;
        }
#pragma unroll
        for (int q = 0; q < kRadixRounds; ++q)
            if (dig[q] >= 0) atomicAdd(&h[dig[q]], 1);
    }
    __syncthreads();
    if (threadIdx.x < 256) {
        int c = 0;
        for (int q = 0; q < kTailWarps; ++q) c += hist[q * 256 + threadIdx.x];
        tot[threadIdx.x] = c;
    }
    __syncthreads();
    if (w == 0) {
        // exclusive scan of the 256 totals: 8 digits per lane, then the lanes
        int c[8], sum = 0, one = 0;
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            c[q] = tot[8 * lane + q];
            sum += c[q];
            one |= c[q] == n;
        }
        int incl = sum;
#pragma unroll
        for (int o = 1; o < kWarp; o <<= 1) {
            const int t = __shfl_up_sync(kFull, incl, o);
            if (lane >= o) incl += t;
        }
        int run = incl - sum;
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            tot[8 * lane + q] = run;
            run += c[q];
        }
        one = __any_sync(kFull, one != 0) ? 1 : 0;
        if (lane == 0) tot[256] = one;
    }
    __syncthreads();
    const bool skip = tot[256] != 0;
    if (!skip && threadIdx.x < 256) {
        int run = tot[threadIdx.x];
        for (int q = 0; q < kTailWarps; ++q) {
            const int c = hist[q * 256 + threadIdx.x];
            hist[q * 256 + threadIdx.x] = run;
            run += c;
        }
    }
    __syncthreads();
    if (skip) return false;
    const unsigned lt = (1u << lane) - 1u;
    for (int base = t0; base < t1; base += kRadixRounds * kWarp) {
        int32_t r[kRadixRounds];
        double v[kRadixRounds];
        long long x[kRadixRounds];
#pragma unroll
        for (int q = 0; q < kRadixRounds; ++q) {
            const int i = base + q * kWarp + lane;
            r[q] = 0;
            v[q] = 0.0;
            x[q] = 0;
            if (i < t1) {
                r[q] = row[i];
                v[q] = val[i];
                if (AUX) x[q] = aux[i];
            }
        }
#pragma unroll
        for (int q = 0; q < kRadixRounds; ++q) {
            const bool valid = base + q * kWarp + lane < t1;
            const int dig = valid ? (VR ? vr_digit(r[q], v[q], d) : rv_digit(r[q], v[q], d)) : 256;
            const unsigned peers = __match_any_sync(kFull, dig);
            const int rank = __popc(peers & lt);
            const int at = valid ? h[dig] + rank : 0;
            __syncwarp();
            if (valid && rank == 0) h[dig] += __popc(peers);
            __syncwarp();
            if (valid) {
                orow[at] = r[q];
                oval[at] = v[q];
                if (AUX) oaux[at] = x[q];
            }
        }
    }
    __syncthreads();
    return true;
}

template <bool VR, bool AUX>
__device__ void tail_radix_sort(int32_t* r_out, double* v_out, long long* x_out, int32_t* r_tmp, double* v_tmp,
                                long long* x_tmp, int n, int dlo, int dhi, int* hist, int* tot) {
    int32_t *r0 = r_out, *r1 = r_tmp;
    double *v0 = v_out, *v1 = v_tmp;
    long long *x0 = x_out, *x1 = x_tmp;
    for (int d = dlo; d < dhi; ++d) {
        if (!tail_radix_pass<VR, AUX>(r0, v0, x0, r1, v1, x1, n, d, hist, tot)) continue;
        int32_t* tr = r0;
        r0 = r1;
        r1 = tr;
        double* tv = v0;
        v0 = v1;
        v1 = tv;
        long long* tx = x0;
        x0 = x1;
        x1 = tx;
    }
    if (r0 != r_out) {
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            r_out[i] = r0[i];
            v_out[i] = v0[i];
            if (AUX) x_out[i] = x0[i];
        }
        __syncthreads();
    }
}

// Exclusive count of the flagged entries before each warp's tile, for an
// order-preserving compaction (warp w holds the tile as in the radix passes).
__device__ __forceinline__ int tail_tile_offset(int count, int* scan) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) scan[w] = count;
    __syncthreads();
    if (threadIdx.x == 0) {
        int run = 0;
        for (int q = 0; q < kTailWarps; ++q) {
            const int c = scan[q];
            scan[q] = run;
            run += c;
        }
        scan[kTailWarps] = run;
    }
    __syncthreads();
    return scan[w];
}

__global__ void __launch_bounds__(kTailThreads, 1) factor_tail_kernel(FactorArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    int* hist = reinterpret_cast<int*>(smem);      // [kTailWarps][256]
    int* tot = hist + kTailWarps * 256;            // [257]
    int* scan = tot + 260;                         // [kTailWarps + 1]
    __shared__ long long sh_base;
    __shared__ int sh_stop;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const unsigned lt = (1u << lane) - 1u;
    long long fills = 0;
    int max_gather = 0;
    __shared__ int32_t sh_k;
    if (threadIdx.x == 0) sh_stop = 0;
    __syncthreads();
    // CTA b works in huge slab b (the persistent kernel, which shares them
    // under locks, has finished)
    Slab s = make_global_slab(a.hscratch + (size_t)blockIdx.x * (size_t)a.hscratch_entries * kGlobalSlabBytes,
                              (int)a.hscratch_entries);
    const unsigned long long t0 = global_timer_ns();
    while (true) {
        // claim the next tail vertex in index order and wait until every
        // column it depends on is eliminated (all have lower indices, so
        // they were claimed earlier by running CTAs); the wait is bounded
        // by time without progress of the eliminated count
        if (threadIdx.x == 0) {
            int32_t k = a.tail + atomicAdd(a.counters + kTailTicket, 1);
            if (k < a.n) {
                unsigned spins = 0;
                int seen = -1;
                unsigned long long since = t0;
                while (ld_acquire(a.dep + k) > 0) {
                    if ((++spins & 63u) == 0) {
                        if (aborted(a)) {
                            k = a.n;
                            break;
                        }
                        const int d = ld_relaxed(a.counters + kDone);
                        const unsigned long long now = global_timer_ns();
                        if (d != seen) {
                            seen = d;
                            since = now;
                        } else if (now - since > a.timeout_ns) {
                            fail(a, kDevTimeout);
                            k = a.n;
                            break;
                        }
                    }
                }
            }
            sh_k = k;
        }
        __syncthreads();
        const int32_t k = sh_k;
        if (k >= a.n) break;
        __threadfence();
        const int nf = ld_relaxed(a.fcnt + k);
        const int oc0 = a.lcolptr[k];
        const int ocnt = a.lcolptr[k + 1] - oc0;
        const int o0 = oc0 + min(ocnt, a.c0);
        const int no = ocnt - min(ocnt, a.c0);
        const int total = nf + no;
        if (a.gsize && threadIdx.x == 0) a.gsize[k] = total;
        if (total == 0) {
            if (threadIdx.x == 0) {
                a.diag[k] = 0.0;
                a.pcnt[k] = 0;
                a.pstart[k] = 0;
                atomicAdd(a.counters + kDone, 1);
            }
            __syncthreads();
            continue;
        }
        if (total > max_gather) max_gather = total;
        if ((int64_t)total > a.hscratch_entries) {
            if (threadIdx.x == 0) fail(a, kDevCapacity);
            break;
        }
        // ---- gather: bucket, overflow chunks, originals
        const int n0 = min(nf, a.c0);
        for (int t = threadIdx.x; t < n0; t += blockDim.x) {
            const size_t o = (size_t)k * (size_t)a.c0 + (size_t)t;
            s.a_row[t] = __ldcg(a.brow + o);
            s.a_val[t] = __ldcg(a.bval + o);
        }
        int rem = nf - n0, pos = n0;
        int chunk = rem > 0 ? ld_relaxed(a.chead + k) : -1;
        bool bad = false;
        for (int lvl = 0; rem > 0; ++lvl) {
            if (chunk < 0 || chunk > a.nchunks - (1 << lvl)) {
                bad = true;
                break;
            }
            const int cnt = min(rem, kChunk << lvl);
            for (int t = threadIdx.x; t < cnt; t += blockDim.x) {
                s.a_row[pos + t] = __ldcg(a.crow + (size_t)chunk * kChunk + t);
                s.a_val[pos + t] = __ldcg(a.cval + (size_t)chunk * kChunk + t);
            }
            pos += cnt;
            rem -= cnt;
            if (rem > 0) chunk = ld_relaxed(a.cnext + chunk);
        }
        if (bad) {
            if (threadIdx.x == 0) fail(a, kDevBadInput);
            break;
        }
        for (int t = threadIdx.x; t < no; t += blockDim.x) {
            s.a_row[nf + t] = a.lrow[o0 + t];
            s.a_val[nf + t] = a.lval[o0 + t];
        }
        __syncthreads();
        // ---- sort by (row, value bits); merge duplicate rows in that order
        tail_radix_sort<false, false>(s.a_row, s.a_val, nullptr, s.t_row, s.t_val, nullptr, total, 0, 12, hist, tot);
        const int tile = ((total + kTailWarps - 1) / kTailWarps + 31) & ~31;
        const int t0 = min(total, w * tile), t1 = min(total, t0 + tile);
        int heads = 0;
        for (int base = t0; base < t1; base += kWarp) {
            const int i = base + lane;
            const bool head = i < t1 && (i == 0 || s.a_row[i - 1] != s.a_row[i]);
            heads += __popc(__ballot_sync(kFull, head));
        }
        int m0 = tail_tile_offset(heads, scan);
        const int m = scan[kTailWarps];
        for (int base = t0; base < t1; base += kWarp) {
            const int i = base + lane;
            const bool valid = i < t1;
            const int32_t ri = valid ? s.a_row[i] : INT_MAX;
            const bool head = valid && (i == 0 || s.a_row[i - 1] != ri);
            const unsigned bal = __ballot_sync(kFull, head);
            if (head) {
                const int rank = m0 + __popc(bal & lt);
                double acc = s.a_val[i];
                int cnt = 1;
                for (int j = i + 1; j < total && s.a_row[j] == ri; ++j) {
                    acc = __dadd_rn(acc, s.a_val[j]);
                    ++cnt;
                }
                s.b_val[rank] = acc;
                s.b_row[rank] = ri;
                s.b_aux[rank] = ((long long)cnt << 32) | (long long)rank;
            }
            m0 += __popc(bal);
        }
        __syncthreads();
        // ---- sort by value (input in row order: the value bytes suffice)
        tail_radix_sort<true, true>(s.b_row, s.b_val, s.b_aux, s.t_row, s.t_val, s.t_aux, m, 4, 12, hist, tot);
        // ---- prefix sums: 32-wide Kogge-Stone chunks (warp c % 32 takes
        // chunk c), the chunk totals in t_val; then the carries chained in
        // chunk order by one thread, as the warp path carries them
        const int nchunk = (m + kWarp - 1) / kWarp;
        for (int c = w; c < nchunk; c += kTailWarps) {
            const int i = c * kWarp + lane;
            double v = i < m ? s.b_val[i] : 0.0;
#pragma unroll
            for (int off = 1; off < kWarp; off <<= 1) {
                const double t = __shfl_up_sync(kFull, v, off);
                if (lane >= off) v = __dadd_rn(v, t);
            }
            if (i < m) s.a_val[i] = v;
            if (lane == kWarp - 1) s.t_val[c] = v;
        }
        __syncthreads();
        if (w == 0) {
            // t_val[c] becomes the carry into chunk c (c >= 1): one lane adds
            // the totals in chunk order, 32 at a time read into registers
            double carry = 0.0;
            for (int c0 = 0; c0 < nchunk; c0 += kWarp) {
                const double tl = c0 + lane < nchunk ? s.t_val[c0 + lane] : 0.0;
                double cin = 0.0;
                for (int q = 0; q < kWarp && c0 + q < nchunk; ++q) {
                    const double tq = __shfl_sync(kFull, tl, q);
                    if (lane == q) cin = carry;  // carry into chunk c0 + q
                    carry = (c0 + q == 0) ? tq : __dadd_rn(carry, tq);
                }
                if (c0 + lane < nchunk) s.t_val[c0 + lane] = cin;
            }
        }
        __syncthreads();
        for (int i = kWarp + threadIdx.x; i < m; i += blockDim.x) s.a_val[i] = __dadd_rn(s.t_val[i / kWarp], s.a_val[i]);
        __syncthreads();
        const double S = s.a_val[m - 1];
        // ---- L column k into the pool (row order), D_k
        if (threadIdx.x == 0) {
            const unsigned long long got = atomicAdd(a.pool_cursor, (unsigned long long)m);
            sh_base = (long long)got;
            if ((int64_t)got + m > a.pool_cap) {
                fail(a, kDevCapacity);
                sh_stop = 1;
            } else {
                a.diag[k] = S;
                a.pstart[k] = (int64_t)got;
                a.pcnt[k] = m;
            }
        }
        __syncthreads();
        if (sh_stop) break;
        const int64_t pbase = sh_base;
        fills += m - 1;
        for (int i = threadIdx.x; i < m; i += blockDim.x) {
            const int p = (int)(s.b_aux[i] & 0xffffffffll);
            a.prow[pbase + p] = s.b_row[i];
            a.pval[pbase + p] = __ddiv_rn(s.b_val[i], S);
        }
        // ---- clique sampling (the same search predicate as the warp path),
        // searching a shared-memory copy of the prefix sums when it fits
        const double* C = s.a_val;
        if (m <= a.tail_cdf_cap) {
            double* cs = reinterpret_cast<double*>(smem + sizeof(int) * kTailIntWords);
            for (int i = threadIdx.x; i < m; i += blockDim.x) cs[i] = s.a_val[i];
            __syncthreads();
            C = cs;
        }
        bool ok = true;
        for (int i = threadIdx.x; i < m - 1; i += blockDim.x) {
            const double ci = C[i];
            const double rem_i = __dsub_rn(S, ci);
            const double target = __dmul_rn(sample_uniform(a.seed, k, i), rem_i);
            int lo = i + 1, hi = m;
            while (lo < hi) {
                const int mid = lo + ((hi - lo) >> 1);
                if (__dsub_rn(C[mid], ci) < target) lo = mid + 1;
                else hi = mid;
            }
            const int j = lo < m ? lo : m - 1;
            const int32_t r_i = s.b_row[i], r_j = s.b_row[j];
            const int32_t grow = r_i > r_j ? r_i : r_j;
            const int32_t gcol = r_i > r_j ? r_j : r_i;
            const double gval = __ddiv_rn(__dmul_rn(s.b_val[i], rem_i), S);
            if (!append_fill(a, gcol, grow, gval)) ok = false;
            atomicAdd(a.dep + grow, 1);
        }
        // rows of L column k are one level below k (the solve schedules)
        const int lk = ld_relaxed(a.level + k) + 1;
        for (int i = threadIdx.x; i < m; i += blockDim.x) atomicMax(a.level + s.b_row[i], lk);
        if (__syncthreads_or(!ok)) {
            if (threadIdx.x == 0) fail(a, kDevCapacity);
            break;
        }
        // fills, pool writes and levels visible before any neighbour is
        // released: each neighbour's counter drops by its multiplicity
        __threadfence();
        __syncthreads();
        for (int i = threadIdx.x; i < m; i += blockDim.x)
            atom_add_acq_rel(a.dep + s.b_row[i], -(int)(s.b_aux[i] >> 32));
        if (threadIdx.x == 0) atomicAdd(a.counters + kDone, 1);
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        atomicMax(a.counters + kMaxGather, max_gather);
        atomicAdd(a.pool_cursor + 1, (unsigned long long)fills);
    }
}

size_t tail_smem_bytes() { return sizeof(int) * (size_t)kTailIntWords + sizeof(double) * (size_t)kTailCdfCap; }

// ---- setup kernels --------------------------------------------------------

// The first c0 strict-lower entries of each column go into its fill bucket
// (fcnt = their count), so that a vertex's gather usually reads one place.
// A thread per column (stencil columns hold a few entries); the cost is the
// bucket writes, a few entries into each column's own c0-slot row.
__global__ void prefill_bucket_kernel(int32_t n, int c0, const int32_t* __restrict__ lcolptr,
                                      const int32_t* __restrict__ lrow, const double* __restrict__ lval,
                                      int32_t* fcnt, int32_t* brow, double* bval) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += stride) {
        const int s = lcolptr[c];
        const int cnt = min(lcolptr[c + 1] - s, c0);
        int32_t* br = brow + (size_t)c * (size_t)c0;
        double* bv = bval + (size_t)c * (size_t)c0;
#pragma unroll 4
        for (int t = 0; t < cnt; ++t) {
            br[t] = lrow[s + t];
            bv[t] = lval[s + t];
        }
        fcnt[c] = cnt;
    }
}

// Per column: entries below the diagonal (lower_cnt) and above it (dep,
// count_minimum_dependencies, pre_process.hpp:474-496).  Columns with at
// most kLaneCol entries are handled by one lane each (32 columns per warp in
// flight); longer ones by the whole warp, one at a time.  Columns longer than
// kHugeCol (a ground vertex joined to every row with a diagonal excess, say)
// would keep one warp busy for thousands of round trips, so they go to a
// list (list[0] = count, then column ids; at most kHugeColCap, the rest stay
// with their warp) with zero counts, and count_huge_kernel adds them up
// with the whole grid.
constexpr int kLaneCol = 32;

__global__ void count_lower_kernel(int32_t n, const int32_t* __restrict__ colptr,
                                   const int32_t* __restrict__ rowind, int32_t* lower_cnt, int32_t* dep,
                                   int32_t* huge) {
    const int lane = threadIdx.x & 31;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t c0 = (((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 32; c0 < n; c0 += nw * 32) {
        const int64_t c = c0 + lane;
        const bool have = c < n;
        const int s = have ? colptr[c] : 0, e = have ? colptr[c + 1] : 0;
        const bool wide = e - s > kLaneCol;
        int lo = 0, up = 0;
        if (!wide) {
#pragma unroll 4
            for (int p = s; p < e; ++p) {
                const int r = rowind[p];
                lo += r > c;
                up += r < c;
            }
        }
        for (unsigned lb = __ballot_sync(kFull, wide); lb; lb &= lb - 1u) {
            const int src = __ffs(lb) - 1;
            const int cs = __shfl_sync(kFull, s, src), ce = __shfl_sync(kFull, e, src);
            const int64_t cc = c0 + src;
            int l2 = 0, u2 = 0;
            int slot = kHugeColCap;
            if (ce - cs > kHugeCol) {
                if (lane == 0) slot = atomicAdd(huge, 1);
                slot = __shfl_sync(kFull, slot, 0);
                if (slot < kHugeColCap && lane == 0) huge[1 + slot] = (int32_t)cc;
            }
            for (int p0 = cs + lane; slot >= kHugeColCap && p0 < ce; p0 += 8 * 32) {
                int r[8];
#pragma unroll
                for (int q = 0; q < 8; ++q) r[q] = p0 + 32 * q < ce ? rowind[p0 + 32 * q] : (int)cc;
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    l2 += r[q] > cc;
                    u2 += r[q] < cc;
                }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                l2 += __shfl_xor_sync(kFull, l2, o);
                u2 += __shfl_xor_sync(kFull, u2, o);
            }
            if (lane == src) {
                lo = l2;
                up = u2;
            }
        }
        if (have) {
            lower_cnt[c] = lo;
            if (dep) dep[c] = up;
        }
    }
}

// The listed long columns, each spread over every thread of the grid; one
// atomic add per block and column onto the zero counts count_lower_kernel
// left (integer sums: the result does not depend on the order).
__global__ void count_huge_kernel(const int32_t* __restrict__ colptr, const int32_t* __restrict__ rowind,
                                  const int32_t* __restrict__ huge, int32_t* lower_cnt, int32_t* dep) {
    __shared__ int red[2][32];
    const int nh = min(huge[0], kHugeColCap);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int q = 0; q < nh; ++q) {
        const int32_t c = huge[1 + q];
        const int64_t s = colptr[c], e = colptr[c + 1];
        int lo = 0, up = 0;
        for (int64_t p = s + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < e; p += stride) {
            const int r = rowind[p];
            lo += r > c;
            up += r < c;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            lo += __shfl_xor_sync(kFull, lo, o);
            up += __shfl_xor_sync(kFull, up, o);
        }
        if (lane == 0) {
            red[0][warp] = lo;
            red[1][warp] = up;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            int tl = 0, tu = 0;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
                tl += red[0][w];
                tu += red[1][w];
            }
            if (tl) atomicAdd(lower_cnt + c, tl);
            if (dep && tu) atomicAdd(dep + c, tu);
        }
        __syncthreads();
    }
}

// Strict lower triangle with |values|, original order within each column
// (make_lower_triangular, pre_process.hpp:785-867).
__global__ void scatter_lower_kernel(int32_t n, const int32_t* __restrict__ colptr,
                                     const int32_t* __restrict__ rowind, const double* __restrict__ val,
                                     const int32_t* __restrict__ lcolptr, int32_t* lrow, double* lval) {
    const int lane = threadIdx.x & 31;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t c0 = (((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 32; c0 < n; c0 += nw * 32) {
        const int64_t c = c0 + lane;
        const bool have = c < n;
        const int s = have ? colptr[c] : 0, e = have ? colptr[c + 1] : 0;
        const int o = have ? lcolptr[c] : 0;
        const int cnt = have ? lcolptr[c + 1] - o : 0;
        // nothing to take (the ground column) or everything (a plain copy)
        const bool wide = e - s > kLaneCol && cnt > 0;
        if (!wide && cnt > 0) {
            int out = o;
#pragma unroll 4
            for (int p = s; p < e; ++p) {
                const int r = rowind[p];
                if (r > c) {
                    lrow[out] = r;
                    lval[out] = fabs(val[p]);
                    ++out;
                }
            }
        }
        for (unsigned lb = __ballot_sync(kFull, wide); lb; lb &= lb - 1u) {
            const int src = __ffs(lb) - 1;
            const int cs = __shfl_sync(kFull, s, src), ce = __shfl_sync(kFull, e, src);
            const int64_t cc = c0 + src;
            int out = __shfl_sync(kFull, o, src);
            if (__shfl_sync(kFull, cnt, src) == ce - cs) {
                for (int p = cs + lane; p < ce; p += 32) {
                    lrow[out + p - cs] = rowind[p];
                    lval[out + p - cs] = fabs(val[p]);
                }
                continue;
            }
            for (int base = cs; base < ce; base += 32) {
                const int p = base + lane;
                const bool take = p < ce && rowind[p] > cc;
                const unsigned bal = __ballot_sync(kFull, take);
                if (take) {
                    const int at = out + __popc(bal & ((1u << lane) - 1u));
                    lrow[at] = rowind[p];
                    lval[at] = fabs(val[p]);
                }
                out += __popc(bal);
            }
        }
    }
}

__global__ void init_queue_kernel(int32_t n, const int32_t* __restrict__ dep, int32_t* queue,
                                  int32_t* counters) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t base = (int64_t)blockIdx.x * blockDim.x; base < n; base += stride) {
        int64_t i = base + threadIdx.x;
        bool ready = i < n && dep[i] == 0;
        unsigned bal = __ballot_sync(kFull, ready);
        int lane = threadIdx.x & 31;
        int pos = 0;
        if (lane == 0 && bal) pos = atomicAdd(counters + kQTail, __popc(bal));
        pos = __shfl_sync(kFull, pos, 0);
        if (ready) queue[pos + __popc(bal & ((1u << lane) - 1u))] = (int32_t)i;
    }
}

}  // namespace

// ---------------------------------------------------------------------------

// count_lower_kernel, then count_huge_kernel for the long columns it listed
// in `huge` (kHugeColCap + 1 words of scratch).
static cudaError_t count_lower(const DevCsc& A, int32_t* lower_cnt, int32_t* dep, int32_t* huge, cudaStream_t s) {
    cudaError_t e = cudaMemsetAsync(huge, 0, sizeof(int32_t), s);
    if (e != cudaSuccess) return e;
    count_lower_kernel<<<grid_for(A.n, 256), 256, 0, s>>>(A.n, A.colptr, A.rowind, lower_cnt, dep, huge);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    count_huge_kernel<<<2 * current_sm_count(), 256, 0, s>>>(A.colptr, A.rowind, huge, lower_cnt, dep);
    return cudaGetLastError();
}

cudaError_t launch_count_lower(const DevCsc& A, int32_t* lower_cnt, int32_t* huge, cudaStream_t s) {
    return count_lower(A, lower_cnt, nullptr, huge, s);
}

cudaError_t launch_lower_and_deps(const DevCsc& A, FactorWork& w, cudaStream_t s) {
    // lower counts go to w.pcnt (scratch), dependency counts to w.dep
    cudaError_t e = count_lower(A, w.pcnt, w.dep, w.hcols, s);
    if (e != cudaSuccess) return e;
    e = exclusive_scan_i32_to_i32(w.pcnt, w.lcolptr, A.n, w.scan_tmp, s);
    if (e != cudaSuccess) return e;
    scatter_lower_kernel<<<grid_for(A.n, 256), 256, 0, s>>>(A.n, A.colptr, A.rowind, A.val, w.lcolptr, w.lrow,
                                                             w.lval);
    return cudaGetLastError();
}

cudaError_t launch_init_factor_state(FactorWork& w, cudaStream_t s) {
    cudaError_t e;
    if ((e = cudaMemsetAsync(w.fcnt, 0, sizeof(int32_t) * (size_t)w.n, s)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(w.chead, 0xff, sizeof(int32_t) * (size_t)w.n, s)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(w.cnext, 0xff, sizeof(int32_t) * (size_t)w.nchunks, s)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(w.queue, 0xff, sizeof(int32_t) * (size_t)w.n, s)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(w.level, 0, sizeof(int32_t) * (size_t)w.n, s)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(w.counters, 0, sizeof(int32_t) * 16, s)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(w.counters64, 0, sizeof(unsigned long long) * 4, s)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(w.hlock, 0, sizeof(int32_t) * w.nhuge, s)) != cudaSuccess) return e;
    prefill_bucket_kernel<<<grid_for(w.n, 256), 256, 0, s>>>(w.n, w.c0, w.lcolptr, w.lrow, w.lval,
                                                                            w.fcnt, w.brow, w.bval);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    init_queue_kernel<<<grid_for(w.n, 256), 256, 0, s>>>(w.n, w.dep, w.queue, w.counters);
    return cudaGetLastError();
}

// per warp: the shared-memory slab, at least 2 KB (radix histogram + CDF index of global slabs)
static int smem_region_bytes(int smem_slab) { return (smem_slab > 64 ? smem_slab : 64) * kSlabBytesPerEntry; }

size_t factor_smem_bytes(int block, int smem_slab) {
    return (size_t)(block / kWarp) * (size_t)smem_region_bytes(smem_slab);
}

int factor_resident_grid(int block, int smem_slab, int device) {
    size_t smem = factor_smem_bytes(block, smem_slab);
    cudaFuncSetAttribute(factor_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, factor_kernel, block, smem) != cudaSuccess)
        return 0;
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    return per_sm * sms;
}

cudaError_t launch_factor(FactorWork& w, const FactorLaunch& cfg, cudaStream_t s) {
    FactorArgs a;
    a.n = w.n;
    a.lcolptr = w.lcolptr;
    a.lrow = w.lrow;
    a.lval = w.lval;
    a.dep = w.dep;
    a.queue = w.queue;
    a.c0 = w.c0;
    a.fcnt = w.fcnt;
    a.brow = w.brow;
    a.bval = w.bval;
    a.chead = w.chead;
    a.cnext = w.cnext;
    a.crow = w.crow;
    a.cval = w.cval;
    a.nchunks = w.nchunks;
    a.pool_cap = w.pool_cap;
    a.prow = w.prow;
    a.pval = w.pval;
    a.pstart = w.pstart;
    a.pcnt = w.pcnt;
    a.diag = w.diag;
    a.level = w.level;
    a.gscratch = w.gscratch;
    a.gscratch_entries = w.gscratch_entries;
    a.hscratch = w.hscratch;
    a.hscratch_entries = w.hscratch_entries;
    a.nhuge = w.nhuge;
    a.hlock = w.hlock;
    a.counters = w.counters;
    a.pool_cursor = w.counters64;
    a.seed = cfg.seed;
    a.smem_slab = cfg.smem_slab;
    a.smem_region = smem_region_bytes(cfg.smem_slab);
    a.timeout_ns = (unsigned long long)(cfg.timeout_s * 1e9);
    a.tail = cfg.tail > 0 && cfg.tail < w.n ? w.n - cfg.tail : w.n;
    a.tail_cdf_cap = kTailCdfCap;
    a.gsize = cfg.gsize;
    size_t smem = factor_smem_bytes(cfg.block, cfg.smem_slab);
    cudaError_t e = cudaFuncSetAttribute(factor_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    factor_kernel<<<cfg.grid, cfg.block, smem, s>>>(a);
    RCHOL_TRY(cudaGetLastError());
    if (a.tail < w.n) {
        // the tail after the rest is eliminated: one CTA per shared slab,
        // each a vertex at a time, claimed in index order
        const size_t tsmem = tail_smem_bytes();
        RCHOL_TRY(cudaFuncSetAttribute(factor_tail_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tsmem));
        factor_tail_kernel<<<w.nhuge, kTailThreads, tsmem, s>>>(a);
        RCHOL_TRY(cudaGetLastError());
    }
    return cudaSuccess;
}

}  // namespace rchol
