// Factor assembly (driver.cu:1309-1548, 1743-1872; driver_physics.cu:1594-1738;
// experiment/driver_local.cpp:880-956): the elimination pool becomes
//   Lc  strict CSC of L  (rows ascending in each column, L_ij = -w/sum),
//   Lr  strict CSR of L  (columns ascending in each row),
//   D   the pivots,
// with the ground vertex (the last one) removed when the input was an SDDM
// converted to a Laplacian.  FP32 copies feed the mixed-precision solve.
#include <algorithm>
#include <climits>

#include "device_common.cuh"
#include "rchol_internal.h"

namespace rchol {

namespace {

constexpr int kSortSlab = 256;  // per-warp shared slab for the row sort (col, val)
// Columns of at most kLaneSeg entries are handled by one lane each (32 in
// flight per warp); longer ones by the whole warp, one at a time.
constexpr int kLaneSeg = 32;

__global__ void col_counts_kernel(int32_t nout, int32_t ground, const int32_t* __restrict__ pcnt,
                                  const int64_t* __restrict__ pstart, const int32_t* __restrict__ prow,
                                  int32_t* cnt) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nout; k += stride) {
        int c = pcnt[k];
        // rows are ascending in the pool, so the ground row is the last one
        if (ground >= 0 && c > 0 && prow[pstart[k] + c - 1] == ground) --c;
        cnt[k] = c;
    }
}

// Lc from the pool (and, when col_of is given, the column of every entry).
__global__ void scatter_cols_kernel(int32_t nout, const int64_t* __restrict__ lc_ptr,
                                    const int64_t* __restrict__ pstart, const int32_t* __restrict__ prow,
                                    const double* __restrict__ pval, int32_t* lc_idx, double* lc_val,
                                    int32_t* row_cnt, int32_t* col_of) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t k = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); k < nout; k += warps) {
        int64_t o = lc_ptr[k], len = lc_ptr[k + 1] - o, src = pstart[k];
        for (int64_t t = lane; t < len; t += 32) {
            int32_t r = prow[src + t];
            lc_idx[o + t] = r;
            lc_val[o + t] = -pval[src + t];
            if (col_of) col_of[o + t] = (int32_t)k;
            atomicAdd(row_cnt + r, 1);
        }
    }
}

// Lr entry q is Lc entry order[q] (Lc's entries stably ordered by row).
__global__ void gather_rows_kernel(int64_t nnz, const int32_t* __restrict__ order, const int32_t* __restrict__ col_of,
                                   const double* __restrict__ lc_val, int32_t* lr_idx, double* lr_val) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < nnz; q += stride) {
        const int32_t p = order[q];
        lr_idx[q] = col_of[p];
        lr_val[q] = lc_val[p];
    }
}

__global__ void transpose_kernel(int32_t nout, const int64_t* __restrict__ lc_ptr, const int32_t* __restrict__ lc_idx,
                                 const double* __restrict__ lc_val, const int64_t* __restrict__ lr_ptr,
                                 int32_t* cursor, int32_t* lr_idx, double* lr_val) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t j = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); j < nout; j += warps) {
        for (int64_t p = lc_ptr[j] + lane; p < lc_ptr[j + 1]; p += 32) {
            int32_t i = lc_idx[p];
            int slot = atomicAdd(cursor + i, 1);
            lr_idx[lr_ptr[i] + slot] = (int32_t)j;
            lr_val[lr_ptr[i] + slot] = lc_val[p];
        }
    }
}

// Sort every row of Lr by column (the atomics above leave arrival order) so
// that the triangular solves sum in a fixed order.  Warp per row; bitonic
// over a padded power of two in a shared slab, or in a per-warp global slab
// for rows longer than the shared one.
__global__ void sort_rows_kernel(int32_t nrows, const int64_t* __restrict__ ptr, int32_t* idx, double* val,
                                 int32_t* long_rows, int32_t* nlong) {
    __shared__ int32_t skey[8][kSortSlab];
    __shared__ double sval[8][kSortSlab];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int64_t gw = (int64_t)blockIdx.x * (blockDim.x >> 5) + wib;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t r = gw; r < nrows; r += warps) {
        const int64_t o = ptr[r];
        const int len = (int)(ptr[r + 1] - o);
        if (len <= 1) continue;
        // already sorted?  (common: columns arrive mostly in order)
        bool sorted = true;
        for (int t = lane; t + 1 < len; t += 32) sorted &= idx[o + t] <= idx[o + t + 1];
        if (__all_sync(kFull, sorted)) continue;
        int P = 1;
        while (P < len) P <<= 1;
        if (P > kSortSlab) {  // left to the block-level sort
            if (lane == 0) long_rows[atomicAdd(nlong, 1)] = (int32_t)r;
            continue;
        }
        int32_t* key = skey[wib];
        double* v = sval[wib];
        for (int t = lane; t < P; t += 32) {
            key[t] = t < len ? idx[o + t] : INT_MAX;
            v[t] = t < len ? val[o + t] : 0.0;
        }
        __syncwarp();
        for (int k = 2; k <= P; k <<= 1) {
            for (int j = k >> 1; j > 0; j >>= 1) {
                for (int i = lane; i < P; i += 32) {
                    int l = i ^ j;
                    if (l > i) {
                        bool asc = (i & k) == 0;
                        if ((key[i] > key[l]) == asc) {
                            int32_t tk = key[i];
                            key[i] = key[l];
                            key[l] = tk;
                            double tv = v[i];
                            v[i] = v[l];
                            v[l] = tv;
                        }
                    }
                }
                __syncwarp();
            }
        }
        for (int t = lane; t < len; t += 32) {
            idx[o + t] = key[t];
            val[o + t] = v[t];
        }
        __syncwarp();
    }
}

// One CTA per long row: bitonic sort over a padded power of two held in
// dynamic shared memory (up to kBlockSortCap entries) or, beyond that, in a
// per-CTA global slab.
constexpr int kBlockSortCap = 8192;

__global__ void sort_long_rows_kernel(const int32_t* __restrict__ rows, int32_t nlong, const int64_t* __restrict__ ptr,
                                      int32_t* idx, double* val, int32_t* gkey, double* gval, int64_t gcap,
                                      int32_t* status) {
    extern __shared__ __align__(16) unsigned char sm[];
    double* sv = reinterpret_cast<double*>(sm);
    int32_t* sk = reinterpret_cast<int32_t*>(sv + kBlockSortCap);
    for (int t = blockIdx.x; t < nlong; t += gridDim.x) {
        const int32_t r = rows[t];
        const int64_t o = ptr[r];
        const int len = (int)(ptr[r + 1] - o);
        int P = 1;
        while (P < len) P <<= 1;
        int32_t* key = sk;
        double* v = sv;
        if (P > kBlockSortCap) {
            if (P > gcap) {
                if (threadIdx.x == 0) raise_error(status, kDevCapacity);
                continue;
            }
            key = gkey + (int64_t)blockIdx.x * gcap;
            v = gval + (int64_t)blockIdx.x * gcap;
        }
        for (int q = threadIdx.x; q < P; q += blockDim.x) {
            key[q] = q < len ? idx[o + q] : INT_MAX;
            v[q] = q < len ? val[o + q] : 0.0;
        }
        __syncthreads();
        for (int k = 2; k <= P; k <<= 1) {
            for (int j = k >> 1; j > 0; j >>= 1) {
                for (int i = threadIdx.x; i < P; i += blockDim.x) {
                    int l = i ^ j;
                    if (l > i) {
                        bool asc = (i & k) == 0;
                        if ((key[i] > key[l]) == asc) {
                            int32_t tk = key[i];
                            key[i] = key[l];
                            key[l] = tk;
                            double tv = v[i];
                            v[i] = v[l];
                            v[l] = tv;
                        }
                    }
                }
                __syncthreads();
            }
        }
        for (int q = threadIdx.x; q < len; q += blockDim.x) {
            idx[o + q] = key[q];
            val[o + q] = v[q];
        }
        __syncthreads();
    }
}

// lane class of a row (log2 of its lane-group size) and its bucket
__device__ __forceinline__ int lane_class(int64_t len, int epl) {
    int64_t need = (len + epl - 1) / epl;
    int c = 0;
    while (c < kLaneClasses - 1 && (1ll << c) < need) ++c;
    return c;
}
__device__ __forceinline__ int sched_key(int level, int64_t len, int epl) {
    return kLaneClasses * level + lane_class(len, epl);
}

// Buckets counted in shared memory first when this many fit (32 KB).
constexpr int kSchedSharedBins = 8192;

// bucket key of every row and the bucket sizes (warp-aggregated counts; with
// nsh > 0 bins, per block in shared memory and then one add per bin, so the
// few buckets that hold most rows, the first level's, are not a hot spot)
__global__ void sched_hist_kernel(const int32_t* __restrict__ level, const int64_t* __restrict__ ptr, int32_t n,
                                  int32_t depth, int backward, int epl, int32_t* key, int32_t* hist, int nsh) {
    extern __shared__ int32_t sh_hist[];
    const int lane = threadIdx.x & 31;
    for (int b = threadIdx.x; b < nsh; b += blockDim.x) sh_hist[b] = 0;
    if (nsh > 0) __syncthreads();
    int32_t* h = nsh > 0 ? sh_hist : hist;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t n_up = ((int64_t)n + 31) / 32 * 32;  // whole warps iterate together
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n_up; i += stride) {
        int k = -1;
        if (i < n) {
            const int l = backward ? depth - 1 - level[i] : level[i];
            k = sched_key(l, ptr[i + 1] - ptr[i], epl);
            key[i] = k;
        }
        const unsigned peers = __match_any_sync(0xffffffffu, k);
        if (k >= 0 && (peers & ((1u << lane) - 1u)) == 0) atomicAdd(h + k, __popc(peers));
    }
    if (nsh == 0) return;
    __syncthreads();
    for (int b = threadIdx.x; b < nsh; b += blockDim.x)
        if (sh_hist[b]) atomicAdd(hist + b, sh_hist[b]);
}

// Longest path from each row to a sink of the L^T solve DAG:
// levb[j] = 1 + max over i in column j of levb[i] (0 for an empty column).
// Rows are visited in the reverse of the forward schedule (a topological
// order of the L^T DAG) by persistent warps round-robin; each waits for the
// levels it needs (-1 = pending), bounded.
__global__ void bwd_level_kernel(int32_t n, const int64_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                                 const int32_t* __restrict__ order_f, int32_t* levb, int32_t* status,
                                 unsigned long long timeout_ns) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const unsigned long long t0 = global_timer_ns();
    bool ok = true;
    for (int64_t t = warp; t < n && ok; t += nwarps) {
        const int32_t j = order_f[n - 1 - t];
        int m = -1;
        for (int64_t p = ptr[j] + lane; p < ptr[j + 1]; p += 32) {
            int v;
            unsigned spins = 0;
            while ((v = ld_relaxed(levb + idx[p])) < 0) {
                if ((++spins & 255u) == 0 && global_timer_ns() - t0 > timeout_ns) {
                    raise_error(status, kDevTimeout);
                    ok = false;
                    break;
                }
            }
            m = max(m, v);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(kFull, m, o));
        if (lane == 0) atomicExch(levb + j, m + 1);
        ok = __all_sync(kFull, ok);
    }
}

// tasks per bucket: rows of class c pack 32 >> c to a warp
__global__ void sched_task_count_kernel(const int32_t* __restrict__ hist, int32_t nb, int32_t* tcount) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += stride) {
        const int per = 32 >> (int)(b % kLaneClasses);
        tcount[b] = (hist[b] + per - 1) / per;
    }
}

__global__ void sched_task_emit_kernel(const int32_t* __restrict__ hist, const int32_t* __restrict__ start,
                                       const int32_t* __restrict__ tstart, int32_t nb, int32_t ntasks, int2* tasks) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < ntasks; t += stride) {
        int lo = 0, hi = nb - 1;  // last bucket with tstart <= t
        while (lo < hi) {
            int mid = (lo + hi + 1) >> 1;
            if (tstart[mid] <= t) lo = mid;
            else hi = mid - 1;
        }
        const int b = lo;
        const int cls = b % kLaneClasses;
        const int per = 32 >> cls;
        const int q = (int)(t - tstart[b]);
        int2 d;
        d.x = start[b] + per * q;
        d.y = min(per, hist[b] - per * q) | (cls << 8);
        tasks[t] = d;
    }
}

__global__ void mask_mul_kernel(const int32_t* __restrict__ a, const int32_t* __restrict__ mask, int32_t* out,
                                int32_t n) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += stride) out[t] = mask[t] ? a[t] : 0;
}

// Entries of the row at schedule position p: ptr[order[p]] .. ptr[order[p] + 1].
__device__ __forceinline__ int64_t pos_len(const int32_t* __restrict__ order, const int64_t* __restrict__ ptr,
                                           int64_t p) {
    const int32_t i = order[p];
    return ptr[i + 1] - ptr[i];
}

// Parts of each scheduled task: 1, or ceil(len / split_len) for a one-row
// task of the widest class whose row is longer than split_min.
__global__ void pack_nsub_kernel(const int2* __restrict__ tasks, int32_t ntasks, const int32_t* __restrict__ order,
                                 const int64_t* __restrict__ ptr, int split_min, int split_len, int32_t* nsub,
                                 int32_t* issplit) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < ntasks; t += stride) {
        const int2 d = tasks[t];
        const int cls = d.y >> 8, cnt = d.y & 0xff;
        const int64_t len = cnt == 1 ? pos_len(order, ptr, d.x) : 0;
        const int np = (cls == kLaneClasses - 1 && len > split_min) ? (int)((len + split_len - 1) / split_len) : 1;
        nsub[t] = np;
        issplit[t] = np > 1 ? 1 : 0;
    }
}

// Expanded tasks {position, d.z bits, part count, part length or 0} and the
// split bookkeeping of part tasks.
__global__ void pack_expand_kernel(const int2* __restrict__ tasks, int32_t ntasks, const int64_t* __restrict__ ptr,
                                   const int32_t* __restrict__ order, int split_len, const int32_t* __restrict__ nsub,
                                   const int32_t* __restrict__ tbase, const int32_t* __restrict__ sid,
                                   const int32_t* __restrict__ pbase, int4* etask, int2* split, int32_t* srow) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < ntasks; t += stride) {
        const int2 d = tasks[t];
        const int np = nsub[t];
        if (np == 1) {
            etask[tbase[t]] = make_int4(d.x, d.y, 1, 0);
            continue;
        }
        const int64_t len = pos_len(order, ptr, d.x);
        srow[sid[t]] = order[d.x];
        for (int q = 0; q < np; ++q) {
            const int plen = (int)min((int64_t)split_len, len - (int64_t)q * split_len);
            etask[tbase[t] + q] = make_int4(d.x, d.y | (1 << 11) | (q << 12), np, plen);
            split[tbase[t] + q] = make_int2(sid[t], pbase[t]);
        }
    }
}

// slots per lane of each expanded task: the longest of its rows (or the
// part's length) over G lanes
__global__ void pack_m_kernel(const int4* __restrict__ etask, int32_t ntasks, const int32_t* __restrict__ order,
                              const int64_t* __restrict__ ptr, int32_t* m) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < ntasks; t += stride) {
        const int4 e = etask[t];
        const int cls = (e.y >> 8) & 7, cnt = e.y & 0xff;
        int64_t longest = e.w;
        if (!((e.y >> 11) & 1))
            for (int r = 0; r < cnt; ++r) longest = max(longest, pos_len(order, ptr, e.x + r));
        m[t] = (int32_t)((longest + (1 << cls) - 1) >> cls);
    }
}

__global__ void pack_desc_kernel(const int4* __restrict__ etask, int32_t ntasks, const int32_t* __restrict__ m,
                                 const int64_t* __restrict__ base, int4* pack) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < ntasks; t += stride) {
        const int4 e = etask[t];
        pack[t] = make_int4(e.x, (int32_t)base[t], e.y, m[t] | (((e.y >> 11) & 1) ? e.z << 8 : 0));
    }
}

// One warp per task: slot (k, lane) <- entry k*G + lane%G of row lane/G,
// except that entry 0 and the row's gate trade places.  The gate is the
// dependency scheduled last (largest sign * level; the first such entry on
// ties): the solve polls it alone before reading the rest of the row.
__global__ void pack_fill_kernel(const int4* __restrict__ pack, int32_t ntasks, const int32_t* __restrict__ order,
                                 const int64_t* __restrict__ ptr, int split_len, const int32_t* __restrict__ sidx,
                                 const double* __restrict__ sval,
                                 const float* __restrict__ sval32, const int32_t* __restrict__ level, int sign,
                                 int32_t* pidx, double* pval, float* pval32) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t t = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); t < ntasks; t += warps) {
        const int4 d = pack[t];
        const int cls = (d.z >> 8) & 7, cnt = d.z & 0xff;
        const int G = 1 << cls;
        const int r = lane >> cls, gl = lane & (G - 1);
        int64_t s = 0, len = 0;
        if (r < cnt) {
            const int32_t i = order[d.x + r];
            s = ptr[i];
            len = ptr[i + 1] - s;
            if ((d.z >> 11) & 1) {  // part task: its window of the row
                const int64_t q0 = (int64_t)(d.z >> 12) * split_len;
                s += q0;
                len = min((int64_t)split_len, len - q0);
            }
        }
        // gate of the row: best (key, entry) over the lane's entries, then over the G lanes
        long long best_key = LLONG_MIN, best_e = 0;
        for (int64_t e = gl; e < len; e += G) {
            const long long key = (long long)sign * level[sidx[s + e]];
            if (key > best_key) {
                best_key = key;
                best_e = e;
            }
        }
        for (int o = 1; o < G; o <<= 1) {
            const long long ok = __shfl_xor_sync(0xffffffffu, best_key, o);
            const long long oe = __shfl_xor_sync(0xffffffffu, best_e, o);
            if (ok > best_key || (ok == best_key && oe < best_e)) {
                best_key = ok;
                best_e = oe;
            }
        }
        const int mslots = d.w & 0xff;
        for (int k = 0; k < mslots; ++k) {
            int64_t e = ((int64_t)k << cls) + gl;
            const size_t o = ((size_t)d.y + k) * 32 + lane;
            const bool have = e < len;
            if (have && e == 0) e = best_e;
            else if (have && e == best_e) e = 0;
            pidx[o] = have ? sidx[s + e] : -1;
            pval[o] = have ? sval[s + e] : 0.0;
            if (pval32) pval32[o] = have ? sval32[s + e] : 0.0f;
        }
    }
}

// rows in schedule order: position p copies row order[p] of (ptr, idx, val)
__global__ void permute_len_kernel(int32_t n, const int32_t* __restrict__ order, const int64_t* __restrict__ ptr,
                                   int32_t* len) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += stride) {
        const int32_t i = order[p];
        len[p] = (int32_t)(ptr[i + 1] - ptr[i]);
    }
}

__global__ void permute_rows_kernel(int32_t n, const int32_t* __restrict__ order, const int64_t* __restrict__ ptr,
                                    const int32_t* __restrict__ idx, const double* __restrict__ val,
                                    const float* __restrict__ val32, const int64_t* __restrict__ optr, int32_t* oidx,
                                    double* oval, float* oval32) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t p = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); p < n; p += warps) {
        const int32_t i = order[p];
        const int64_t s = ptr[i], len = ptr[i + 1] - s, o = optr[p];
        for (int64_t q = lane; q < len; q += 32) {
            oidx[o + q] = idx[s + q];
            oval[o + q] = val[s + q];
            if (val32) oval32[o + q] = val32[s + q];
        }
    }
}

// flag = 1 unless colptr[0] = 0, colptr[n] = nnz and colptr never decreases
__global__ void colptr_check_kernel(const int32_t* __restrict__ colptr, int32_t n, int32_t nnz, int32_t* flag) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i <= n; i += stride) {
        const int32_t c = colptr[i];
        const bool bad = (i == 0 && c != 0) || (i == n && c != nnz) || (i < n && colptr[i + 1] < c);
        if (bad) *flag = 1;
    }
}

__global__ void max_kernel(const int32_t* __restrict__ a, int64_t n, int32_t* out) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    int32_t m = 0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) m = max(m, a[i]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(kFull, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

__global__ void to_f32_kernel(const double* __restrict__ in, float* out, int64_t n) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) out[i] = (float)in[i];
}

__global__ void trim_count_kernel(int32_t nout, const int32_t* __restrict__ colptr, const int32_t* __restrict__ rowind,
                                  int32_t* cnt) {
    const int lane = threadIdx.x & 31;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t c0 = (((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 32; c0 < nout; c0 += nw * 32) {
        const int64_t c = c0 + lane;
        const bool have = c < nout;
        const int s = have ? colptr[c] : 0, e = have ? colptr[c + 1] : 0;
        const bool wide = e - s > kLaneSeg;
        int k = 0;
        if (!wide) {
#pragma unroll 4
            for (int p = s; p < e; ++p) k += rowind[p] < nout;
        }
        for (unsigned lb = __ballot_sync(kFull, wide); lb; lb &= lb - 1u) {
            const int sl = __ffs(lb) - 1;
            const int ws = __shfl_sync(kFull, s, sl), we = __shfl_sync(kFull, e, sl);
            int k2 = 0;
#pragma unroll 8
            for (int p = ws + lane; p < we; p += 32) k2 += rowind[p] < nout;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) k2 += __shfl_xor_sync(kFull, k2, o);
            if (lane == sl) k = k2;
        }
        if (have) cnt[c] = k;
    }
}

__global__ void trim_scatter_kernel(int32_t nout, const int32_t* __restrict__ colptr, const int32_t* __restrict__ rowind,
                                    const double* __restrict__ val, const int32_t* __restrict__ ocolptr,
                                    int32_t* orow, double* oval) {
    const int lane = threadIdx.x & 31;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t c0 = (((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 32; c0 < nout; c0 += nw * 32) {
        const int64_t c = c0 + lane;
        const bool have = c < nout;
        const int s = have ? colptr[c] : 0, e = have ? colptr[c + 1] : 0;
        const int o = have ? ocolptr[c] : 0;
        const bool wide = e - s > kLaneSeg;
        if (!wide) {
            int out = o;
#pragma unroll 4
            for (int p = s; p < e; ++p) {
                const int r = rowind[p];
                if (r < nout) {
                    orow[out] = r;
                    oval[out] = val[p];
                    ++out;
                }
            }
        }
        for (unsigned lb = __ballot_sync(kFull, wide); lb; lb &= lb - 1u) {
            const int sl = __ffs(lb) - 1;
            const int ws = __shfl_sync(kFull, s, sl), we = __shfl_sync(kFull, e, sl);
            int out = __shfl_sync(kFull, o, sl);
#pragma unroll 8
            for (int base = ws; base < we; base += 32) {
                const int p = base + lane;
                const bool take = p < we && rowind[p] < nout;
                const unsigned bal = __ballot_sync(kFull, take);
                if (take) {
                    const int q = out + __popc(bal & ((1u << lane) - 1u));
                    orow[q] = rowind[p];
                    oval[q] = val[p];
                }
                out += __popc(bal);
            }
        }
    }
}

template <typename T>
cudaError_t dmalloc(T** p, int64_t n) {
    return cudaMalloc((void**)p, sizeof(T) * (size_t)(n > 0 ? n : 1));
}

// Level table of the backward schedule's first lvcap levels: lv[l] = {first
// task, first slab unit, first position} of level l, written by the task that
// opens the level (levels are contiguous in task order), plus the end of
// the last level when it falls inside the table.  split_min receives the
// lowest level holding a part task.
__global__ void head_level_kernel(int32_t npt, const int4* __restrict__ pack, const int32_t* __restrict__ order,
                                  const int32_t* __restrict__ level, int32_t n, int32_t lvcap, int4* lv,
                                  int32_t* split_min) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < npt; t += stride) {
        const int4 d = pack[t];
        const int32_t l = level[order[d.x]];
        if (l > lvcap) continue;
        if (t == 0 || level[order[pack[t - 1].x]] != l) lv[l] = make_int4((int)t, d.y, d.x, 0);
        if (((d.z >> 11) & 1) && l < lvcap) atomicMin(split_min, l);
        if (t == npt - 1 && l + 1 <= lvcap) lv[l + 1] = make_int4(npt, d.y + (d.w & 0xff), n, 0);
    }
}

__global__ void invert_order_kernel(int32_t n, const int32_t* __restrict__ order, int32_t* pos) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += stride) pos[order[p]] = (int32_t)p;
}

// Head slab slots with row indices replaced by positions in order_b; a
// position outside the head (which the level structure rules out) sets bad.
__global__ void head_idx_kernel(int64_t nslots, const int32_t* __restrict__ pidx, const int32_t* __restrict__ pos,
                                int32_t rows, int32_t* out, int32_t* bad) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < nslots; s += stride) {
        const int32_t j = pidx[s];
        int32_t q = -1;
        if (j >= 0) {
            q = pos[j];
            if (q >= rows) {
                *bad = 1;
                q = -1;
            }
        }
        out[s] = q;
    }
}

}  // namespace

// (Re)allocate a persistent buffer that shares the capacity `cap` with its
// siblings: kept when present and the shared capacity did not grow.
template <typename T>
static cudaError_t realloc_if(T** p, bool grow, int64_t cap) {
    if (*p && !grow) return cudaSuccess;
    cudaFree(*p);
    *p = nullptr;
    return cudaMalloc((void**)p, sizeof(T) * (size_t)(cap > 0 ? cap : 1));
}

// Reuse a buffer with its own capacity when it suffices, else reallocate.
template <typename T>
static cudaError_t ensure(T** p, int64_t& cap, int64_t need) {
    if (*p && cap >= need) return cudaSuccess;
    cudaFree(*p);
    *p = nullptr;
    cap = 0;
    cudaError_t e = cudaMalloc((void**)p, sizeof(T) * (size_t)(need > 0 ? need : 1));
    if (e == cudaSuccess) cap = need;
    return e;
}

cudaError_t assemble_factor(const FactorWork& w, bool trim_ground, bool make_fp32, int epl, bool exact_bwd,
                            bool bwd_head, double timeout_s, Scratch& sc, DevFactor& f, cudaStream_t s) {
    const int32_t nout = trim_ground ? w.n - 1 : w.n;
    const int32_t ground = trim_ground ? w.n - 1 : -1;
    f.n = nout;
    sc.reset();
    // temporaries of this call: counts, scan scratch, long-row list, status
    RCHOL_TRY(sc.reserve((size_t)nout * 40 + 4 * scan_tmp_bytes(nout) + (16u << 20)));
    int32_t *cnt = nullptr, *dsc = nullptr, *long_rows = nullptr;
    void* tmp = nullptr;
    RCHOL_TRY(sc.get(&cnt, nout));
    RCHOL_TRY(sc.get(&long_rows, nout));
    RCHOL_TRY(sc.get(&dsc, 4));
    RCHOL_TRY(sc.get((char**)&tmp, (int64_t)scan_tmp_bytes(nout)));
    // per-row arrays share cap_n (n+1 entries)
    const bool grow_n = f.cap_n < (int64_t)nout + 1;
    const int64_t capn = std::max<int64_t>(f.cap_n, (int64_t)nout + 1);
    RCHOL_TRY(realloc_if(&f.lc_ptr, grow_n, capn));
    RCHOL_TRY(realloc_if(&f.lr_ptr, grow_n, capn));
    RCHOL_TRY(realloc_if(&f.diag, grow_n, capn));
    RCHOL_TRY(realloc_if(&f.order_f, grow_n, capn));
    RCHOL_TRY(realloc_if(&f.order_b, grow_n, capn));
    if (make_fp32) RCHOL_TRY(realloc_if(&f.diag32, grow_n, capn));
    f.cap_n = capn;
    col_counts_kernel<<<grid_for(nout, 256), 256, 0, s>>>(nout, ground, w.pcnt, w.pstart, w.prow, cnt);
    RCHOL_TRY(cudaGetLastError());
    RCHOL_TRY(exclusive_scan_i32_to_i64(cnt, f.lc_ptr, nout, tmp, s));
    int64_t nnz = 0;
    RCHOL_TRY(cudaMemcpyAsync(&nnz, f.lc_ptr + nout, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    RCHOL_TRY(cudaStreamSynchronize(s));
    f.nnz = nnz;
    // per-entry arrays share cap_nnz
    const bool grow_z = f.cap_nnz < nnz;
    const int64_t capz = std::max<int64_t>(f.cap_nnz, nnz);
    RCHOL_TRY(realloc_if(&f.lc_idx, grow_z, capz));
    RCHOL_TRY(realloc_if(&f.lc_val, grow_z, capz));
    RCHOL_TRY(realloc_if(&f.lr_idx, grow_z, capz));
    RCHOL_TRY(realloc_if(&f.lr_val, grow_z, capz));
    if (make_fp32) {
        RCHOL_TRY(realloc_if(&f.lc_val32, grow_z, capz));
        RCHOL_TRY(realloc_if(&f.lr_val32, grow_z, capz));
    } else {
        cudaFree(f.lc_val32);
        cudaFree(f.lr_val32);
        cudaFree(f.diag32);
        f.lc_val32 = f.lr_val32 = nullptr;
        f.diag32 = nullptr;
    }
    f.cap_nnz = capz;
    // Lr: a stable sort of Lc's entries (columns ascending) by row leaves
    // every row's columns ascending, with no atomics and no row sort; the
    // atomic transpose plus row sorts is kept for more than 2^31 - 1 entries
    const bool by_sort = nnz <= (int64_t)INT_MAX;
    int32_t *col_of = nullptr, *eorder = nullptr;
    if (by_sort) {
        RCHOL_TRY(sc.get(&col_of, nnz));
        RCHOL_TRY(sc.get(&eorder, nnz));
    }
    RCHOL_TRY(cudaMemsetAsync(cnt, 0, sizeof(int32_t) * (size_t)(nout > 0 ? nout : 1), s));
    scatter_cols_kernel<<<grid_for((int64_t)nout * 32, 256), 256, 0, s>>>(nout, f.lc_ptr, w.pstart, w.prow, w.pval,
                                                                          f.lc_idx, f.lc_val, cnt, col_of);
    RCHOL_TRY(cudaGetLastError());
    RCHOL_TRY(exclusive_scan_i32_to_i64(cnt, f.lr_ptr, nout, tmp, s));
    if (by_sort) {
        RCHOL_TRY(stable_key_order_carried(f.lc_idx, (int32_t)nnz, nout, eorder, sc, s));
        gather_rows_kernel<<<grid_for(nnz, 256), 256, 0, s>>>(nnz, eorder, col_of, f.lc_val, f.lr_idx, f.lr_val);
        RCHOL_TRY(cudaGetLastError());
    } else {
        RCHOL_TRY(cudaMemsetAsync(cnt, 0, sizeof(int32_t) * (size_t)(nout > 0 ? nout : 1), s));
        transpose_kernel<<<grid_for((int64_t)nout * 32, 256), 256, 0, s>>>(nout, f.lc_ptr, f.lc_idx, f.lc_val,
                                                                           f.lr_ptr, cnt, f.lr_idx, f.lr_val);
        RCHOL_TRY(cudaGetLastError());
    }
    // deterministic row order: warp sort for short rows, CTA sort for long ones
    const int sort_block = 256;
    const int sort_grid = current_sm_count() * 4;
    RCHOL_TRY(cudaMemsetAsync(dsc, 0, sizeof(int32_t) * 4, s));  // long rows, max row, max level
    max_kernel<<<grid_for(nout, 256), 256, 0, s>>>(cnt, nout, dsc + 1);
    max_kernel<<<grid_for(nout, 256), 256, 0, s>>>(w.level, nout, dsc + 2);
    if (!by_sort) {
        sort_rows_kernel<<<sort_grid, sort_block, 0, s>>>(nout, f.lr_ptr, f.lr_idx, f.lr_val, long_rows, dsc);
        RCHOL_TRY(cudaGetLastError());
    }
    int32_t hs[4] = {0, 0, 0, 0};
    RCHOL_TRY(cudaMemcpyAsync(hs, dsc, sizeof(hs), cudaMemcpyDeviceToHost, s));
    RCHOL_TRY(cudaStreamSynchronize(s));
    int32_t* gkey = nullptr;
    double* gval = nullptr;
    int64_t gcap = 1;
    const int lgrid = hs[0] > 0 ? std::min(hs[0], current_sm_count() * 2) : 1;
    if (hs[0] > 0 && hs[1] > kBlockSortCap) {
        while (gcap < hs[1]) gcap <<= 1;
        RCHOL_TRY(sc.get(&gkey, (int64_t)lgrid * gcap));
        RCHOL_TRY(sc.get(&gval, (int64_t)lgrid * gcap));
    }
    if (hs[0] > 0) {
        const size_t smem = (size_t)kBlockSortCap * 12;
        RCHOL_TRY(cudaFuncSetAttribute(sort_long_rows_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        sort_long_rows_kernel<<<lgrid, 512, smem, s>>>(long_rows, hs[0], f.lr_ptr, f.lr_idx, f.lr_val, gkey, gval,
                                                        gcap, w.counters + 3);
        RCHOL_TRY(cudaGetLastError());
    }
    f.depth = hs[2] + 1;
    if (epl <= 0) epl = auto_sched_epl(hs[1]);
    RCHOL_TRY(cudaMemcpyAsync(f.diag, w.diag, sizeof(double) * (size_t)nout, cudaMemcpyDeviceToDevice, s));
    if (make_fp32) {
        to_f32_kernel<<<grid_for(nnz, 256), 256, 0, s>>>(f.lc_val, f.lc_val32, nnz);
        to_f32_kernel<<<grid_for(nnz, 256), 256, 0, s>>>(f.lr_val, f.lr_val32, nnz);
        to_f32_kernel<<<grid_for(nout, 256), 256, 0, s>>>(f.diag, f.diag32, nout);
        RCHOL_TRY(cudaGetLastError());
    }
    RCHOL_TRY(build_solve_schedule(f, w.level, epl, exact_bwd, bwd_head, timeout_s, sc, s));
    RCHOL_TRY(cudaStreamSynchronize(s));
    sc.reset();
    return cudaSuccess;
}

// Orders the rows by (level, lane class, row) into `order` (capacity n,
// owned by the factor) and emits the task list into `*tasks` (grown as
// needed).
static cudaError_t build_one_schedule(const int32_t* level, const int64_t* ptr, int32_t n, int32_t depth, int backward,
                                      int epl, Scratch& sc, int32_t* order, int2** tasks, int64_t& tcap,
                                      int32_t* ntasks, cudaStream_t s) {
    const int32_t nb = kLaneClasses * depth;
    int32_t *hist = nullptr, *start = nullptr, *tcount = nullptr, *tstart = nullptr, *key = nullptr;
    void* tmp = nullptr;
    RCHOL_TRY(sc.get(&key, std::max<int32_t>(n, 1)));
    RCHOL_TRY(sc.get(&hist, nb));
    RCHOL_TRY(sc.get(&start, (int64_t)nb + 1));
    RCHOL_TRY(sc.get(&tcount, nb));
    RCHOL_TRY(sc.get(&tstart, (int64_t)nb + 1));
    RCHOL_TRY(sc.get((char**)&tmp, (int64_t)scan_tmp_bytes(nb)));
    RCHOL_TRY(cudaMemsetAsync(hist, 0, sizeof(int32_t) * (size_t)nb, s));
    {
        const int nsh = nb <= kSchedSharedBins ? nb : 0;
        const int grid = nsh > 0 ? grid_for(n, 256, 4) : grid_for(n, 256);
        sched_hist_kernel<<<grid, 256, sizeof(int32_t) * (size_t)nsh, s>>>(level, ptr, n, depth, backward, epl,
                                                                           key, hist, nsh);
    }
    RCHOL_TRY(exclusive_scan_i32_to_i32(hist, start, nb, tmp, s));
    sched_task_count_kernel<<<grid_for(nb, 256), 256, 0, s>>>(hist, nb, tcount);
    RCHOL_TRY(exclusive_scan_i32_to_i32(tcount, tstart, nb, tmp, s));
    int32_t nt = 0;
    RCHOL_TRY(cudaMemcpyAsync(&nt, tstart + nb, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    RCHOL_TRY(cudaStreamSynchronize(s));
    *ntasks = nt;
    RCHOL_TRY(ensure(tasks, tcap, (int64_t)nt));
    sched_task_emit_kernel<<<grid_for(nt, 256), 256, 0, s>>>(hist, start, tstart, nb, nt, *tasks);
    RCHOL_TRY(cudaGetLastError());
    return stable_key_order(key, n, nb, order, sc, s);
}

static cudaError_t build_layout(int32_t n, const int32_t* order, const int64_t* ptr, const int32_t* idx,
                                const double* val, const float* val32, int64_t* optr, int32_t* oidx, double* oval,
                                float* oval32, Scratch& sc, cudaStream_t s) {
    int32_t* len = nullptr;
    void* tmp = nullptr;
    RCHOL_TRY(sc.get(&len, n));
    RCHOL_TRY(sc.get((char**)&tmp, (int64_t)scan_tmp_bytes(n)));
    permute_len_kernel<<<grid_for(n, 256), 256, 0, s>>>(n, order, ptr, len);
    RCHOL_TRY(exclusive_scan_i32_to_i64(len, optr, n, tmp, s));
    permute_rows_kernel<<<grid_for((int64_t)n * 32, 256), 256, 0, s>>>(n, order, ptr, idx, val, val32, optr, oidx,
                                                                        oval, oval32);
    return cudaGetLastError();
}

// Output arrays of one direction's task slabs.
struct PackOut {
    int4** pack;
    int64_t* cap_d;
    int32_t** pidx;
    int64_t* cap_i;
    double** pval;
    int64_t* cap_v;
    float** pval32;
    int64_t* cap_w;
    int64_t* slots;
    int32_t* npt;
    int32_t* nsplit;
    int2** split;
    int64_t* cap_s;
    double** psum;
    int64_t* cap_q;
    int32_t** pcount;
    int64_t* cap_c;
    int32_t** srow;
    int64_t* cap_r;
};

// Task slabs of one direction from its task list and row order over L's
// rows (ptr, sidx, sval by row id); rows longer than split_min are split
// into part tasks first.
static cudaError_t build_pack(int32_t ntasks, const int2* tasks, const int32_t* order, const int64_t* ptr,
                              const int32_t* sidx, const double* sval, const float* sval32, const int32_t* level,
                              int sign, int split_min, int split_len, const PackOut& o, Scratch& sc, cudaStream_t s) {
    const int64_t nt = std::max<int32_t>(ntasks, 1);
    int32_t *nsub = nullptr, *issplit = nullptr, *tbase = nullptr, *sid = nullptr, *pbase = nullptr;
    void* tmp = nullptr;
    RCHOL_TRY(sc.get(&nsub, nt));
    RCHOL_TRY(sc.get(&issplit, nt));
    RCHOL_TRY(sc.get(&tbase, nt + 1));
    RCHOL_TRY(sc.get(&sid, nt + 1));
    RCHOL_TRY(sc.get(&pbase, nt + 1));
    RCHOL_TRY(sc.get((char**)&tmp, (int64_t)scan_tmp_bytes(nt)));
    *o.npt = 0;
    *o.nsplit = 0;
    *o.slots = 0;
    if (ntasks == 0) {
        RCHOL_TRY(ensure(o.pack, *o.cap_d, 1));
        return cudaSuccess;
    }
    pack_nsub_kernel<<<grid_for(ntasks, 256), 256, 0, s>>>(tasks, ntasks, order, ptr, split_min, split_len, nsub,
                                                           issplit);
    RCHOL_TRY(exclusive_scan_i32_to_i32(nsub, tbase, ntasks, tmp, s));
    RCHOL_TRY(exclusive_scan_i32_to_i32(issplit, sid, ntasks, tmp, s));
    int32_t hs[2] = {0, 0};
    RCHOL_TRY(cudaMemcpyAsync(&hs[0], tbase + ntasks, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    RCHOL_TRY(cudaMemcpyAsync(&hs[1], sid + ntasks, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    RCHOL_TRY(cudaStreamSynchronize(s));
    const int32_t ne = hs[0], nsp = hs[1];
    // first partial of each split task: exclusive scan of its part count
    int32_t nparts = 0;
    if (nsp > 0) {
        int32_t* psub = nullptr;
        RCHOL_TRY(sc.get(&psub, nt));
        mask_mul_kernel<<<grid_for(ntasks, 256), 256, 0, s>>>(nsub, issplit, psub, ntasks);
        RCHOL_TRY(exclusive_scan_i32_to_i32(psub, pbase, ntasks, tmp, s));
        RCHOL_TRY(cudaMemcpyAsync(&nparts, pbase + ntasks, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
        RCHOL_TRY(cudaStreamSynchronize(s));
    }
    int4* etask = nullptr;
    int32_t* m = nullptr;
    int64_t* base = nullptr;
    void* tmp2 = nullptr;
    RCHOL_TRY(sc.get(&etask, ne));
    RCHOL_TRY(sc.get(&m, ne));
    RCHOL_TRY(sc.get(&base, (int64_t)ne + 1));
    RCHOL_TRY(sc.get((char**)&tmp2, (int64_t)scan_tmp_bytes(ne)));
    RCHOL_TRY(ensure(o.pack, *o.cap_d, (int64_t)ne));
    RCHOL_TRY(ensure(o.split, *o.cap_s, std::max<int64_t>(ne, 1)));
    RCHOL_TRY(ensure(o.psum, *o.cap_q, std::max<int64_t>(nparts, 1)));
    RCHOL_TRY(ensure(o.pcount, *o.cap_c, std::max<int64_t>(nsp, 1)));
    RCHOL_TRY(ensure(o.srow, *o.cap_r, std::max<int64_t>(nsp, 1)));
    RCHOL_TRY(cudaMemsetAsync(*o.pcount, 0, sizeof(int32_t) * (size_t)std::max<int32_t>(nsp, 1), s));
    pack_expand_kernel<<<grid_for(ntasks, 256), 256, 0, s>>>(tasks, ntasks, ptr, order, split_len, nsub, tbase, sid,
                                                             pbase, etask, *o.split, *o.srow);
    pack_m_kernel<<<grid_for(ne, 256), 256, 0, s>>>(etask, ne, order, ptr, m);
    RCHOL_TRY(exclusive_scan_i32_to_i64(m, base, ne, tmp2, s));
    int64_t units = 0;
    RCHOL_TRY(cudaMemcpyAsync(&units, base + ne, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    RCHOL_TRY(cudaStreamSynchronize(s));
    if (units >= (int64_t)INT32_MAX) return cudaErrorInvalidValue;  // slab offsets are int32 units
    const int64_t nslots = std::max<int64_t>(units * 32, 32);
    *o.slots = units * 32;
    *o.npt = ne;
    *o.nsplit = nsp;
    RCHOL_TRY(ensure(o.pidx, *o.cap_i, nslots));
    RCHOL_TRY(ensure(o.pval, *o.cap_v, nslots));
    if (sval32) {
        RCHOL_TRY(ensure(o.pval32, *o.cap_w, nslots));
    } else {
        cudaFree(*o.pval32);
        *o.pval32 = nullptr;
        *o.cap_w = 0;
    }
    pack_desc_kernel<<<grid_for(ne, 256), 256, 0, s>>>(etask, ne, m, base, *o.pack);
    pack_fill_kernel<<<grid_for((int64_t)ne * 32, 256), 256, 0, s>>>(
        *o.pack, ne, order, ptr, split_len, sidx, sval, sval32, level, sign, *o.pidx, *o.pval,
        sval32 ? *o.pval32 : nullptr);
    return cudaGetLastError();
}

// The task slabs of both directions for the orders already built, read
// from the rows of Lr (forward) and Lc (backward); FP32 values are copied
// when the factor has them.
static cudaError_t build_packs(DevFactor& f, const int32_t* level_f, const int32_t* level_b, int sign_b,
                                 Scratch& sc, cudaStream_t s) {
    const PackOut of{&f.pack_f, &f.cap_pdf, &f.pf_idx, &f.cap_pif, &f.pf_val, &f.cap_pvf, &f.pf_val32, &f.cap_pwf,
                     &f.slots_f, &f.npt_f, &f.nsplit_f, &f.split_f, &f.cap_sf, &f.psum_f, &f.cap_qf, &f.pcount_f,
                     &f.cap_cf, &f.srow_f, &f.cap_rf};
    const PackOut ob{&f.pack_b, &f.cap_pdb, &f.pb_idx, &f.cap_pib, &f.pb_val, &f.cap_pvb, &f.pb_val32, &f.cap_pwb,
                     &f.slots_b, &f.npt_b, &f.nsplit_b, &f.split_b, &f.cap_sb, &f.psum_b, &f.cap_qb, &f.pcount_b,
                     &f.cap_cb, &f.srow_b, &f.cap_rb};
    // Forward gates: the dependency of greatest position in the forward
    // schedule (greatest level, then dealt last), which lands last more
    // often than the level alone tells (c2 forward 0.517 -> 0.508 ms per
    // launch).  The backward keeps greatest level, then least entry: its
    // position form was slower (0.544 -> 0.561 ms).
    int32_t* pos_f = nullptr;
    RCHOL_TRY(sc.get(&pos_f, std::max<int32_t>(f.n, 1)));
    (void)level_f;
    invert_order_kernel<<<grid_for(f.n, 256), 256, 0, s>>>(f.n, f.order_f, pos_f);
    RCHOL_TRY(cudaGetLastError());
    RCHOL_TRY(build_pack(f.ntasks_f, f.tasks_f, f.order_f, f.lr_ptr, f.lr_idx, f.lr_val, f.lr_val32, pos_f, 1,
                         kSplitMinF, kSplitLenF, of, sc, s));
    RCHOL_TRY(build_pack(f.ntasks_b, f.tasks_b, f.order_b, f.lc_ptr, f.lc_idx, f.lc_val, f.lc_val32, level_b, sign_b,
                         kSplitMinB, kSplitLenB, ob, sc, s));
    return cudaSuccess;
}

// The backward head (see DevFactor::hb_nlev): levels from the first while
// each holds at most kHeadMaxRows rows, kHeadMaxTasks tasks and no part
// task, and the head's rows, level table and largest stage (FP64 values, so
// that either value type fits) fit the kernel's shared memory.  Fewer than
// kHeadMinLevels such levels leave the head empty.
static cudaError_t build_bwd_head(DevFactor& f, const int32_t* levb, Scratch& sc, cudaStream_t s) {
    f.hb_nlev = f.hb_ntask = f.hb_rows = f.hb_stage = 0;
    const int32_t lvcap = std::min<int32_t>(f.depth_b, kHeadMaxLevels);
    if (f.npt_b == 0 || lvcap < kHeadMinLevels) return cudaSuccess;
    int4* lv = nullptr;
    int32_t* flags = nullptr;  // [0] lowest split level, [1] bad index
    RCHOL_TRY(sc.get(&lv, (int64_t)lvcap + 1));
    RCHOL_TRY(sc.get(&flags, 2));
    const int32_t init[2] = {INT32_MAX, 0};
    RCHOL_TRY(cudaMemcpyAsync(flags, init, sizeof(init), cudaMemcpyHostToDevice, s));
    head_level_kernel<<<grid_for(f.npt_b, 256), 256, 0, s>>>(f.npt_b, f.pack_b, f.order_b, levb, f.n, lvcap, lv,
                                                             flags);
    RCHOL_TRY(cudaGetLastError());
    std::vector<int4> h((size_t)lvcap + 1);
    int32_t hf[2] = {0, 0};
    RCHOL_TRY(cudaMemcpyAsync(h.data(), lv, sizeof(int4) * h.size(), cudaMemcpyDeviceToHost, s));
    RCHOL_TRY(cudaMemcpyAsync(hf, flags, sizeof(hf), cudaMemcpyDeviceToHost, s));
    RCHOL_TRY(cudaStreamSynchronize(s));
    int nlev = 0, stage = 0;
    for (int l = 0; l < lvcap && l < hf[0]; ++l) {
        const int ntask = h[l + 1].x - h[l].x, units = h[l + 1].y - h[l].y, rows = h[l + 1].z - h[l].z;
        if (rows > kHeadMaxRows || ntask > kHeadMaxTasks) break;
        const int st = std::max(stage, head_stage_bytes(ntask, units, rows, 8));
        if (head_smem_bytes(h[l + 1].z, st) > kHeadSmem) break;
        stage = st;
        nlev = l + 1;
    }
    if (nlev < kHeadMinLevels) return cudaSuccess;
    const int32_t rows = h[nlev].z;
    const int64_t nslots = (int64_t)h[nlev].y * 32;
    int32_t* pos = nullptr;
    RCHOL_TRY(sc.get(&pos, f.n));
    RCHOL_TRY(ensure(&f.hb_lv, f.cap_hl, (int64_t)kHeadMaxLevels + 1));
    RCHOL_TRY(ensure(&f.hb_idx, f.cap_hi, std::max<int64_t>(nslots, 32)));
    invert_order_kernel<<<grid_for(f.n, 256), 256, 0, s>>>(f.n, f.order_b, pos);
    head_idx_kernel<<<grid_for(nslots, 256), 256, 0, s>>>(nslots, f.pb_idx, pos, rows, f.hb_idx, flags + 1);
    RCHOL_TRY(cudaGetLastError());
    RCHOL_TRY(cudaMemcpyAsync(f.hb_lv, lv, sizeof(int4) * ((size_t)nlev + 1), cudaMemcpyDeviceToDevice, s));
    RCHOL_TRY(cudaMemcpyAsync(&hf[1], flags + 1, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    RCHOL_TRY(cudaStreamSynchronize(s));
    if (hf[1] != 0) return cudaSuccess;  // not a head after all: leave it empty
    f.hb_nlev = nlev;
    f.hb_ntask = h[nlev].x;
    f.hb_rows = rows;
    f.hb_stage = stage;
    return cudaSuccess;
}

cudaError_t build_solve_layouts(DevFactor& f, Scratch& sc, cudaStream_t s) {
    if (f.lay_ready) return cudaSuccess;
    const bool grow_n = f.cap_ln < (int64_t)f.n + 1;
    const int64_t capn = std::max<int64_t>(f.cap_ln, (int64_t)f.n + 1);
    RCHOL_TRY(realloc_if(&f.sf_ptr, grow_n, capn));
    RCHOL_TRY(realloc_if(&f.sb_ptr, grow_n, capn));
    f.cap_ln = capn;
    const bool fp32 = f.lr_val32 != nullptr;
    const bool grow_z = f.cap_lz < f.nnz || (fp32 && !f.sf_val32);
    const int64_t capz = std::max<int64_t>(f.cap_lz, f.nnz);
    RCHOL_TRY(realloc_if(&f.sf_idx, grow_z, capz));
    RCHOL_TRY(realloc_if(&f.sf_val, grow_z, capz));
    RCHOL_TRY(realloc_if(&f.sb_idx, grow_z, capz));
    RCHOL_TRY(realloc_if(&f.sb_val, grow_z, capz));
    if (fp32) {
        RCHOL_TRY(realloc_if(&f.sf_val32, grow_z, capz));
        RCHOL_TRY(realloc_if(&f.sb_val32, grow_z, capz));
    } else {
        cudaFree(f.sf_val32);
        cudaFree(f.sb_val32);
        f.sf_val32 = f.sb_val32 = nullptr;
    }
    f.cap_lz = capz;
    sc.reset();
    RCHOL_TRY(build_layout(f.n, f.order_f, f.lr_ptr, f.lr_idx, f.lr_val, f.lr_val32, f.sf_ptr, f.sf_idx, f.sf_val,
                           f.sf_val32, sc, s));
    RCHOL_TRY(build_layout(f.n, f.order_b, f.lc_ptr, f.lc_idx, f.lc_val, f.lc_val32, f.sb_ptr, f.sb_idx, f.sb_val,
                           f.sb_val32, sc, s));
    RCHOL_TRY(cudaStreamSynchronize(s));
    sc.reset();
    f.lay_ready = true;
    return cudaSuccess;
}

cudaError_t build_solve_schedule(DevFactor& f, const int32_t* level, int epl, bool exact_bwd, bool bwd_head,
                                 double timeout_s, Scratch& sc, cudaStream_t s) {
    if (epl < 1) epl = 1;
    f.hb_nlev = f.hb_ntask = f.hb_rows = f.hb_stage = 0;
    f.lay_ready = false;
    {
        const bool grow_n = f.cap_n < (int64_t)f.n + 1;
        const int64_t capn = std::max<int64_t>(f.cap_n, (int64_t)f.n + 1);
        RCHOL_TRY(realloc_if(&f.order_f, grow_n, capn));
        RCHOL_TRY(realloc_if(&f.order_b, grow_n, capn));
        if (grow_n && f.cap_n > 0) return cudaErrorInvalidValue;  // siblings would be undersized
        f.cap_n = capn;
    }
    // forward: rows of Lr; backward: rows of L^T = columns of Lc
    RCHOL_TRY(build_one_schedule(level, f.lr_ptr, f.n, f.depth, 0, epl, sc, f.order_f, &f.tasks_f, f.cap_tf,
                                 &f.ntasks_f, s));
    f.depth_b = f.depth;
    if (!exact_bwd || f.n == 0) {
        RCHOL_TRY(build_one_schedule(level, f.lc_ptr, f.n, f.depth, 1, epl, sc, f.order_b, &f.tasks_b, f.cap_tb,
                                     &f.ntasks_b, s));
        // reversed forward levels: the backward gate is the dependency of least forward level
        RCHOL_TRY(build_packs(f, level, level, -1, sc, s));
        return cudaStreamSynchronize(s);
    }
    // true backward levels, visited in the reversed forward order
    int32_t *levb = nullptr, *st = nullptr;
    RCHOL_TRY(sc.get(&levb, f.n));
    RCHOL_TRY(sc.get(&st, 2));
    RCHOL_TRY(cudaMemsetAsync(levb, 0xff, sizeof(int32_t) * (size_t)f.n, s));
    RCHOL_TRY(cudaMemsetAsync(st, 0, sizeof(int32_t) * 2, s));
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, bwd_level_kernel, 256, 0);
    bwd_level_kernel<<<std::max(1, per_sm * sms), 256, 0, s>>>(f.n, f.lc_ptr, f.lc_idx, f.order_f, levb, st,
                                                              (unsigned long long)(timeout_s * 1e9));
    RCHOL_TRY(cudaGetLastError());
    max_kernel<<<grid_for(f.n, 256), 256, 0, s>>>(levb, f.n, st + 1);
    int32_t hs[2] = {0, 0};
    RCHOL_TRY(cudaMemcpyAsync(hs, st, sizeof(hs), cudaMemcpyDeviceToHost, s));
    RCHOL_TRY(cudaStreamSynchronize(s));
    if (hs[0] != 0) return cudaErrorLaunchTimeout;
    f.depth_b = hs[1] + 1;
    RCHOL_TRY(build_one_schedule(levb, f.lc_ptr, f.n, f.depth_b, 0, epl, sc, f.order_b, &f.tasks_b, f.cap_tb,
                                 &f.ntasks_b, s));
    RCHOL_TRY(build_packs(f, level, levb, 1, sc, s));
    if (bwd_head) RCHOL_TRY(build_bwd_head(f, levb, sc, s));
    return cudaStreamSynchronize(s);
}

cudaError_t max_i32(const int32_t* v, int64_t n, int32_t* out, cudaStream_t s) {
    max_kernel<<<grid_for(n, 256), 256, 0, s>>>(v, n, out);
    return cudaGetLastError();
}

cudaError_t check_colptr(const int32_t* colptr, int32_t n, int32_t nnz, int32_t* flag, cudaStream_t s) {
    RCHOL_TRY(cudaMemsetAsync(flag, 0, sizeof(int32_t), s));
    colptr_check_kernel<<<grid_for((int64_t)n + 1, 256), 256, 0, s>>>(colptr, n, nnz, flag);
    return cudaGetLastError();
}

cudaError_t trim_matrix(const DevCsc& A, DevCsc& out, Scratch& sc, cudaStream_t s) {
    const int32_t nout = A.n - 1;
    int32_t* cnt = nullptr;
    void* tmp = nullptr;
    RCHOL_TRY(sc.get(&cnt, nout));
    RCHOL_TRY(sc.get((char**)&tmp, (int64_t)scan_tmp_bytes(nout)));
    // colptr keeps its size for a matrix of the same order; rowind / val are
    // sized for all of A's entries, so any matrix with as many fits
    if (out.colptr && out.n != nout) {
        cudaFree(out.colptr);
        out.colptr = nullptr;
    }
    out.n = nout;
    if (!out.colptr) RCHOL_TRY(dmalloc(&out.colptr, (int64_t)nout + 1));
    if (out.cap < A.nnz) {
        cudaFree(out.rowind);
        cudaFree(out.val);
        out.rowind = nullptr;
        out.val = nullptr;
        out.cap = 0;
        RCHOL_TRY(dmalloc(&out.rowind, A.nnz));
        RCHOL_TRY(dmalloc(&out.val, A.nnz));
        out.cap = A.nnz;
    }
    trim_count_kernel<<<grid_for(nout, 256), 256, 0, s>>>(nout, A.colptr, A.rowind, cnt);
    RCHOL_TRY(cudaGetLastError());
    RCHOL_TRY(exclusive_scan_i32_to_i32(cnt, out.colptr, nout, tmp, s));
    int32_t nnz = 0;
    RCHOL_TRY(cudaMemcpyAsync(&nnz, out.colptr + nout, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    trim_scatter_kernel<<<grid_for(nout, 256), 256, 0, s>>>(nout, A.colptr, A.rowind, A.val, out.colptr,
                                                            out.rowind, out.val);
    RCHOL_TRY(cudaGetLastError());
    RCHOL_TRY(cudaStreamSynchronize(s));
    out.nnz = nnz;
    return cudaSuccess;
}

}  // namespace rchol
