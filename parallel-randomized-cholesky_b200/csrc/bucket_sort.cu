// Stable ordering of 0..n-1 by an integer key (LSD radix, 8-bit digits).
//
// Used by the solve schedules, whose row order inside a (level, lane class)
// bucket must not depend on thread timing: the per-thread partial sums of
// the PCG reductions follow the schedule, so a timing-dependent order
// would make the solver's rounding differ between identical runs.
//
// Each pass is a stable counting sort of the current order by one digit:
//   radix_hist_kernel     digit counts of every 2048-item tile, stored
//                         digit-major so one exclusive scan yields every
//                         (digit, tile) output offset;
//   radix_scatter_kernel  each tile re-reads its items in order and places
//                         them at offset + rank, the rank built from warp
//                         match masks and per-warp digit counts, so equal
//                         digits keep their input order.
#include <cstdint>

#include "device_common.cuh"
#include "rchol_internal.h"

namespace rchol {

namespace {

constexpr int kRadix = 256;
constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kItemsPerThread = 8;
constexpr int kSortTile = kSortThreads * kItemsPerThread;

__global__ void __launch_bounds__(kSortThreads) radix_hist_kernel(const int32_t* __restrict__ key,
                                                                  const int32_t* __restrict__ in, int32_t n, int shift,
                                                                  int32_t ntiles, int32_t* hist) {
    __shared__ int32_t h[kRadix];
    for (int d = threadIdx.x; d < kRadix; d += blockDim.x) h[d] = 0;
    __syncthreads();
    const int64_t base = (int64_t)blockIdx.x * kSortTile;
    for (int r = 0; r < kItemsPerThread; ++r) {
        const int64_t t = base + (int64_t)r * kSortThreads + threadIdx.x;
        if (t < n) {
            const int32_t i = in ? in[t] : (int32_t)t;
            atomicAdd(&h[(key[i] >> shift) & (kRadix - 1)], 1);
        }
    }
    __syncthreads();
    for (int d = threadIdx.x; d < kRadix; d += blockDim.x) hist[(int64_t)d * ntiles + blockIdx.x] = h[d];
}

__global__ void __launch_bounds__(kSortThreads) radix_scatter_kernel(const int32_t* __restrict__ key,
                                                                     const int32_t* __restrict__ in, int32_t n,
                                                                     int shift, int32_t ntiles,
                                                                     const int32_t* __restrict__ offs, int32_t* out) {
    __shared__ int32_t run[kRadix];               // next output position per digit
    __shared__ int32_t wcnt[kSortWarps][kRadix];  // per-warp counts, then per-warp offsets
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int d = threadIdx.x; d < kRadix; d += blockDim.x) run[d] = offs[(int64_t)d * ntiles + blockIdx.x];
    const int64_t base = (int64_t)blockIdx.x * kSortTile;
    for (int r = 0; r < kItemsPerThread; ++r) {
        for (int q = threadIdx.x; q < kSortWarps * kRadix; q += blockDim.x) (&wcnt[0][0])[q] = 0;
        __syncthreads();
        const int64_t t = base + (int64_t)r * kSortThreads + threadIdx.x;
        const bool have = t < n;
        int32_t item = 0;
        int d = kRadix;  // lanes without an item form their own group
        if (have) {
            item = in ? in[t] : (int32_t)t;
            d = (key[item] >> shift) & (kRadix - 1);
        }
        const unsigned peers = __match_any_sync(kFull, d);
        const int rank = __popc(peers & ((1u << lane) - 1u));
        if (have && rank == 0) wcnt[warp][d] = __popc(peers);
        __syncthreads();
        for (int dd = threadIdx.x; dd < kRadix; dd += blockDim.x) {
            int32_t s = run[dd];
            for (int w = 0; w < kSortWarps; ++w) {
                const int32_t c = wcnt[w][dd];
                wcnt[w][dd] = s;
                s += c;
            }
            run[dd] = s;
        }
        __syncthreads();
        if (have) out[wcnt[warp][d] + rank] = item;
        __syncthreads();
    }
}

// The same passes with the keys carried along (read and written in tile
// order) instead of read through the item index: for large n, where
// key[item] would be a scattered read in every pass after the first.
__global__ void __launch_bounds__(kSortThreads) radix_hist_carried_kernel(const int32_t* __restrict__ kin, int32_t n,
                                                                          int shift, int32_t ntiles, int32_t* hist) {
    __shared__ int32_t h[kRadix];
    for (int d = threadIdx.x; d < kRadix; d += blockDim.x) h[d] = 0;
    __syncthreads();
    const int64_t base = (int64_t)blockIdx.x * kSortTile;
    for (int r = 0; r < kItemsPerThread; ++r) {
        const int64_t t = base + (int64_t)r * kSortThreads + threadIdx.x;
        if (t < n) atomicAdd(&h[(kin[t] >> shift) & (kRadix - 1)], 1);
    }
    __syncthreads();
    for (int d = threadIdx.x; d < kRadix; d += blockDim.x) hist[(int64_t)d * ntiles + blockIdx.x] = h[d];
}

__global__ void __launch_bounds__(kSortThreads) radix_scatter_carried_kernel(const int32_t* __restrict__ kin,
                                                                             const int32_t* __restrict__ in, int32_t n,
                                                                             int shift, int32_t ntiles,
                                                                             const int32_t* __restrict__ offs,
                                                                             int32_t* kout, int32_t* out) {
    __shared__ int32_t run[kRadix];
    __shared__ int32_t wcnt[kSortWarps][kRadix];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int d = threadIdx.x; d < kRadix; d += blockDim.x) run[d] = offs[(int64_t)d * ntiles + blockIdx.x];
    const int64_t base = (int64_t)blockIdx.x * kSortTile;
    for (int r = 0; r < kItemsPerThread; ++r) {
        for (int q = threadIdx.x; q < kSortWarps * kRadix; q += blockDim.x) (&wcnt[0][0])[q] = 0;
        __syncthreads();
        const int64_t t = base + (int64_t)r * kSortThreads + threadIdx.x;
        const bool have = t < n;
        int32_t item = 0, k = 0;
        int d = kRadix;
        if (have) {
            item = in ? in[t] : (int32_t)t;
            k = kin[t];
            d = (k >> shift) & (kRadix - 1);
        }
        const unsigned peers = __match_any_sync(kFull, d);
        const int rank = __popc(peers & ((1u << lane) - 1u));
        if (have && rank == 0) wcnt[warp][d] = __popc(peers);
        __syncthreads();
        for (int dd = threadIdx.x; dd < kRadix; dd += blockDim.x) {
            int32_t s = run[dd];
            for (int w = 0; w < kSortWarps; ++w) {
                const int32_t c = wcnt[w][dd];
                wcnt[w][dd] = s;
                s += c;
            }
            run[dd] = s;
        }
        __syncthreads();
        if (have) {
            const int32_t at = wcnt[warp][d] + rank;
            out[at] = item;
            if (kout) kout[at] = k;
        }
        __syncthreads();
    }
}

}  // namespace

cudaError_t stable_key_order_carried(const int32_t* key, int32_t n, int32_t nkeys, int32_t* order, Scratch& sc,
                                     cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    int bits = 0;
    while (bits < 31 && (1ll << bits) < (int64_t)nkeys) ++bits;
    const int passes = bits <= 8 ? 1 : (bits + 7) / 8;
    const int32_t ntiles = (int32_t)((n + kSortTile - 1) / kSortTile);
    const int64_t nh = (int64_t)kRadix * ntiles;
    int32_t *hist = nullptr, *offs = nullptr, *buf = nullptr, *kb0 = nullptr, *kb1 = nullptr;
    void* tmp = nullptr;
    RCHOL_TRY(sc.get(&hist, nh));
    RCHOL_TRY(sc.get(&offs, nh + 1));
    RCHOL_TRY(sc.get((char**)&tmp, (int64_t)scan_tmp_bytes(nh)));
    if (passes > 1) {
        RCHOL_TRY(sc.get(&buf, n));
        RCHOL_TRY(sc.get(&kb0, n));
        if (passes > 2) RCHOL_TRY(sc.get(&kb1, n));
    }
    const int32_t* in = nullptr;
    const int32_t* kin = key;
    for (int p = 0; p < passes; ++p) {
        int32_t* out = ((passes - 1 - p) % 2 == 0) ? order : buf;
        int32_t* kout = p + 1 < passes ? (p % 2 == 0 ? kb0 : kb1) : nullptr;
        radix_hist_carried_kernel<<<ntiles, kSortThreads, 0, s>>>(kin, n, 8 * p, ntiles, hist);
        RCHOL_TRY(cudaGetLastError());
        RCHOL_TRY(exclusive_scan_i32_to_i32(hist, offs, nh, tmp, s));
        radix_scatter_carried_kernel<<<ntiles, kSortThreads, 0, s>>>(kin, in, n, 8 * p, ntiles, offs, kout, out);
        RCHOL_TRY(cudaGetLastError());
        in = out;
        kin = kout;
    }
    return cudaSuccess;
}

cudaError_t stable_key_order(const int32_t* key, int32_t n, int32_t nkeys, int32_t* order, Scratch& sc,
                             cudaStream_t s) {
    return stable_key_order_from(key, nullptr, n, nkeys, order, sc, s);
}

cudaError_t stable_key_order_from(const int32_t* key, const int32_t* in0, int32_t n, int32_t nkeys, int32_t* order,
                                  Scratch& sc, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    int bits = 0;
    while (bits < 31 && (1ll << bits) < (int64_t)nkeys) ++bits;
    const int passes = bits <= 8 ? 1 : (bits + 7) / 8;
    const int32_t ntiles = (int32_t)((n + kSortTile - 1) / kSortTile);
    const int64_t nh = (int64_t)kRadix * ntiles;
    int32_t *hist = nullptr, *offs = nullptr, *buf = nullptr;
    void* tmp = nullptr;
    RCHOL_TRY(sc.get(&hist, nh));
    RCHOL_TRY(sc.get(&offs, nh + 1));
    RCHOL_TRY(sc.get((char**)&tmp, (int64_t)scan_tmp_bytes(nh)));
    if (passes > 1) RCHOL_TRY(sc.get(&buf, n));
    // ping-pong so that the last pass writes `order` (which may alias in0)
    if (in0 && in0 == order) {
        int32_t* copy = nullptr;
        RCHOL_TRY(sc.get(&copy, n));
        RCHOL_TRY(cudaMemcpyAsync(copy, in0, sizeof(int32_t) * (size_t)n, cudaMemcpyDeviceToDevice, s));
        in0 = copy;
    }
    const int32_t* in = in0;
    for (int p = 0; p < passes; ++p) {
        int32_t* out = ((passes - 1 - p) % 2 == 0) ? order : buf;
        radix_hist_kernel<<<ntiles, kSortThreads, 0, s>>>(key, in, n, 8 * p, ntiles, hist);
        RCHOL_TRY(cudaGetLastError());
        RCHOL_TRY(exclusive_scan_i32_to_i32(hist, offs, nh, tmp, s));
        radix_scatter_kernel<<<ntiles, kSortThreads, 0, s>>>(key, in, n, 8 * p, ntiles, offs, out);
        RCHOL_TRY(cudaGetLastError());
        in = out;
    }
    return cudaSuccess;
}

}  // namespace rchol
