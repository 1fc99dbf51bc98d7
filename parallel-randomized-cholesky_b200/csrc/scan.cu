// Exclusive prefix sums for the setup and assembly phases: three passes
// (tile sums, scan of tile sums, tile scan + offset).  int64 accumulation.
#include "device_common.cuh"
#include "rchol_internal.h"

namespace rchol {

namespace {

constexpr int kScanBlock = 256;
constexpr int kScanItems = 8;
constexpr int kTile = kScanBlock * kScanItems;

__device__ __forceinline__ long long block_inclusive_scan(long long v, long long* warp_tot) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        long long t = __shfl_up_sync(kFull, v, o);
        if (lane >= o) v += t;
    }
    if (lane == 31) warp_tot[w] = v;
    __syncthreads();
    if (w == 0) {
        long long x = lane < (kScanBlock / 32) ? warp_tot[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            long long t = __shfl_up_sync(kFull, x, o);
            if (lane >= o) x += t;
        }
        if (lane < (kScanBlock / 32)) warp_tot[lane] = x;
    }
    __syncthreads();
    if (w > 0) v += warp_tot[w - 1];
    __syncthreads();
    return v;
}

__global__ void tile_sum_kernel(const int32_t* __restrict__ in, int64_t n, long long* tile_sums) {
    __shared__ long long wt[kScanBlock / 32];
    int64_t base = (int64_t)blockIdx.x * kTile;
    long long s = 0;
    for (int i = 0; i < kScanItems; ++i) {
        int64_t idx = base + (int64_t)i * kScanBlock + threadIdx.x;
        if (idx < n) s += in[idx];
    }
    long long inc = block_inclusive_scan(s, wt);
    if (threadIdx.x == kScanBlock - 1) tile_sums[blockIdx.x] = inc;
}

__global__ void scan_tile_sums_kernel(long long* tile_sums, int64_t ntiles) {
    __shared__ long long wt[kScanBlock / 32];
    long long carry = 0;
    for (int64_t base = 0; base < ntiles; base += kScanBlock) {
        int64_t idx = base + threadIdx.x;
        long long v = idx < ntiles ? tile_sums[idx] : 0;
        long long inc = block_inclusive_scan(v, wt);
        if (idx < ntiles) tile_sums[idx] = carry + inc - v;  // exclusive
        __shared__ long long last;
        if (threadIdx.x == kScanBlock - 1) last = inc;
        __syncthreads();
        carry += last;
        __syncthreads();
    }
}

template <typename OutT>
__global__ void tile_scan_kernel(const int32_t* __restrict__ in, int64_t n, const long long* tile_sums,
                                 OutT* out) {
    __shared__ long long wt[kScanBlock / 32];
    int64_t base = (int64_t)blockIdx.x * kTile + (int64_t)threadIdx.x * kScanItems;
    long long vals[kScanItems];
    long long s = 0;
    for (int i = 0; i < kScanItems; ++i) {
        int64_t idx = base + i;
        vals[i] = idx < n ? in[idx] : 0;
        s += vals[i];
    }
    long long inc = block_inclusive_scan(s, wt);
    long long run = tile_sums[blockIdx.x] + inc - s;
    for (int i = 0; i < kScanItems; ++i) {
        int64_t idx = base + i;
        if (idx < n) out[idx] = (OutT)run;
        run += vals[i];
    }
    // the total goes to out[n]
    if (blockIdx.x == gridDim.x - 1 && threadIdx.x == kScanBlock - 1) out[n] = (OutT)run;
}

template <typename OutT>
cudaError_t exclusive_scan(const int32_t* in, OutT* out, int64_t n, void* tmp, cudaStream_t s) {
    int64_t ntiles = ceil_div(n > 0 ? n : 1, kTile);
    long long* ts = reinterpret_cast<long long*>(tmp);
    tile_sum_kernel<<<(unsigned)ntiles, kScanBlock, 0, s>>>(in, n, ts);
    scan_tile_sums_kernel<<<1, kScanBlock, 0, s>>>(ts, ntiles);
    tile_scan_kernel<OutT><<<(unsigned)ntiles, kScanBlock, 0, s>>>(in, n, ts, out);
    return cudaGetLastError();
}

}  // namespace

size_t scan_tmp_bytes(int64_t n) { return (size_t)(ceil_div(n > 0 ? n : 1, kTile) + 1) * sizeof(long long); }

cudaError_t exclusive_scan_i32_to_i64(const int32_t* in, int64_t* out, int64_t n, void* tmp, cudaStream_t s) {
    return exclusive_scan<int64_t>(in, out, n, tmp, s);
}

cudaError_t exclusive_scan_i32_to_i32(const int32_t* in, int32_t* out, int64_t n, void* tmp, cudaStream_t s) {
    return exclusive_scan<int32_t>(in, out, n, tmp, s);
}

}  // namespace rchol
