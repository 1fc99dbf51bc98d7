// Sliced-ELL copy of the solve matrix for the one-RHS SpMV.
//
// Rows are cut into slices of 32 consecutive rows.  Slice s stores w_s
// columns of 32 slots (w_s = longest row of the slice), column-major: slot
// (sptr[s] + k) * 32 + lane holds entry k of row 32 s + lane, index -1 and
// value 0 past the row's end.  A warp then reads every column of its slice
// with one coalesced load per array and no row-pointer round trip, and each
// lane adds its own row's products in CSR entry order.
//
// Rows longer than kLongRow get no slots (each has a CTA of its own in the
// solver).  The copy is only made when the padding is small.
#include <cstdint>

#include "device_common.cuh"
#include "rchol_internal.h"

namespace rchol {

namespace {

constexpr int kSellBlock = 256;

// width[s] = longest row of slice s (a warp per slice)
__global__ void __launch_bounds__(kSellBlock) sell_width_kernel(const int32_t* __restrict__ ptr, int32_t n,
                                                                int32_t nslices, int32_t* width) {
    const int lane = threadIdx.x & 31;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t s = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; s < nslices; s += nw) {
        const int64_t i = s * 32 + lane;
        int len = i < n ? ptr[i + 1] - ptr[i] : 0;
        if (len > kLongRow) len = 0;  // done by spmv_long_kernel
        const int w = __reduce_max_sync(kFull, len);
        if (lane == 0) width[s] = w;
    }
}

__global__ void __launch_bounds__(kSellBlock) sell_fill_kernel(const int32_t* __restrict__ ptr,
                                                               const int32_t* __restrict__ idx,
                                                               const double* __restrict__ val, int32_t n,
                                                               int32_t nslices, const int64_t* __restrict__ sptr,
                                                               int32_t* sidx, double* sval) {
    const int lane = threadIdx.x & 31;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t s = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; s < nslices; s += nw) {
        const int64_t i = s * 32 + lane;
        const int ps = i < n ? ptr[i] : 0;
        int len = i < n ? ptr[i + 1] - ps : 0;
        if (len > kLongRow) len = 0;  // done by spmv_long_kernel
        const int64_t base = sptr[s], w = sptr[s + 1] - base;
        for (int64_t k = 0; k < w; ++k) {
            const int64_t slot = (base + k) * 32 + lane;
            const bool have = k < len;
            sidx[slot] = have ? idx[ps + k] : -1;
            sval[slot] = have ? val[ps + k] : 0.0;
        }
    }
}

}  // namespace

cudaError_t build_sell(const DevCsc& A, double max_fill, DevSell& out, Scratch& sc, cudaStream_t s) {
    out.n = 0;
    out.nslices = 0;
    out.slots = 0;
    if (A.n <= 0 || A.nnz <= 0) return cudaSuccess;
    const int32_t nslices = (int32_t)(((int64_t)A.n + 31) / 32);
    int32_t* width = nullptr;
    void* tmp = nullptr;
    int sms = 0, dev = 0;
    RCHOL_TRY(cudaGetDevice(&dev));
    RCHOL_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    RCHOL_TRY(sc.get(&width, nslices));
    RCHOL_TRY(sc.get((char**)&tmp, (int64_t)scan_tmp_bytes(nslices)));
    if (out.cap_slices < (int64_t)nslices + 1) {
        cudaFree(out.sptr);
        out.sptr = nullptr;
        out.cap_slices = 0;
        RCHOL_TRY(cudaMalloc(&out.sptr, sizeof(int64_t) * ((size_t)nslices + 1)));
        out.cap_slices = (int64_t)nslices + 1;
    }
    const int64_t want_blocks = ((int64_t)nslices * 32 + kSellBlock - 1) / kSellBlock;
    const int grid = (int)(want_blocks < (int64_t)sms * 16 ? want_blocks : (int64_t)sms * 16);
    sell_width_kernel<<<grid, kSellBlock, 0, s>>>(A.colptr, A.n, nslices, width);
    RCHOL_TRY(cudaGetLastError());
    RCHOL_TRY(exclusive_scan_i32_to_i64(width, out.sptr, nslices, tmp, s));
    int64_t cols = 0;
    RCHOL_TRY(cudaMemcpyAsync(&cols, out.sptr + nslices, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    RCHOL_TRY(cudaStreamSynchronize(s));
    const int64_t slots = cols * 32;
    if ((double)slots > max_fill * (double)A.nnz) return cudaSuccess;  // too much padding: no copy
    if (out.cap_slots < slots) {
        cudaFree(out.sidx);
        cudaFree(out.sval);
        out.sidx = nullptr;
        out.sval = nullptr;
        out.cap_slots = 0;
        RCHOL_TRY(cudaMalloc(&out.sidx, sizeof(int32_t) * (size_t)slots));
        RCHOL_TRY(cudaMalloc(&out.sval, sizeof(double) * (size_t)slots));
        out.cap_slots = slots;
    }
    sell_fill_kernel<<<grid, kSellBlock, 0, s>>>(A.colptr, A.rowind, A.val, A.n, nslices, out.sptr, out.sidx,
                                                  out.sval);
    RCHOL_TRY(cudaGetLastError());
    out.n = A.n;
    out.nslices = nslices;
    out.slots = slots;
    return cudaSuccess;
}

void free_sell(DevSell& m) {
    cudaFree(m.sptr);
    cudaFree(m.sidx);
    cudaFree(m.sval);
    m = DevSell();
}

}  // namespace rchol
