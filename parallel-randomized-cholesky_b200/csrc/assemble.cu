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

__global__ void scatter_cols_kernel(int32_t nout, const int64_t* __restrict__ lc_ptr,
                                    const int64_t* __restrict__ pstart, const int32_t* __restrict__ prow,
                                    const double* __restrict__ pval, int32_t* lc_idx, double* lc_val,
                                    int32_t* row_cnt) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t k = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); k < nout; k += warps) {
        int64_t o = lc_ptr[k], len = lc_ptr[k + 1] - o, src = pstart[k];
        for (int64_t t = lane; t < len; t += 32) {
            int32_t r = prow[src + t];
            lc_idx[o + t] = r;
            lc_val[o + t] = -pval[src + t];
            atomicAdd(row_cnt + r, 1);
        }
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

__global__ void level_hist_kernel(const int32_t* __restrict__ level, int32_t n, int32_t* hist) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) atomicAdd(hist + level[i], 1);
}

__global__ void level_scatter_kernel(const int32_t* __restrict__ level, int32_t n, const int32_t* __restrict__ start,
                                     int32_t* cursor, int32_t* order) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        int l = level[i];
        order[start[l] + atomicAdd(cursor + l, 1)] = (int32_t)i;
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
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t c = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); c < nout; c += warps) {
        int k = 0;
        for (int p = colptr[c] + lane; p < colptr[c + 1]; p += 32) k += rowind[p] < nout;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) k += __shfl_xor_sync(kFull, k, o);
        if (lane == 0) cnt[c] = k;
    }
}

__global__ void trim_scatter_kernel(int32_t nout, const int32_t* __restrict__ colptr, const int32_t* __restrict__ rowind,
                                    const double* __restrict__ val, const int32_t* __restrict__ ocolptr,
                                    int32_t* orow, double* oval) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t c = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); c < nout; c += warps) {
        int out = ocolptr[c];
        for (int base = colptr[c]; base < colptr[c + 1]; base += 32) {
            int p = base + lane;
            bool take = p < colptr[c + 1] && rowind[p] < nout;
            unsigned bal = __ballot_sync(kFull, take);
            if (take) {
                int q = out + __popc(bal & ((1u << lane) - 1u));
                orow[q] = rowind[p];
                oval[q] = val[p];
            }
            out += __popc(bal);
        }
    }
}

int grid_for(int64_t work, int block) {
    int64_t g = ceil_div(work, block);
    if (g < 1) g = 1;
    if (g > 148 * 32) g = 148 * 32;
    return (int)g;
}

template <typename T>
cudaError_t dmalloc(T** p, int64_t n) {
    return cudaMalloc((void**)p, sizeof(T) * (size_t)(n > 0 ? n : 1));
}

}  // namespace

#define RCHOL_TRY(x)                        \
    do {                                    \
        cudaError_t e__ = (x);              \
        if (e__ != cudaSuccess) return e__; \
    } while (0)

cudaError_t assemble_factor(const FactorWork& w, bool trim_ground, bool make_fp32, DevFactor& f, cudaStream_t s) {
    const int32_t nout = trim_ground ? w.n - 1 : w.n;
    const int32_t ground = trim_ground ? w.n - 1 : -1;
    f.n = nout;
    int32_t* cnt = nullptr;
    void* tmp = nullptr;
    RCHOL_TRY(dmalloc(&cnt, nout));
    RCHOL_TRY(cudaMalloc(&tmp, scan_tmp_bytes(nout)));
    RCHOL_TRY(dmalloc(&f.lc_ptr, (int64_t)nout + 1));
    col_counts_kernel<<<grid_for(nout, 256), 256, 0, s>>>(nout, ground, w.pcnt, w.pstart, w.prow, cnt);
    RCHOL_TRY(cudaGetLastError());
    RCHOL_TRY(exclusive_scan_i32_to_i64(cnt, f.lc_ptr, nout, tmp, s));
    int64_t nnz = 0;
    RCHOL_TRY(cudaMemcpyAsync(&nnz, f.lc_ptr + nout, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    RCHOL_TRY(cudaStreamSynchronize(s));
    f.nnz = nnz;
    RCHOL_TRY(dmalloc(&f.lc_idx, nnz));
    RCHOL_TRY(dmalloc(&f.lc_val, nnz));
    RCHOL_TRY(dmalloc(&f.lr_idx, nnz));
    RCHOL_TRY(dmalloc(&f.lr_val, nnz));
    RCHOL_TRY(dmalloc(&f.lr_ptr, (int64_t)nout + 1));
    RCHOL_TRY(dmalloc(&f.diag, nout));
    RCHOL_TRY(cudaMemsetAsync(cnt, 0, sizeof(int32_t) * (size_t)(nout > 0 ? nout : 1), s));
    scatter_cols_kernel<<<grid_for((int64_t)nout * 32, 256), 256, 0, s>>>(nout, f.lc_ptr, w.pstart, w.prow, w.pval,
                                                                          f.lc_idx, f.lc_val, cnt);
    RCHOL_TRY(cudaGetLastError());
    RCHOL_TRY(exclusive_scan_i32_to_i64(cnt, f.lr_ptr, nout, tmp, s));
    RCHOL_TRY(cudaMemsetAsync(cnt, 0, sizeof(int32_t) * (size_t)(nout > 0 ? nout : 1), s));
    transpose_kernel<<<grid_for((int64_t)nout * 32, 256), 256, 0, s>>>(nout, f.lc_ptr, f.lc_idx, f.lc_val, f.lr_ptr,
                                                                       cnt, f.lr_idx, f.lr_val);
    RCHOL_TRY(cudaGetLastError());
    // deterministic row order: warp sort for short rows, CTA sort for long ones
    const int sort_block = 256;
    const int sort_grid = 148 * 4;
    int32_t* dsc = nullptr;  // [0] long-row count, [1] max row length, [2] max level
    int32_t* long_rows = nullptr;
    RCHOL_TRY(dmalloc(&dsc, 4));
    RCHOL_TRY(dmalloc(&long_rows, nout));
    RCHOL_TRY(cudaMemsetAsync(dsc, 0, sizeof(int32_t) * 4, s));
    max_kernel<<<grid_for(nout, 256), 256, 0, s>>>(cnt, nout, dsc + 1);
    max_kernel<<<grid_for(nout, 256), 256, 0, s>>>(w.level, nout, dsc + 2);
    sort_rows_kernel<<<sort_grid, sort_block, 0, s>>>(nout, f.lr_ptr, f.lr_idx, f.lr_val, long_rows, dsc);
    RCHOL_TRY(cudaGetLastError());
    int32_t hs[4] = {0, 0, 0, 0};
    RCHOL_TRY(cudaMemcpyAsync(hs, dsc, sizeof(hs), cudaMemcpyDeviceToHost, s));
    RCHOL_TRY(cudaStreamSynchronize(s));
    int32_t* gkey = nullptr;
    double* gval = nullptr;
    int64_t gcap = 1;
    const int lgrid = hs[0] > 0 ? std::min(hs[0], 148 * 2) : 1;
    if (hs[1] > kBlockSortCap) {
        while (gcap < hs[1]) gcap <<= 1;
        RCHOL_TRY(dmalloc(&gkey, (int64_t)lgrid * gcap));
        RCHOL_TRY(dmalloc(&gval, (int64_t)lgrid * gcap));
    }
    if (hs[0] > 0) {
        const size_t smem = (size_t)kBlockSortCap * 12;
        RCHOL_TRY(cudaFuncSetAttribute(sort_long_rows_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        sort_long_rows_kernel<<<lgrid, 512, smem, s>>>(long_rows, hs[0], f.lr_ptr, f.lr_idx, f.lr_val, gkey, gval,
                                                        gcap, w.counters + 3);
        RCHOL_TRY(cudaGetLastError());
    }
    // rows in non-decreasing forward level
    const int32_t depth = hs[2] + 1;
    f.depth = depth;
    int32_t *hist = nullptr, *lstart = nullptr;
    RCHOL_TRY(dmalloc(&hist, depth));
    RCHOL_TRY(dmalloc(&lstart, (int64_t)depth + 1));
    RCHOL_TRY(dmalloc(&f.order, nout));
    void* tmp2 = nullptr;
    RCHOL_TRY(cudaMalloc(&tmp2, scan_tmp_bytes(depth)));
    RCHOL_TRY(cudaMemsetAsync(hist, 0, sizeof(int32_t) * (size_t)depth, s));
    level_hist_kernel<<<grid_for(nout, 256), 256, 0, s>>>(w.level, nout, hist);
    RCHOL_TRY(exclusive_scan_i32_to_i32(hist, lstart, depth, tmp2, s));
    RCHOL_TRY(cudaMemsetAsync(hist, 0, sizeof(int32_t) * (size_t)depth, s));
    level_scatter_kernel<<<grid_for(nout, 256), 256, 0, s>>>(w.level, nout, lstart, hist, f.order);
    RCHOL_TRY(cudaGetLastError());
    RCHOL_TRY(cudaMemcpyAsync(f.diag, w.diag, sizeof(double) * (size_t)nout, cudaMemcpyDeviceToDevice, s));
    if (make_fp32) {
        RCHOL_TRY(dmalloc(&f.lc_val32, nnz));
        RCHOL_TRY(dmalloc(&f.lr_val32, nnz));
        RCHOL_TRY(dmalloc(&f.diag32, nout));
        to_f32_kernel<<<grid_for(nnz, 256), 256, 0, s>>>(f.lc_val, f.lc_val32, nnz);
        to_f32_kernel<<<grid_for(nnz, 256), 256, 0, s>>>(f.lr_val, f.lr_val32, nnz);
        to_f32_kernel<<<grid_for(nout, 256), 256, 0, s>>>(f.diag, f.diag32, nout);
        RCHOL_TRY(cudaGetLastError());
    }
    RCHOL_TRY(cudaStreamSynchronize(s));
    cudaFree(gkey);
    cudaFree(gval);
    cudaFree(cnt);
    cudaFree(tmp);
    cudaFree(tmp2);
    cudaFree(hist);
    cudaFree(lstart);
    cudaFree(dsc);
    cudaFree(long_rows);
    return cudaSuccess;
}

cudaError_t trim_matrix(const DevCsc& A, DevCsc& out, cudaStream_t s) {
    const int32_t nout = A.n - 1;
    out.n = nout;
    int32_t* cnt = nullptr;
    void* tmp = nullptr;
    RCHOL_TRY(dmalloc(&cnt, nout));
    RCHOL_TRY(cudaMalloc(&tmp, scan_tmp_bytes(nout)));
    RCHOL_TRY(dmalloc(&out.colptr, (int64_t)nout + 1));
    trim_count_kernel<<<grid_for((int64_t)nout * 32, 256), 256, 0, s>>>(nout, A.colptr, A.rowind, cnt);
    RCHOL_TRY(cudaGetLastError());
    RCHOL_TRY(exclusive_scan_i32_to_i32(cnt, out.colptr, nout, tmp, s));
    int32_t nnz = 0;
    RCHOL_TRY(cudaMemcpyAsync(&nnz, out.colptr + nout, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    RCHOL_TRY(cudaStreamSynchronize(s));
    out.nnz = nnz;
    RCHOL_TRY(dmalloc(&out.rowind, nnz));
    RCHOL_TRY(dmalloc(&out.val, nnz));
    trim_scatter_kernel<<<grid_for((int64_t)nout * 32, 256), 256, 0, s>>>(nout, A.colptr, A.rowind, A.val,
                                                                          out.colptr, out.rowind, out.val);
    RCHOL_TRY(cudaGetLastError());
    RCHOL_TRY(cudaStreamSynchronize(s));
    cudaFree(cnt);
    cudaFree(tmp);
    return cudaSuccess;
}

}  // namespace rchol
