// SDDM -> ordered Laplacian on the device: the physics preprocessing of the
// reference (cpu_implementation/write_graph.jl:98-183, physics_produce), which
// the reference runs offline in Julia before its drivers read the result.
//
//   1. signs: off-diagonals -|v|, diagonal |v| (a diagonal of sum |off| per
//      column when the input has none), as the drivers' preprocessing does
//      (gpu_implementation/pre_process.hpp:189-306);
//   2. ordering (write_graph.jl:112-128): "nnz-sort" = a seeded random
//      permutation, then a stable sort by column nnz; "random" = the seeded
//      permutation alone; "given" = none.  The permutation sorts vertices by
//      a 64-bit counter-based key (splitmix64 of (seed, stream 4, vertex)),
//      ties by vertex, so it is the same permutation as the library's
//      synthetic generator draws;
//   3. ground vertex (write_graph.jl:153-163): with column sums c_j (summed in
//      row order) and their total above 1e-9, one vertex is appended whose
//      column holds -c_j for every c_j > 0 and, on the diagonal, the sum of
//      those c_j (summed in column order on the host); a total below -1e-9
//      is not diagonally dominant and is rejected.  A c_j within the
//      rounding bound of its own sum counts as zero (see col_sum_kernel).
// The result is a CSC (rows ascending per column) in the scratch arena.
#include <cmath>
#include <cstdint>
#include <vector>

#include "device_common.cuh"
#include "rchol_internal.h"

namespace rchol {

namespace {

__device__ __forceinline__ uint64_t order_mix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

// The ordering key of vertex i (stream 4 of the counter-based streams).
__device__ __forceinline__ uint64_t order_key(uint64_t seed, uint64_t i) {
    return order_mix64(order_mix64(order_mix64(seed) ^ (4ull * 0xD1B54A32D192ED03ull)) ^ i);
}

// bad index -> flags[0]; diagonal present -> flags[1]; column counts
__global__ void sddm_scan_kernel(int32_t n, int64_t nnz, const int32_t* __restrict__ rows,
                                 const int32_t* __restrict__ cols, int32_t* cnt, int32_t* flags) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nnz; k += stride) {
        const int32_t r = rows[k], c = cols[k];
        if (r < 0 || r >= n || c < 0 || c >= n) {
            flags[0] = 1;
            continue;
        }
        if (r == c) flags[1] = 1;
        atomicAdd(cnt + c, 1);
    }
}

// keys of the random permutation: low and high 32 bits of the 64-bit key
__global__ void order_keys_kernel(int32_t n, uint64_t seed, int32_t* lo, int32_t* hi) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const uint64_t k = order_key(seed, (uint64_t)i);
        lo[i] = (int32_t)(uint32_t)k;
        hi[i] = (int32_t)(uint32_t)(k >> 32);
    }
}

__global__ void invert_kernel(int32_t n, const int32_t* __restrict__ order, int32_t* pos) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += stride) pos[order[k]] = (int32_t)k;
}

__global__ void iota_kernel(int32_t n, int32_t* v) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += stride) v[k] = (int32_t)k;
}

// permuted, sign-normalised entries; with append_diag, entry nnz + j is a
// placeholder for the diagonal of input vertex j (filled after the CSC)
__global__ void permute_entries_kernel(int32_t n, int64_t nnz, int append_diag, const int32_t* __restrict__ rows,
                                       const int32_t* __restrict__ cols, const double* __restrict__ vals,
                                       const int32_t* __restrict__ pos, int32_t* prow, int32_t* pcol, double* pval) {
    const int64_t total = nnz + (append_diag ? n : 0);
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < total; k += stride) {
        if (k < nnz) {
            const int32_t r = rows[k], c = cols[k];
            prow[k] = pos[r];
            pcol[k] = pos[c];
            pval[k] = r == c ? fabs(vals[k]) : -fabs(vals[k]);
        } else {
            const int32_t j = pos[k - nnz];
            prow[k] = j;
            pcol[k] = j;
            pval[k] = 0.0;
        }
    }
}

__global__ void count_cols_kernel(int64_t total, const int32_t* __restrict__ pcol, int32_t* cnt) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < total; k += stride) atomicAdd(cnt + pcol[k], 1);
}

__global__ void gather_csc_kernel(int64_t total, const int32_t* __restrict__ ord, const int32_t* __restrict__ prow,
                                  const double* __restrict__ pval, int32_t* rowind, double* val) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < total; k += stride) {
        const int32_t e = ord[k];
        rowind[k] = prow[e];
        val[k] = pval[e];
    }
}

// the appended diagonal of column j: sum |off| in row order (one thread per
// column; the column's only diagonal entry is the placeholder)
__global__ void fill_diag_kernel(int32_t n, const int32_t* __restrict__ colptr, const int32_t* __restrict__ rowind,
                                 double* val) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += stride) {
        double s = 0.0;
        int32_t d = -1;
        for (int32_t p = colptr[j]; p < colptr[j + 1]; ++p) {
            if (rowind[p] == j) d = p;
            else s += fabs(val[p]);
        }
        if (d >= 0) val[d] = s;
    }
}

// Column sums in row order (one thread per column).  flag: c_j above the
// rounding bound of its own sum, m_j * 2^-52 * sum |a_ij| -- a column whose
// excess is zero sums to a few ulps of either sign, and a ground edge of that
// size would only add entries (write_graph.jl:158 keeps every c_j > 0).
__global__ void col_sum_kernel(int32_t n, const int32_t* __restrict__ colptr, const double* __restrict__ val,
                               double* csum, int32_t* pos_flag) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += stride) {
        double s = 0.0, a = 0.0;
        for (int32_t p = colptr[j]; p < colptr[j + 1]; ++p) {
            s += val[p];
            a += fabs(val[p]);
        }
        csum[j] = s;
        pos_flag[j] = s > (double)(colptr[j + 1] - colptr[j]) * 0x1p-52 * a ? 1 : 0;
    }
}

// total of the column sums (the threshold test only; any order)
__global__ void total_kernel(int32_t n, const double* __restrict__ csum, double* total) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t n_up = ((int64_t)n + 31) / 32 * 32;
    double s = 0.0;
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n_up; j += stride)
        if (j < n) s += csum[j];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(kFull, s, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(total, s);
}

// The matrix with the ground vertex n: every column j with c_j > 0 gains
// (n, -c_j) after its entries (n is the largest row); column n lists those
// j ascending and then its diagonal (value written by the host).
__global__ void ground_append_kernel(int32_t n, const int32_t* __restrict__ colptr, const int32_t* __restrict__ rowind,
                                     const double* __restrict__ val, const double* __restrict__ csum,
                                     const int32_t* __restrict__ gpre, int32_t* ocolptr, int32_t* orow, double* oval,
                                     double* gpos) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int32_t nnz = colptr[n], ng = gpre[n];
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += stride) {
        const int32_t s = colptr[j], e = colptr[j + 1], o = s + gpre[j];
        ocolptr[j] = o;
        for (int32_t p = s; p < e; ++p) {
            orow[o + (p - s)] = rowind[p];
            oval[o + (p - s)] = val[p];
        }
        if (gpre[j + 1] > gpre[j]) {
            orow[o + (e - s)] = n;
            oval[o + (e - s)] = -csum[j];
            orow[nnz + ng + gpre[j]] = (int32_t)j;
            oval[nnz + ng + gpre[j]] = -csum[j];
            gpos[gpre[j]] = csum[j];
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        ocolptr[n] = nnz + ng;
        ocolptr[n + 1] = nnz + 2 * ng + 1;
        orow[nnz + 2 * ng] = n;
    }
}

}  // namespace

cudaError_t sddm_to_laplacian(int32_t n, int64_t nnz, const int32_t* rows, const int32_t* cols, const double* vals,
                              int ordering, uint64_t seed, Scratch& sc, cudaStream_t s, SddmResult& res,
                              const int32_t* order_in) {
    res = SddmResult();
    if (n <= 0 || nnz < 0 || nnz + 2 * (int64_t)n + 2 >= (int64_t)INT32_MAX) return cudaErrorInvalidValue;
    if (ordering != kOrderGiven && ordering != kOrderNnzSort && ordering != kOrderRandom &&
        !(ordering == kOrderExternal && order_in))
        return cudaErrorInvalidValue;
    int32_t *cnt = nullptr, *flags = nullptr, *order = nullptr;
    RCHOL_TRY(sc.get(&cnt, n));
    RCHOL_TRY(sc.get(&flags, 2));
    RCHOL_TRY(sc.get(&order, n));
    RCHOL_TRY(sc.get(&res.perm, n));
    RCHOL_TRY(cudaMemsetAsync(cnt, 0, sizeof(int32_t) * (size_t)n, s));
    RCHOL_TRY(cudaMemsetAsync(flags, 0, sizeof(int32_t) * 2, s));
    sddm_scan_kernel<<<grid_for(nnz, 256), 256, 0, s>>>(n, nnz, rows, cols, cnt, flags);
    RCHOL_TRY(cudaGetLastError());
    int32_t hf[2] = {0, 0};
    RCHOL_TRY(cudaMemcpyAsync(hf, flags, sizeof(hf), cudaMemcpyDeviceToHost, s));
    RCHOL_TRY(cudaStreamSynchronize(s));
    if (hf[0]) {
        res.status = SddmResult::kBadIndex;
        return cudaSuccess;
    }
    const int append_diag = hf[1] ? 0 : 1;  // (every column then gains one: the count order is unchanged)
    // the permutation: order[k] = input vertex placed at position k
    if (ordering == kOrderExternal) {
        RCHOL_TRY(cudaMemcpyAsync(order, order_in, sizeof(int32_t) * (size_t)n, cudaMemcpyDeviceToDevice, s));
    } else {
        iota_kernel<<<grid_for(n, 256), 256, 0, s>>>(n, order);
        RCHOL_TRY(cudaGetLastError());
    }
    if (ordering == kOrderNnzSort || ordering == kOrderRandom) {
        int32_t *klo = nullptr, *khi = nullptr;
        RCHOL_TRY(sc.get(&klo, n));
        RCHOL_TRY(sc.get(&khi, n));
        order_keys_kernel<<<grid_for(n, 256), 256, 0, s>>>(n, seed, klo, khi);
        RCHOL_TRY(cudaGetLastError());
        // LSD over (column count, key high word, key low word), ties by vertex
        RCHOL_TRY(stable_key_order_from(klo, nullptr, n, INT32_MAX, order, sc, s));
        RCHOL_TRY(stable_key_order_from(khi, order, n, INT32_MAX, order, sc, s));
        if (ordering == kOrderNnzSort) {
            int32_t maxc = 0;
            int32_t* dmax = nullptr;
            RCHOL_TRY(sc.get(&dmax, 1));
            RCHOL_TRY(cudaMemsetAsync(dmax, 0, sizeof(int32_t), s));
            RCHOL_TRY(max_i32(cnt, n, dmax, s));
            RCHOL_TRY(cudaMemcpyAsync(&maxc, dmax, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
            RCHOL_TRY(cudaStreamSynchronize(s));
            RCHOL_TRY(stable_key_order_from(cnt, order, n, maxc + 1, order, sc, s));
        }
    }
    invert_kernel<<<grid_for(n, 256), 256, 0, s>>>(n, order, res.perm);
    RCHOL_TRY(cudaGetLastError());
    // permuted, sign-normalised entries, then the CSC by (column, row)
    const int64_t total = nnz + (append_diag ? n : 0);
    int32_t *prow = nullptr, *pcol = nullptr, *ord = nullptr, *ccnt = nullptr, *colptr = nullptr, *rowind = nullptr;
    double *pval = nullptr, *val = nullptr;
    void* tmp = nullptr;
    RCHOL_TRY(sc.get(&prow, total));
    RCHOL_TRY(sc.get(&pcol, total));
    RCHOL_TRY(sc.get(&pval, total));
    RCHOL_TRY(sc.get(&ord, total));
    RCHOL_TRY(sc.get(&ccnt, n));
    RCHOL_TRY(sc.get(&colptr, (int64_t)n + 1));
    RCHOL_TRY(sc.get(&rowind, total));
    RCHOL_TRY(sc.get(&val, total));
    RCHOL_TRY(sc.get((char**)&tmp, (int64_t)scan_tmp_bytes((int64_t)n + 2)));
    permute_entries_kernel<<<grid_for(total, 256), 256, 0, s>>>(n, nnz, append_diag, rows, cols, vals, res.perm, prow,
                                                                pcol, pval);
    RCHOL_TRY(cudaGetLastError());
    RCHOL_TRY(stable_key_order_from(prow, nullptr, (int32_t)total, n, ord, sc, s));
    RCHOL_TRY(stable_key_order_from(pcol, ord, (int32_t)total, n, ord, sc, s));
    RCHOL_TRY(cudaMemsetAsync(ccnt, 0, sizeof(int32_t) * (size_t)n, s));
    count_cols_kernel<<<grid_for(total, 256), 256, 0, s>>>(total, pcol, ccnt);
    RCHOL_TRY(cudaGetLastError());
    RCHOL_TRY(exclusive_scan_i32_to_i32(ccnt, colptr, n, tmp, s));
    gather_csc_kernel<<<grid_for(total, 256), 256, 0, s>>>(total, ord, prow, pval, rowind, val);
    RCHOL_TRY(cudaGetLastError());
    if (append_diag) {
        fill_diag_kernel<<<grid_for(n, 256), 256, 0, s>>>(n, colptr, rowind, val);
        RCHOL_TRY(cudaGetLastError());
    }
    // column sums and the ground vertex
    double *csum = nullptr, *dtot = nullptr;
    int32_t *flag = nullptr, *gpre = nullptr;
    RCHOL_TRY(sc.get(&csum, n));
    RCHOL_TRY(sc.get(&dtot, 1));
    RCHOL_TRY(sc.get(&flag, n));
    RCHOL_TRY(sc.get(&gpre, (int64_t)n + 1));
    col_sum_kernel<<<grid_for(n, 256), 256, 0, s>>>(n, colptr, val, csum, flag);
    RCHOL_TRY(cudaMemsetAsync(dtot, 0, sizeof(double), s));
    total_kernel<<<grid_for(n, 256), 256, 0, s>>>(n, csum, dtot);
    RCHOL_TRY(cudaGetLastError());
    RCHOL_TRY(exclusive_scan_i32_to_i32(flag, gpre, n, tmp, s));
    double htot = 0.0;
    int32_t ng = 0;
    RCHOL_TRY(cudaMemcpyAsync(&htot, dtot, sizeof(double), cudaMemcpyDeviceToHost, s));
    RCHOL_TRY(cudaMemcpyAsync(&ng, gpre + n, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    RCHOL_TRY(cudaStreamSynchronize(s));
    res.total = htot;
    if (htot < -1e-9) {
        res.status = SddmResult::kNotDominant;
        return cudaSuccess;
    }
    if (!(htot > 1e-9)) {
        res.n = n;
        res.nnz = total;
        res.colptr = colptr;
        res.rowind = rowind;
        res.val = val;
        return cudaSuccess;
    }
    // ground vertex n
    const int64_t nnz2 = total + 2 * (int64_t)ng + 1;
    int32_t *ocolptr = nullptr, *orow = nullptr;
    double *oval = nullptr, *gpos = nullptr;
    RCHOL_TRY(sc.get(&ocolptr, (int64_t)n + 2));
    RCHOL_TRY(sc.get(&orow, nnz2));
    RCHOL_TRY(sc.get(&oval, nnz2));
    RCHOL_TRY(sc.get(&gpos, std::max<int64_t>(ng, 1)));
    ground_append_kernel<<<grid_for(n, 256), 256, 0, s>>>(n, colptr, rowind, val, csum, gpre, ocolptr, orow, oval,
                                                          gpos);
    RCHOL_TRY(cudaGetLastError());
    // the ground diagonal: the positive column sums added in column order
    std::vector<double> hpos((size_t)ng);
    if (ng > 0)
        RCHOL_TRY(cudaMemcpyAsync(hpos.data(), gpos, sizeof(double) * (size_t)ng, cudaMemcpyDeviceToHost, s));
    RCHOL_TRY(cudaStreamSynchronize(s));
    double gd = 0.0;
    for (double x : hpos) gd += x;
    RCHOL_TRY(cudaMemcpyAsync(oval + nnz2 - 1, &gd, sizeof(double), cudaMemcpyHostToDevice, s));
    RCHOL_TRY(cudaStreamSynchronize(s));
    res.n = n + 1;
    res.nnz = nnz2;
    res.ground = true;
    res.colptr = ocolptr;
    res.rowind = orow;
    res.val = oval;
    return cudaSuccess;
}

}  // namespace rchol
