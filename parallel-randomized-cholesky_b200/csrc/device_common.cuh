// Device helpers shared by the factor, assembly and solve kernels (sm_100a).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace rchol {

constexpr int kWarp = 32;
constexpr unsigned kFull = 0xffffffffu;

// Bit pattern that marks "value not produced yet" in the sync-free
// triangular solves: a quiet NaN with a payload that no arithmetic result
// carries.  A real solution component is never NaN unless the input was.
constexpr unsigned long long kPendingBits = 0x7ff4dead0000beefull;

// ---- memory-model primitives (PTX ISA 8.x memory consistency model) ----

__device__ __forceinline__ int ld_acquire(const int* p) {
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ int ld_relaxed(const int* p) {
    int v;
    asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ unsigned long long ld_relaxed_u64(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ double ld_relaxed_f64(const double* p) {
    return __longlong_as_double((long long)ld_relaxed_u64((const unsigned long long*)p));
}
__device__ __forceinline__ void st_release(int* p, int v) {
    asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void st_relaxed_f64(double* p, double v) {
    asm volatile("st.relaxed.gpu.global.f64 [%0], %1;" ::"l"(p), "d"(v) : "memory");
}
__device__ __forceinline__ int atom_add_acq_rel(int* p, int v) {
    int old;
    asm volatile("atom.acq_rel.gpu.global.add.s32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}
__device__ __forceinline__ unsigned long long global_timer_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

// First error wins; later errors keep the first code.
__device__ __forceinline__ void raise_error(int* status, int code) { atomicCAS(status, 0, code); }

// ---- Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11) ------------------

__host__ __device__ __forceinline__ void philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                                                       uint32_t k0, uint32_t k1, uint32_t out[4]) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        if (r > 0) {
            k0 += 0x9E3779B9u;
            k1 += 0xBB67AE85u;
        }
        uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ c1 ^ k0;
        uint32_t n2 = hi0 ^ c3 ^ k1;
        c0 = n0;
        c1 = lo1;
        c2 = n2;
        c3 = lo0;
    }
    out[0] = c0;
    out[1] = c1;
    out[2] = c2;
    out[3] = c3;
}

// The clique-sampling uniform for (vertex, slot): counter (vertex, slot/2,0,0),
// key = seed; words 2*(slot%2) and 2*(slot%2)+1 give 53 bits in [0,1).
__host__ __device__ __forceinline__ double sample_uniform(uint64_t seed, int32_t vertex, int32_t slot) {
    uint32_t o[4];
    philox4x32_10((uint32_t)vertex, (uint32_t)slot >> 1, 0u, 0u, (uint32_t)seed, (uint32_t)(seed >> 32), o);
    uint32_t a = o[2 * (slot & 1)], b = o[2 * (slot & 1) + 1];
    return ((double)(a >> 5) * 67108864.0 + (double)(b >> 6)) * (1.0 / 9007199254740992.0);
}

// ---- small launch helpers ----------------------------------------------

__host__ __device__ __forceinline__ int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }

// Streaming multiprocessors of the current device, queried once per device
// ordinal (1 if the query fails: launches stay correct, only smaller).
inline int current_sm_count() {
    static int cached[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) return 1;
    if (dev < 64 && cached[dev] > 0) return cached[dev];
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) return 1;
    if (dev < 64) cached[dev] = sms;
    return sms;
}

// Grid for a grid-stride loop over `work` items: enough blocks for one item
// per thread, capped at `per_sm` blocks per SM of the current device.
inline int grid_for(int64_t work, int block, int per_sm = 32) {
    int64_t g = ceil_div(work, block);
    const int64_t cap = (int64_t)current_sm_count() * per_sm;
    if (g > cap) g = cap;
    if (g < 1) g = 1;
    return (int)g;
}

}  // namespace rchol
