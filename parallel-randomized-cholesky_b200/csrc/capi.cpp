// C-ABI implementation (include/rchol.h): context, matrix upload, factor
// orchestration with capacity retries, PCG, the reference drop-ins.
#include <algorithm>
#include <mutex>
#include <map>
#include <chrono>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/rchol.h"
#include "host_io.h"
#include "rchol_internal.h"

using rchol::DevCsc;
using rchol::DevFactor;
using rchol::FactorWork;

struct rchol_ctx {
    rchol_opts o;
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    DevCsc A;        // as loaded (ground vertex included when trim)
    DevCsc At;       // the matrix of the solve (A itself when not trimmed)
    rchol::DevSell sell;     // sliced-ELL copy of At for the one-RHS SpMV (built on first use)
    bool sell_tried = false;
    bool trim = false;
    bool have = false;
    int32_t max_lower = 0;  // largest strict-lower column of A (bounds the first gathers)
    FactorWork w;
    bool w_ready = false;
    // solver cache
    rchol::PcgSolver* solver = nullptr;
    const rchol_factor_t* solver_f = nullptr;
    bool matrix_new = true;  // the solve matrix changed since the solver saw it
    int solver_k = 0, solver_fp32 = -1, solver_stop = -1, solver_maxit = -1, solver_poll = -1;
    double solver_tol = -1;
    // batched systems (block-diagonal stacking)
    std::vector<int64_t> batch_off;
    rchol::BatchSolver* bsolver = nullptr;
    const rchol_factor_t* bsolver_f = nullptr;
    int bsolver_k = 0;
    // assembly temporaries and the buffers of the last released factor
    rchol::Scratch scratch;
    DevFactor spare;
    // device staging for solves (row-major blocks)
    double* dB = nullptr;
    double* dX = nullptr;
    size_t stage_elems = 0;
    // factors made by this context and not yet freed: rchol_destroy detaches
    // them, so that a factor freed after its context does not touch it
    std::vector<rchol_factor_t*> live;
    // the autotuner's record of each vertex's gathered entries (device, n)
    int32_t* gsize = nullptr;
    // device flag of the input checks
    int32_t* dflag = nullptr;
    // second stream: input checks and counts under the value upload
    cudaStream_t side = nullptr;
    cudaEvent_t ev_struct = nullptr;
};

struct rchol_factor {
    rchol_ctx* ctx = nullptr;  // null once the context is destroyed
    int device = 0;
    DevFactor F;
    rchol_factor_info info;
};

namespace {

rchol_status fail(rchol_ctx* c, rchol_status s, const std::string& msg) {
    if (c) c->err = msg;
    return s;
}

rchol_status cuda_fail(rchol_ctx* c, cudaError_t e, const char* where) {
    return fail(c, RCHOL_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

#define CK(call, where)                                   \
    do {                                                  \
        cudaError_t e__ = (call);                         \
        if (e__ != cudaSuccess) return cuda_fail(ctx, e__, where); \
    } while (0)

template <typename T>
cudaError_t dalloc(T** p, int64_t n) {
    return cudaMalloc((void**)p, sizeof(T) * (size_t)(n > 0 ? n : 1));
}

void free_csc(DevCsc& a) {
    cudaFree(a.colptr);
    cudaFree(a.rowind);
    cudaFree(a.val);
    a = DevCsc();
}

void free_work(FactorWork& w) {
    void* ps[] = {w.lcolptr, w.lrow,  w.lval, w.dep,  w.queue,  w.fcnt,   w.brow,     w.bval,       w.chead,
                  w.cnext,   w.crow,  w.cval, w.prow, w.pval,   w.pstart, w.pcnt,     w.diag,       w.gscratch,
                  w.counters, w.counters64, w.scan_tmp, w.level, w.hscratch, w.hlock, w.hcols};
    for (void* p : ps) cudaFree(p);
    w = FactorWork();
}

void free_factor(DevFactor& f) {
    void* ps[] = {f.lc_ptr, f.lc_idx,  f.lc_val,  f.lc_val32, f.lr_ptr,  f.lr_idx, f.lr_val,
                  f.lr_val32, f.diag, f.diag32, f.order_f, f.order_b, f.tasks_f, f.tasks_b,
                  f.pack_f, f.pack_b, f.pf_idx, f.pf_val, f.pf_val32, f.pb_idx, f.pb_val, f.pb_val32,
                  f.split_f, f.split_b, f.psum_f, f.psum_b, f.pcount_f, f.pcount_b, f.srow_f, f.srow_b,
                  f.hb_lv, f.hb_idx, f.sf_ptr, f.sf_idx, f.sf_val, f.sf_val32, f.sb_ptr, f.sb_idx, f.sb_val,
                  f.sb_val32};
    for (void* p : ps) cudaFree(p);
    f = DevFactor();
}

int64_t pow2_ge(int64_t x) {
    int64_t p = 1;
    while (p < x) p <<= 1;
    return p;
}

bool has_device() {
    int n = 0;
    return cudaGetDeviceCount(&n) == cudaSuccess && n > 0;
}

// Sizes of the factor work pools.
struct PoolPlan {
    int c0;
    int32_t nchunks;
    int64_t pool_cap;
    int64_t gscratch_entries;
    int64_t hscratch_entries;
    int grid, block;
};

rchol_status alloc_work(rchol_ctx* ctx, const PoolPlan& pp) {
    FactorWork& w = ctx->w;
    const int32_t n = ctx->A.n;
    w.n = n;
    w.c0 = pp.c0;
    w.nchunks = pp.nchunks;
    w.pool_cap = pp.pool_cap;
    w.gscratch_entries = pp.gscratch_entries;
    w.hscratch_entries = pp.hscratch_entries;
    const int64_t warps = (int64_t)pp.grid * (pp.block / 32);
    CK(dalloc(&w.lcolptr, (int64_t)n + 1), "alloc lcolptr");
    CK(dalloc(&w.lrow, w.lnnz), "alloc lrow");
    CK(dalloc(&w.lval, w.lnnz), "alloc lval");
    CK(dalloc(&w.dep, n), "alloc dep");
    CK(dalloc(&w.queue, n), "alloc queue");
    CK(dalloc(&w.fcnt, n), "alloc fcnt");
    CK(dalloc(&w.brow, (int64_t)n * w.c0), "alloc bucket rows");
    CK(dalloc(&w.bval, (int64_t)n * w.c0), "alloc bucket values");
    CK(dalloc(&w.chead, n), "alloc chunk heads");
    CK(dalloc(&w.cnext, w.nchunks), "alloc chunk links");
    CK(dalloc(&w.crow, (int64_t)w.nchunks * 64), "alloc chunk rows");
    CK(dalloc(&w.cval, (int64_t)w.nchunks * 64), "alloc chunk values");
    CK(dalloc(&w.prow, w.pool_cap), "alloc pool rows");
    CK(dalloc(&w.pval, w.pool_cap), "alloc pool values");
    CK(dalloc(&w.pstart, n), "alloc pool starts");
    CK(dalloc(&w.pcnt, n), "alloc pool counts");
    CK(dalloc(&w.hcols, rchol::kHugeColCap + 1), "alloc long-column list");
    CK(dalloc(&w.diag, n), "alloc diag");
    CK(dalloc(&w.level, n), "alloc levels");
    CK(cudaMalloc((void**)&w.gscratch, (size_t)warps * (size_t)w.gscratch_entries * rchol::kGlobalSlabBytes),
       "alloc slab scratch");
    {
        const size_t slab = (size_t)w.hscratch_entries * rchol::kGlobalSlabBytes;
        w.nhuge = (int32_t)std::max<size_t>(rchol::kHugeSlabsMin,
                                            std::min<size_t>(rchol::kHugeSlabsMax, rchol::kHugeSlabBudget / slab));
    }
    CK(cudaMalloc((void**)&w.hscratch, (size_t)w.nhuge * (size_t)w.hscratch_entries * rchol::kGlobalSlabBytes),
       "alloc shared slabs");
    CK(dalloc(&w.hlock, w.nhuge), "alloc slab locks");
    CK(cudaMemset(w.hlock, 0, sizeof(int32_t) * w.nhuge), "clear slab locks");
    CK(dalloc(&w.counters, 16), "alloc counters");
    CK(dalloc(&w.counters64, 4), "alloc counters64");
    CK(cudaMalloc(&w.scan_tmp, rchol::scan_tmp_bytes(n)), "alloc scan scratch");
    return RCHOL_OK;
}

// Strict-lower nnz of the loaded matrix (device count + scan).
rchol_status lower_nnz(rchol_ctx* ctx, int64_t* out, cudaStream_t st = nullptr) {
    const int32_t n = ctx->A.n;
    if (!st) st = ctx->stream;
    int32_t* cnt = nullptr;
    int32_t* huge = nullptr;
    int64_t* ptr = nullptr;
    void* tmp = nullptr;
    // temporaries from the context's scratch arena (released on return)
    struct Release {
        rchol::Scratch& sc;
        ~Release() { sc.reset(); }
    } release{ctx->scratch};
    CK(ctx->scratch.get(&cnt, n), "alloc counts");
    CK(ctx->scratch.get(&huge, rchol::kHugeColCap + 1), "alloc long-column list");
    CK(ctx->scratch.get(&ptr, (int64_t)n + 1), "alloc ptr");
    CK(ctx->scratch.get((char**)&tmp, (int64_t)rchol::scan_tmp_bytes(n)), "alloc scan");
    CK(rchol::launch_count_lower(ctx->A, cnt, huge, st), "count lower");
    CK(rchol::exclusive_scan_i32_to_i64(cnt, ptr, n, tmp, st), "scan lower");
    CK(cudaMemcpyAsync(out, ptr + n, sizeof(int64_t), cudaMemcpyDeviceToHost, st), "copy lnnz");
    CK(cudaStreamSynchronize(st), "sync lnnz");
    // the largest strict-lower column (the scan scratch's first word holds it)
    int32_t* dmax = reinterpret_cast<int32_t*>(tmp);
    int32_t hmax = 0;
    CK(cudaMemsetAsync(dmax, 0, sizeof(int32_t), st), "clear max");
    CK(rchol::max_i32(cnt, n, dmax, st), "max lower");
    CK(cudaMemcpyAsync(&hmax, dmax, sizeof(int32_t), cudaMemcpyDeviceToHost, st), "copy max");
    CK(cudaStreamSynchronize(st), "sync max");
    ctx->max_lower = hmax;
    return RCHOL_OK;
}

rchol_status install_host_csc(rchol_ctx* ctx, const rchol::HostCsc& h, int trim_ground) {
    if (trim_ground && h.n < 2)
        return fail(ctx, RCHOL_ERR_INVALID, "trim_ground needs at least two vertices");
    for (double v : h.val)
        if (!std::isfinite(v)) return fail(ctx, RCHOL_ERR_NUMERIC, "non-finite matrix entry");
    return rchol_set_csc(ctx, h.n, h.colptr.data(), h.rowind.data(), h.val.data(), 0, trim_ground);
}

void drop_sell(rchol_ctx* ctx) {
    rchol::free_sell(ctx->sell);
    ctx->sell_tried = false;
}

void drop_solver(rchol_ctx* ctx) {
    if (ctx->solver) rchol::pcg_destroy(ctx->solver);
    ctx->solver = nullptr;
    ctx->solver_f = nullptr;
    if (ctx->bsolver) rchol::batch_destroy(ctx->bsolver);
    ctx->bsolver = nullptr;
    ctx->bsolver_f = nullptr;
}

rchol_status ensure_stage(rchol_ctx* ctx, size_t elems) {
    if (ctx->stage_elems >= elems) return RCHOL_OK;
    cudaFree(ctx->dB);
    cudaFree(ctx->dX);
    ctx->dB = ctx->dX = nullptr;
    ctx->stage_elems = 0;
    CK(cudaMalloc(&ctx->dB, sizeof(double) * elems), "alloc rhs staging");
    CK(cudaMalloc(&ctx->dX, sizeof(double) * elems), "alloc solution staging");
    ctx->stage_elems = elems;
    return RCHOL_OK;
}

}  // namespace

// ===========================================================================
// context
// ===========================================================================

extern "C" rchol_status rchol_opts_default(rchol_opts* o) {
    if (!o) return RCHOL_ERR_INVALID;
    std::memset(o, 0, sizeof(*o));
    o->precision = RCHOL_PREC_FP64;
    o->seed = 1;
    o->num_blocks = 0;
    o->warps_per_block = 8;
    o->slab_entries = 256;
    o->bucket_cap = 64;
    o->pool_mult = 6.0;
    o->max_iter = 1000;
    o->tol = 1e-6;
    o->stop_rule = RCHOL_STOP_RELRES;
    o->unroll = 4;
    o->use_graph = 1;
    o->device = 0;
    o->timeout_s = 30.0;
    o->verbose = 0;
    o->poll_ns = 0;
    o->sched_epl = 0;
    o->exact_bwd_levels = 1;
    o->spmv_layout = RCHOL_SPMV_AUTO;
    o->tail_vertices = 0;
    o->rhs_block = 0;
    o->bwd_head = 1;
    return RCHOL_OK;
}

static rchol_status check_opts(const rchol_opts* o, std::string& why) {
    if (o->precision != RCHOL_PREC_FP64 && o->precision != RCHOL_PREC_FP32_FACTOR) why = "precision";
    else if (o->warps_per_block < 1 || o->warps_per_block > 8) why = "warps_per_block must be 1..8";
    else if (o->slab_entries < 32 || (o->slab_entries & (o->slab_entries - 1))) why = "slab_entries must be a power of two >= 32";
    else if (o->bucket_cap < 1) why = "bucket_cap must be positive";
    else if (!(o->pool_mult >= 1.0)) why = "pool_mult must be >= 1";
    else if (o->max_iter < 1) why = "max_iter must be positive";
    else if (!(o->tol > 0.0)) why = "tol must be positive";
    else if (o->stop_rule < 0 || o->stop_rule > 2) why = "stop_rule";
    else if (o->unroll < 1 || o->unroll > 64) why = "unroll must be 1..64";
    else if (!(o->timeout_s > 0.0)) why = "timeout_s must be positive";
    else if (o->poll_ns < 0 || o->poll_ns > 100000) why = "poll_ns must be 0..100000";
    else if (o->sched_epl < 0 || o->sched_epl > 64) why = "sched_epl must be 0 (automatic) or 1..64";
    else if (o->spmv_layout != RCHOL_SPMV_AUTO && o->spmv_layout != RCHOL_SPMV_CSR) why = "spmv_layout";
    else if (o->tail_vertices < 0) why = "tail_vertices must be >= 0";
    else if (o->rhs_block != 0 && o->rhs_block != 1 && o->rhs_block != 2 && o->rhs_block != 4 && o->rhs_block != 8 &&
             o->rhs_block != 16 && o->rhs_block != 32)
        why = "rhs_block must be 0 or 1, 2, 4, 8, 16, 32";
    else if (o->bwd_head != 0 && o->bwd_head != 1) why = "bwd_head must be 0 or 1";
    else return RCHOL_OK;
    return RCHOL_ERR_INVALID;
}

extern "C" rchol_status rchol_create(rchol_ctx** out, const rchol_opts* opts) {
    if (!out) return RCHOL_ERR_INVALID;
    *out = nullptr;
    rchol_opts o;
    if (opts) o = *opts;
    else rchol_opts_default(&o);
    std::string why;
    if (check_opts(&o, why) != RCHOL_OK) return RCHOL_ERR_INVALID;
    if (!has_device()) return RCHOL_ERR_NO_DEVICE;
    if (cudaSetDevice(o.device) != cudaSuccess) return RCHOL_ERR_NO_DEVICE;
    rchol_ctx* ctx = new rchol_ctx();
    ctx->o = o;
    ctx->device = o.device;
    if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete ctx;
        return RCHOL_ERR_CUDA;
    }
    *out = ctx;
    return RCHOL_OK;
}

extern "C" void rchol_destroy(rchol_ctx* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    for (rchol_factor_t* f : ctx->live) f->ctx = nullptr;
    drop_solver(ctx);
    drop_sell(ctx);
    free_work(ctx->w);
    free_factor(ctx->spare);
    ctx->scratch.release();
    if (ctx->trim) free_csc(ctx->At);
    free_csc(ctx->A);
    cudaFree(ctx->dB);
    cudaFree(ctx->dX);
    cudaFree(ctx->gsize);
    cudaFree(ctx->dflag);
    if (ctx->ev_struct) cudaEventDestroy(ctx->ev_struct);
    if (ctx->side) cudaStreamDestroy(ctx->side);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
}

extern "C" rchol_status rchol_set_opts(rchol_ctx* ctx, const rchol_opts* o) {
    if (!ctx || !o) return RCHOL_ERR_INVALID;
    std::string why;
    if (check_opts(o, why) != RCHOL_OK) return fail(ctx, RCHOL_ERR_INVALID, "bad option: " + why);
    if (o->device != ctx->device) return fail(ctx, RCHOL_ERR_INVALID, "device cannot change");
    bool pools = o->bucket_cap != ctx->o.bucket_cap || o->pool_mult != ctx->o.pool_mult ||
                 o->slab_entries != ctx->o.slab_entries || o->warps_per_block != ctx->o.warps_per_block ||
                 o->num_blocks != ctx->o.num_blocks;
    ctx->o = *o;
    if (pools) {
        free_work(ctx->w);
        ctx->w_ready = false;
    }
    drop_solver(ctx);
    return RCHOL_OK;
}

extern "C" const char* rchol_status_string(rchol_status s) {
    switch (s) {
        case RCHOL_OK: return "ok";
        case RCHOL_ERR_INVALID: return "invalid argument";
        case RCHOL_ERR_IO: return "i/o error";
        case RCHOL_ERR_CUDA: return "CUDA error";
        case RCHOL_ERR_CAPACITY: return "device pool capacity exceeded";
        case RCHOL_ERR_TIMEOUT: return "device wait timed out";
        case RCHOL_ERR_NOT_CONVERGED: return "PCG did not converge";
        case RCHOL_ERR_NO_DEVICE: return "no CUDA device";
        case RCHOL_ERR_NUMERIC: return "non-finite or invalid numeric input";
        case RCHOL_ERR_NO_MATRIX: return "no matrix loaded";
    }
    return "unknown status";
}

extern "C" const char* rchol_last_error(const rchol_ctx* ctx) { return ctx ? ctx->err.c_str() : ""; }

// ===========================================================================
// input
// ===========================================================================

extern "C" rchol_status rchol_set_csc(rchol_ctx* ctx, int n, const int* colptr, const int* rowind,
                                      const double* val, int on_device, int trim_ground) {
    if (!ctx || n <= 0 || !colptr || !rowind || !val) return fail(ctx, RCHOL_ERR_INVALID, "bad CSC arguments");
    if (trim_ground && n < 2) return fail(ctx, RCHOL_ERR_INVALID, "trim_ground needs n >= 2");
    cudaSetDevice(ctx->device);
    int32_t nnz32 = 0;
    if (on_device) {
        CK(cudaMemcpy(&nnz32, colptr + n, sizeof(int32_t), cudaMemcpyDeviceToHost), "read nnz");
    } else {
        nnz32 = colptr[n];
    }
    if (nnz32 < 0) return fail(ctx, RCHOL_ERR_INVALID, "negative nnz");
    // a matrix of the same shape reuses every device buffer (new values or a
    // new pattern of the same size); the factor work is kept when the strict
    // lower triangle keeps its size
    const bool same = ctx->have && ctx->A.n == n && ctx->A.nnz == nnz32 && ctx->trim == (trim_ground != 0);
    const int64_t old_lnnz = ctx->w.lnnz;
    // the PCG solver, the trimmed matrix and the sliced-ELL copy keep their
    // buffers for a matrix of the same shape (refilled below / on first use)
    ctx->sell_tried = false;
    ctx->solver_f = nullptr;
    ctx->matrix_new = true;
    ctx->batch_off.clear();
    if (ctx->bsolver) drop_solver(ctx);
    DevCsc A;
    if (same) {
        A = ctx->A;
    } else {
        drop_solver(ctx);
        drop_sell(ctx);
        if (ctx->trim) free_csc(ctx->At);
        ctx->At = DevCsc();
        free_work(ctx->w);
        ctx->w_ready = false;
        free_csc(ctx->A);
        A.n = n;
        A.nnz = nnz32;
        CK(dalloc(&A.colptr, (int64_t)n + 1), "alloc colptr");
        CK(dalloc(&A.rowind, A.nnz), "alloc rowind");
        CK(dalloc(&A.val, A.nnz), "alloc val");
    }
    ctx->have = false;
    const cudaMemcpyKind kind = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    if (!ctx->dflag) CK(cudaMalloc(&ctx->dflag, sizeof(int32_t)), "alloc flag");
    if (!ctx->side) CK(cudaStreamCreateWithFlags(&ctx->side, cudaStreamNonBlocking), "side stream");
    if (!ctx->ev_struct) CK(cudaEventCreateWithFlags(&ctx->ev_struct, cudaEventDisableTiming), "event");
    CK(cudaMemcpyAsync(A.colptr, colptr, sizeof(int32_t) * ((size_t)n + 1), kind, ctx->stream), "copy colptr");
    CK(cudaMemcpyAsync(A.rowind, rowind, sizeof(int32_t) * (size_t)A.nnz, kind, ctx->stream), "copy rowind");
    CK(cudaEventRecord(ctx->ev_struct, ctx->stream), "record");
    CK(cudaMemcpyAsync(A.val, val, sizeof(double) * (size_t)A.nnz, kind, ctx->stream), "copy val");
    ctx->A = A;
    // under the value upload, on the side stream: colptr checked on the
    // device (the host arrays are not walked), then the strict-lower counts
    // that decide whether the factor work can be kept
    int32_t bad = 0;
    CK(cudaStreamWaitEvent(ctx->side, ctx->ev_struct, 0), "wait structure");
    CK(rchol::check_colptr(A.colptr, n, nnz32, ctx->dflag, ctx->side), "check colptr");
    CK(cudaMemcpyAsync(&bad, ctx->dflag, sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->side), "read flag");
    CK(cudaStreamSynchronize(ctx->side), "sync check");
    const bool recount = same && ctx->w_ready && !bad;
    int64_t lnnz = 0;
    rchol_status ls = recount ? lower_nnz(ctx, &lnnz, ctx->side) : RCHOL_OK;
    CK(cudaStreamSynchronize(ctx->stream), "sync upload");
    if (bad) return fail(ctx, RCHOL_ERR_INVALID, "colptr is not monotone (or colptr[0] != 0)");
    if (ls != RCHOL_OK) return ls;
    ctx->trim = trim_ground != 0;
    if (ctx->trim) {
        rchol::DevCsc At = ctx->At;
        const cudaError_t et = rchol::trim_matrix(ctx->A, At, ctx->scratch, ctx->stream);
        ctx->scratch.reset();
        ctx->At = At;
        CK(et, "trim matrix");
    } else {
        ctx->At = ctx->A;
    }
    CK(cudaStreamSynchronize(ctx->stream), "sync upload");
    ctx->have = true;
    if (recount) {
        if (lnnz != old_lnnz || 4 * (int64_t)ctx->max_lower > ctx->w.hscratch_entries) {
            free_work(ctx->w);
            ctx->w_ready = false;
        }
    }
    return RCHOL_OK;
}

extern "C" rchol_status rchol_set_triplets(rchol_ctx* ctx, int n, long long nnz, const int* rows, const int* cols,
                                           const double* vals, int trim_ground) {
    if (!ctx || n <= 0 || nnz < 0 || (nnz > 0 && (!rows || !cols || !vals)))
        return fail(ctx, RCHOL_ERR_INVALID, "bad triplet arguments");
    rchol::Triplets t;
    t.n = n;
    t.rows.assign(rows, rows + nnz);
    t.cols.assign(cols, cols + nnz);
    t.vals.assign(vals, vals + nnz);
    rchol::HostCsc h;
    std::string err;
    if (!rchol::triplets_to_csc(t, h, err)) return fail(ctx, RCHOL_ERR_INVALID, err);
    return install_host_csc(ctx, h, trim_ground);
}

extern "C" rchol_status rchol_set_sddm(rchol_ctx* ctx, int n, long long nnz, const int* rows, const int* cols,
                                       const double* vals, int on_device, int ordering, unsigned long long order_seed,
                                       int* perm, int* has_ground) {
    if (!ctx || n <= 0 || nnz < 0 || (nnz > 0 && (!rows || !cols || !vals)))
        return fail(ctx, RCHOL_ERR_INVALID, "bad triplet arguments");
    if (ordering != RCHOL_ORDER_GIVEN && ordering != RCHOL_ORDER_NNZ_SORT && ordering != RCHOL_ORDER_RANDOM &&
        ordering != RCHOL_ORDER_RCM && ordering != RCHOL_ORDER_ND)
        return fail(ctx, RCHOL_ERR_INVALID, "ordering must be one of RCHOL_ORDER_*");
    if (nnz + 2 * (long long)n + 2 >= (long long)INT32_MAX)
        return fail(ctx, RCHOL_ERR_INVALID, "matrix too large for int32 indices");
    cudaSetDevice(ctx->device);
    if (!on_device) {
        for (long long k = 0; k < nnz; ++k)
            if (!std::isfinite(vals[k])) return fail(ctx, RCHOL_ERR_NUMERIC, "non-finite matrix entry");
    }
    struct Release {
        rchol::Scratch& sc;
        ~Release() { sc.reset(); }
    } release{ctx->scratch};
    const int32_t* drows = rows;
    const int32_t* dcols = cols;
    const double* dvals = vals;
    if (!on_device) {
        int32_t *r = nullptr, *c = nullptr;
        double* v = nullptr;
        CK(ctx->scratch.get(&r, nnz), "alloc triplets");
        CK(ctx->scratch.get(&c, nnz), "alloc triplets");
        CK(ctx->scratch.get(&v, nnz), "alloc triplets");
        if (nnz > 0) {
            CK(cudaMemcpyAsync(r, rows, sizeof(int32_t) * (size_t)nnz, cudaMemcpyHostToDevice, ctx->stream), "upload");
            CK(cudaMemcpyAsync(c, cols, sizeof(int32_t) * (size_t)nnz, cudaMemcpyHostToDevice, ctx->stream), "upload");
            CK(cudaMemcpyAsync(v, vals, sizeof(double) * (size_t)nnz, cudaMemcpyHostToDevice, ctx->stream), "upload");
        }
        drows = r;
        dcols = c;
        dvals = v;
    }
    // RCM and nested dissection are computed on the host from the pattern
    int32_t* dorder = nullptr;
    int dev_ordering = ordering;
    if (ordering == RCHOL_ORDER_RCM || ordering == RCHOL_ORDER_ND) {
        std::vector<int32_t> hr, hc;
        const int32_t *pr = rows, *pc = cols;
        if (on_device) {
            hr.resize((size_t)nnz);
            hc.resize((size_t)nnz);
            if (nnz > 0) {
                CK(cudaMemcpy(hr.data(), rows, sizeof(int32_t) * (size_t)nnz, cudaMemcpyDeviceToHost), "copy pattern");
                CK(cudaMemcpy(hc.data(), cols, sizeof(int32_t) * (size_t)nnz, cudaMemcpyDeviceToHost), "copy pattern");
            }
            pr = hr.data();
            pc = hc.data();
        }
        std::vector<int32_t> ord;
        std::string err;
        if (!rchol::host_ordering(ordering == RCHOL_ORDER_RCM ? rchol::kHostOrderRcm : rchol::kHostOrderNd, n, nnz, pr,
                                  pc, ord, err))
            return fail(ctx, RCHOL_ERR_INVALID, err);
        CK(ctx->scratch.get(&dorder, n), "alloc order");
        CK(cudaMemcpyAsync(dorder, ord.data(), sizeof(int32_t) * (size_t)n, cudaMemcpyHostToDevice, ctx->stream),
           "upload order");
        CK(cudaStreamSynchronize(ctx->stream), "upload order");
        dev_ordering = rchol::kOrderExternal;
    }
    rchol::SddmResult res;
    CK(rchol::sddm_to_laplacian(n, nnz, drows, dcols, dvals, dev_ordering, order_seed, ctx->scratch, ctx->stream, res,
                                dorder),
       "sddm conversion");
    if (res.status == rchol::SddmResult::kBadIndex) return fail(ctx, RCHOL_ERR_INVALID, "triplet index out of range");
    if (res.status == rchol::SddmResult::kNotDominant)
        return fail(ctx, RCHOL_ERR_NUMERIC, "not diagonally dominant: the entries sum to " + std::to_string(res.total));
    if (perm) CK(cudaMemcpy(perm, res.perm, sizeof(int32_t) * (size_t)n, cudaMemcpyDeviceToHost), "copy permutation");
    if (has_ground) *has_ground = res.ground ? 1 : 0;
    return rchol_set_csc(ctx, res.n, res.colptr, res.rowind, res.val, 1, res.ground ? 1 : 0);
}

extern "C" rchol_status rchol_ordering(int kind, int n, long long nnz, const int* rows, const int* cols, int* order) {
    if (n <= 0 || nnz < 0 || (nnz > 0 && (!rows || !cols)) || !order) return RCHOL_ERR_INVALID;
    if (kind != RCHOL_ORDER_RCM && kind != RCHOL_ORDER_ND) return RCHOL_ERR_INVALID;
    std::vector<int32_t> ord;
    std::string err;
    if (!rchol::host_ordering(kind == RCHOL_ORDER_RCM ? rchol::kHostOrderRcm : rchol::kHostOrderNd, n, nnz, rows, cols,
                              ord, err))
        return RCHOL_ERR_INVALID;
    std::memcpy(order, ord.data(), sizeof(int) * (size_t)n);
    return RCHOL_OK;
}

extern "C" rchol_status rchol_write_bin(const char* path, int n, const int* colptr, const int* rowind,
                                        const double* val, int trim_ground) {
    if (!path || n <= 0 || !colptr || !rowind || !val) return RCHOL_ERR_INVALID;
    std::string err;
    return rchol::write_csc_bin(path, n, colptr, rowind, val, trim_ground, err) ? RCHOL_OK : RCHOL_ERR_IO;
}

extern "C" rchol_status rchol_read_bin(const char* path, int* n, long long* nnz, int** colptr, int** rowind,
                                       double** val, int* trim_ground) {
    if (!path || !n || !nnz || !colptr || !rowind || !val) return RCHOL_ERR_INVALID;
    rchol::HostCsc h;
    int trim = 0;
    std::string err;
    if (!rchol::read_csc_bin(path, h, trim, err)) return RCHOL_ERR_IO;
    const size_t nz = h.rowind.size();
    *colptr = (int*)std::malloc(sizeof(int) * ((size_t)h.n + 1));
    *rowind = (int*)std::malloc(sizeof(int) * std::max<size_t>(nz, 1));
    *val = (double*)std::malloc(sizeof(double) * std::max<size_t>(nz, 1));
    if (!*colptr || !*rowind || !*val) {
        std::free(*colptr);
        std::free(*rowind);
        std::free(*val);
        return RCHOL_ERR_CAPACITY;
    }
    std::memcpy(*colptr, h.colptr.data(), sizeof(int) * ((size_t)h.n + 1));
    std::memcpy(*rowind, h.rowind.data(), sizeof(int) * nz);
    std::memcpy(*val, h.val.data(), sizeof(double) * nz);
    *n = h.n;
    *nnz = (long long)nz;
    if (trim_ground) *trim_ground = trim;
    return RCHOL_OK;
}

extern "C" rchol_status rchol_load_bin(rchol_ctx* ctx, const char* path) {
    if (!ctx || !path) return fail(ctx, RCHOL_ERR_INVALID, "null path");
    rchol::HostCsc h;
    int trim = 0;
    std::string err;
    if (!rchol::read_csc_bin(path, h, trim, err)) return fail(ctx, RCHOL_ERR_IO, err);
    return install_host_csc(ctx, h, trim);
}

extern "C" rchol_status rchol_save_bin(const rchol_ctx* ctx, const char* path) {
    if (!ctx || !path) return RCHOL_ERR_INVALID;
    if (!ctx->have) return RCHOL_ERR_NO_MATRIX;
    cudaSetDevice(ctx->device);
    std::vector<int32_t> cp((size_t)ctx->A.n + 1), ri((size_t)ctx->A.nnz);
    std::vector<double> v((size_t)ctx->A.nnz);
    if (cudaMemcpy(cp.data(), ctx->A.colptr, sizeof(int32_t) * cp.size(), cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(ri.data(), ctx->A.rowind, sizeof(int32_t) * ri.size(), cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(v.data(), ctx->A.val, sizeof(double) * v.size(), cudaMemcpyDeviceToHost) != cudaSuccess)
        return RCHOL_ERR_CUDA;
    std::string err;
    return rchol::write_csc_bin(path, ctx->A.n, cp.data(), ri.data(), v.data(), ctx->trim ? 1 : 0, err)
               ? RCHOL_OK
               : RCHOL_ERR_IO;
}

extern "C" rchol_status rchol_load_mtx(rchol_ctx* ctx, const char* path, int trim_ground) {
    if (!ctx || !path) return fail(ctx, RCHOL_ERR_INVALID, "null path");
    rchol::Triplets t;
    std::string err;
    if (!rchol::read_mtx(path, t, err)) return fail(ctx, RCHOL_ERR_IO, err);
    rchol::HostCsc h;
    if (!rchol::triplets_to_csc(t, h, err)) return fail(ctx, RCHOL_ERR_INVALID, err);
    return install_host_csc(ctx, h, trim_ground);
}

extern "C" rchol_status rchol_matrix_info(const rchol_ctx* ctx, int* n, long long* nnz) {
    if (!ctx) return RCHOL_ERR_INVALID;
    if (!ctx->have) return RCHOL_ERR_NO_MATRIX;
    if (n) *n = ctx->A.n;
    if (nnz) *nnz = ctx->A.nnz;
    return RCHOL_OK;
}

extern "C" rchol_status rchol_matrix_copy_to_host(const rchol_ctx* cctx, int* colptr, int* rowind, double* val) {
    rchol_ctx* ctx = const_cast<rchol_ctx*>(cctx);
    if (!ctx) return RCHOL_ERR_INVALID;
    if (!ctx->have) return RCHOL_ERR_NO_MATRIX;
    if (colptr) CK(cudaMemcpy(colptr, ctx->A.colptr, sizeof(int32_t) * ((size_t)ctx->A.n + 1), cudaMemcpyDeviceToHost), "copy");
    if (rowind) CK(cudaMemcpy(rowind, ctx->A.rowind, sizeof(int32_t) * (size_t)ctx->A.nnz, cudaMemcpyDeviceToHost), "copy");
    if (val) CK(cudaMemcpy(val, ctx->A.val, sizeof(double) * (size_t)ctx->A.nnz, cudaMemcpyDeviceToHost), "copy");
    return RCHOL_OK;
}

// ===========================================================================
// factorization
// ===========================================================================

extern "C" rchol_status rchol_factor(rchol_ctx* ctx, rchol_factor_t** out) {
    if (!ctx || !out) return fail(ctx, RCHOL_ERR_INVALID, "null argument");
    *out = nullptr;
    if (!ctx->have) return fail(ctx, RCHOL_ERR_NO_MATRIX, "no matrix loaded");
    cudaSetDevice(ctx->device);
    const rchol_opts& o = ctx->o;
    const int block = 32 * o.warps_per_block;
    const int max_grid = rchol::factor_resident_grid(block, o.slab_entries, ctx->device);
    if (max_grid <= 0) return fail(ctx, RCHOL_ERR_CUDA, "factor kernel does not fit on the device");
    int grid = max_grid;
    if (o.num_blocks > 0) grid = std::max(1, std::min(max_grid, (o.num_blocks + o.warps_per_block - 1) / o.warps_per_block));

    if (!ctx->w_ready) {
        int64_t lnnz = 0;
        rchol_status s = lower_nnz(ctx, &lnnz);
        if (s != RCHOL_OK) return s;
        ctx->w.lnnz = lnnz;
        PoolPlan pp;
        pp.c0 = o.bucket_cap;
        pp.nchunks = (int32_t)std::min<int64_t>(INT32_MAX / 64, std::max<int64_t>(4096, lnnz / 16 + ctx->A.n / 8));
        pp.pool_cap = (int64_t)(o.pool_mult * (double)lnnz) + ctx->A.n + (int64_t)max_grid * (block / 32) * 1024;
        // per-warp scratch up to 4096 entries; larger gathers share nhuge slabs
        const int64_t want = std::max<int64_t>(1024, pow2_ge(4 * (int64_t)ctx->max_lower));
        pp.gscratch_entries = std::min<int64_t>(want, 4096);
        pp.hscratch_entries = want;
        pp.grid = max_grid;
        pp.block = block;
        s = alloc_work(ctx, pp);
        if (s != RCHOL_OK) return s;
        ctx->w_ready = true;
    }
    FactorWork& w = ctx->w;
    cudaEvent_t ev[4];
    for (auto& e : ev) CK(cudaEventCreate(&e), "event");
    rchol_factor_info info;
    std::memset(&info, 0, sizeof(info));
    int32_t counters[16];
    unsigned long long c64[4];
    int attempt = 0;
    for (;; ++attempt) {
        CK(cudaEventRecord(ev[0], ctx->stream), "record");
        CK(rchol::launch_lower_and_deps(ctx->A, w, ctx->stream), "lower triangle");
        CK(rchol::launch_init_factor_state(w, ctx->stream), "init factor state");
        CK(cudaEventRecord(ev[1], ctx->stream), "record");
        rchol::FactorLaunch fl;
        fl.grid = grid;
        fl.block = block;
        fl.smem_slab = o.slab_entries;
        fl.seed = o.seed;
        fl.timeout_s = o.timeout_s;
        fl.tail = std::min<int32_t>(std::max(0, o.tail_vertices), ctx->A.n);
        fl.gsize = ctx->gsize;
        CK(rchol::launch_factor(w, fl, ctx->stream), "factor launch");
        CK(cudaEventRecord(ev[2], ctx->stream), "record");
        CK(cudaMemcpyAsync(counters, w.counters, sizeof(counters), cudaMemcpyDeviceToHost, ctx->stream), "counters");
        CK(cudaMemcpyAsync(c64, w.counters64, sizeof(c64), cudaMemcpyDeviceToHost, ctx->stream), "counters");
        CK(cudaStreamSynchronize(ctx->stream), "factor");
        const int st = counters[3];
        if (st == 0) break;
        if (st == rchol::kDevTimeout) return fail(ctx, RCHOL_ERR_TIMEOUT, "factor: a device wait timed out");
        if (st != rchol::kDevCapacity || attempt >= 6)
            return fail(ctx, st == rchol::kDevCapacity ? RCHOL_ERR_CAPACITY : RCHOL_ERR_INVALID,
                        "factor: device status " + std::to_string(st));
        // grow the pool that ran out and retry from scratch
        PoolPlan pp{w.c0, w.nchunks, w.pool_cap, w.gscratch_entries, w.hscratch_entries, max_grid, block};
        if (counters[2] >= w.nchunks) pp.nchunks = (int32_t)std::min<int64_t>(INT32_MAX / 64, 2ll * w.nchunks + 1024);
        if ((int64_t)c64[0] > w.pool_cap) pp.pool_cap = 2 * w.pool_cap;
        if ((int64_t)counters[6] > w.hscratch_entries) pp.hscratch_entries = pow2_ge(2 * (int64_t)counters[6]);
        if (pp.nchunks == w.nchunks && pp.pool_cap == w.pool_cap && pp.hscratch_entries == w.hscratch_entries) {
            pp.nchunks = (int32_t)std::min<int64_t>(INT32_MAX / 64, 2ll * w.nchunks);
            pp.pool_cap *= 2;
            pp.hscratch_entries *= 2;
        }
        int64_t lnnz = w.lnnz;
        free_work(w);
        w.lnnz = lnnz;
        rchol_status s = alloc_work(ctx, pp);
        if (s != RCHOL_OK) return s;
    }
    rchol_factor_t* f = new rchol_factor_t();
    f->ctx = ctx;
    f->device = ctx->device;
    ctx->live.push_back(f);
    f->F = ctx->spare;  // reuse the buffers of the last released factor
    ctx->spare = DevFactor();
    cudaError_t e = rchol::assemble_factor(w, ctx->trim, o.precision == RCHOL_PREC_FP32_FACTOR, o.sched_epl,
                                           o.exact_bwd_levels != 0, o.bwd_head != 0, o.timeout_s, ctx->scratch,
                                           f->F, ctx->stream);
    if (e != cudaSuccess) {
        free_factor(f->F);
        delete f;
        return cuda_fail(ctx, e, "assemble");
    }
    CK(cudaEventRecord(ev[3], ctx->stream), "record");
    CK(cudaEventSynchronize(ev[3]), "sync");
    int32_t sort_status = 0;
    CK(cudaMemcpy(&sort_status, w.counters + 3, sizeof(int32_t), cudaMemcpyDeviceToHost), "status");
    if (sort_status != 0) {
        free_factor(f->F);
        delete f;
        return fail(ctx, RCHOL_ERR_CAPACITY, "assembly: row sort scratch too small");
    }
    cudaEventElapsedTime(&info.ms_setup, ev[0], ev[1]);
    cudaEventElapsedTime(&info.ms_factor, ev[1], ev[2]);
    cudaEventElapsedTime(&info.ms_assemble, ev[2], ev[3]);
    for (auto& x : ev) cudaEventDestroy(x);
    info.n = f->F.n;
    info.n_factored = ctx->A.n;
    info.nnz_strict = f->F.nnz;
    info.nnz_lower_a = w.lnnz;
    info.max_gather = counters[6];
    info.big_vertices = counters[5];
    info.overflow_fills = counters[7];
    info.chunks_used = counters[2];
    info.factor_grid = grid;
    info.attempts = attempt + 1;
    info.solve_depth = f->F.depth;
    info.solve_depth_b = f->F.depth_b;
    info.bwd_head_levels = f->F.hb_nlev;
    info.bwd_head_rows = f->F.hb_rows;
    // setup (count, 3-pass scan, scatter, queue) + elimination + assembly
    // (counts, scans, scatter, transpose, maxima, row sorts, level order)
    info.kernel_launches = 6 + 1 + 1 + 3 + 1 + 3 + 1 + 2 + 1 + 1 + 1 + 3 + 1 +
                           (o.precision == RCHOL_PREC_FP32_FACTOR ? 3 : 0);
    info.lc_ptr = reinterpret_cast<const long long*>(f->F.lc_ptr);
    info.lc_idx = f->F.lc_idx;
    info.lc_val = f->F.lc_val;
    info.lr_ptr = reinterpret_cast<const long long*>(f->F.lr_ptr);
    info.lr_idx = f->F.lr_idx;
    info.lr_val = f->F.lr_val;
    info.diag = f->F.diag;
    info.fills = (long long)c64[1];
    info.tail_vertices = std::min<int32_t>(std::max(0, o.tail_vertices), ctx->A.n);
    if (info.tail_vertices > 0) ++info.kernel_launches;
    // backward head: level table, then (when built) the inverse order and its slab indices
    if (o.exact_bwd_levels && o.bwd_head) info.kernel_launches += 1 + (f->F.hb_nlev > 0 ? 2 : 0);
    f->info = info;
    *out = f;
    return RCHOL_OK;
}

extern "C" rchol_status rchol_factor_get_info(const rchol_factor_t* f, rchol_factor_info* info) {
    if (!f || !info) return RCHOL_ERR_INVALID;
    *info = f->info;
    return RCHOL_OK;
}

extern "C" rchol_status rchol_factor_copy_to_host(const rchol_factor_t* f, long long* colptr, int* rowind,
                                                  double* val, double* diag) {
    if (!f) return RCHOL_ERR_INVALID;
    rchol_ctx* ctx = f->ctx;
    cudaSetDevice(f->device);
    const DevFactor& F = f->F;
    if (colptr) CK(cudaMemcpy(colptr, F.lc_ptr, sizeof(int64_t) * ((size_t)F.n + 1), cudaMemcpyDeviceToHost), "copy");
    if (rowind) CK(cudaMemcpy(rowind, F.lc_idx, sizeof(int32_t) * (size_t)F.nnz, cudaMemcpyDeviceToHost), "copy");
    if (val) CK(cudaMemcpy(val, F.lc_val, sizeof(double) * (size_t)F.nnz, cudaMemcpyDeviceToHost), "copy");
    if (diag) CK(cudaMemcpy(diag, F.diag, sizeof(double) * (size_t)F.n, cudaMemcpyDeviceToHost), "copy");
    return RCHOL_OK;
}

extern "C" rchol_status rchol_factor_write(const rchol_factor_t* f, const char* prefix) {
    if (!f || !prefix) return RCHOL_ERR_INVALID;
    rchol_ctx* ctx = f->ctx;
    const DevFactor& F = f->F;
    std::vector<int64_t> cp((size_t)F.n + 1);
    std::vector<int32_t> ri((size_t)F.nnz);
    std::vector<double> v((size_t)F.nnz), d((size_t)F.n);
    rchol_status s = rchol_factor_copy_to_host(f, reinterpret_cast<long long*>(cp.data()), ri.data(), v.data(), d.data());
    if (s != RCHOL_OK) return s;
    std::string err;
    if (!rchol::write_factor_files(prefix, F.n, cp, ri, v, d, err)) return fail(ctx, RCHOL_ERR_IO, err);
    return RCHOL_OK;
}

namespace {

// Build a DevFactor from a host strict CSC of L and D (transpose on device).
rchol_status factor_from_host_csc(rchol_ctx* ctx, int32_t n, const std::vector<int64_t>& cp,
                                  const std::vector<int32_t>& ri, const std::vector<double>& v,
                                  const std::vector<double>& d, rchol_factor_t** out) {
    // host transpose (the adopted factor is a one-off input)
    const int64_t nnz = cp[(size_t)n];
    std::vector<int64_t> rp((size_t)n + 1, 0);
    for (int64_t p = 0; p < nnz; ++p) rp[(size_t)ri[(size_t)p] + 1]++;
    for (int32_t i = 0; i < n; ++i) rp[(size_t)i + 1] += rp[(size_t)i];
    std::vector<int64_t> cur(rp.begin(), rp.end() - 1);
    std::vector<int32_t> ci((size_t)nnz);
    std::vector<double> cv((size_t)nnz);
    for (int32_t j = 0; j < n; ++j)
        for (int64_t p = cp[(size_t)j]; p < cp[(size_t)j + 1]; ++p) {
            int64_t q = cur[(size_t)ri[(size_t)p]]++;
            ci[(size_t)q] = j;
            cv[(size_t)q] = v[(size_t)p];
        }
    rchol_factor_t* f = new rchol_factor_t();
    f->ctx = ctx;
    f->device = ctx->device;
    ctx->live.push_back(f);
    DevFactor& F = f->F;
    F.n = n;
    F.nnz = nnz;
    std::vector<float> v32(v.begin(), v.end()), cv32(cv.begin(), cv.end()), d32(d.begin(), d.end());
    // forward levels of the solve DAG and the rows sorted by level
    std::vector<int32_t> lev((size_t)n, 0);
    for (int32_t j = 0; j < n; ++j)
        for (int64_t p = cp[(size_t)j]; p < cp[(size_t)j + 1]; ++p)
            lev[(size_t)ri[(size_t)p]] = std::max(lev[(size_t)ri[(size_t)p]], lev[(size_t)j] + 1);
    int32_t depth = 0;
    for (int32_t x : lev) depth = std::max(depth, x + 1);
    auto up = [&](auto** dst, const auto& src) -> cudaError_t {
        using T = typename std::remove_reference<decltype(src)>::type::value_type;
        cudaError_t e = cudaMalloc((void**)dst, sizeof(T) * std::max<size_t>(src.size(), 1));
        if (e != cudaSuccess) return e;
        return cudaMemcpy(*dst, src.data(), sizeof(T) * src.size(), cudaMemcpyHostToDevice);
    };
    cudaError_t e = cudaSuccess;
    if (e == cudaSuccess) e = up(&F.lc_ptr, cp);
    if (e == cudaSuccess) e = up(&F.lc_idx, ri);
    if (e == cudaSuccess) e = up(&F.lc_val, v);
    if (e == cudaSuccess) e = up(&F.lc_val32, v32);
    if (e == cudaSuccess) e = up(&F.lr_ptr, rp);
    if (e == cudaSuccess) e = up(&F.lr_idx, ci);
    if (e == cudaSuccess) e = up(&F.lr_val, cv);
    if (e == cudaSuccess) e = up(&F.lr_val32, cv32);
    if (e == cudaSuccess) e = up(&F.diag, d);
    if (e == cudaSuccess) e = up(&F.diag32, d32);
    F.depth = depth;
    int32_t* dlev = nullptr;
    if (e == cudaSuccess) e = up(&dlev, lev);
    if (e == cudaSuccess) {
        ctx->scratch.reset();
        int epl = ctx->o.sched_epl;
        if (epl <= 0) {
            int64_t longest = 0;
            for (int32_t i = 0; i < n; ++i) longest = std::max(longest, rp[(size_t)i + 1] - rp[(size_t)i]);
            epl = rchol::auto_sched_epl(longest);
        }
        e = rchol::build_solve_schedule(F, dlev, epl, ctx->o.exact_bwd_levels != 0, ctx->o.bwd_head != 0,
                                        ctx->o.timeout_s,
                                        ctx->scratch, ctx->stream);
        ctx->scratch.reset();
    }
    cudaFree(dlev);
    if (e != cudaSuccess) {
        free_factor(F);
        delete f;
        return cuda_fail(ctx, e, "upload factor");
    }
    std::memset(&f->info, 0, sizeof(f->info));
    f->info.n = n;
    f->info.n_factored = n;
    f->info.nnz_strict = nnz;
    f->info.lc_ptr = reinterpret_cast<const long long*>(F.lc_ptr);
    f->info.lc_idx = F.lc_idx;
    f->info.lc_val = F.lc_val;
    f->info.lr_ptr = reinterpret_cast<const long long*>(F.lr_ptr);
    f->info.lr_idx = F.lr_idx;
    f->info.lr_val = F.lr_val;
    f->info.diag = F.diag;
    f->info.solve_depth = depth;
    f->info.solve_depth_b = F.depth_b;
    f->info.bwd_head_levels = F.hb_nlev;
    f->info.bwd_head_rows = F.hb_rows;
    *out = f;
    return RCHOL_OK;
}

}  // namespace

extern "C" rchol_status rchol_factor_read(rchol_ctx* ctx, const char* prefix, rchol_factor_t** out) {
    if (!ctx || !prefix || !out) return fail(ctx, RCHOL_ERR_INVALID, "null argument");
    cudaSetDevice(ctx->device);
    int32_t n = 0;
    std::vector<int64_t> cp;
    std::vector<int32_t> ri;
    std::vector<double> v, d;
    std::string err;
    if (!rchol::read_factor_files(prefix, n, cp, ri, v, d, err)) return fail(ctx, RCHOL_ERR_IO, err);
    if (ctx->have && ctx->trim && n == ctx->A.n) {
        // a factor written before the ground trim: drop the last vertex
        std::vector<int64_t> cp2((size_t)n, 0);
        std::vector<int32_t> ri2;
        std::vector<double> v2;
        for (int32_t j = 0; j + 1 < n; ++j) {
            for (int64_t p = cp[(size_t)j]; p < cp[(size_t)j + 1]; ++p)
                if (ri[(size_t)p] < n - 1) {
                    ri2.push_back(ri[(size_t)p]);
                    v2.push_back(v[(size_t)p]);
                }
            cp2[(size_t)j + 1] = (int64_t)ri2.size();
        }
        d.resize((size_t)n - 1);
        return factor_from_host_csc(ctx, n - 1, cp2, ri2, v2, d, out);
    }
    return factor_from_host_csc(ctx, n, cp, ri, v, d, out);
}

extern "C" rchol_status rchol_factor_from_csr_upper(rchol_ctx* ctx, int n, const int* rowptr, const int* colind,
                                                    const double* val, const double* diag, int on_device,
                                                    rchol_factor_t** out) {
    if (!ctx || n <= 0 || !rowptr || !colind || !val || !diag || !out)
        return fail(ctx, RCHOL_ERR_INVALID, "null argument");
    cudaSetDevice(ctx->device);
    std::vector<int32_t> rp((size_t)n + 1);
    const cudaMemcpyKind k = cudaMemcpyDeviceToHost;
    if (on_device) CK(cudaMemcpy(rp.data(), rowptr, sizeof(int32_t) * rp.size(), k), "copy rowptr");
    else std::memcpy(rp.data(), rowptr, sizeof(int32_t) * rp.size());
    const int64_t nz = rp[(size_t)n];
    std::vector<int32_t> ci((size_t)nz);
    std::vector<double> cv((size_t)nz), d((size_t)n);
    if (on_device) {
        CK(cudaMemcpy(ci.data(), colind, sizeof(int32_t) * ci.size(), k), "copy colind");
        CK(cudaMemcpy(cv.data(), val, sizeof(double) * cv.size(), k), "copy val");
        CK(cudaMemcpy(d.data(), diag, sizeof(double) * d.size(), k), "copy diag");
    } else {
        std::memcpy(ci.data(), colind, sizeof(int32_t) * ci.size());
        std::memcpy(cv.data(), val, sizeof(double) * cv.size());
        std::memcpy(d.data(), diag, sizeof(double) * d.size());
    }
    // row r of L^T = column r of L; drop the unit diagonal, sort rows
    std::vector<int64_t> cp((size_t)n + 1, 0);
    std::vector<int32_t> ri;
    std::vector<double> v;
    ri.reserve((size_t)nz);
    v.reserve((size_t)nz);
    for (int32_t j = 0; j < n; ++j) {
        std::vector<std::pair<int32_t, double>> col;
        for (int32_t p = rp[(size_t)j]; p < rp[(size_t)j + 1]; ++p) {
            if (ci[(size_t)p] < j) return fail(ctx, RCHOL_ERR_INVALID, "factor is not upper triangular");
            if (ci[(size_t)p] == j) continue;
            col.emplace_back(ci[(size_t)p], cv[(size_t)p]);
        }
        std::sort(col.begin(), col.end());
        for (auto& e : col) {
            ri.push_back(e.first);
            v.push_back(e.second);
        }
        cp[(size_t)j + 1] = (int64_t)ri.size();
    }
    return factor_from_host_csc(ctx, n, cp, ri, v, d, out);
}

extern "C" void rchol_factor_free(rchol_factor_t* f) {
    if (!f) return;
    rchol_ctx* ctx = f->ctx;
    cudaSetDevice(f->device);
    if (ctx) {
        ctx->live.erase(std::remove(ctx->live.begin(), ctx->live.end(), f), ctx->live.end());
        // the PCG solver stays for the next factor (rchol::pcg_rebind)
        if (ctx->solver_f == f) ctx->solver_f = nullptr;
        if (ctx->bsolver_f == f) drop_solver(ctx);
        if (!ctx->spare.lc_ptr && f->F.cap_n > 0) {  // keep the buffers for the next factor
            ctx->spare = f->F;
            f->F = DevFactor();
        }
    }
    free_factor(f->F);
    delete f;
}

// ===========================================================================
// solve
// ===========================================================================

namespace {

bool valid_k(int k) { return k == 1 || k == 2 || k == 4 || k == 8 || k == 16 || k == 32; }

// The multi-RHS layouts of a factor (rchol::build_solve_layouts), built on
// its first k > 1 use: a cache of the factor's rows, so a const factor is
// extended in place.  Uses the context's scratch, which holds nothing here.
rchol_status ensure_layouts(rchol_ctx* ctx, const rchol_factor_t* f) {
    rchol_factor_t* mf = const_cast<rchol_factor_t*>(f);
    if (mf->F.lay_ready) return RCHOL_OK;
    const cudaError_t e = rchol::build_solve_layouts(mf->F, ctx->scratch, ctx->stream);
    ctx->scratch.reset();
    CK(e, "multi-RHS layouts");
    return RCHOL_OK;
}

rchol_status get_solver(rchol_ctx* ctx, const rchol_factor_t* f, int k) {
    const rchol_opts& o = ctx->o;
    if (k > 1) {
        const rchol_status ls = ensure_layouts(ctx, f);
        if (ls != RCHOL_OK) return ls;
    }
    const int fp32 = o.precision == RCHOL_PREC_FP32_FACTOR;
    const bool want_sell = k == 1 && o.spmv_layout == RCHOL_SPMV_AUTO;
    if (want_sell && !ctx->sell_tried) {
        ctx->sell_tried = true;
        cudaError_t e = rchol::build_sell(ctx->At, 1.25, ctx->sell, ctx->scratch, ctx->stream);
        ctx->scratch.reset();
        if (e == cudaErrorMemoryAllocation) {  // no room for the copy: CSR SpMV
            cudaGetLastError();
            drop_sell(ctx);
            ctx->sell_tried = true;
        } else if (e != cudaSuccess) {
            return cuda_fail(ctx, e, "sliced-ELL copy");
        }
    }
    const rchol::DevSell* sell = want_sell && ctx->sell.slots > 0 ? &ctx->sell : nullptr;
    if (ctx->solver && ctx->solver_k == k && ctx->solver_fp32 == fp32 && ctx->solver_stop == o.stop_rule &&
        ctx->solver_maxit == o.max_iter && ctx->solver_tol == o.tol && ctx->solver_poll == o.poll_ns) {
        if (ctx->solver_f == f) return RCHOL_OK;
        // another factor, or a new matrix of the same shape: keep the
        // solver's vectors and graph
        if (rchol::pcg_rebind(ctx->solver, ctx->At, sell, f->F, ctx->matrix_new) == cudaSuccess) {
            ctx->matrix_new = false;
            ctx->solver_f = f;
            return RCHOL_OK;
        }
    }
    drop_solver(ctx);
    rchol::SolveConfig cfg;
    cfg.k = k;
    cfg.fp32_factor = fp32 != 0;
    cfg.tol = o.tol;
    cfg.max_iter = o.max_iter;
    cfg.stop_rule = o.stop_rule;
    cfg.unroll = o.unroll;
    cfg.use_graph = o.use_graph != 0;
    cfg.timeout_s = o.timeout_s;
    cfg.poll_ns = o.poll_ns;
    if (cfg.fp32_factor && !f->F.lr_val32)
        return fail(ctx, RCHOL_ERR_INVALID, "factor has no FP32 copy (factor with RCHOL_PREC_FP32_FACTOR)");
    cudaError_t e = cudaSuccess;
    ctx->solver = rchol::pcg_create(ctx->At, f->F, cfg, ctx->device, ctx->stream, &e, sell);
    if (!ctx->solver) return cuda_fail(ctx, e, "create solver");
    ctx->matrix_new = false;
    ctx->solver_f = f;
    ctx->solver_k = k;
    ctx->solver_fp32 = fp32;
    ctx->solver_stop = o.stop_rule;
    ctx->solver_maxit = o.max_iter;
    ctx->solver_tol = o.tol;
    ctx->solver_poll = o.poll_ns;
    return RCHOL_OK;
}

// Bring a column-major block (host or device) into the row-major staging buffer.
rchol_status stage_in(rchol_ctx* ctx, const double* B, int ldb, int k, int on_device, double* dst) {
    const int32_t n = ctx->At.n;
    if (k == 1 && on_device) {
        CK(cudaMemcpyAsync(dst, B, sizeof(double) * (size_t)n, cudaMemcpyDeviceToDevice, ctx->stream), "copy rhs");
        return RCHOL_OK;
    }
    if (on_device) {
        CK(rchol::cm_to_rm(B, ldb, dst, n, k, ctx->stream), "layout");
        return RCHOL_OK;
    }
    // host: upload column by column into the X staging (as column-major), then transpose
    double* tmp = dst == ctx->dB ? ctx->dX : ctx->dB;
    for (int c = 0; c < k; ++c)
        CK(cudaMemcpyAsync(tmp + (size_t)c * n, B + (size_t)c * ldb, sizeof(double) * (size_t)n,
                           cudaMemcpyHostToDevice, ctx->stream),
           "upload rhs");
    if (k == 1) {
        CK(cudaMemcpyAsync(dst, tmp, sizeof(double) * (size_t)n, cudaMemcpyDeviceToDevice, ctx->stream), "copy");
    } else {
        CK(rchol::cm_to_rm(tmp, n, dst, n, k, ctx->stream), "layout");
    }
    return RCHOL_OK;
}

rchol_status stage_out(rchol_ctx* ctx, const double* src, double* X, int ldb, int k, int on_device) {
    const int32_t n = ctx->At.n;
    if (on_device) {
        if (k == 1) CK(cudaMemcpyAsync(X, src, sizeof(double) * (size_t)n, cudaMemcpyDeviceToDevice, ctx->stream), "copy");
        else CK(rchol::rm_to_cm(src, X, ldb, n, k, ctx->stream), "layout");
        return RCHOL_OK;
    }
    const double* cm = src;
    if (k > 1) {
        double* tmp = src == ctx->dX ? ctx->dB : ctx->dX;
        CK(rchol::rm_to_cm(src, tmp, n, n, k, ctx->stream), "layout");
        cm = tmp;
    }
    for (int c = 0; c < k; ++c)
        CK(cudaMemcpyAsync(X + (size_t)c * ldb, cm + (size_t)c * n, sizeof(double) * (size_t)n,
                           cudaMemcpyDeviceToHost, ctx->stream),
           "download solution");
    return RCHOL_OK;
}

}  // namespace

static rchol_status pcg_solve_block(rchol_ctx* ctx, const rchol_factor_t* f, int k, const double* B, double* X,
                                    int ldb, int on_device, rchol_solve_info* info);

extern "C" rchol_status rchol_pcg_solve(rchol_ctx* ctx, const rchol_factor_t* f, int k, const double* B, double* X,
                                        int ldb, int on_device, rchol_solve_info* info) {
    const int blk = ctx ? ctx->o.rhs_block : 0;
    if (!ctx || !f || !B || !X || blk <= 0 || k <= blk) return pcg_solve_block(ctx, f, k, B, X, ldb, on_device, info);
    if (!valid_k(k)) return fail(ctx, RCHOL_ERR_INVALID, "k must be 1, 2, 4, 8, 16 or 32");
    // k right-hand sides in blocks of rhs_block columns (column-major: block
    // j starts at column j * blk), each its own PCG; the statistics merge
    rchol_solve_info tot;
    std::memset(&tot, 0, sizeof(tot));
    tot.converged = 1;
    rchol_status worst = RCHOL_OK;
    for (int c0 = 0; c0 < k; c0 += blk) {
        rchol_solve_info bi;
        std::memset(&bi, 0, sizeof(bi));
        const rchol_status s = pcg_solve_block(ctx, f, blk, B + (size_t)c0 * ldb, X + (size_t)c0 * ldb, ldb,
                                               on_device, &bi);
        if (s != RCHOL_OK && s != RCHOL_ERR_NOT_CONVERGED) return s;
        if (s != RCHOL_OK) worst = s;
        tot.iterations = std::max(tot.iterations, bi.iterations);
        tot.converged = tot.converged && bi.converged;
        tot.device_status = tot.device_status ? tot.device_status : bi.device_status;
        tot.relres_true = std::max(tot.relres_true, bi.relres_true);
        tot.relres_rec = std::max(tot.relres_rec, bi.relres_rec);
        tot.precond_ratio = std::max(tot.precond_ratio, bi.precond_ratio);
        tot.ms_total += bi.ms_total;
        tot.ms_iterations += bi.ms_iterations;
        tot.kernel_launches += bi.kernel_launches;
        tot.graph_launches += bi.graph_launches;
    }
    if (info) *info = tot;
    return worst == RCHOL_OK ? RCHOL_OK : fail(ctx, worst, "pcg did not reach the tolerance");
}

static rchol_status pcg_solve_block(rchol_ctx* ctx, const rchol_factor_t* f, int k, const double* B, double* X,
                                    int ldb, int on_device, rchol_solve_info* info) {
    if (!ctx || !f || !B || !X) return fail(ctx, RCHOL_ERR_INVALID, "null argument");
    if (!ctx->have) return fail(ctx, RCHOL_ERR_NO_MATRIX, "no matrix loaded");
    if (!valid_k(k)) return fail(ctx, RCHOL_ERR_INVALID, "k must be 1, 2, 4, 8, 16 or 32");
    if (f->F.n != ctx->At.n) return fail(ctx, RCHOL_ERR_INVALID, "factor and matrix sizes differ");
    if (ldb < ctx->At.n) return fail(ctx, RCHOL_ERR_INVALID, "ldb < n");
    cudaSetDevice(ctx->device);
    rchol_status s = get_solver(ctx, f, k);
    if (s != RCHOL_OK) return s;
    s = ensure_stage(ctx, (size_t)ctx->At.n * (size_t)k);
    if (s != RCHOL_OK) return s;
    s = stage_in(ctx, B, ldb, k, on_device, ctx->dB);
    if (s != RCHOL_OK) return s;
    rchol::SolveResult r;
    cudaError_t e = rchol::pcg_solve(ctx->solver, ctx->dB, ctx->dX, &r);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "pcg");
    s = stage_out(ctx, ctx->dX, X, ldb, k, on_device);
    if (s != RCHOL_OK) return s;
    CK(cudaStreamSynchronize(ctx->stream), "sync solve");
    if (info) {
        info->iterations = r.iterations;
        info->converged = r.converged;
        info->device_status = r.status;
        info->relres_true = r.relres_true;
        info->relres_rec = r.relres_rec;
        info->precond_ratio = r.precond_ratio;
        info->ms_total = r.ms_total;
        info->ms_iterations = r.ms_iterations;
        info->kernel_launches = r.kernel_launches;
        info->graph_launches = r.graph_launches;
    }
    if (r.status == rchol::kDevTimeout) return fail(ctx, RCHOL_ERR_TIMEOUT, "pcg: a device wait timed out");
    if (!r.converged) return fail(ctx, RCHOL_ERR_NOT_CONVERGED, "pcg did not reach the tolerance");
    return RCHOL_OK;
}

extern "C" rchol_status rchol_precond_apply(rchol_ctx* ctx, const rchol_factor_t* f, int k, const double* R,
                                            double* Z, int ldb, int on_device, int fp32) {
    if (!ctx || !f || !R || !Z) return fail(ctx, RCHOL_ERR_INVALID, "null argument");
    if (!valid_k(k)) return fail(ctx, RCHOL_ERR_INVALID, "k must be 1, 2, 4, 8, 16 or 32");
    if (ldb < f->F.n) return fail(ctx, RCHOL_ERR_INVALID, "ldb < n");
    if (fp32 && !f->F.lr_val32) return fail(ctx, RCHOL_ERR_INVALID, "factor has no FP32 copy");
    if (!ctx->have || ctx->At.n != f->F.n) return fail(ctx, RCHOL_ERR_INVALID, "factor does not match the matrix");
    cudaSetDevice(ctx->device);
    const size_t elems = (size_t)f->F.n * (size_t)k;
    rchol_status s = k > 1 ? ensure_layouts(ctx, f) : RCHOL_OK;
    if (s != RCHOL_OK) return s;
    s = ensure_stage(ctx, 2 * elems);
    if (s != RCHOL_OK) return s;
    s = stage_in(ctx, R, ldb, k, on_device, ctx->dB);
    if (s != RCHOL_OK) return s;
    int status = 0;
    // ctx->dX holds z, its second half the y work vector
    CK(rchol::precond_apply(f->F, ctx->dB, ctx->dX, ctx->dX + elems, k, fp32 != 0, &status, ctx->o.timeout_s,
                            ctx->stream),
       "precond apply");
    if (status != 0) return fail(ctx, RCHOL_ERR_TIMEOUT, "precond apply: a device wait timed out");
    s = stage_out(ctx, ctx->dX, Z, ldb, k, on_device);
    if (s != RCHOL_OK) return s;
    CK(cudaStreamSynchronize(ctx->stream), "sync");
    return RCHOL_OK;
}

extern "C" rchol_status rchol_precond_apply_noalloc(const rchol_factor_t* f, int k, const double* R, double* Z,
                                                    int fp32, void* stream) {
    if (!f) return RCHOL_ERR_INVALID;
    rchol_ctx* ctx = f->ctx;
    if (!R || !Z) return fail(ctx, RCHOL_ERR_INVALID, "null argument");
    if (!valid_k(k)) return fail(ctx, RCHOL_ERR_INVALID, "k must be 1, 2, 4, 8, 16 or 32");
    if (fp32 && !f->F.lr_val32) return fail(ctx, RCHOL_ERR_INVALID, "factor has no FP32 copy");
    if ((long long)f->F.n * k > rchol::kNoAllocMaxElems)
        return fail(ctx, RCHOL_ERR_INVALID,
                    "precond_apply_noalloc: n * k = " + std::to_string((long long)f->F.n * k) +
                        " exceeds the allocation-free limit of " + std::to_string(rchol::kNoAllocMaxElems) +
                        " elements");
    cudaSetDevice(f->device);
    int status = 0;
    CK(rchol::precond_apply_noalloc(f->F, R, Z, k, fp32 != 0, &status, ctx ? ctx->o.timeout_s : 30.0,
                                    (cudaStream_t)stream),
       "precond apply (no alloc)");
    if (status != 0) return fail(ctx, RCHOL_ERR_TIMEOUT, "precond apply: a device wait timed out");
    return RCHOL_OK;
}

// ---- autotuner ----------------------------------------------------------------
// Picks, for the loaded matrix on this GPU: the tail of vertices eliminated
// by the cooperative CTA pass (tail_vertices), the first fill-chunk size per
// column (bucket_cap) and the right-hand-side block width of multi-RHS
// solves (rhs_block).  One factorization records every vertex's gathered
// entries; the candidates come from that profile and each is kept only when
// a timed trial beats the options it started from.  Results are cached per
// process, keyed by the matrix fingerprint (n, nnz, trim, a hash of the
// column-length histogram), the GPU, the precision and max_rhs.

namespace {
std::mutex g_tune_mu;
std::map<std::string, rchol_tune_result> g_tune_cache;

// Factor once with `o` and return its factor time (ms), or < 0 on failure.
float timed_factor(rchol_ctx* ctx, const rchol_opts& o, rchol_status* st) {
    *st = rchol_set_opts(ctx, &o);
    if (*st != RCHOL_OK) return -1.0f;
    rchol_factor_t* f = nullptr;
    *st = rchol_factor(ctx, &f);
    if (*st != RCHOL_OK) return -1.0f;
    const float ms = f->info.ms_factor;
    rchol_factor_free(f);
    return ms;
}
}  // namespace

extern "C" rchol_status rchol_autotune(rchol_ctx* ctx, int max_rhs, rchol_tune_result* out) {
    if (!ctx || !out) return fail(ctx, RCHOL_ERR_INVALID, "null argument");
    if (!ctx->have) return fail(ctx, RCHOL_ERR_NO_MATRIX, "no matrix loaded");
    if (max_rhs < 1 || max_rhs > 32) return fail(ctx, RCHOL_ERR_INVALID, "max_rhs must be 1..32");
    cudaSetDevice(ctx->device);
    std::memset(out, 0, sizeof(*out));
    const int32_t n = ctx->A.n;
    // fingerprint
    std::vector<int32_t> cp((size_t)n + 1);
    CK(cudaMemcpy(cp.data(), ctx->A.colptr, sizeof(int32_t) * cp.size(), cudaMemcpyDeviceToHost), "copy colptr");
    std::map<int32_t, int64_t> hist;
    for (int32_t j = 0; j < n; ++j) hist[cp[(size_t)j + 1] - cp[(size_t)j]]++;
    uint64_t h = 1469598103934665603ull;
    for (auto& kv : hist) {
        h = (h ^ (uint64_t)(uint32_t)kv.first) * 1099511628211ull;
        h = (h ^ (uint64_t)kv.second) * 1099511628211ull;
    }
    cudaDeviceProp prop;
    CK(cudaGetDeviceProperties(&prop, ctx->device), "device properties");
    const std::string key = std::to_string(n) + "/" + std::to_string(ctx->A.nnz) + "/" + std::to_string(ctx->trim) +
                            "/" + std::to_string(h) + "/" + prop.name + "/" + std::to_string(ctx->o.precision) + "/" +
                            std::to_string(max_rhs);
    rchol_opts base = ctx->o;
    {
        std::lock_guard<std::mutex> guard(g_tune_mu);
        auto it = g_tune_cache.find(key);
        if (it != g_tune_cache.end()) {
            *out = it->second;
            out->from_cache = 1;
            rchol_opts o = base;
            o.tail_vertices = out->tail_vertices;
            o.bucket_cap = out->bucket_cap;
            o.rhs_block = out->rhs_block;
            return rchol_set_opts(ctx, &o);
        }
    }
    // 1. profile: every vertex's gathered entries, no cooperative tail
    rchol_opts o = base;
    o.tail_vertices = 0;
    rchol_status st = rchol_set_opts(ctx, &o);
    if (st != RCHOL_OK) return st;
    CK(cudaMalloc(&ctx->gsize, sizeof(int32_t) * (size_t)n), "alloc gather record");
    CK(cudaMemset(ctx->gsize, 0, sizeof(int32_t) * (size_t)n), "clear gather record");
    rchol_factor_t* f0 = nullptr;
    st = rchol_factor(ctx, &f0);
    std::vector<int32_t> g((size_t)n);
    if (st == RCHOL_OK) {
        out->ms_factor_default = f0->info.ms_factor;
        out->max_gather = f0->info.max_gather;
        if (cudaMemcpy(g.data(), ctx->gsize, sizeof(int32_t) * (size_t)n, cudaMemcpyDeviceToHost) != cudaSuccess)
            st = RCHOL_ERR_CUDA;
        rchol_factor_free(f0);
    }
    cudaFree(ctx->gsize);
    ctx->gsize = nullptr;
    if (st != RCHOL_OK) return st;
    float best = out->ms_factor_default;
    // 2. tail: the longest suffix in which at least 3/4 of the vertices
    // gather >= 1024 entries (at least 64 vertices long)
    int32_t tail = 0, big = 0;
    for (int32_t L = 1; L <= n; ++L) {
        big += g[(size_t)(n - L)] >= 1024;
        if (4 * big >= 3 * L) tail = L;
    }
    if (tail < 64) tail = 0;
    if (tail > 0) {
        o.tail_vertices = tail;
        const float ms = timed_factor(ctx, o, &st);
        if (st != RCHOL_OK) return st;
        if (ms < best) best = ms;
        else o.tail_vertices = 0;
    }
    // 3. bucket capacity: the power of two covering 95% of the gathers,
    // then twice and four times that (fewer overflow-chunk walks for the
    // big gathers), while the buckets fit a quarter of the free memory
    std::vector<int32_t> sorted(g);
    std::sort(sorted.begin(), sorted.end());
    const int32_t p95 = sorted.empty() ? 0 : sorted[(size_t)((sorted.size() - 1) * 95 / 100)];
    int cap = 8;
    while (cap < p95 && cap < 64) cap <<= 1;
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) free_b = 0;
    for (int c = cap; c <= std::min(4 * cap, 128); c <<= 1) {
        if (c == o.bucket_cap) continue;
        const double bytes = (double)n * (double)(c - o.bucket_cap) * 12.0;
        if (bytes > 0.25 * (double)free_b) break;
        rchol_opts t = o;
        t.bucket_cap = c;
        const float ms = timed_factor(ctx, t, &st);
        if (st != RCHOL_OK) return st;
        if (ms < best) {
            best = ms;
            o = t;
        }
    }
    out->ms_factor_tuned = best;
    // 4. right-hand-side block: the width with the least iteration time per RHS
    o.rhs_block = 0;
    if (max_rhs > 1) {
        st = rchol_set_opts(ctx, &o);
        if (st != RCHOL_OK) return st;
        rchol_factor_t* f = nullptr;
        st = rchol_factor(ctx, &f);
        if (st != RCHOL_OK) return st;
        float best_rhs = 0.0f;
        int kbest = 1;
        for (int q = 0, kk = 1; kk <= max_rhs && q < 6; ++q, kk <<= 1) {
            float ms3[3] = {0, 0, 0};
            st = rchol_profile_solve(ctx, f, kk, 3, ms3);
            if (st != RCHOL_OK) break;
            out->per_rhs_ms[q] = (ms3[0] + ms3[1] + ms3[2]) / (float)kk;
            if (kk == 1 || out->per_rhs_ms[q] < best_rhs) {
                best_rhs = out->per_rhs_ms[q];
                kbest = kk;
            }
        }
        rchol_factor_free(f);
        if (st != RCHOL_OK) return st;
        o.rhs_block = kbest;
    }
    out->tail_vertices = o.tail_vertices;
    out->bucket_cap = o.bucket_cap;
    out->rhs_block = o.rhs_block;
    st = rchol_set_opts(ctx, &o);
    if (st != RCHOL_OK) return st;
    std::lock_guard<std::mutex> guard(g_tune_mu);
    g_tune_cache[key] = *out;
    return RCHOL_OK;
}

extern "C" rchol_status rchol_profile_solve(rchol_ctx* ctx, const rchol_factor_t* f, int k, int reps,
                                            float* ms_out) {
    if (!ctx || !f || !ms_out || reps < 1) return fail(ctx, RCHOL_ERR_INVALID, "bad argument");
    if (!valid_k(k)) return fail(ctx, RCHOL_ERR_INVALID, "k must be 1, 2, 4, 8, 16 or 32");
    if (!ctx->have || ctx->At.n != f->F.n) return fail(ctx, RCHOL_ERR_INVALID, "factor does not match the matrix");
    cudaSetDevice(ctx->device);
    rchol_status s = get_solver(ctx, f, k);
    if (s != RCHOL_OK) return s;
    const size_t elems = (size_t)f->F.n * (size_t)k;
    s = ensure_stage(ctx, elems);
    if (s != RCHOL_OK) return s;
    std::vector<double> b(elems);
    std::mt19937_64 g(12345);
    std::normal_distribution<double> nd(0.0, 1.0);
    for (int c = 0; c < k; ++c) {
        double mean = 0;
        for (int32_t i = 0; i < f->F.n; ++i) mean += (b[(size_t)i * k + c] = nd(g));
        mean /= f->F.n;
        for (int32_t i = 0; i < f->F.n; ++i) b[(size_t)i * k + c] -= mean;
    }
    CK(cudaMemcpyAsync(ctx->dB, b.data(), sizeof(double) * elems, cudaMemcpyHostToDevice, ctx->stream), "upload");
    CK(rchol::pcg_profile(ctx->solver, ctx->dB, ctx->dX, reps, ms_out), "profile");
    CK(cudaStreamSynchronize(ctx->stream), "sync");
    return RCHOL_OK;
}

extern "C" rchol_status rchol_hop_latency(rchol_ctx* ctx, int rounds, double* ns_per_hop, int* sm_pair) {
    if (!ctx || !ns_per_hop || rounds < 64 || rounds > (1 << 20)) return fail(ctx, RCHOL_ERR_INVALID, "bad argument");
    cudaSetDevice(ctx->device);
    const cudaError_t e = rchol::hop_latency(rounds, ns_per_hop, sm_pair);
    if (e == cudaErrorTimeout) return fail(ctx, RCHOL_ERR_TIMEOUT, "hop probe: a wait ran out (2 s)");
    CK(e, "hop probe");
    return RCHOL_OK;
}

extern "C" rchol_status rchol_spmv(rchol_ctx* ctx, int k, const double* X, double* Y, int ldb, int on_device) {
    if (!ctx || !X || !Y) return fail(ctx, RCHOL_ERR_INVALID, "null argument");
    if (!ctx->have) return fail(ctx, RCHOL_ERR_NO_MATRIX, "no matrix loaded");
    if (!valid_k(k)) return fail(ctx, RCHOL_ERR_INVALID, "k must be 1, 2, 4, 8, 16 or 32");
    if (ldb < ctx->At.n) return fail(ctx, RCHOL_ERR_INVALID, "ldb < n");
    cudaSetDevice(ctx->device);
    const size_t elems = (size_t)ctx->At.n * (size_t)k;
    rchol_status s = ensure_stage(ctx, elems);
    if (s != RCHOL_OK) return s;
    s = stage_in(ctx, X, ldb, k, on_device, ctx->dB);
    if (s != RCHOL_OK) return s;
    CK(rchol::spmv_f64(ctx->At, ctx->dB, ctx->dX, k, ctx->stream), "spmv");
    s = stage_out(ctx, ctx->dX, Y, ldb, k, on_device);
    if (s != RCHOL_OK) return s;
    CK(cudaStreamSynchronize(ctx->stream), "sync");
    return RCHOL_OK;
}

// ===========================================================================
// reference drop-ins
// ===========================================================================

namespace {

// generate_zero_sum_vector (solver.hpp:43-61): libstdc++'s std::mt19937 and
// uniform_real_distribution, as the reference.
void zero_sum_rhs(std::vector<double>& b, size_t n, unsigned long seed) {
    std::mt19937 gen(seed);
    std::uniform_real_distribution<double> dist(0.0, 1.0);
    double sum = 0.0;
    b.resize(n);
    for (size_t i = 0; i < n; ++i) {
        b[i] = dist(gen);
        sum += b[i];
    }
    double mean = sum / (double)n;
    for (size_t i = 0; i < n; ++i) b[i] -= mean;
}

// generate_random_vector (solver.hpp:29-41): U(-1,1), seed 0
void random_vec(std::vector<double>& v, size_t n, unsigned long seed) {
    std::mt19937 gen(seed);
    std::uniform_real_distribution<double> dist(-1.0, 1.0);
    v.resize(n);
    for (size_t i = 0; i < n; ++i) v[i] = dist(gen);
}

}  // namespace

extern "C" rchol_status rchol_batch_set(rchol_ctx* ctx, int nsys, const rchol_system* sys, long long* offsets) {
    if (!ctx || nsys < 1 || !sys) return fail(ctx, RCHOL_ERR_INVALID, "bad batch arguments");
    std::vector<int64_t> off((size_t)nsys + 1, 0);
    for (int s = 0; s < nsys; ++s) {
        if (sys[s].n < 32 || !sys[s].colptr || !sys[s].rowind || !sys[s].val)
            return fail(ctx, RCHOL_ERR_INVALID, "every batched system needs >= 32 vertices and CSC arrays");
        off[(size_t)s + 1] = off[(size_t)s] + sys[s].n;
    }
    if (off[(size_t)nsys] > INT32_MAX) return fail(ctx, RCHOL_ERR_INVALID, "batch too large");
    int64_t nnz = 0;
    for (int s = 0; s < nsys; ++s) nnz += sys[s].colptr[sys[s].n];
    if (nnz > INT32_MAX) return fail(ctx, RCHOL_ERR_INVALID, "batch has more than 2^31-1 entries");
    const int32_t n = (int32_t)off[(size_t)nsys];
    std::vector<int32_t> cp((size_t)n + 1), ri((size_t)nnz);
    std::vector<double> v((size_t)nnz);
    int64_t pos = 0;
    for (int s = 0; s < nsys; ++s) {
        const int32_t o = (int32_t)off[(size_t)s];
        const int32_t ns = sys[s].n;
        for (int32_t j = 0; j < ns; ++j) {
            cp[(size_t)o + j] = (int32_t)pos;
            for (int32_t p = sys[s].colptr[j]; p < sys[s].colptr[j + 1]; ++p) {
                const int32_t r = sys[s].rowind[p];
                if (r < 0 || r >= ns) return fail(ctx, RCHOL_ERR_INVALID, "row index out of range in a system");
                ri[(size_t)pos] = o + r;
                v[(size_t)pos] = sys[s].val[p];
                ++pos;
            }
        }
    }
    cp[(size_t)n] = (int32_t)pos;
    rchol_status st = rchol_set_csc(ctx, n, cp.data(), ri.data(), v.data(), 0, 0);
    if (st != RCHOL_OK) return st;
    ctx->batch_off = off;
    if (offsets)
        for (int s = 0; s <= nsys; ++s) offsets[s] = off[(size_t)s];
    return RCHOL_OK;
}

extern "C" rchol_status rchol_batch_solve(rchol_ctx* ctx, const rchol_factor_t* f, int k, const double* B, double* X,
                                          int ldb, int on_device, rchol_solve_info* per_system,
                                          rchol_solve_info* total) {
    if (!ctx || !f || !B || !X) return fail(ctx, RCHOL_ERR_INVALID, "null argument");
    if (ctx->batch_off.empty()) return fail(ctx, RCHOL_ERR_NO_MATRIX, "no batch loaded (rchol_batch_set)");
    if (!valid_k(k)) return fail(ctx, RCHOL_ERR_INVALID, "k must be 1, 2, 4, 8, 16 or 32");
    if (f->F.n != ctx->At.n || ldb < ctx->At.n) return fail(ctx, RCHOL_ERR_INVALID, "factor/ldb mismatch");
    cudaSetDevice(ctx->device);
    const rchol_opts& o = ctx->o;
    const int nsys = (int)ctx->batch_off.size() - 1;
    if (k > 1) {
        const rchol_status ls = ensure_layouts(ctx, f);
        if (ls != RCHOL_OK) return ls;
    }
    if (!(ctx->bsolver && ctx->bsolver_f == f && ctx->bsolver_k == k)) {
        drop_solver(ctx);
        rchol::SolveConfig cfg;
        cfg.k = k;
        cfg.fp32_factor = o.precision == RCHOL_PREC_FP32_FACTOR;
        cfg.tol = o.tol;
        cfg.max_iter = o.max_iter;
        cfg.stop_rule = o.stop_rule;
        cfg.unroll = o.unroll;
        cfg.use_graph = o.use_graph != 0;
        cfg.timeout_s = o.timeout_s;
        cfg.poll_ns = o.poll_ns;
        if (cfg.fp32_factor && !f->F.lr_val32) return fail(ctx, RCHOL_ERR_INVALID, "factor has no FP32 copy");
        cudaError_t e = cudaSuccess;
        ctx->bsolver = rchol::batch_create(ctx->At, f->F, cfg, ctx->device, ctx->stream, ctx->batch_off.data(), nsys, &e);
        if (!ctx->bsolver) return cuda_fail(ctx, e, "create batch solver");
        ctx->bsolver_f = f;
        ctx->bsolver_k = k;
    }
    rchol_status s = ensure_stage(ctx, (size_t)ctx->At.n * (size_t)k);
    if (s != RCHOL_OK) return s;
    s = stage_in(ctx, B, ldb, k, on_device, ctx->dB);
    if (s != RCHOL_OK) return s;
    rchol::BatchResult r;
    cudaError_t e = rchol::batch_solve(ctx->bsolver, ctx->dB, ctx->dX, &r);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "batch pcg");
    s = stage_out(ctx, ctx->dX, X, ldb, k, on_device);
    if (s != RCHOL_OK) return s;
    CK(cudaStreamSynchronize(ctx->stream), "sync");
    int maxit = 0;
    double maxrel = 0.0;
    for (int q = 0; q < nsys; ++q) {
        maxit = std::max(maxit, r.iterations[(size_t)q]);
        maxrel = std::max(maxrel, r.relres[(size_t)q]);
        if (per_system) {
            std::memset(&per_system[q], 0, sizeof(rchol_solve_info));
            per_system[q].iterations = r.iterations[(size_t)q];
            per_system[q].relres_true = r.relres[(size_t)q];
            per_system[q].converged = o.stop_rule != RCHOL_STOP_RELRES || r.relres[(size_t)q] <= o.tol;
            per_system[q].device_status = r.status;
        }
    }
    if (total) {
        std::memset(total, 0, sizeof(*total));
        total->iterations = maxit;
        total->relres_true = maxrel;
        total->converged = r.converged;
        total->device_status = r.status;
        total->ms_total = r.ms_total;
        total->ms_iterations = r.ms_iterations;
        total->kernel_launches = r.kernel_launches;
        total->graph_launches = r.graph_launches;
    }
    if (r.status == rchol::kDevTimeout) return fail(ctx, RCHOL_ERR_TIMEOUT, "batch pcg: a device wait timed out");
    if (!r.converged) return fail(ctx, RCHOL_ERR_NOT_CONVERGED, "batch pcg did not reach the tolerance");
    return RCHOL_OK;
}

extern "C" rchol_status rchol_factorization_driver(const char* path, int num_blocks, int check_solve, double tol,
                                                   int physics) {
    rchol_opts o;
    rchol_opts_default(&o);
    o.num_blocks = num_blocks;
    o.tol = tol;
    o.stop_rule = RCHOL_STOP_PRECOND;
    o.max_iter = 300;
    o.verbose = 1;
    rchol_ctx* ctx = nullptr;
    rchol_status s = rchol_create(&ctx, &o);
    if (s != RCHOL_OK) {
        std::fprintf(stderr, "rchol: %s\n", rchol_status_string(s));
        return s;
    }
    std::printf("problem: %s\n", path);
    auto t0 = std::chrono::high_resolution_clock::now();
    s = rchol_load_mtx(ctx, path, physics);
    if (s != RCHOL_OK) {
        std::fprintf(stderr, "rchol: %s: %s\n", rchol_status_string(s), rchol_last_error(ctx));
        rchol_destroy(ctx);
        return s;
    }
    auto t1 = std::chrono::high_resolution_clock::now();
    std::printf("number of nodes: %d\nnumber of nonzeros: %lld\n", ctx->A.n, (long long)ctx->A.nnz);
    std::printf("initial preprocessing time (read, sort, upload; not part of the algorithm): %lld milliseconds\n",
                (long long)std::chrono::duration_cast<std::chrono::milliseconds>(t1 - t0).count());
    rchol_factor_t* f = nullptr;
    s = rchol_factor(ctx, &f);
    if (s != RCHOL_OK) {
        std::fprintf(stderr, "rchol: %s: %s\n", rchol_status_string(s), rchol_last_error(ctx));
        rchol_destroy(ctx);
        return s;
    }
    std::printf("Kernel execution time: %f ms\n", f->info.ms_factor);
    std::printf("total conversion time: %f milliseconds\n", f->info.ms_assemble + f->info.ms_setup);
    std::printf("nnz ratio: %f, factor nnz: %lld, original lower triangular nnz (exclude diagonal): %lld\n",
                (double)(f->info.nnz_strict + f->info.n) / (double)std::max<long long>(1, f->info.nnz_lower_a),
                f->info.nnz_strict + f->info.n, f->info.nnz_lower_a);
    if (check_solve) {
        const int32_t n = ctx->At.n;
        std::vector<double> b, x((size_t)n, 0.0);
        zero_sum_rhs(b, (size_t)n, 0);
        rchol_solve_info si;
        s = rchol_pcg_solve(ctx, f, 1, b.data(), x.data(), n, 0, &si);
        std::printf("final iteration: %d, residual: %e\n", si.iterations, si.precond_ratio);
        std::printf("pcg time: %f ms\n", si.ms_total);
        std::printf("normalized diff norm: %.16f\n", si.relres_true);
        if (s == RCHOL_ERR_NOT_CONVERGED) s = RCHOL_OK;  // the reference reports and exits normally
    }
    rchol_factor_free(f);
    rchol_destroy(ctx);
    return s;
}

extern "C" rchol_status rchol_prepare_and_solve(int lap_n, long long lap_nnz, const int* lap_rowptr,
                                                const int* lap_colind, const double* lap_val, const int* csr_rowptr,
                                                const double* csr_val, const int* csr_colind, const double* diag,
                                                double tol, int physics, long long factor_nnz, int removal, double* X,
                                                rchol_solve_info* info) {
    (void)factor_nnz;
    (void)removal;  // unused by the reference as well (solver.hpp:236-593)
    if (lap_n <= 0 || !lap_rowptr || !lap_colind || !lap_val || !csr_rowptr || !csr_val || !csr_colind || !diag)
        return RCHOL_ERR_INVALID;
    int dev = 0;
    cudaGetDevice(&dev);
    rchol_opts o;
    rchol_opts_default(&o);
    o.device = dev;
    o.tol = tol;
    o.stop_rule = RCHOL_STOP_PRECOND;
    o.max_iter = 300;
    rchol_ctx* ctx = nullptr;
    rchol_status s = rchol_create(&ctx, &o);
    if (s != RCHOL_OK) return s;
    (void)lap_nnz;
    s = rchol_set_csc(ctx, lap_n, lap_rowptr, lap_colind, lap_val, 1, 0);
    rchol_factor_t* f = nullptr;
    if (s == RCHOL_OK) s = rchol_factor_from_csr_upper(ctx, lap_n, csr_rowptr, csr_colind, csr_val, diag, 1, &f);
    std::vector<double> b;
    if (s == RCHOL_OK) {
        if (physics) {
            zero_sum_rhs(b, (size_t)lap_n, 0);
        } else {
            std::vector<double> v;
            random_vec(v, (size_t)lap_n, 0);
            b.resize((size_t)lap_n);
            s = rchol_spmv(ctx, 1, v.data(), b.data(), lap_n, 0);
        }
    }
    if (s == RCHOL_OK) {
        std::vector<double> x((size_t)lap_n, 0.0);
        rchol_solve_info si;
        s = rchol_pcg_solve(ctx, f, 1, b.data(), x.data(), lap_n, 0, &si);
        if (info) *info = si;
        if (X) cudaMemcpy(X, x.data(), sizeof(double) * (size_t)lap_n, cudaMemcpyHostToDevice);
        if (s == RCHOL_ERR_NOT_CONVERGED) s = RCHOL_OK;
    }
    if (f) rchol_factor_free(f);
    rchol_destroy(ctx);
    return s;
}

// ===========================================================================
// synthetic inputs
// ===========================================================================

extern "C" rchol_status rchol_generate(const char* kind, const long long* dims, int ndims, double wlo, double whi,
                                       int log_weights, double aniso_z, double excess_frac, double excess_lo,
                                       double excess_hi, int ordering, unsigned long long seed, int* n_out,
                                       long long* nnz_out, int** rows, int** cols, double** vals, int* has_ground) {
    if (!kind || !dims || ndims <= 0 || !n_out || !nnz_out || !rows || !cols || !vals) return RCHOL_ERR_INVALID;
    rchol::GenSpec sp;
    sp.kind = kind;
    sp.dims.assign(dims, dims + ndims);
    sp.wlo = wlo;
    sp.whi = whi;
    sp.log_weights = log_weights != 0;
    sp.aniso_z = aniso_z;
    sp.excess_frac = excess_frac;
    sp.excess_lo = excess_lo;
    sp.excess_hi = excess_hi;
    sp.ordering = ordering;
    sp.seed = seed;
    rchol::Triplets t;
    bool g = false;
    std::string err;
    if (!rchol::generate(sp, t, g, err)) {
        std::fprintf(stderr, "rchol_generate: %s\n", err.c_str());
        return RCHOL_ERR_INVALID;
    }
    const size_t nz = t.rows.size();
    *rows = (int*)std::malloc(sizeof(int) * std::max<size_t>(nz, 1));
    *cols = (int*)std::malloc(sizeof(int) * std::max<size_t>(nz, 1));
    *vals = (double*)std::malloc(sizeof(double) * std::max<size_t>(nz, 1));
    if (!*rows || !*cols || !*vals) return RCHOL_ERR_INVALID;
    std::memcpy(*rows, t.rows.data(), sizeof(int) * nz);
    std::memcpy(*cols, t.cols.data(), sizeof(int) * nz);
    std::memcpy(*vals, t.vals.data(), sizeof(double) * nz);
    *n_out = t.n;
    *nnz_out = (long long)nz;
    if (has_ground) *has_ground = g ? 1 : 0;
    return RCHOL_OK;
}

extern "C" void rchol_free_host(void* p) { std::free(p); }

extern "C" rchol_status rchol_csc_from_triplets(int n, long long nnz, const int* rows, const int* cols,
                                                const double* vals, int* colptr, int* rowind, double* val,
                                                long long* nnz_out) {
    if (n <= 0 || nnz < 0 || (nnz > 0 && (!rows || !cols || !vals)) || !nnz_out) return RCHOL_ERR_INVALID;
    rchol::Triplets t;
    t.n = n;
    t.rows.assign(rows, rows + nnz);
    t.cols.assign(cols, cols + nnz);
    t.vals.assign(vals, vals + nnz);
    rchol::HostCsc h;
    std::string err;
    if (!rchol::triplets_to_csc(t, h, err)) return err.find("finite") != std::string::npos ? RCHOL_ERR_NUMERIC
                                                                                          : RCHOL_ERR_INVALID;
    *nnz_out = (long long)h.rowind.size();
    if (colptr) {
        if (!rowind || !val) return RCHOL_ERR_INVALID;
        std::memcpy(colptr, h.colptr.data(), sizeof(int) * h.colptr.size());
        std::memcpy(rowind, h.rowind.data(), sizeof(int) * h.rowind.size());
        std::memcpy(val, h.val.data(), sizeof(double) * h.val.size());
    }
    return RCHOL_OK;
}

extern "C" rchol_status rchol_zero_sum_vector(int n, unsigned int seed, double* out) {
    if (n < 0 || (n > 0 && !out)) return RCHOL_ERR_INVALID;
    std::vector<double> b;
    zero_sum_rhs(b, (size_t)n, (unsigned long)seed);
    if (n > 0) std::memcpy(out, b.data(), sizeof(double) * (size_t)n);
    return RCHOL_OK;
}

extern "C" rchol_status rchol_read_mtx(const char* path, int* n, long long* nnz, int** rows, int** cols,
                                       double** vals) {
    if (!path || !n || !nnz || !rows || !cols || !vals) return RCHOL_ERR_INVALID;
    rchol::Triplets t;
    std::string err;
    if (!rchol::read_mtx(path, t, err)) return RCHOL_ERR_IO;
    const size_t nz = t.rows.size();
    *rows = (int*)std::malloc(sizeof(int) * std::max<size_t>(nz, 1));
    *cols = (int*)std::malloc(sizeof(int) * std::max<size_t>(nz, 1));
    *vals = (double*)std::malloc(sizeof(double) * std::max<size_t>(nz, 1));
    if (!*rows || !*cols || !*vals) return RCHOL_ERR_INVALID;
    std::memcpy(*rows, t.rows.data(), sizeof(int) * nz);
    std::memcpy(*cols, t.cols.data(), sizeof(int) * nz);
    std::memcpy(*vals, t.vals.data(), sizeof(double) * nz);
    *n = t.n;
    *nnz = (long long)nz;
    return RCHOL_OK;
}

extern "C" rchol_status rchol_write_mtx(const char* path, int n, long long nnz, const int* rows, const int* cols,
                                        const double* vals) {
    if (!path || n <= 0 || nnz < 0) return RCHOL_ERR_INVALID;
    std::string err;
    if (!rchol::write_mtx(path, n, nnz, rows, cols, vals, err)) return RCHOL_ERR_IO;
    return RCHOL_OK;
}
