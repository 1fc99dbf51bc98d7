// Command-line drivers with the reference's argv forms.
//
//   driver          <matrix.mtx> <num_blocks> <solve 0|1> <tolerance> [--key=value ...]
//   driver_physics  <matrix.mtx> <num_blocks> <solve 0|1> <tolerance> [--key=value ...]
//       gpu_implementation/driver.cu:2148-2160 and driver_physics.cu:2120-2129
//       (driver_physics trims the appended ground vertex).
//   driver_local    <matrix.mtx> <num_blocks> <out_prefix> [1] [--key=value ...]
//       experiment/driver_local.cpp:1274-1296: writes <prefix>l_sol.mtx and
//       <prefix>sol_diag.txt when the prefix is non-empty, a trailing "1"
//       trims the ground vertex, then solves as example_pcg_solver does
//       (custom_cg.hpp:65-265: zero-sum right-hand side, ||r||^2 <= 2e-7,
//       at most 400 iterations).  The factor runs on the GPU; the second
//       argument sizes its launch as <num_blocks> does for the GPU drivers.
//
// Extras: --precision=fp64|fp32  --seed=N  --k=N (right-hand sides)
//         --stop=relres|precond|abs  --max_iter=N  --bucket=N  --slab=N
//         --warps=N  --unroll=N  --timeout=S
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/rchol.h"

#ifndef RCHOL_DRIVER_MODE
#define RCHOL_DRIVER_MODE 0  // 0 driver, 1 driver_physics, 2 driver_local
#endif

namespace {

bool parse_extra(const char* a, rchol_opts& o, int& k) {
    std::string s(a);
    if (s.rfind("--", 0) != 0) return false;
    size_t eq = s.find('=');
    if (eq == std::string::npos) return false;
    std::string key = s.substr(2, eq - 2), v = s.substr(eq + 1);
    if (key == "precision") o.precision = (v == "fp32") ? RCHOL_PREC_FP32_FACTOR : RCHOL_PREC_FP64;
    else if (key == "seed") o.seed = std::strtoull(v.c_str(), nullptr, 10);
    else if (key == "k") k = std::atoi(v.c_str());
    else if (key == "stop") o.stop_rule = v == "precond" ? RCHOL_STOP_PRECOND : (v == "abs" ? RCHOL_STOP_ABS_R2 : RCHOL_STOP_RELRES);
    else if (key == "max_iter") o.max_iter = std::atoi(v.c_str());
    else if (key == "bucket") o.bucket_cap = std::atoi(v.c_str());
    else if (key == "slab") o.slab_entries = std::atoi(v.c_str());
    else if (key == "warps") o.warps_per_block = std::atoi(v.c_str());
    else if (key == "unroll") o.unroll = std::atoi(v.c_str());
    else if (key == "timeout") o.timeout_s = std::atof(v.c_str());
    else if (key == "sddm" || key == "order_seed") return true;  // read by main
    else return false;
    return true;
}

int die(rchol_ctx* ctx, rchol_status s, const char* what) {
    std::fprintf(stderr, "%s: %s%s%s\n", what, rchol_status_string(s), ctx ? ": " : "",
                 ctx ? rchol_last_error(ctx) : "");
    if (ctx) rchol_destroy(ctx);
    return 1;
}

}  // namespace

int main(int argc, char** argv) {
    const int mode = RCHOL_DRIVER_MODE;
    int npos = 0;
    for (int i = 1; i < argc; ++i)
        if (std::strncmp(argv[i], "--", 2) != 0) ++npos;
    if ((mode < 2 && npos != 4) || (mode == 2 && npos != 3 && npos != 4)) {
        std::printf("argument count not correct\n");
        if (mode < 2) std::printf("usage: %s <matrix.mtx> <num_blocks> <solve 0|1> <tolerance> [--key=value]\n", argv[0]);
        else std::printf("usage: %s <matrix.mtx> <num_blocks> <out_prefix> [1] [--key=value]\n", argv[0]);
        return 1;
    }
    std::vector<const char*> pos;
    rchol_opts o;
    rchol_opts_default(&o);
    int k = 1;
    for (int i = 1; i < argc; ++i) {
        if (std::strncmp(argv[i], "--", 2) == 0) {
            if (!parse_extra(argv[i], o, k)) {
                std::fprintf(stderr, "unknown option %s\n", argv[i]);
                return 1;
            }
        } else {
            pos.push_back(argv[i]);
        }
    }
    const char* path = pos[0];
    o.num_blocks = std::atoi(pos[1]);
    if (mode < 2) {
        // reference GPU stop rule unless overridden: sqrt(r.z/r0.z0) <= tol, 300 iterations
        bool stop_given = false, iter_given = false;
        for (int i = 1; i < argc; ++i) {
            stop_given |= std::strncmp(argv[i], "--stop=", 7) == 0;
            iter_given |= std::strncmp(argv[i], "--max_iter=", 11) == 0;
        }
        if (!stop_given) o.stop_rule = RCHOL_STOP_PRECOND;
        if (!iter_given) o.max_iter = 300;
        o.tol = std::atof(pos[3]);
    } else {
        o.stop_rule = RCHOL_STOP_ABS_R2;
        o.tol = 2e-7;
        o.max_iter = 400;
        for (int i = 1; i < argc; ++i) {
            if (std::strncmp(argv[i], "--stop=", 7) == 0) parse_extra(argv[i], o, k);
        }
    }
    const int solve = mode < 2 ? std::atoi(pos[2]) : 1;
    const int trim = mode == 1 ? 1 : (mode == 2 ? (pos.size() > 3) : 0);
    // --sddm=nnz|random|given: the input is an SDDM (or Laplacian) in its own
    // order, converted and ordered on the device as write_graph.jl does
    // offline; a .rchb input is the binary matrix cache
    int sddm = -1;
    unsigned long long order_seed = 0;
    for (int i = 1; i < argc; ++i) {
        if (std::strncmp(argv[i], "--sddm=", 7) == 0) {
            const std::string m = argv[i] + 7;
            sddm = m == "random" ? RCHOL_ORDER_RANDOM : (m == "given" ? RCHOL_ORDER_GIVEN : RCHOL_ORDER_NNZ_SORT);
        } else if (std::strncmp(argv[i], "--order_seed=", 13) == 0) {
            order_seed = std::strtoull(argv[i] + 13, nullptr, 10);
        }
    }
    rchol_ctx* ctx = nullptr;
    rchol_status s = rchol_create(&ctx, &o);
    if (s != RCHOL_OK) return die(nullptr, s, "create");
    std::printf("problem: %s\n", path);
    const size_t plen = std::strlen(path);
    if (plen > 5 && std::strcmp(path + plen - 5, ".rchb") == 0) {
        s = rchol_load_bin(ctx, path);
    } else if (sddm >= 0) {
        int n0 = 0, has_ground = 0;
        long long nz0 = 0;
        int *rr = nullptr, *cc = nullptr;
        double* vv = nullptr;
        s = rchol_read_mtx(path, &n0, &nz0, &rr, &cc, &vv);
        if (s == RCHOL_OK) s = rchol_set_sddm(ctx, n0, nz0, rr, cc, vv, 0, sddm, order_seed, nullptr, &has_ground);
        rchol_free_host(rr);
        rchol_free_host(cc);
        rchol_free_host(vv);
        if (s == RCHOL_OK) std::printf("converted on the device: %s ground vertex\n", has_ground ? "with" : "no");
    } else {
        s = rchol_load_mtx(ctx, path, trim);
    }
    if (s != RCHOL_OK) return die(ctx, s, "load");
    int n = 0;
    long long nnz = 0;
    rchol_matrix_info(ctx, &n, &nnz);
    std::printf("number of nodes: %d\nnumber of nonzeros: %lld\n", n, nnz);
    rchol_factor_t* f = nullptr;
    s = rchol_factor(ctx, &f);
    if (s != RCHOL_OK) return die(ctx, s, "factor");
    rchol_factor_info fi;
    rchol_factor_get_info(f, &fi);
    std::printf("Kernel execution time: %f ms\n", fi.ms_factor);
    std::printf("Factorization execution time: %f seconds\n", fi.ms_factor / 1000.0);
    std::printf("total conversion time: %f milliseconds\n", fi.ms_setup + fi.ms_assemble);
    std::printf("nnz ratio: %f, factor nnz: %lld, original lower triangular nnz (exclude diagonal): %lld\n",
                (double)(fi.nnz_strict + fi.n) / (double)(fi.nnz_lower_a > 0 ? fi.nnz_lower_a : 1),
                fi.nnz_strict + fi.n, fi.nnz_lower_a);
    if (mode == 2 && std::strlen(pos[2]) > 0) {
        s = rchol_factor_write(f, pos[2]);
        if (s != RCHOL_OK) return die(ctx, s, "write factor");
    }
    int rc = 0;
    if (solve) {
        const int ns = fi.n;
        if (k < 1) k = 1;
        std::vector<double> b((size_t)ns * k), x((size_t)ns * k, 0.0);
        // column c: the reference right-hand side generate_zero_sum_vector(seed c)
        for (int c = 0; c < k; ++c) rchol_zero_sum_vector(ns, (unsigned)c, b.data() + (size_t)c * ns);
        rchol_solve_info si;
        s = rchol_pcg_solve(ctx, f, k, b.data(), x.data(), ns, 0, &si);
        if (s != RCHOL_OK && s != RCHOL_ERR_NOT_CONVERGED) return die(ctx, s, "solve");
        std::printf("final iteration: %d, residual: %e\n", si.iterations, si.precond_ratio);
        std::printf("pcg time: %f ms\n", si.ms_total);
        std::printf("Solve time taken: %.0f milliseconds\n", si.ms_total);
        std::printf("normalized diff norm: %.16f\n", si.relres_true);
        std::printf("relative residual: %.12f\n", si.relres_true);
        if (!si.converged) std::printf("warning: PCG stopped at the iteration cap\n");
    }
    rchol_factor_free(f);
    rchol_destroy(ctx);
    return rc;
}
