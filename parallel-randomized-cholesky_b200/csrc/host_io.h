// Host-side input handling: MatrixMarket IO, preprocessing into CSC, the
// factor file format, and the synthetic benchmark generators.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace rchol {

struct Triplets {
    int32_t n = 0;
    std::vector<int32_t> rows, cols;
    std::vector<double> vals;
};

struct HostCsc {
    int32_t n = 0;
    std::vector<int32_t> colptr;  // [n+1]
    std::vector<int32_t> rowind;
    std::vector<double> val;
};

// MatrixMarket coordinate reader (real/integer/pattern; symmetric,
// skew-symmetric and hermitian files generalised).  Returns false with a
// message in `err` on failure.
bool read_mtx(const std::string& path, Triplets& t, std::string& err);
bool write_mtx(const std::string& path, int32_t n, int64_t nnz, const int32_t* rows, const int32_t* cols,
               const double* vals, std::string& err);

// Binary matrix cache (a preprocessed CSC, read with one fread per array):
// magic "RCHOLCSC", uint32 version 1, int32 trim flag, int64 n, int64 nnz,
// then colptr (int32, n+1), rowind (int32, nnz), val (float64, nnz), in the
// host's byte order (little-endian on the supported hosts).
bool write_csc_bin(const std::string& path, int32_t n, const int32_t* colptr, const int32_t* rowind,
                   const double* val, int trim, std::string& err);
bool read_csc_bin(const std::string& path, HostCsc& out, int& trim, std::string& err);

// Host orderings of a symmetric pattern (0-based triplets, diagonal ignored):
// order[k] = vertex placed at position k (host_order.cpp).
constexpr int kHostOrderRcm = 3;  // reverse Cuthill-McKee
constexpr int kHostOrderNd = 4;   // nested dissection by level-structure bisection
bool host_ordering(int kind, int32_t n, int64_t nnz, const int32_t* rows, const int32_t* cols,
                   std::vector<int32_t>& order, std::string& err);

// sparse_matrix_processor preprocessing (pre_process.hpp:189-306, 338-356):
// off-diagonals -> -|v|, diagonal -> |v|, diagonal appended as the column
// sum of |off-diagonals| when the input has none, CSC sorted by (col,row),
// duplicates kept.  Validates finiteness and squareness.
bool triplets_to_csc(const Triplets& t, HostCsc& out, std::string& err);

// Factor files: <prefix>l_sol.mtx holds the CSC of L with its unit diagonal
// (1-based "row col value", column-major, 16 significant digits) and
// <prefix>sol_diag.txt one D value per line (experiment/driver_local.cpp:958-988;
// D is written with 17 significant digits, a superset of the reference's 6).
bool write_factor_files(const std::string& prefix, int32_t n, const std::vector<int64_t>& colptr,
                        const std::vector<int32_t>& rowind, const std::vector<double>& val,
                        const std::vector<double>& diag, std::string& err);
// Reads them back as a strict CSC (unit diagonal dropped) plus D.
bool read_factor_files(const std::string& prefix, int32_t& n, std::vector<int64_t>& colptr,
                       std::vector<int32_t>& rowind, std::vector<double>& val, std::vector<double>& diag,
                       std::string& err);

struct GenSpec {
    std::string kind;                 // grid2d, grid3d, grid3d27, chunglu
    std::vector<long long> dims;
    double wlo = 1.0, whi = 1.0;
    bool log_weights = false;
    double aniso_z = 1.0;
    double excess_frac = 0.0, excess_lo = 0.0, excess_hi = 0.0;
    int ordering = 0;                 // 0 ascending nnz, 1 random, 2 natural
    uint64_t seed = 0;
};

// Builds the (reordered) Laplacian triplets, appending a ground vertex when
// the operator is an SDDM (write_graph.jl:98-183).
bool generate(const GenSpec& spec, Triplets& out, bool& has_ground, std::string& err);

}  // namespace rchol
