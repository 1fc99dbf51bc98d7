// Minimal MatrixMarket reader/writer exposing the names that the reference
// CPU factor (cpu_implementation/pre_process.hpp:346 and
// cpu_implementation/driver_local.cpp:972-983) calls from the third-party
// header-only library fast_matrix_market (github.com/alugowski/fast_matrix_market,
// un-vendored, unpinned: the reference README clones its HEAD).
//
// Own-written test infrastructure: it exists only so that the reference's own
// CPU factor can be compiled from its sources as the oracle and the timed CPU
// baseline.  Semantics follow fast_matrix_market's documented defaults:
//   * coordinate format, field real / integer / pattern (pattern -> 1.0);
//   * symmetric / skew-symmetric / hermitian files are generalized (the
//     mirrored off-diagonal entry is appended after all file entries), which is
//     the library's `generalize_symmetry = true` default;
//   * indices are converted from 1-based to 0-based;
//   * write_matrix_market_csc writes a coordinate/real/general file, column by
//     column, 1-based "row col value" lines, values with `precision`
//     significant digits (shortest round-trip form when precision < 0).
#pragma once

#include <algorithm>
#include <cctype>
#include <chrono>
#include <climits>
#include <cmath>
#include <iostream>
#include <numeric>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <istream>
#include <iterator>
#include <ostream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace fast_matrix_market {

enum object_type { matrix, vector };
enum format_type { array, coordinate };
enum field_type { real, double_, complex, integer, pattern, unsigned_integer };
enum symmetry_type { general, symmetric, skew_symmetric, hermitian };

struct matrix_market_header {
    object_type object = matrix;
    format_type format = coordinate;
    field_type field = real;
    symmetry_type symmetry = general;
    int64_t nrows = 0, ncols = 0, vector_length = 0, nnz = 0;
    std::string comment;
    matrix_market_header() = default;
    matrix_market_header(int64_t r, int64_t c) : nrows(r), ncols(c) {}
};

struct read_options {
    bool generalize_symmetry = true;
};

struct write_options {
    int precision = -1;
};

namespace detail {

inline std::string lower(std::string s) {
    for (auto& ch : s) ch = (char)std::tolower((unsigned char)ch);
    return s;
}

inline void format_value(char* buf, size_t len, double v, int precision) {
    if (precision < 0) {
        // shortest representation that round-trips
        for (int p = 1; p <= 17; ++p) {
            std::snprintf(buf, len, "%.*g", p, v);
            if (std::strtod(buf, nullptr) == v) return;
        }
        std::snprintf(buf, len, "%.17g", v);
    } else {
        std::snprintf(buf, len, "%.*g", precision == 0 ? 1 : precision, v);
    }
}

}  // namespace detail

template <typename IT, typename VT>
void read_matrix_market_triplet(std::istream& in, IT& nrows, IT& ncols,
                                std::vector<IT>& rows, std::vector<IT>& cols,
                                std::vector<VT>& vals,
                                const read_options& opts = {}) {
    // whole file in one read when the stream is seekable
    std::string text;
    in.seekg(0, std::ios::end);
    const std::streamoff fsize = in.good() ? (std::streamoff)in.tellg() : (std::streamoff)-1;
    if (fsize > 0) {
        text.resize((size_t)fsize);
        in.seekg(0, std::ios::beg);
        in.read(&text[0], fsize);
        text.resize((size_t)in.gcount());
    } else {
        in.clear();
        in.seekg(0, std::ios::beg);
        text.assign((std::istreambuf_iterator<char>(in)), std::istreambuf_iterator<char>());
    }
    const char* p = text.c_str();
    const char* end = p + text.size();
    // banner
    const char* eol = (const char*)std::memchr(p, '\n', (size_t)(end - p));
    if (!eol) eol = end;
    std::string banner = detail::lower(std::string(p, eol));
    if (banner.rfind("%%matrixmarket", 0) != 0)
        throw std::runtime_error("not a MatrixMarket file");
    if (banner.find("coordinate") == std::string::npos)
        throw std::runtime_error("only coordinate MatrixMarket files are supported");
    bool is_pattern = banner.find("pattern") != std::string::npos;
    bool is_complex = banner.find("complex") != std::string::npos;
    if (is_complex) throw std::runtime_error("complex MatrixMarket files are not supported");
    symmetry_type sym = general;
    if (banner.find("skew-symmetric") != std::string::npos) sym = skew_symmetric;
    else if (banner.find("symmetric") != std::string::npos) sym = symmetric;
    else if (banner.find("hermitian") != std::string::npos) sym = hermitian;
    p = eol < end ? eol + 1 : end;
    // comments
    while (p < end && (*p == '%' || *p == '\n' || *p == '\r')) {
        const char* e = (const char*)std::memchr(p, '\n', (size_t)(end - p));
        p = e ? e + 1 : end;
    }
    char* q = nullptr;
    long long r0 = std::strtoll(p, &q, 10); p = q;
    long long c0 = std::strtoll(p, &q, 10); p = q;
    long long nz = std::strtoll(p, &q, 10); p = q;
    nrows = (IT)r0;
    ncols = (IT)c0;
    rows.clear(); cols.clear(); vals.clear();
    rows.reserve((size_t)nz * (sym == general ? 1 : 2));
    cols.reserve(rows.capacity());
    vals.reserve(rows.capacity());
    rows.resize((size_t)nz);
    cols.resize((size_t)nz);
    vals.resize((size_t)nz);
    // The body is split into line-aligned chunks parsed in parallel (the
    // library parses in parallel too); each chunk first counts its entry
    // lines, so entries keep their file order.
    while (p < end && *p != '\n') ++p;  // rest of the size line
    const char* body = p;
    int nchunks = 1;
#ifdef _OPENMP
    nchunks = std::max(1, omp_get_max_threads());
#endif
    std::vector<const char*> cut((size_t)nchunks + 1, end);
    cut[0] = body;
    for (int t = 1; t < nchunks; ++t) {
        const char* s = body + (end - body) * t / nchunks;
        if (s < cut[(size_t)t - 1]) s = cut[(size_t)t - 1];
        while (s < end && *s != '\n') ++s;
        cut[(size_t)t] = s;
    }
    auto is_entry_line = [](const char* s, const char* e) {
        while (s < e && (*s == ' ' || *s == '\t' || *s == '\r')) ++s;
        return s < e && *s != '\n' && *s != '%';
    };
    std::vector<long long> count((size_t)nchunks + 1, 0);
#pragma omp parallel for schedule(static, 1)
    for (int t = 0; t < nchunks; ++t) {
        long long c = 0;
        for (const char* s = cut[(size_t)t]; s < cut[(size_t)t + 1];) {
            const char* e = (const char*)std::memchr(s, '\n', (size_t)(cut[(size_t)t + 1] - s));
            if (!e) e = cut[(size_t)t + 1];
            if (is_entry_line(s, e)) ++c;
            s = e + 1;
        }
        count[(size_t)t + 1] = c;
    }
    for (int t = 0; t < nchunks; ++t) count[(size_t)t + 1] += count[(size_t)t];
    if (count[(size_t)nchunks] < nz) throw std::runtime_error("MatrixMarket file has fewer entries than its header");
#pragma omp parallel for schedule(static, 1)
    for (int t = 0; t < nchunks; ++t) {
        long long k = count[(size_t)t];
        char* qq = nullptr;
        for (const char* s = cut[(size_t)t]; s < cut[(size_t)t + 1] && k < nz;) {
            const char* e = (const char*)std::memchr(s, '\n', (size_t)(cut[(size_t)t + 1] - s));
            if (!e) e = cut[(size_t)t + 1];
            if (is_entry_line(s, e)) {
                const char* z = s;
                long long r = std::strtoll(z, &qq, 10); z = qq;
                long long c = std::strtoll(z, &qq, 10); z = qq;
                double v = 1.0;
                if (!is_pattern) v = std::strtod(z, &qq);
                rows[(size_t)k] = (IT)(r - 1);
                cols[(size_t)k] = (IT)(c - 1);
                vals[(size_t)k] = (VT)v;
                ++k;
            }
            s = e + 1;
        }
    }
    if (sym != general && opts.generalize_symmetry) {
        size_t base = rows.size();
        for (size_t k = 0; k < base; ++k) {
            if (rows[k] == cols[k]) continue;
            VT v = vals[k];
            if (sym == skew_symmetric) v = -v;
            rows.push_back(cols[k]);
            cols.push_back(rows[k]);
            vals.push_back(v);
        }
    }
}

template <typename PT, typename IT, typename VT>
void write_matrix_market_csc(std::ostream& out, const matrix_market_header& header,
                             const std::vector<PT>& indptr, const std::vector<IT>& indices,
                             const std::vector<VT>& values, bool is_csr,
                             const write_options& opts = {}) {
    const int64_t nnz = indptr.empty() ? 0 : (int64_t)indptr.back();
    std::string buf;
    buf.reserve(1 << 20);
    buf += "%%MatrixMarket matrix coordinate real general\n";
    buf += std::to_string(header.nrows) + " " + std::to_string(header.ncols) + " " +
           std::to_string(nnz) + "\n";
    char line[128], num[64];
    const size_t outer = indptr.empty() ? 0 : indptr.size() - 1;
    for (size_t j = 0; j < outer; ++j) {
        for (int64_t k = (int64_t)indptr[j]; k < (int64_t)indptr[j + 1]; ++k) {
            long long row = is_csr ? (long long)j : (long long)indices[(size_t)k];
            long long col = is_csr ? (long long)indices[(size_t)k] : (long long)j;
            detail::format_value(num, sizeof(num), (double)values[(size_t)k], opts.precision);
            int n = std::snprintf(line, sizeof(line), "%lld %lld %s\n", row + 1, col + 1, num);
            buf.append(line, (size_t)n);
            if (buf.size() > (1u << 20)) { out << buf; buf.clear(); }
        }
    }
    out << buf;
}

}  // namespace fast_matrix_market
