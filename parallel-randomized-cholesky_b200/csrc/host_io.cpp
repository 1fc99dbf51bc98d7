// Host-side input handling (see host_io.h).
#include "host_io.h"

#include <algorithm>
#include <climits>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <numeric>
#include <sstream>

#include <omp.h>

namespace rchol {

namespace {

std::string lower(std::string s) {
    for (auto& c : s) c = (char)std::tolower((unsigned char)c);
    return s;
}

bool slurp(const std::string& path, std::string& out, std::string& err) {
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) {
        err = "cannot open " + path + ": " + std::strerror(errno);
        return false;
    }
    std::fseek(f, 0, SEEK_END);
    long sz = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    out.resize(sz > 0 ? (size_t)sz : 0);
    size_t got = sz > 0 ? std::fread(&out[0], 1, (size_t)sz, f) : 0;
    std::fclose(f);
    if ((long)got != sz) {
        err = "short read on " + path;
        return false;
    }
    return true;
}

// splitmix64 finaliser: a counter-based stream for the generators
inline uint64_t mix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}
inline uint64_t hash3(uint64_t seed, uint64_t stream, uint64_t i) {
    return mix64(mix64(mix64(seed) ^ (stream * 0xD1B54A32D192ED03ull)) ^ i);
}
inline double unit(uint64_t h) { return (double)(h >> 11) * (1.0 / 9007199254740992.0); }

enum Stream : uint64_t { kWeight = 1, kExcessPick = 2, kExcessVal = 3, kOrder = 4, kDegree = 5, kEdgeU = 6,
                         kEdgeV = 7 };

}  // namespace

bool read_mtx(const std::string& path, Triplets& t, std::string& err) {
    std::string text;
    if (!slurp(path, text, err)) return false;
    const char* p = text.c_str();
    const char* end = p + text.size();
    const char* eol = (const char*)std::memchr(p, '\n', (size_t)(end - p));
    if (!eol) eol = end;
    std::string banner = lower(std::string(p, eol));
    if (banner.rfind("%%matrixmarket", 0) != 0) {
        err = path + ": missing %%MatrixMarket banner";
        return false;
    }
    if (banner.find("coordinate") == std::string::npos) {
        err = path + ": only coordinate MatrixMarket files are supported";
        return false;
    }
    if (banner.find("complex") != std::string::npos) {
        err = path + ": complex matrices are not supported";
        return false;
    }
    const bool pattern = banner.find("pattern") != std::string::npos;
    int sym = 0;  // 0 general, 1 symmetric, 2 skew, 3 hermitian
    if (banner.find("skew-symmetric") != std::string::npos) sym = 2;
    else if (banner.find("symmetric") != std::string::npos) sym = 1;
    else if (banner.find("hermitian") != std::string::npos) sym = 3;
    p = eol < end ? eol + 1 : end;
    while (p < end && (*p == '%' || *p == '\n' || *p == '\r' || *p == ' ' || *p == '\t')) {
        if (*p == '%') {
            const char* e = (const char*)std::memchr(p, '\n', (size_t)(end - p));
            p = e ? e + 1 : end;
        } else {
            ++p;
        }
    }
    char* q = nullptr;
    long long nr = std::strtoll(p, &q, 10);
    p = q;
    long long nc = std::strtoll(p, &q, 10);
    p = q;
    long long nz = std::strtoll(p, &q, 10);
    p = q;
    if (nr <= 0 || nr != nc || nz < 0 || nr > INT32_MAX) {
        err = path + ": matrix must be square with a positive size";
        return false;
    }
    t.n = (int32_t)nr;
    size_t reserve = (size_t)nz * (sym ? 2 : 1);
    t.rows.clear();
    t.cols.clear();
    t.vals.clear();
    t.rows.reserve(reserve);
    t.cols.reserve(reserve);
    t.vals.reserve(reserve);
    t.rows.resize((size_t)nz);
    t.cols.resize((size_t)nz);
    t.vals.resize((size_t)nz);
    // The entry lines are parsed in parallel: the body is cut into
    // line-aligned chunks, each chunk counts its entry lines, and a prefix
    // sum gives every chunk its first entry, so the entries keep file order.
    while (p < end && *p != '\n') ++p;  // rest of the size line
    const char* body = p;
    const int nchunks = std::max(1, std::min(omp_get_max_threads() * 4, (int)((end - body) / 65536) + 1));
    std::vector<const char*> cut((size_t)nchunks + 1, end);
    cut[0] = body;
    for (int c = 1; c < nchunks; ++c) {
        const char* q0 = body + (end - body) * c / nchunks;
        if (q0 < cut[(size_t)c - 1]) q0 = cut[(size_t)c - 1];
        while (q0 < end && *q0 != '\n') ++q0;
        cut[(size_t)c] = q0;
    }
    auto entry_line = [](const char* a, const char* b) {
        while (a < b && (*a == ' ' || *a == '\t' || *a == '\r' || *a == '\n')) ++a;
        return a < b && *a != '%';
    };
    std::vector<long long> first((size_t)nchunks + 1, 0);
#pragma omp parallel for schedule(dynamic, 1)
    for (int c = 0; c < nchunks; ++c) {
        long long cnt = 0;
        for (const char* a = cut[(size_t)c]; a < cut[(size_t)c + 1];) {
            const char* e = (const char*)std::memchr(a, '\n', (size_t)(cut[(size_t)c + 1] - a));
            if (!e) e = cut[(size_t)c + 1];
            if (entry_line(a, e)) ++cnt;
            a = e + 1;
        }
        first[(size_t)c + 1] = cnt;
    }
    for (int c = 0; c < nchunks; ++c) first[(size_t)c + 1] += first[(size_t)c];
    if (first[(size_t)nchunks] < nz) {
        err = path + ": truncated entry list";
        return false;
    }
    int bad = 0;  // 1: malformed entry, 2: index out of range
#pragma omp parallel for schedule(dynamic, 1) reduction(| : bad)
    for (int c = 0; c < nchunks; ++c) {
        long long k = first[(size_t)c];
        char* qq = nullptr;
        for (const char* a = cut[(size_t)c]; a < cut[(size_t)c + 1] && k < nz;) {
            const char* e = (const char*)std::memchr(a, '\n', (size_t)(cut[(size_t)c + 1] - a));
            if (!e) e = cut[(size_t)c + 1];
            if (entry_line(a, e)) {
                const char* z = a;
                long long r = std::strtoll(z, &qq, 10);
                if (qq == z) bad |= 1;
                z = qq;
                long long cc = std::strtoll(z, &qq, 10);
                if (qq == z) bad |= 1;
                z = qq;
                double v = 1.0;
                if (!pattern) {
                    v = std::strtod(z, &qq);
                    if (qq == z) bad |= 1;
                }
                if (r < 1 || r > nr || cc < 1 || cc > nc) bad |= 2;
                t.rows[(size_t)k] = (int32_t)(r - 1);
                t.cols[(size_t)k] = (int32_t)(cc - 1);
                t.vals[(size_t)k] = v;
                ++k;
            }
            a = e + 1;
        }
    }
    if (bad & 1) {
        err = path + ": truncated entry list";
        return false;
    }
    if (bad & 2) {
        err = path + ": index out of range";
        return false;
    }
    if (sym) {
        size_t base = t.rows.size();
        for (size_t k = 0; k < base; ++k) {
            if (t.rows[k] == t.cols[k]) continue;
            t.rows.push_back(t.cols[k]);
            t.cols.push_back(t.rows[k]);
            t.vals.push_back(sym == 2 ? -t.vals[k] : t.vals[k]);
        }
    }
    return true;
}

bool write_mtx(const std::string& path, int32_t n, int64_t nnz, const int32_t* rows, const int32_t* cols,
               const double* vals, std::string& err) {
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) {
        err = "cannot write " + path;
        return false;
    }
    std::fprintf(f, "%%%%MatrixMarket matrix coordinate real general\n%d %d %lld\n", n, n, (long long)nnz);
    std::vector<char> buf;
    buf.reserve(1 << 22);
    char line[96];
    for (int64_t k = 0; k < nnz; ++k) {
        int len = std::snprintf(line, sizeof(line), "%d %d %.17g\n", rows[k] + 1, cols[k] + 1, vals[k]);
        buf.insert(buf.end(), line, line + len);
        if (buf.size() > (1u << 22) - 128) {
            std::fwrite(buf.data(), 1, buf.size(), f);
            buf.clear();
        }
    }
    std::fwrite(buf.data(), 1, buf.size(), f);
    bool ok = std::fclose(f) == 0;
    if (!ok) err = "write failed on " + path;
    return ok;
}

// pre_process.hpp:189-306.  Stable: equal (col,row) keys keep input order.
bool triplets_to_csc(const Triplets& t, HostCsc& out, std::string& err) {
    const int32_t n = t.n;
    const size_t nz = t.rows.size();
    if (t.cols.size() != nz || t.vals.size() != nz) {
        err = "triplet arrays differ in length";
        return false;
    }
    bool has_diag = false;
    for (size_t k = 0; k < nz; ++k) {
        if (t.rows[k] < 0 || t.rows[k] >= n || t.cols[k] < 0 || t.cols[k] >= n) {
            err = "triplet index out of range";
            return false;
        }
        if (!std::isfinite(t.vals[k])) {
            err = "non-finite matrix entry";
            return false;
        }
        if (t.rows[k] == t.cols[k]) has_diag = true;
    }
    const size_t total = nz + (has_diag ? 0 : (size_t)n);
    if (total > (size_t)INT32_MAX) {
        err = "matrix has more than 2^31-1 entries";
        return false;
    }
    out.n = n;
    out.colptr.assign((size_t)n + 1, 0);
    for (size_t k = 0; k < nz; ++k) out.colptr[(size_t)t.cols[k] + 1]++;
    if (!has_diag)
        for (int32_t i = 0; i < n; ++i) out.colptr[(size_t)i + 1]++;
    for (int32_t i = 0; i < n; ++i) out.colptr[(size_t)i + 1] += out.colptr[i];
    // bucket by column keeping input order, diagonal appended last
    std::vector<int32_t> cursor(out.colptr.begin(), out.colptr.end() - 1);
    std::vector<int64_t> src(total);
    for (size_t k = 0; k < nz; ++k) src[(size_t)cursor[t.cols[k]]++] = (int64_t)k;
    if (!has_diag)
        for (int32_t i = 0; i < n; ++i) src[(size_t)cursor[i]++] = -1 - (int64_t)i;
    std::vector<double> dsum;
    if (!has_diag) {
        dsum.assign((size_t)n, 0.0);
        for (size_t k = 0; k < nz; ++k) dsum[(size_t)t.cols[k]] += std::fabs(t.vals[k]);
    }
    out.rowind.resize(total);
    out.val.resize(total);
#pragma omp parallel for schedule(dynamic, 4096)
    for (int32_t c = 0; c < n; ++c) {
        const int32_t b = out.colptr[c], e = out.colptr[(size_t)c + 1];
        auto key = [&](int64_t s) { return s >= 0 ? t.rows[(size_t)s] : (int32_t)(-1 - s); };
        std::stable_sort(src.begin() + b, src.begin() + e,
                         [&](int64_t x, int64_t y) { return key(x) < key(y); });
        for (int32_t p = b; p < e; ++p) {
            int64_t s = src[(size_t)p];
            if (s >= 0) {
                const int32_t r = t.rows[(size_t)s];
                out.rowind[(size_t)p] = r;
                out.val[(size_t)p] = (r != c) ? -std::fabs(t.vals[(size_t)s]) : std::fabs(t.vals[(size_t)s]);
            } else {
                out.rowind[(size_t)p] = c;
                out.val[(size_t)p] = dsum[(size_t)c];
            }
        }
    }
    return true;
}

namespace {
constexpr char kBinMagic[8] = {'R', 'C', 'H', 'O', 'L', 'C', 'S', 'C'};
}

bool write_csc_bin(const std::string& path, int32_t n, const int32_t* colptr, const int32_t* rowind,
                   const double* val, int trim, std::string& err) {
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) {
        err = "cannot write " + path + ": " + std::strerror(errno);
        return false;
    }
    const uint32_t version = 1;
    const int32_t tr = trim ? 1 : 0;
    const int64_t n64 = n, nnz = colptr[n];
    bool ok = std::fwrite(kBinMagic, 1, 8, f) == 8 && std::fwrite(&version, 4, 1, f) == 1 &&
              std::fwrite(&tr, 4, 1, f) == 1 && std::fwrite(&n64, 8, 1, f) == 1 && std::fwrite(&nnz, 8, 1, f) == 1;
    ok = ok && std::fwrite(colptr, 4, (size_t)n + 1, f) == (size_t)n + 1;
    ok = ok && std::fwrite(rowind, 4, (size_t)nnz, f) == (size_t)nnz;
    ok = ok && std::fwrite(val, 8, (size_t)nnz, f) == (size_t)nnz;
    if (std::fclose(f) != 0 || !ok) {
        err = "write failed on " + path;
        return false;
    }
    return true;
}

bool read_csc_bin(const std::string& path, HostCsc& out, int& trim, std::string& err) {
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) {
        err = "cannot open " + path + ": " + std::strerror(errno);
        return false;
    }
    char magic[8];
    uint32_t version = 0;
    int32_t tr = 0;
    int64_t n = 0, nnz = 0;
    bool ok = std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, kBinMagic, 8) == 0 &&
              std::fread(&version, 4, 1, f) == 1 && version == 1 && std::fread(&tr, 4, 1, f) == 1 &&
              std::fread(&n, 8, 1, f) == 1 && std::fread(&nnz, 8, 1, f) == 1 && n > 0 && n <= INT32_MAX &&
              nnz >= 0 && nnz <= INT32_MAX;
    if (!ok) {
        std::fclose(f);
        err = path + ": not a binary matrix file of version 1";
        return false;
    }
    out.n = (int32_t)n;
    out.colptr.resize((size_t)n + 1);
    out.rowind.resize((size_t)nnz);
    out.val.resize((size_t)nnz);
    ok = std::fread(out.colptr.data(), 4, (size_t)n + 1, f) == (size_t)n + 1 &&
         std::fread(out.rowind.data(), 4, (size_t)nnz, f) == (size_t)nnz &&
         std::fread(out.val.data(), 8, (size_t)nnz, f) == (size_t)nnz;
    std::fclose(f);
    if (!ok) {
        err = "short read on " + path;
        return false;
    }
    // structure checks: monotone pointers ending at nnz, indices in range
    if (out.colptr[0] != 0 || out.colptr[(size_t)n] != nnz) ok = false;
    for (int64_t j = 0; j < n && ok; ++j) ok = out.colptr[(size_t)j] <= out.colptr[(size_t)j + 1];
    for (int64_t k = 0; k < nnz && ok; ++k) ok = out.rowind[(size_t)k] >= 0 && out.rowind[(size_t)k] < n;
    if (!ok) {
        err = path + ": corrupt matrix structure";
        return false;
    }
    trim = tr;
    return true;
}

bool write_factor_files(const std::string& prefix, int32_t n, const std::vector<int64_t>& colptr,
                        const std::vector<int32_t>& rowind, const std::vector<double>& val,
                        const std::vector<double>& diag, std::string& err) {
    const std::string lpath = prefix + "l_sol.mtx";
    FILE* f = std::fopen(lpath.c_str(), "wb");
    if (!f) {
        err = "cannot write " + lpath;
        return false;
    }
    const long long nnz = (long long)colptr[(size_t)n] + n;
    std::fprintf(f, "%%%%MatrixMarket matrix coordinate real general\n%d %d %lld\n", n, n, nnz);
    // columns are formatted in parallel, a block of columns per buffer, and
    // the buffers written in column order
    const int32_t block = 16384;
    const int32_t nblocks = (n + block - 1) / block;
    bool ok = true;
    for (int32_t b0 = 0; b0 < nblocks && ok; b0 += 64) {
        const int32_t b1 = std::min(nblocks, b0 + 64);
        std::vector<std::string> out((size_t)(b1 - b0));
#pragma omp parallel for schedule(dynamic, 1)
        for (int32_t b = b0; b < b1; ++b) {
            std::string& o = out[(size_t)(b - b0)];
            char line[96];
            const int32_t j0 = b * block, j1 = std::min(n, j0 + block);
            o.reserve((size_t)(colptr[(size_t)j1] - colptr[(size_t)j0] + (j1 - j0)) * 36);
            for (int32_t j = j0; j < j1; ++j) {
                int len = std::snprintf(line, sizeof(line), "%d %d 1\n", j + 1, j + 1);  // unit diagonal first
                o.append(line, (size_t)len);
                for (int64_t p = colptr[(size_t)j]; p < colptr[(size_t)j + 1]; ++p) {
                    len = std::snprintf(line, sizeof(line), "%d %d %.16g\n", rowind[(size_t)p] + 1, j + 1,
                                        val[(size_t)p]);
                    o.append(line, (size_t)len);
                }
            }
        }
        for (const std::string& o : out)
            if (std::fwrite(o.data(), 1, o.size(), f) != o.size()) ok = false;
    }
    if (std::fclose(f) != 0 || !ok) {
        err = "write failed on " + lpath;
        return false;
    }
    const std::string dpath = prefix + "sol_diag.txt";
    FILE* g = std::fopen(dpath.c_str(), "wb");
    if (!g) {
        err = "cannot write " + dpath;
        return false;
    }
    for (int32_t i = 0; i < n; ++i) std::fprintf(g, "%.17g\n", diag[(size_t)i]);
    if (std::fclose(g) != 0) {
        err = "write failed on " + dpath;
        return false;
    }
    return true;
}

bool read_factor_files(const std::string& prefix, int32_t& n, std::vector<int64_t>& colptr,
                       std::vector<int32_t>& rowind, std::vector<double>& val, std::vector<double>& diag,
                       std::string& err) {
    Triplets t;
    if (!read_mtx(prefix + "l_sol.mtx", t, err)) return false;
    n = t.n;
    // bucket by column, keep strictly-lower entries, sort rows per column
    colptr.assign((size_t)n + 1, 0);
    for (size_t k = 0; k < t.rows.size(); ++k) {
        if (t.rows[k] < t.cols[k]) {
            err = "factor file has an entry above the diagonal";
            return false;
        }
        if (t.rows[k] > t.cols[k]) colptr[(size_t)t.cols[k] + 1]++;
    }
    for (int32_t i = 0; i < n; ++i) colptr[(size_t)i + 1] += colptr[(size_t)i];
    std::vector<int64_t> cur(colptr.begin(), colptr.end() - 1);
    rowind.assign((size_t)colptr[(size_t)n], 0);
    val.assign((size_t)colptr[(size_t)n], 0.0);
    for (size_t k = 0; k < t.rows.size(); ++k) {
        if (t.rows[k] <= t.cols[k]) continue;
        int64_t p = cur[(size_t)t.cols[k]]++;
        rowind[(size_t)p] = t.rows[k];
        val[(size_t)p] = t.vals[k];
    }
    for (int32_t j = 0; j < n; ++j) {
        std::vector<std::pair<int32_t, double>> v;
        for (int64_t p = colptr[(size_t)j]; p < colptr[(size_t)j + 1]; ++p)
            v.emplace_back(rowind[(size_t)p], val[(size_t)p]);
        std::sort(v.begin(), v.end());
        for (size_t q = 0; q < v.size(); ++q) {
            rowind[(size_t)colptr[(size_t)j] + q] = v[q].first;
            val[(size_t)colptr[(size_t)j] + q] = v[q].second;
        }
    }
    std::string text;
    if (!slurp(prefix + "sol_diag.txt", text, err)) return false;
    diag.clear();
    const char* p = text.c_str();
    char* q = nullptr;
    while (true) {
        double d = std::strtod(p, &q);
        if (q == p) break;
        diag.push_back(d);
        p = q;
    }
    if ((int32_t)diag.size() != n) {
        err = "sol_diag.txt length does not match l_sol.mtx";
        return false;
    }
    return true;
}

// ---------------------------------------------------------------------------
// generators
// ---------------------------------------------------------------------------

namespace {

struct EdgeList {
    int64_t n = 0;
    std::vector<int64_t> a, b;
    std::vector<double> w;
};

double draw_weight(const GenSpec& s, uint64_t e) {
    double u = unit(hash3(s.seed, kWeight, e));
    if (s.log_weights) return std::exp(std::log(s.wlo) + u * (std::log(s.whi) - std::log(s.wlo)));
    return s.wlo + u * (s.whi - s.wlo);
}

void grid_edges(const GenSpec& s, EdgeList& E, bool p27) {
    const bool is3 = s.dims.size() >= 3;
    const int64_t nx = s.dims[0], ny = s.dims.size() > 1 ? s.dims[1] : s.dims[0], nz = is3 ? s.dims[2] : 1;
    E.n = nx * ny * nz;
    auto id = [&](int64_t x, int64_t y, int64_t z) { return x + nx * (y + ny * z); };
    std::vector<int> offs;  // dx,dy,dz triples with a positive first nonzero component
    if (p27) {
        for (int dz = -1; dz <= 1; ++dz)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx) {
                    int first = dz != 0 ? dz : (dy != 0 ? dy : dx);
                    if (first > 0) {
                        offs.push_back(dx);
                        offs.push_back(dy);
                        offs.push_back(dz);
                    }
                }
    } else {
        int o[] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
        offs.assign(o, o + (is3 ? 9 : 6));
    }
    const size_t no = offs.size() / 3;
    uint64_t e = 0;
    for (int64_t z = 0; z < nz; ++z)
        for (int64_t y = 0; y < ny; ++y)
            for (int64_t x = 0; x < nx; ++x)
                for (size_t k = 0; k < no; ++k) {
                    int dx = offs[3 * k], dy = offs[3 * k + 1], dz = offs[3 * k + 2];
                    int64_t X = x + dx, Y = y + dy, Z = z + dz;
                    if (X < 0 || X >= nx || Y < 0 || Y >= ny || Z < 0 || Z >= nz) continue;
                    double base = 1.0;
                    if (s.aniso_z != 1.0) {
                        // per-axis conductances (1, 1, aniso_z), weighted by
                        // direction and damped by the squared edge length
                        double d2 = (double)(dx * dx + dy * dy + dz * dz);
                        base = ((double)(dx * dx) + (double)(dy * dy) + s.aniso_z * (double)(dz * dz)) / (d2 * d2);
                    } else if (p27) {
                        double d2 = (double)(dx * dx + dy * dy + dz * dz);
                        base = 1.0 / d2;
                    }
                    E.a.push_back(id(x, y, z));
                    E.b.push_back(id(X, Y, Z));
                    E.w.push_back(base * draw_weight(s, e));
                    ++e;
                }
}

bool chunglu_edges(const GenSpec& s, EdgeList& E, std::string& err) {
    if (s.dims.size() < 4) {
        err = "chunglu needs dims {n, m, dmin, dmax}";
        return false;
    }
    const int64_t n = s.dims[0], m = s.dims[1];
    const double dmin = (double)s.dims[2], dmax = (double)s.dims[3];
    const double g = 2.3, a = std::pow(dmin, 1.0 - g), b = std::pow(dmax, 1.0 - g);
    std::vector<double> cdf((size_t)n);
    double acc = 0.0;
    for (int64_t i = 0; i < n; ++i) {
        double u = unit(hash3(s.seed, kDegree, (uint64_t)i));
        double w = std::pow(a - u * (a - b), 1.0 / (1.0 - g));
        acc += w;
        cdf[(size_t)i] = acc;
    }
    auto pick = [&](double u) {
        double t = u * acc;
        return (int64_t)(std::upper_bound(cdf.begin(), cdf.end(), t) - cdf.begin());
    };
    std::vector<std::pair<int64_t, int64_t>> ed;
    ed.reserve((size_t)m);
    for (int64_t e = 0; e < m; ++e) {
        int64_t u = std::min<int64_t>(pick(unit(hash3(s.seed, kEdgeU, (uint64_t)e))), n - 1);
        int64_t v = std::min<int64_t>(pick(unit(hash3(s.seed, kEdgeV, (uint64_t)e))), n - 1);
        if (u == v) continue;
        ed.emplace_back(std::min(u, v), std::max(u, v));
    }
    std::sort(ed.begin(), ed.end());
    ed.erase(std::unique(ed.begin(), ed.end()), ed.end());
    // largest connected component (union-find)
    std::vector<int64_t> par((size_t)n);
    std::iota(par.begin(), par.end(), 0);
    auto find = [&](int64_t x) {
        while (par[(size_t)x] != x) {
            par[(size_t)x] = par[(size_t)par[(size_t)x]];
            x = par[(size_t)x];
        }
        return x;
    };
    for (auto& p : ed) {
        int64_t ra = find(p.first), rb = find(p.second);
        if (ra != rb) par[(size_t)std::max(ra, rb)] = std::min(ra, rb);
    }
    std::vector<int64_t> sz((size_t)n, 0);
    for (int64_t i = 0; i < n; ++i) sz[(size_t)find(i)]++;
    int64_t best = (int64_t)(std::max_element(sz.begin(), sz.end()) - sz.begin());
    std::vector<int64_t> relabel((size_t)n, -1);
    int64_t nn = 0;
    for (int64_t i = 0; i < n; ++i)
        if (find(i) == best) relabel[(size_t)i] = nn++;
    E.n = nn;
    uint64_t e = 0;
    for (auto& p : ed) {
        if (relabel[(size_t)p.first] < 0) continue;
        E.a.push_back(relabel[(size_t)p.first]);
        E.b.push_back(relabel[(size_t)p.second]);
        E.w.push_back(draw_weight(s, e++));
    }
    return true;
}

}  // namespace

bool generate(const GenSpec& s, Triplets& out, bool& has_ground, std::string& err) {
    EdgeList E;
    if (s.kind == "grid2d" || s.kind == "grid3d") {
        if (s.dims.empty()) {
            err = "grid needs side lengths";
            return false;
        }
        grid_edges(s, E, false);
    } else if (s.kind == "grid3d27") {
        grid_edges(s, E, true);
    } else if (s.kind == "chunglu") {
        if (!chunglu_edges(s, E, err)) return false;
    } else {
        err = "unknown generator kind " + s.kind;
        return false;
    }
    const int64_t n = E.n;
    if (n <= 0 || n + 1 > INT32_MAX) {
        err = "generator size out of range";
        return false;
    }
    std::vector<double> wdeg((size_t)n, 0.0);
    std::vector<int64_t> deg((size_t)n, 0);
    for (size_t k = 0; k < E.a.size(); ++k) {
        wdeg[(size_t)E.a[k]] += E.w[k];
        wdeg[(size_t)E.b[k]] += E.w[k];
        deg[(size_t)E.a[k]]++;
        deg[(size_t)E.b[k]]++;
    }
    std::vector<double> excess((size_t)n, 0.0);
    has_ground = false;
    if (s.excess_frac > 0.0) {
        for (int64_t i = 0; i < n; ++i) {
            if (unit(hash3(s.seed, kExcessPick, (uint64_t)i)) < s.excess_frac) {
                double u = unit(hash3(s.seed, kExcessVal, (uint64_t)i));
                excess[(size_t)i] = (s.excess_lo + u * (s.excess_hi - s.excess_lo)) * wdeg[(size_t)i];
                if (excess[(size_t)i] > 0.0) has_ground = true;
            }
        }
    }
    // ordering of the SDDM (write_graph.jl:112-128): random permutation, then
    // a stable sort by column nnz (degree + diagonal)
    std::vector<int64_t> order((size_t)n);
    std::iota(order.begin(), order.end(), 0);
    if (s.ordering == 0 || s.ordering == 1) {
        std::vector<uint64_t> key((size_t)n);
        for (int64_t i = 0; i < n; ++i) key[(size_t)i] = hash3(s.seed, kOrder, (uint64_t)i);
        std::sort(order.begin(), order.end(), [&](int64_t x, int64_t y) {
            return key[(size_t)x] != key[(size_t)y] ? key[(size_t)x] < key[(size_t)y] : x < y;
        });
        if (s.ordering == 0)
            std::stable_sort(order.begin(), order.end(),
                             [&](int64_t x, int64_t y) { return deg[(size_t)x] < deg[(size_t)y]; });
    }
    std::vector<int32_t> pos((size_t)n);
    for (int64_t i = 0; i < n; ++i) pos[(size_t)order[(size_t)i]] = (int32_t)i;
    const int32_t N = (int32_t)(n + (has_ground ? 1 : 0));
    out.n = N;
    size_t ne = E.a.size();
    size_t ng = 0;
    if (has_ground)
        for (int64_t i = 0; i < n; ++i) ng += excess[(size_t)i] > 0.0;
    out.rows.clear();
    out.cols.clear();
    out.vals.clear();
    out.rows.reserve(2 * ne + 2 * ng + (size_t)N);
    out.cols.reserve(out.rows.capacity());
    out.vals.reserve(out.rows.capacity());
    for (size_t k = 0; k < ne; ++k) {
        int32_t u = pos[(size_t)E.a[k]], v = pos[(size_t)E.b[k]];
        out.rows.push_back(u);
        out.cols.push_back(v);
        out.vals.push_back(-E.w[k]);
        out.rows.push_back(v);
        out.cols.push_back(u);
        out.vals.push_back(-E.w[k]);
    }
    double gsum = 0.0;
    if (has_ground) {
        // write_graph.jl:153-163: the appended row/column is -max(0, colsum)
        for (int64_t i = 0; i < n; ++i) {
            double x = excess[(size_t)i];
            if (x <= 0.0) continue;
            int32_t u = pos[(size_t)i];
            out.rows.push_back(u);
            out.cols.push_back(N - 1);
            out.vals.push_back(-x);
            out.rows.push_back(N - 1);
            out.cols.push_back(u);
            out.vals.push_back(-x);
            gsum += x;
        }
    }
    for (int64_t i = 0; i < n; ++i) {
        int32_t u = pos[(size_t)i];
        out.rows.push_back(u);
        out.cols.push_back(u);
        out.vals.push_back(wdeg[(size_t)i] + excess[(size_t)i]);
    }
    if (has_ground) {
        out.rows.push_back(N - 1);
        out.cols.push_back(N - 1);
        out.vals.push_back(gsum);
    }
    return true;
}

}  // namespace rchol
