// Fill-reducing and bandwidth orderings on the host (the reference's
// write_graph.jl:61-75 offers "amd", "random" and "nd" besides "nnz-sort",
// through Julia's AMD and Metis packages, which are not part of this build).
// Two orderings restated here from their published descriptions:
//   * reverse Cuthill-McKee (Cuthill & McKee 1969; George & Liu 1981): per
//     connected component, a breadth-first search from a pseudo-peripheral
//     vertex visiting neighbours by ascending degree; the whole order is
//     then reversed;
//   * nested dissection by level-structure bisection (George 1973; George &
//     Liu 1981, ch. 8): a region's breadth-first levels from a
//     pseudo-peripheral vertex are cut at the level holding its median
//     vertex; that level is the separator, numbered after the two halves,
//     which are dissected the same way down to kNdLeaf vertices.
#include "host_io.h"

#include <algorithm>
#include <numeric>
#include <vector>

namespace rchol {

namespace {

struct Graph {
    int32_t n = 0;
    std::vector<int64_t> ptr;
    std::vector<int32_t> adj;
};

// symmetric off-diagonal pattern (duplicates kept: they only repeat a visit)
Graph build_graph(int32_t n, int64_t nnz, const int32_t* rows, const int32_t* cols) {
    Graph g;
    g.n = n;
    g.ptr.assign((size_t)n + 1, 0);
    for (int64_t k = 0; k < nnz; ++k)
        if (rows[k] != cols[k]) g.ptr[(size_t)cols[k] + 1]++;
    for (int32_t i = 0; i < n; ++i) g.ptr[(size_t)i + 1] += g.ptr[(size_t)i];
    g.adj.resize((size_t)g.ptr[(size_t)n]);
    std::vector<int64_t> cur(g.ptr.begin(), g.ptr.end() - 1);
    for (int64_t k = 0; k < nnz; ++k)
        if (rows[k] != cols[k]) g.adj[(size_t)cur[(size_t)cols[k]]++] = rows[k];
    return g;
}

// Breadth-first levels from `root` inside region `reg` (mark[v] == reg).
// Returns the visit order; level_of[v] is set for visited vertices.
int32_t bfs(const Graph& g, int32_t root, const std::vector<int32_t>& mark, int32_t reg, std::vector<int32_t>& level_of,
            std::vector<int32_t>& order, bool by_degree, const std::vector<int32_t>& deg) {
    order.clear();
    order.push_back(root);
    level_of[(size_t)root] = 0;
    int32_t depth = 0;
    std::vector<int32_t> nb;
    for (size_t h = 0; h < order.size(); ++h) {
        const int32_t v = order[h];
        nb.clear();
        for (int64_t p = g.ptr[(size_t)v]; p < g.ptr[(size_t)v + 1]; ++p) {
            const int32_t u = g.adj[(size_t)p];
            if (mark[(size_t)u] == reg && level_of[(size_t)u] < 0) {
                level_of[(size_t)u] = level_of[(size_t)v] + 1;
                nb.push_back(u);
            }
        }
        if (by_degree)
            std::stable_sort(nb.begin(), nb.end(),
                             [&](int32_t x, int32_t y) { return deg[(size_t)x] < deg[(size_t)y]; });
        for (int32_t u : nb) {
            order.push_back(u);
            depth = std::max(depth, level_of[(size_t)u]);
        }
    }
    return depth;
}

// A pseudo-peripheral vertex of the component of `start` in region `reg`:
// repeat a search from the least-degree vertex of the last level while the
// eccentricity grows (Gibbs, Poole & Stockmeyer 1976).
int32_t peripheral(const Graph& g, int32_t start, const std::vector<int32_t>& mark, int32_t reg,
                   std::vector<int32_t>& level_of, std::vector<int32_t>& order, const std::vector<int32_t>& deg) {
    int32_t root = start, best = -1;
    for (int it = 0; it < 8; ++it) {
        for (int32_t v : order) level_of[(size_t)v] = -1;
        level_of[(size_t)root] = -1;
        const int32_t depth = bfs(g, root, mark, reg, level_of, order, false, deg);
        if (depth <= best) break;
        best = depth;
        int32_t cand = root;
        for (int32_t v : order)
            if (level_of[(size_t)v] == depth && (cand == root || deg[(size_t)v] < deg[(size_t)cand])) cand = v;
        if (cand == root) break;
        root = cand;
    }
    for (int32_t v : order) level_of[(size_t)v] = -1;
    return root;
}

constexpr int32_t kNdLeaf = 64;

}  // namespace

bool host_ordering(int kind, int32_t n, int64_t nnz, const int32_t* rows, const int32_t* cols,
                   std::vector<int32_t>& order, std::string& err) {
    if (kind != kHostOrderRcm && kind != kHostOrderNd) {
        err = "unknown host ordering";
        return false;
    }
    for (int64_t k = 0; k < nnz; ++k)
        if (rows[k] < 0 || rows[k] >= n || cols[k] < 0 || cols[k] >= n) {
            err = "triplet index out of range";
            return false;
        }
    const Graph g = build_graph(n, nnz, rows, cols);
    std::vector<int32_t> deg((size_t)n);
    for (int32_t v = 0; v < n; ++v) deg[(size_t)v] = (int32_t)(g.ptr[(size_t)v + 1] - g.ptr[(size_t)v]);
    std::vector<int32_t> level_of((size_t)n, -1), visit;
    order.clear();
    order.reserve((size_t)n);
    if (kind == kHostOrderRcm) {
        std::vector<int32_t> mark((size_t)n, 0);  // 0: unnumbered, 1: numbered
        for (int32_t s = 0; s < n; ++s) {
            if (mark[(size_t)s] != 0) continue;
            const int32_t root = peripheral(g, s, mark, 0, level_of, visit, deg);
            bfs(g, root, mark, 0, level_of, visit, true, deg);
            for (int32_t v : visit) {
                mark[(size_t)v] = 1;
                order.push_back(v);
            }
        }
        std::reverse(order.begin(), order.end());
        return true;
    }
    // nested dissection: regions on an explicit stack; each region's vertices
    // are numbered after its two halves (the stack keeps the separators to
    // append once both halves are done)
    std::vector<int32_t> mark((size_t)n, 0);
    int32_t next_reg = 1;
    struct Item {
        std::vector<int32_t> verts;  // region vertices, or a separator to append
        bool separator;
    };
    std::vector<Item> stack;
    {
        std::vector<int32_t> all((size_t)n);
        std::iota(all.begin(), all.end(), 0);
        stack.push_back({std::move(all), false});
    }
    while (!stack.empty()) {
        Item it = std::move(stack.back());
        stack.pop_back();
        if (it.separator || (int32_t)it.verts.size() <= kNdLeaf) {
            order.insert(order.end(), it.verts.begin(), it.verts.end());
            continue;
        }
        const int32_t reg = next_reg++;
        for (int32_t v : it.verts) mark[(size_t)v] = reg;
        // one component at a time: the levels of the first vertex's component
        const int32_t root = peripheral(g, it.verts[0], mark, reg, level_of, visit, deg);
        const int32_t depth = bfs(g, root, mark, reg, level_of, visit, false, deg);
        std::vector<int32_t> rest;  // vertices of other components of the region
        if (visit.size() < it.verts.size()) {
            for (int32_t v : it.verts)
                if (level_of[(size_t)v] < 0) rest.push_back(v);
        }
        std::vector<int32_t> a, b, sep;
        if (depth < 2) {
            a = visit;  // too shallow to cut: number the component as is
        } else {
            std::vector<int32_t> cnt((size_t)depth + 1, 0);
            for (int32_t v : visit) cnt[(size_t)level_of[(size_t)v]]++;
            int32_t cut = 1, acc = 0;
            for (int32_t l = 0; l <= depth; ++l) {
                acc += cnt[(size_t)l];
                if (2 * acc >= (int32_t)visit.size()) {
                    cut = std::min(std::max(l, 1), depth - 1);
                    break;
                }
            }
            for (int32_t v : visit) {
                const int32_t l = level_of[(size_t)v];
                (l < cut ? a : (l > cut ? b : sep)).push_back(v);
            }
        }
        for (int32_t v : visit) level_of[(size_t)v] = -1;
        for (int32_t v : it.verts) mark[(size_t)v] = 0;
        // numbered in this order: rest, then a, b, then the separator
        stack.push_back({std::move(sep), true});
        if (!b.empty()) stack.push_back({std::move(b), false});
        if (depth < 2) {
            stack.push_back({std::move(a), true});
        } else if (!a.empty()) {
            stack.push_back({std::move(a), false});
        }
        if (!rest.empty()) stack.push_back({std::move(rest), false});
    }
    if ((int32_t)order.size() != n) {
        err = "nested dissection lost vertices";
        return false;
    }
    return true;
}

}  // namespace rchol
