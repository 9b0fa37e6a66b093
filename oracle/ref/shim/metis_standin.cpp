// METIS stand-in (see metis.h).  TEST INFRASTRUCTURE ONLY.
#include "metis.h"

#include <cstdio>
#include <cstdlib>
#include <deque>
#include <vector>

extern "C" int METIS_SetDefaultOptions(idx_t* options)
{
    for (int i = 0; i < METIS_NOPTIONS; ++i) options[i] = -1;
    return METIS_OK;
}

namespace {
// recursive bisection of a breadth-first order of the vertices of each part
void bisect(const idx_t* xadj, const idx_t* adj, std::vector<idx_t>& verts, idx_t first, idx_t np, idx_t* part,
            std::vector<int>& mark, int& stamp)
{
    if (np == 1) {
        for (idx_t v : verts) part[v] = first;
        return;
    }
    ++stamp;
    for (idx_t v : verts) mark[v] = stamp;
    // start from a vertex of minimum degree inside the part (a corner of a grid)
    idx_t start = verts[0];
    int best = 1 << 30;
    for (idx_t v : verts) {
        int d = 0;
        for (idx_t e = xadj[v]; e < xadj[v + 1]; ++e) d += mark[adj[e]] == stamp;
        if (d < best) { best = d; start = v; }
    }
    std::vector<idx_t> order;
    order.reserve(verts.size());
    ++stamp;
    const int seen = stamp;
    std::vector<idx_t> pending(verts.begin(), verts.end());
    size_t next_seed = 0;
    std::deque<idx_t> q;
    auto inside = [&](idx_t v) { return mark[v] == seen - 1 || mark[v] == seen; };
    mark[start] = seen;
    q.push_back(start);
    while (order.size() < verts.size()) {
        if (q.empty()) {
            while (mark[pending[next_seed]] == seen) ++next_seed;
            mark[pending[next_seed]] = seen;
            q.push_back(pending[next_seed]);
        }
        idx_t v = q.front();
        q.pop_front();
        order.push_back(v);
        for (idx_t e = xadj[v]; e < xadj[v + 1]; ++e) {
            idx_t w = adj[e];
            if (inside(w) && mark[w] != seen) { mark[w] = seen; q.push_back(w); }
        }
    }
    idx_t k = np / 2;
    size_t cut = (size_t)((double)k / np * order.size() + 0.5);
    std::vector<idx_t> a(order.begin(), order.begin() + cut), b(order.begin() + cut, order.end());
    bisect(xadj, adj, a, first, k, part, mark, stamp);
    bisect(xadj, adj, b, first + k, np - k, part, mark, stamp);
}
}  // namespace

extern "C" int METIS_PartGraphKway(idx_t* nvtxs, idx_t*, idx_t* xadj, idx_t* adjncy, idx_t*, idx_t*, idx_t*,
                                   idx_t* nparts, real_t*, real_t*, idx_t*, idx_t* edgecut, idx_t* part)
{
    const idx_t n = *nvtxs;
    if (const char* f = std::getenv("S2L_PART_FILE")) {
        FILE* fp = std::fopen(f, "rb");
        if (!fp) { std::fprintf(stderr, "metis stand-in: cannot open %s\n", f); return METIS_ERROR_INPUT; }
        size_t got = std::fread(part, sizeof(idx_t), (size_t)n, fp);
        std::fclose(fp);
        if (got != (size_t)n) { std::fprintf(stderr, "metis stand-in: %s has %zu of %d entries\n", f, got, n); return METIS_ERROR_INPUT; }
        for (idx_t i = 0; i < n; ++i)
            if (part[i] < 0 || part[i] >= *nparts) return METIS_ERROR_INPUT;
    } else {
        std::vector<idx_t> verts(n);
        for (idx_t i = 0; i < n; ++i) verts[i] = i;
        std::vector<int> mark(n, 0);
        int stamp = 0;
        bisect(xadj, adjncy, verts, 0, *nparts, part, mark, stamp);
    }
    idx_t cut = 0;
    for (idx_t v = 0; v < n; ++v)
        for (idx_t e = xadj[v]; e < xadj[v + 1]; ++e) cut += part[v] != part[adjncy[e]];
    if (edgecut) *edgecut = cut / 2;
    return METIS_OK;
}
