// Invariants of build_row_tiles on seeded random banded symmetric patterns: tiles cover
// the rows in order, every union is sorted, unique and within the cap, every entry's slot
// names its column, each tile's order is a permutation of its rows by decreasing length,
// and a row longer than the cap disables the tiles. Prints "ok" or the first violation.
#include <algorithm>
#include <cstdio>
#include <random>
#include <vector>

#include "host/tree_builder.hpp"

static int check(int rows, int band, int max_rows, int cap, int threads, unsigned seed)
{
    std::mt19937 rng(seed);
    std::vector<std::vector<int>> adj(rows);
    std::uniform_int_distribution<int> off(1, band);
    for (int i = 0; i < rows; ++i)
        for (int t = 0; t < band / 2; ++t) {
            const int j = std::min(rows - 1, i + off(rng));
            if (j != i) { adj[i].push_back(j); adj[j].push_back(i); }
        }
    std::vector<int64_t> rp(rows + 1, 0);
    std::vector<int> ci;
    for (int i = 0; i < rows; ++i) {
        std::sort(adj[i].begin(), adj[i].end());
        adj[i].erase(std::unique(adj[i].begin(), adj[i].end()), adj[i].end());
        ci.insert(ci.end(), adj[i].begin(), adj[i].end());
        rp[i + 1] = static_cast<int64_t>(ci.size());
    }
    rpb::RowTiles T;
    rpb::build_row_tiles(rp.data(), ci.data(), rows, rows, max_rows, cap, threads, T);
    int64_t longest = 0;
    for (int i = 0; i < rows; ++i) longest = std::max(longest, rp[i + 1] - rp[i]);
    if (longest > cap) {
        if (T.valid) { std::printf("tiles valid although a row exceeds the cap\n"); return 1; }
        return 0;
    }
    if (!T.valid) { std::printf("tiles invalid\n"); return 1; }
    if (T.row0.front() != 0 || T.row0.back() != rows) { std::printf("row range\n"); return 1; }
    for (int b = 0; b < T.tiles(); ++b) {
        const int r0 = T.row0[b], r1 = T.row0[b + 1];
        if (r1 <= r0 || r1 - r0 > max_rows) { std::printf("tile %d rows %d..%d\n", b, r0, r1); return 1; }
        const int u0 = T.cols_rp[b], un = T.cols_rp[b + 1] - u0;
        if (un > cap || un > T.max_union) { std::printf("tile %d union %d\n", b, un); return 1; }
        for (int u = 1; u < un; ++u)
            if (T.cols[u0 + u] <= T.cols[u0 + u - 1]) { std::printf("tile %d union not ascending\n", b); return 1; }
        std::vector<int> seen(rows, 0);
        for (int k = r0; k < r1; ++k) {
            const int i = T.order[k];
            if (i < r0 || i >= r1 || seen[i]++) { std::printf("tile %d order\n", b); return 1; }
            if (k > r0) {
                const int h = T.order[k - 1];
                if (rp[h + 1] - rp[h] < rp[i + 1] - rp[i]) { std::printf("tile %d order not by length\n", b); return 1; }
            }
            for (int64_t e = rp[i]; e < rp[i + 1]; ++e)
                if (T.slot[e] >= un || T.cols[u0 + T.slot[e]] != ci[e]) { std::printf("slot of entry %ld\n", (long)e); return 1; }
        }
    }
    return 0;
}

int main()
{
    int bad = 0;
    bad |= check(10000, 40, 64, 1024, 4, 1u);
    bad |= check(10000, 40, 64, 60, 3, 2u);          // small cap: tiles close early
    bad |= check(5000, 200, 128, 150, 2, 3u);        // rows longer than the cap: tiles off
    bad |= check(1, 1, 64, 1024, 1, 4u);             // a single row without entries
    bad |= check(70000, 12, 128, 1536, 8, 5u);       // several chunks of 4096 rows
    if (!bad) std::printf("ok\n");
    return bad;
}
