// Invariants of build_row_tiles on seeded random banded symmetric patterns: tiles cover
// the rows in order and stay within the row, entry and union bounds, every union is
// sorted and unique, every entry's slot names its column, each tile's order is a
// permutation of its rows, and the lane map gives every row one aligned power-of-two
// group inside a warp (each lane at most once), smaller than twice its row. A row longer than
// the cap disables the tiles. Prints "ok" or the first violation.
#include <algorithm>
#include <cstdio>
#include <random>
#include <vector>

#include "host/tree_builder.hpp"

static int check(int rows, int band, int lanes, int cap, int threads, unsigned seed)
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
    const int64_t target = std::max<int64_t>(1, rp[rows] / std::max(1, rows / 100));
    rpb::build_row_tiles(rp.data(), ci.data(), rows, rows, lanes, target, cap, threads, T);
    int64_t longest = 0;
    for (int i = 0; i < rows; ++i) longest = std::max(longest, rp[i + 1] - rp[i]);
    if (longest > cap) {
        if (T.valid) { std::printf("tiles valid although a row exceeds the cap\n"); return 1; }
        return 0;
    }
    if (!T.valid) { std::printf("tiles invalid\n"); return 1; }
    if (T.row0.front() != 0 || T.row0.back() != rows) { std::printf("row range\n"); return 1; }
    if (static_cast<int>(T.lane_map.size()) != T.tiles() * lanes) { std::printf("lane map size\n"); return 1; }
    for (int b = 0; b < T.tiles(); ++b) {
        const int r0 = T.row0[b], r1 = T.row0[b + 1];
        if (r1 <= r0 || r1 - r0 > lanes) { std::printf("tile %d rows %d..%d\n", b, r0, r1); return 1; }
        if (rp[r1 - 1] - rp[r0] >= target && r1 - r0 > 1) { std::printf("tile %d over the entry target\n", b); return 1; }
        const int u0 = T.cols_rp[b], un = T.cols_rp[b + 1] - u0;
        if (un > cap || un > T.max_union) { std::printf("tile %d union %d\n", b, un); return 1; }
        for (int u = 1; u < un; ++u)
            if (T.cols[u0 + u] <= T.cols[u0 + u - 1]) { std::printf("tile %d union not ascending\n", b); return 1; }
        std::vector<int> seen(rows, 0), group_size(r1 - r0, 0);
        std::vector<int64_t> group_lanes(r1 - r0, 0);
        for (int k = r0; k < r1; ++k) {
            const int i = T.order[k];
            if (i < r0 || i >= r1 || seen[i]++) { std::printf("tile %d order\n", b); return 1; }
            for (int64_t e = rp[i]; e < rp[i + 1]; ++e)
                if (T.slot[e] >= un || T.cols[u0 + T.slot[e]] != ci[e]) { std::printf("slot of entry %ld\n", (long)e); return 1; }
        }
        for (int t = 0; t < lanes; ++t) {
            const int m = T.lane_map[static_cast<size_t>(b) * lanes + t];
            if (m < 0) continue;
            const int q = m >> 10, size = ((m >> 5) & 31) + 1, sub = m & 31;
            if (q >= r1 - r0 || sub >= size) { std::printf("tile %d lane %d map\n", b, t); return 1; }
            const int start = t - sub;
            if ((size & (size - 1)) != 0 || start % size != 0 || start / 32 != (start + size - 1) / 32) {
                std::printf("tile %d group alignment\n", b);
                return 1;
            }
            if (group_size[q] == 0) group_size[q] = size;
            else if (group_size[q] != size) { std::printf("tile %d group size\n", b); return 1; }
            group_lanes[q] += int64_t(1) << sub;   // each lane of the group exactly once
        }
        for (int q = 0; q < r1 - r0; ++q) {
            if (group_size[q] == 0 || group_lanes[q] != static_cast<int64_t>((1ull << group_size[q]) - 1)) {
                std::printf("tile %d row %d lanes\n", b, q);
                return 1;
            }
            const int64_t len = rp[T.order[r0 + q] + 1] - rp[T.order[r0 + q]];
            if (group_size[q] > 1 && group_size[q] >= 2 * len) {
                std::printf("tile %d row %d group twice its row\n", b, q);
                return 1;
            }
        }
    }
    return 0;
}

int main()
{
    int bad = 0;
    bad |= check(10000, 40, 288, 1024, 4, 1u);
    bad |= check(10000, 40, 288, 60, 3, 2u);         // small cap: tiles close early
    bad |= check(5000, 200, 288, 150, 2, 3u);        // rows longer than the cap: tiles off
    bad |= check(1, 1, 288, 1024, 1, 4u);            // a single row without entries
    bad |= check(70000, 12, 256, 1536, 8, 5u);       // many tiles, short rows
    bad |= check(3000, 120, 64, 4096, 2, 6u);        // long rows, few lanes
    if (!bad) std::printf("ok\n");
    return bad;
}
