// Cluster tree and block cluster tree on the B200. The block cluster tree: the dual
// traversal of the cluster tree that classifies every block pair as far field (admissible
// cluster pair), near field, very near or intersecting
// (src/ClusterTreePairTraversor/Traverse_DepthFirst.hpp:52-258 with
// src/BlockClusterTree/BlockSplit_Kernel.hpp:164-251), and the full symmetric CSR patterns
// (src/BlockClusterTree.hpp:306-326). The cluster tree (build_cluster_tree_device, at the
// end of this file): the longest-axis splits level by level with the reference's
// permutation, the median fallback's reordering done on the host.
//
// The traversal runs breadth first: one launch per level of block pairs, one thread per
// pair, children and results appended through atomic counters. The decisions come from
// host/bct_rules.hpp, the same code the host builder runs, and this file is compiled
// without fused multiply-adds, so the pair sets equal the host builder's bit for bit
// (the order of discovery differs; the CSR rows are sorted). Rows and columns are then
// sorted on the device (CUB radix sort of 64-bit (row, column) keys).
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "host/bct_rules.hpp"
#include "host/tree_builder.hpp"
#include "rpb_internal.cuh"
#include "rpb_mesh.cuh"

namespace rpb {

namespace {

struct BctTree {
    int dom, size, ps;
    const double* C_box;       // NC x 7
    const int* C_left;
    const int* C_right;
    const int* C_begin;
    const double* P;           // N x ps serialized polytopes, tree order
    const int* S;              // original simplices
    const int* perm;           // tree position -> simplex
    double far_t2, near_t2;
};

// lists: 0 far (cluster pairs), 1 near, 2 very near, 3 intersecting (primitive pairs)
struct BctOut {
    int2* next;
    unsigned long long* n_next;
    unsigned long long cap_next;
    int2* list[4];
    unsigned long long* count;  // 4 counters
    unsigned long long cap[4];
};

__device__ __forceinline__ void emit(const BctOut& O, int k, int a, int b)
{
    const unsigned long long pos = atomicAdd(O.count + k, 1ull);
    if (pos < O.cap[k]) O.list[k][pos] = make_int2(a, b);
}

__device__ __forceinline__ bool adjacent(const BctTree& T, int pi, int pj)
{
    const int* a = T.S + static_cast<int64_t>(T.size) * T.perm[pi];
    const int* b = T.S + static_cast<int64_t>(T.size) * T.perm[pj];
    for (int u = 0; u < T.size; ++u)
        for (int v = 0; v < T.size; ++v)
            if (a[u] == b[v]) return true;
    return false;
}

__global__ void __launch_bounds__(256) k_bct_level(BctTree T, const int2* in, long long n_in, BctOut O)
{
    const long long t = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= n_in) return;
    const int i = in[t].x, j = in[t].y;
    if (i != j && bct::boxes_admissible(T.C_box + 7 * static_cast<int64_t>(i), T.C_box + 7 * static_cast<int64_t>(j),
                                        T.far_t2)) {
        emit(O, 0, i < j ? i : j, i < j ? j : i);
        return;
    }
    const int Li = T.C_left[i], Lj = T.C_left[j];
    if (Li >= 0 || Lj >= 0) {
        const int Ri = T.C_right[i], Rj = T.C_right[j];
        const double si = Li >= 0 ? T.C_box[7 * static_cast<int64_t>(i)] : 0.0;
        const double sj = Lj >= 0 ? T.C_box[7 * static_cast<int64_t>(j)] : 0.0;
        int2 c[4];
        int n = 0;
        if (si == sj && si > 0) {
            if (i == j) { c[0] = make_int2(Li, Rj); c[1] = make_int2(Ri, Rj); c[2] = make_int2(Li, Lj); n = 3; }
            else { c[0] = make_int2(Ri, Rj); c[1] = make_int2(Li, Rj); c[2] = make_int2(Ri, Lj); c[3] = make_int2(Li, Lj); n = 4; }
        } else if (si > sj) {
            c[0] = make_int2(Ri, j); c[1] = make_int2(Li, j); n = 2;
        } else {
            c[0] = make_int2(i, Rj); c[1] = make_int2(i, Lj); n = 2;
        }
        const unsigned long long pos = atomicAdd(O.n_next, static_cast<unsigned long long>(n));
        if (pos + n <= O.cap_next)
            for (int k = 0; k < n; ++k) O.next[pos + k] = c[k];
        return;
    }
    if (i == j) return;
    const int ii = T.C_begin[i], jj = T.C_begin[j];
    const int a = ii < jj ? ii : jj, b = ii < jj ? jj : ii;
    if (adjacent(T, a, b)) { emit(O, 1, a, b); return; }
    const int cls = bct::classify_leaf(T.dom, T.P + static_cast<int64_t>(T.ps) * a, T.P + static_cast<int64_t>(T.ps) * b,
                                       T.near_t2);
    emit(O, 1 + cls, a, b);
}

// both orientations of every pair as (row << 32 | column) keys
__global__ void k_pair_keys(long long n, const int2* pairs, unsigned long long* keys)
{
    const long long t = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int2 p = pairs[t];
    keys[2 * t] = (static_cast<unsigned long long>(p.x) << 32) | static_cast<unsigned int>(p.y);
    keys[2 * t + 1] = (static_cast<unsigned long long>(p.y) << 32) | static_cast<unsigned int>(p.x);
}

// columns and, from the sorted keys, the first entry of every row (rows without entries
// repeat the next row start; rp[rows] = nnz)
__global__ void k_keys_to_csr(long long nnz, int rows, const unsigned long long* keys, int* ci, int64_t* rp)
{
    const long long t = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t > nnz) return;
    const int row = t < nnz ? static_cast<int>(keys[t] >> 32) : rows;
    const int prev = t > 0 ? static_cast<int>(keys[t - 1] >> 32) : -1;
    if (t < nnz) ci[t] = static_cast<int>(keys[t] & 0xffffffffull);
    for (int r = prev + 1; r <= row; ++r) rp[r] = t;
}

cudaError_t sym_pattern(const int2* pairs, long long n, int rows, SymPattern& P, cudaStream_t s)
{
    P = SymPattern();
    P.rows = rows;
    P.rp.assign(static_cast<size_t>(rows) + 1, 0);
    if (n == 0) { P.diag.assign(rows, 0); return cudaSuccess; }
    const long long nnz = 2 * n;
    DevBuf<unsigned long long> keys, sorted;
    DevBuf<int> ci;
    DevBuf<int64_t> rp;
    DevBuf<unsigned char> temp;
    cudaError_t e;
    if ((e = keys.alloc(nnz)) != cudaSuccess || (e = sorted.alloc(nnz)) != cudaSuccess ||
        (e = ci.alloc(nnz)) != cudaSuccess || (e = rp.alloc(rows + 1)) != cudaSuccess)
        return e;
    k_pair_keys<<<static_cast<unsigned>((n + 255) / 256), 256, 0, s>>>(n, pairs, keys.ptr);
    size_t bytes = 0;
    int end_bit = 32;
    while (end_bit < 64 && (1ll << (end_bit - 32)) <= rows) ++end_bit;
    if ((e = cub::DeviceRadixSort::SortKeys(nullptr, bytes, keys.ptr, sorted.ptr, nnz, 0, end_bit, s)) != cudaSuccess) return e;
    if ((e = temp.alloc(bytes)) != cudaSuccess) return e;
    if ((e = cub::DeviceRadixSort::SortKeys(temp.ptr, bytes, keys.ptr, sorted.ptr, nnz, 0, end_bit, s)) != cudaSuccess) return e;
    k_keys_to_csr<<<static_cast<unsigned>((nnz + 1 + 255) / 256), 256, 0, s>>>(nnz, rows, sorted.ptr, ci.ptr, rp.ptr);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    P.ci.resize(nnz);
    if ((e = cudaMemcpyAsync(P.rp.data(), rp.ptr, rp.bytes(), cudaMemcpyDeviceToHost, s)) != cudaSuccess) return e;
    if ((e = cudaMemcpyAsync(P.ci.data(), ci.ptr, ci.bytes(), cudaMemcpyDeviceToHost, s)) != cudaSuccess) return e;
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return e;
    P.diag.resize(rows);
    for (int i = 0; i < rows; ++i) {
        const auto b = P.ci.begin() + P.rp[i], en = P.ci.begin() + P.rp[i + 1];
        P.diag[i] = std::upper_bound(b, en, i) - P.ci.begin();
    }
    return cudaSuccess;
}

}  // namespace

// The four patterns of T from the serialized polytopes P (tree order) on the device;
// false (with T untouched) if the device work failed.
bool build_block_cluster_tree_device(HostTree& T, const std::vector<double>& P, const int* S, const TreeSettings& set,
                                     cudaStream_t s, std::string& err)
{
    const int N = T.N, NC = T.NC, ps = 1 + 3 + T.size * 3;
    DevBuf<double> d_box, d_P;
    DevBuf<int> d_left, d_right, d_begin, d_S, d_perm;
    auto fail = [&](cudaError_t e) {
        err = std::string("device block cluster tree: ") + cudaGetErrorString(e);
        return false;
    };
    cudaError_t e;
#define RPB_UP(buf, vec)                                                                                     \
    if ((e = buf.alloc((vec).size())) != cudaSuccess ||                                                      \
        (e = cudaMemcpyAsync(buf.ptr, (vec).data(), buf.bytes(), cudaMemcpyHostToDevice, s)) != cudaSuccess) \
        return fail(e);
    RPB_UP(d_box, T.C_box);
    RPB_UP(d_P, P);
    RPB_UP(d_left, T.C_left);
    RPB_UP(d_right, T.C_right);
    RPB_UP(d_begin, T.C_begin);
    RPB_UP(d_perm, T.perm);
#undef RPB_UP
    if ((e = d_S.alloc(static_cast<size_t>(T.size) * N)) != cudaSuccess ||
        (e = cudaMemcpyAsync(d_S.ptr, S, d_S.bytes(), cudaMemcpyHostToDevice, s)) != cudaSuccess)
        return fail(e);
    BctTree bt{T.dom, T.size, ps, d_box.ptr, d_left.ptr, d_right.ptr, d_begin.ptr, d_P.ptr, d_S.ptr, d_perm.ptr,
               set.theta_far * set.theta_far, set.theta_near * set.theta_near};

    // result capacities from the mesh size, grown to the exact counts if a pass overflows
    unsigned long long cap[4] = {40ull * NC + 1024, 80ull * N + 1024, 1ull * N + 1024, 1ull * N + 1024};
    DevBuf<int2> lists[4];
    DevBuf<unsigned long long> counters;   // 4 list counts, next count
    if ((e = counters.alloc(5)) != cudaSuccess) return fail(e);
    unsigned long long counts[5];
    for (int attempt = 0; attempt < 2; ++attempt) {
        for (int k = 0; k < 4; ++k)
            if ((e = lists[k].alloc(cap[k])) != cudaSuccess) return fail(e);
        if ((e = cudaMemsetAsync(counters.ptr, 0, counters.bytes(), s)) != cudaSuccess) return fail(e);
        unsigned long long cap_front = 4096;
        DevBuf<int2> front, next;
        if ((e = front.alloc(cap_front)) != cudaSuccess || (e = next.alloc(cap_front)) != cudaSuccess) return fail(e);
        const int2 root = make_int2(0, 0);
        if ((e = cudaMemcpyAsync(front.ptr, &root, sizeof(root), cudaMemcpyHostToDevice, s)) != cudaSuccess) return fail(e);
        long long n_front = 1;
        for (int level = 0; n_front > 0 && level < 4096; ++level) {
            // list counts before the level, restored if the next frontier overflows
            unsigned long long before[5];
            if ((e = cudaMemcpyAsync(before, counters.ptr, sizeof(before), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
                (e = cudaStreamSynchronize(s)) != cudaSuccess)
                return fail(e);
            for (;;) {
                before[4] = 0;
                if ((e = cudaMemcpyAsync(counters.ptr, before, sizeof(before), cudaMemcpyHostToDevice, s)) != cudaSuccess)
                    return fail(e);
                BctOut O{next.ptr, counters.ptr + 4, next.n, {lists[0].ptr, lists[1].ptr, lists[2].ptr, lists[3].ptr},
                         counters.ptr, {cap[0], cap[1], cap[2], cap[3]}};
                k_bct_level<<<static_cast<unsigned>((n_front + 255) / 256), 256, 0, s>>>(bt, front.ptr, n_front, O);
                if ((e = cudaGetLastError()) != cudaSuccess) return fail(e);
                if ((e = cudaMemcpyAsync(counts, counters.ptr, sizeof(counts), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
                    (e = cudaStreamSynchronize(s)) != cudaSuccess)
                    return fail(e);
                if (counts[4] <= next.n) break;
                if ((e = next.alloc(counts[4] + counts[4] / 4)) != cudaSuccess) return fail(e);
            }
            std::swap(front.ptr, next.ptr);
            std::swap(front.n, next.n);
            n_front = static_cast<long long>(counts[4]);
            if (next.n < front.n && (e = next.alloc(front.n)) != cudaSuccess) return fail(e);
        }
        if (n_front > 0) { err = "device block cluster tree: traversal did not finish"; return false; }
        bool overflow = false;
        for (int k = 0; k < 4; ++k)
            if (counts[k] > cap[k]) { cap[k] = counts[k]; overflow = true; }
        if (!overflow) break;
        if (attempt == 1) { err = "device block cluster tree: result lists overflowed twice"; return false; }
    }
    HostTree R = T;
    const int rows[4] = {NC, N, N, N};
    SymPattern* out[4] = {&R.far, &R.near, &R.verynear, &R.inter};
    for (int k = 0; k < 4; ++k)
        if ((e = sym_pattern(lists[k].ptr, static_cast<long long>(counts[k]), rows[k], *out[k], s)) != cudaSuccess)
            return fail(e);
    T = std::move(R);
    return true;
}

// ----------------------------------------------------------------------------------------
// Cluster tree on the device: the longest-axis splits of AABB_LongestAxisSplit::split
// (src/BoundingVolumes/AABB_LongestAxisSplit.hpp:134-253) for all clusters of one level at
// once, and the depth-first numbering of Serialize_Thread.hpp:273-314, with the same
// permutation, ranges and boxes as the host builder (host/tree_builder.cpp).
//
// The reference partitions a cluster's range [b, e) by one in-place pass: scanning i
// upwards, a primitive whose centre lies below the box centre along the longest axis is
// swapped to the front (position s, then s + 1, ...). Its result has a closed form that
// needs no sequential pass: with nL primitives below the centre and i_r the position of
// the r-th of them (r = 0, 1, ...),
//   * the r-th primitive below the centre ends at b + r;
//   * a primitive above it at a position p >= b + nL stays at p;
//   * one above it at p < b + nL moves to i_p, from there (if i_p < b + nL) to i_{i_p},
//     and so on until the position reaches b + nL or beyond
// (each swap of the scan moves the element at the front of the block of upper primitives
// to the position of the primitive it swaps with). The chains are followed directly for up
// to CT_CHAIN steps and, when a chain is longer, after pointer jumping on i.
// A cluster whose primitives all lie on one side of the centre takes the reference's median
// fallback (std::nth_element of the centres, then the permutation applied); those clusters
// are collected on the device and reordered on the host by the same library call the host
// builder makes, then copied back.
// With split threshold 1 a cluster of m primitives has 2m - 1 clusters in its subtree, so
// the depth-first numbers follow from the split alone: left child g + 1, right child
// g + 2 (s - b). This file is compiled without fused multiply-adds: centres, radii and
// boxes round exactly like the host builder's.
// ----------------------------------------------------------------------------------------
namespace {

constexpr int CT_BLOCK = 256;
constexpr int CT_CHAIN = 64;

inline unsigned ct_grid(long long n) { return static_cast<unsigned>((n + CT_BLOCK - 1) / CT_BLOCK); }

// Per primitive (original index): centre, squared radius about it (serialize_polytope) and
// the bounding box of its vertices.
__global__ void k_ct_prims(int size, int N, const double* __restrict__ V, const int* __restrict__ S, double* cen,
                           double* rad2, double* plo, double* phi)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= N) return;
    double h[3][3];
    for (int a = 0; a < size; ++a) {
        const int v = S[static_cast<int64_t>(size) * j + a];
        for (int k = 0; k < 3; ++k) h[a][k] = V[3 * static_cast<int64_t>(v) + k];
    }
    const double w = 1.0 / size;
    double c[3];
    for (int k = 0; k < 3; ++k) {
        double acc = h[0][k];
        for (int a = 1; a < size; ++a) acc += h[a][k];
        c[k] = acc * w;
    }
    double r2 = 0.0;
    for (int a = 0; a < size; ++a) {
        double d = h[a][0] - c[0];
        double sq = d * d;
        for (int k = 1; k < 3; ++k) {
            d = h[a][k] - c[k];
            sq += d * d;
        }
        r2 = (r2 < sq) ? sq : r2;
    }
    rad2[j] = r2;
    for (int k = 0; k < 3; ++k) {
        double lo = h[0][k], hi = h[0][k];
        for (int a = 1; a < size; ++a) {
            lo = (h[a][k] < lo) ? h[a][k] : lo;
            hi = (hi < h[a][k]) ? h[a][k] : hi;
        }
        cen[3 * static_cast<int64_t>(j) + k] = c[k];
        plo[3 * static_cast<int64_t>(j) + k] = lo;
        phi[3 * static_cast<int64_t>(j) + k] = hi;
    }
}

// Boxes of clusters (one warp each): [r2, centre, half-lengths] of the vertex bounding box
// of the primitives ord[C_begin[g] .. C_end[g]) (aabb_of_range).
__global__ void k_ct_boxes(int n, int N, const int* __restrict__ ids, const int* __restrict__ C_begin,
                           const int* __restrict__ C_end, const int* __restrict__ ord, const double* __restrict__ plo,
                           const double* __restrict__ phi, double* C_box, unsigned* error)
{
    const long long w = (static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= n) return;
    const int g = ids[w];
    const int b = C_begin[g], e = C_end[g];
    double lo[3], hi[3];
    for (int k = 0; k < 3; ++k) {
        lo[k] = 1.7976931348623157e308;
        hi[k] = -1.7976931348623157e308;
    }
    for (int i = b + lane; i < e; i += 32) {
        const int64_t j = ord[i];
        if (j < 0 || j >= N) {
            atomicAdd(error, 1u);
            continue;
        }
        for (int k = 0; k < 3; ++k) {
            const double l = plo[3 * j + k], h = phi[3 * j + k];
            lo[k] = (l < lo[k]) ? l : lo[k];
            hi[k] = (hi[k] < h) ? h : hi[k];
        }
    }
    for (int off = 16; off > 0; off >>= 1)
        for (int k = 0; k < 3; ++k) {
            const double l = __shfl_xor_sync(0xffffffffu, lo[k], off);
            const double h = __shfl_xor_sync(0xffffffffu, hi[k], off);
            lo[k] = (l < lo[k]) ? l : lo[k];
            hi[k] = (hi[k] < h) ? h : hi[k];
        }
    if (lane == 0) {
        double* box = C_box + 7 * static_cast<int64_t>(g);
        double r2 = 0.0;
        for (int k = 0; k < 3; ++k) {
            const double half = 0.5 * (hi[k] - lo[k]);
            r2 += half * half;
            box[1 + k] = lo[k] + half;
            box[4 + k] = half;
        }
        box[0] = r2;
    }
}

// Clusters of one level being split: DFS number and range of each, the cluster of every
// position (index into the level's list, -1 for finished leaves) and per-cluster results.
struct CtLevel {
    int n;                 // clusters in the level
    const int* g;          // DFS numbers
    const int* b;          // ranges [b, e)
    const int* e;
    const int* cl;         // position -> cluster of the level or -1
    int* dir;              // longest axis
    double* mid;           // box centre along it
    int* nL;               // primitives below the centre (-1: median fallback)
    int* split;            // first position of the right child
};

__global__ void k_ct_dirs(CtLevel L, const double* __restrict__ C_box)
{
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= L.n) return;
    const double* box = C_box + 7 * static_cast<int64_t>(L.g[a]);
    int d = 0;
    double lmax = box[4];
    for (int k = 1; k < 3; ++k)
        if (box[4 + k] > lmax) {
            lmax = box[4 + k];
            d = k;
        }
    L.dir[a] = d;
    L.mid[a] = box[1 + d];
}

// (an order entry outside [0, N) would mean a broken permutation: counted in *error, the
// entry skipped)
__global__ void k_ct_flags(CtLevel L, int N, const int* __restrict__ ord, const double* __restrict__ cen, int* flag,
                           unsigned* error)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const int a = L.cl[i];
    const int j = ord[i];
    if (j < 0 || j >= N) {
        atomicAdd(error, 1u);
        flag[i] = 0;
        return;
    }
    flag[i] = (a >= 0 && cen[3 * static_cast<int64_t>(j) + L.dir[a]] < L.mid[a]) ? 1 : 0;
}

// split position of every cluster; clusters with all primitives on one side of the centre
// are appended to fb as (begin, end, axis) for the host's median fallback
__global__ void k_ct_split(CtLevel L, const int* __restrict__ excl, int4* fb, unsigned* n_fb)
{
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= L.n) return;
    const int b = L.b[a], e = L.e[a];
    const int nl = excl[e] - excl[b];
    const bool median = nl == 0 || nl == e - b;
    L.nL[a] = median ? -1 : nl;
    L.split[a] = median ? b + (e - b) / 2 : b + nl;
    if (median) {
        const unsigned k = atomicAdd(n_fb, 1u);
        fb[k] = make_int4(b, e, L.dir[a], a);
    }
}

// ipos[b + r] = position of the r-th primitive below the centre (partitioned clusters)
__global__ void k_ct_lower_positions(CtLevel L, int N, const int* __restrict__ flag, const int* __restrict__ excl,
                                     int* ipos)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const int a = L.cl[i];
    if (a < 0 || L.nL[a] < 0 || !flag[i]) return;
    const int b = L.b[a];
    ipos[b + excl[i] - excl[b]] = i;
}

// Destination of every position of a partitioned cluster; a chain longer than CT_CHAIN
// steps stores -2 - (where it stopped) and counts itself in *pending.
__global__ void k_ct_dest(CtLevel L, int N, const int* __restrict__ flag, const int* __restrict__ excl,
                          const int* __restrict__ ipos, int* dest, unsigned* pending)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const int a = L.cl[i];
    if (a < 0 || L.nL[a] < 0) return;
    const int b = L.b[a], lim = b + L.nL[a];
    if (flag[i]) { dest[i] = b + excl[i] - excl[b]; return; }
    int p = i;
    for (int step = 0; step < CT_CHAIN && p < lim; ++step) p = ipos[p];
    if (p < lim) {
        dest[i] = -2 - p;
        atomicAdd(pending, 1u);
    } else {
        dest[i] = p;
    }
}

// One round of pointer jumping on ipos inside each partitioned cluster's lower block
// (only when some chain was left pending). Updating in place is safe: every value read or
// written is a later element of the same chain, so a round advances at least as far as a
// synchronous one, and ceil(log2 n) rounds reach the end of every chain of length n.
__global__ void k_ct_jump(CtLevel L, int N, const unsigned* pending, int* ipos)
{
    if (*pending == 0) return;
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= N) return;
    const int a = L.cl[q];
    if (a < 0 || L.nL[a] < 0) return;
    const int lim = L.b[a] + L.nL[a];
    if (q >= lim) return;
    const int r = ipos[q];
    if (r < lim) ipos[q] = ipos[r];
}

// finishes the pending chains after the jumps; a chain that still does not end is an error
__global__ void k_ct_dest_finish(CtLevel L, int N, const unsigned* pending, const int* __restrict__ ipos, int* dest,
                                 unsigned* error)
{
    if (*pending == 0) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const int a = L.cl[i];
    if (a < 0 || L.nL[a] < 0 || dest[i] > -2) return;
    const int lim = L.b[a] + L.nL[a];
    int p = -2 - dest[i];
    for (int step = 0; step < CT_CHAIN && p < lim; ++step) p = ipos[p];
    if (p < lim) atomicAdd(error, 1u);
    else dest[i] = p;
}

__global__ void k_ct_scatter(CtLevel L, int N, const int* __restrict__ dest, const int* __restrict__ ord, int* ord_new,
                             unsigned* error)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const int a = L.cl[i];
    if (a < 0 || L.nL[a] < 0) {
        ord_new[i] = ord[i];
        return;
    }
    const int d = dest[i];
    if (d < L.b[a] || d >= L.e[a]) {   // an unfinished chain (already counted) or a broken one
        atomicAdd(error, 1u);
        return;
    }
    ord_new[d] = ord[i];
}

struct CtTree {
    int* C_begin; int* C_end; int* C_left; int* C_right; int* C_parent; int* C_depth; int* leaf_of;
};

// children of every cluster of the level: DFS numbers, ranges, links; the ones with more
// than one primitive are appended to the next level (g, b, e) and remember their index
__global__ void k_ct_children(CtLevel L, int depth, CtTree T, int* kids, int* ng, int* nb, int* ne, unsigned* n_next,
                              int* next_index)
{
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= L.n) return;
    const int g = L.g[a], b = L.b[a], e = L.e[a], s = L.split[a];
    const int c[2] = {g + 1, g + 2 * (s - b)};
    const int cb[2] = {b, s}, ce[2] = {s, e};
    T.C_left[g] = c[0];
    T.C_right[g] = c[1];
    for (int k = 0; k < 2; ++k) {
        T.C_begin[c[k]] = cb[k];
        T.C_end[c[k]] = ce[k];
        T.C_parent[c[k]] = g;
        T.C_depth[c[k]] = depth + 1;
        kids[2 * a + k] = c[k];
        if (ce[k] - cb[k] == 1) {
            T.leaf_of[cb[k]] = c[k];
        } else {
            const unsigned x = atomicAdd(n_next, 1u);
            ng[x] = c[k];
            nb[x] = cb[k];
            ne[x] = ce[k];
            next_index[c[k]] = static_cast<int>(x);
        }
    }
}

// cluster of every position in the next level
__global__ void k_ct_next_cl(CtLevel L, int N, const int* __restrict__ next_index, int* cl_next)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const int a = L.cl[i];
    int out = -1;
    if (a >= 0) {
        const int g = L.g[a], b = L.b[a], e = L.e[a], s = L.split[a];
        const bool left = i < s;
        if ((left ? s - b : e - s) > 1) out = next_index[left ? g + 1 : g + 2 * (s - b)];
    }
    cl_next[i] = out;
}

// serialized polytopes in tree order: [r2, centre, hull]
__global__ void k_ct_serialize(int size, int N, const double* __restrict__ V, const int* __restrict__ S,
                               const int* __restrict__ ord, const double* __restrict__ cen,
                               const double* __restrict__ rad2, double* P, unsigned* error)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const int ps = 1 + 3 + 3 * size;
    const int64_t j = ord[i];
    if (j < 0 || j >= N) {
        atomicAdd(error, 1u);
        return;
    }
    double* o = P + static_cast<int64_t>(ps) * i;
    o[0] = rad2[j];
    for (int k = 0; k < 3; ++k) o[1 + k] = cen[3 * j + k];
    for (int a = 0; a < size; ++a) {
        const int64_t v = S[size * j + a];
        for (int k = 0; k < 3; ++k) o[4 + 3 * a + k] = V[3 * v + k];
    }
}

}  // namespace

bool build_cluster_tree_device(int dom, const double* V, int nV, const int* S, int N, HostTree& T_out,
                               std::vector<double>& P_out, cudaStream_t s, std::string& err)
{
    if (dom != 1 && dom != 2) { err = "domain dimension must be 1 or 2"; return false; }
    if (nV <= 0 || N <= 0) { err = "empty mesh"; return false; }
    const int size = dom + 1;
    for (int64_t k = 0; k < static_cast<int64_t>(N) * size; ++k)
        if (S[k] < 0 || S[k] >= nV) { err = "simplex vertex index out of range"; return false; }
    for (int64_t k = 0; k < 3 * static_cast<int64_t>(nV); ++k)
        if (!std::isfinite(V[k])) { err = "non-finite vertex coordinate"; return false; }
    const int NC = 2 * N - 1;
    cudaError_t e = cudaSuccess;
    auto fail = [&](cudaError_t ce) {
        err = std::string("device cluster tree: ") + cudaGetErrorString(ce);
        return false;
    };
    DevBuf<double> d_V, cen, rad2, plo, phi, C_box;
    DevBuf<int> d_S, ord, ord_new, flag, excl, ipos, dest, cl, cl_next, kids, next_index;
    DevBuf<int> Cb, Ce, Cl, Cr, Cp, Cd, leaf;
    DevBuf<int> lg[2], lb[2], le[2], ldir, lnl, lsplit;
    DevBuf<double> lmid;
    DevBuf<int4> fb;
    DevBuf<unsigned> counters;   // 0 fallbacks, 1 next level, 2 pending chains, 3 errors
    DevBuf<unsigned char> temp;
    if ((e = d_V.alloc(3 * static_cast<size_t>(nV))) || (e = d_S.alloc(static_cast<size_t>(size) * N)) ||
        (e = cen.alloc(3 * static_cast<size_t>(N))) || (e = rad2.alloc(N)) || (e = plo.alloc(3 * static_cast<size_t>(N))) ||
        (e = phi.alloc(3 * static_cast<size_t>(N))) || (e = C_box.alloc(7 * static_cast<size_t>(NC))) ||
        (e = ord.alloc(N)) || (e = ord_new.alloc(N)) || (e = flag.alloc(N + 1)) || (e = excl.alloc(N + 1)) ||
        (e = ipos.alloc(N)) || (e = dest.alloc(N)) || (e = cl.alloc(N)) || (e = cl_next.alloc(N)) ||
        (e = kids.alloc(N)) || (e = next_index.alloc(NC)) || (e = Cb.alloc(NC)) || (e = Ce.alloc(NC)) ||
        (e = Cl.alloc(NC)) || (e = Cr.alloc(NC)) || (e = Cp.alloc(NC)) || (e = Cd.alloc(NC)) || (e = leaf.alloc(N)) ||
        (e = lg[0].alloc(N)) || (e = lg[1].alloc(N)) || (e = lb[0].alloc(N)) || (e = lb[1].alloc(N)) ||
        (e = le[0].alloc(N)) || (e = le[1].alloc(N)) || (e = ldir.alloc(N)) || (e = lnl.alloc(N)) ||
        (e = lsplit.alloc(N)) || (e = lmid.alloc(N)) || (e = fb.alloc(N)) || (e = counters.alloc(4)))
        return fail(e);
    size_t temp_bytes = 0;
    if ((e = cub::DeviceScan::ExclusiveSum(nullptr, temp_bytes, flag.ptr, excl.ptr, N + 1, s)) ||
        (e = temp.alloc(std::max<size_t>(temp_bytes, 16))))
        return fail(e);
    if ((e = cudaMemcpyAsync(d_V.ptr, V, d_V.bytes(), cudaMemcpyHostToDevice, s)) ||
        (e = cudaMemcpyAsync(d_S.ptr, S, d_S.bytes(), cudaMemcpyHostToDevice, s)) ||
        (e = cudaMemsetAsync(Cl.ptr, 0xff, Cl.bytes(), s)) || (e = cudaMemsetAsync(Cr.ptr, 0xff, Cr.bytes(), s)) ||
        (e = cudaMemsetAsync(Cp.ptr, 0xff, Cp.bytes(), s)) || (e = cudaMemsetAsync(Cd.ptr, 0, Cd.bytes(), s)) ||
        (e = cudaMemsetAsync(flag.ptr, 0, flag.bytes(), s)) || (e = cudaMemsetAsync(cl.ptr, 0, cl.bytes(), s)) ||
        (e = cudaMemsetAsync(counters.ptr, 0, counters.bytes(), s)))
        return fail(e);
    // identity order, the root [0, N) with DFS number 0
    {
        std::vector<int> iota(N);
        for (int i = 0; i < N; ++i) iota[i] = i;
        const int zero = 0;
        if ((e = cudaMemcpyAsync(ord.ptr, iota.data(), ord.bytes(), cudaMemcpyHostToDevice, s)) ||
            (e = cudaMemcpyAsync(Cb.ptr, &zero, sizeof(int), cudaMemcpyHostToDevice, s)) ||
            (e = cudaMemcpyAsync(Ce.ptr, &N, sizeof(int), cudaMemcpyHostToDevice, s)) ||
            (e = cudaMemcpyAsync(lg[0].ptr, &zero, sizeof(int), cudaMemcpyHostToDevice, s)) ||
            (e = cudaMemcpyAsync(lb[0].ptr, &zero, sizeof(int), cudaMemcpyHostToDevice, s)) ||
            (e = cudaMemcpyAsync(le[0].ptr, &N, sizeof(int), cudaMemcpyHostToDevice, s)) ||
            (e = cudaStreamSynchronize(s)))   // the host vector and constants leave scope
            return fail(e);
    }
    k_ct_prims<<<ct_grid(N), CT_BLOCK, 0, s>>>(size, N, d_V.ptr, d_S.ptr, cen.ptr, rad2.ptr, plo.ptr, phi.ptr);
    k_ct_boxes<<<1, 32, 0, s>>>(1, N, lg[0].ptr, Cb.ptr, Ce.ptr, ord.ptr, plo.ptr, phi.ptr, C_box.ptr,
                                counters.ptr + 3);
    if (N == 1) {
        if ((e = cudaMemsetAsync(leaf.ptr, 0, sizeof(int), s)) || (e = cudaMemsetAsync(cl.ptr, 0xff, cl.bytes(), s)))
            return fail(e);
    }
    if ((e = cudaGetLastError())) return fail(e);

    // centres on the host for the median fallback (the same rounding as the device's)
    std::vector<double> hcen(3 * static_cast<size_t>(N));
    {
        const double w = 1.0 / size;
        for (int j = 0; j < N; ++j)
            for (int k = 0; k < 3; ++k) {
                double acc = V[3 * static_cast<int64_t>(S[static_cast<int64_t>(size) * j]) + k];
                for (int a = 1; a < size; ++a) acc += V[3 * static_cast<int64_t>(S[static_cast<int64_t>(size) * j + a]) + k];
                hcen[3 * static_cast<size_t>(j) + k] = acc * w;
            }
    }
    std::vector<int> h_ord, lperm, linv;
    std::vector<double> score;
    std::vector<int4> h_fb;
    int cur = 0;
    int n_level = (N > 1) ? 1 : 0;
    int rounds = 1;
    while ((1ll << rounds) < N) ++rounds;
    ++rounds;
    for (int depth = 0; n_level > 0; ++depth) {
        if (depth > N) { err = "device cluster tree: level loop did not finish"; return false; }
        CtLevel L{n_level, lg[cur].ptr, lb[cur].ptr, le[cur].ptr, cl.ptr, ldir.ptr, lmid.ptr, lnl.ptr, lsplit.ptr};
        if ((e = cudaMemsetAsync(counters.ptr, 0, 3 * sizeof(unsigned), s))) return fail(e);
        k_ct_dirs<<<ct_grid(n_level), CT_BLOCK, 0, s>>>(L, C_box.ptr);
        k_ct_flags<<<ct_grid(N), CT_BLOCK, 0, s>>>(L, N, ord.ptr, cen.ptr, flag.ptr, counters.ptr + 3);
        if ((e = cub::DeviceScan::ExclusiveSum(temp.ptr, temp_bytes, flag.ptr, excl.ptr, N + 1, s))) return fail(e);
        k_ct_split<<<ct_grid(n_level), CT_BLOCK, 0, s>>>(L, excl.ptr, fb.ptr, counters.ptr);
        k_ct_lower_positions<<<ct_grid(N), CT_BLOCK, 0, s>>>(L, N, flag.ptr, excl.ptr, ipos.ptr);
        k_ct_dest<<<ct_grid(N), CT_BLOCK, 0, s>>>(L, N, flag.ptr, excl.ptr, ipos.ptr, dest.ptr, counters.ptr + 2);
        for (int r = 0; r < rounds; ++r) k_ct_jump<<<ct_grid(N), CT_BLOCK, 0, s>>>(L, N, counters.ptr + 2, ipos.ptr);
        k_ct_dest_finish<<<ct_grid(N), CT_BLOCK, 0, s>>>(L, N, counters.ptr + 2, ipos.ptr, dest.ptr, counters.ptr + 3);
        k_ct_scatter<<<ct_grid(N), CT_BLOCK, 0, s>>>(L, N, dest.ptr, ord.ptr, ord_new.ptr, counters.ptr + 3);
        CtTree CT{Cb.ptr, Ce.ptr, Cl.ptr, Cr.ptr, Cp.ptr, Cd.ptr, leaf.ptr};
        const int nxt = 1 - cur;
        k_ct_children<<<ct_grid(n_level), CT_BLOCK, 0, s>>>(L, depth, CT, kids.ptr, lg[nxt].ptr, lb[nxt].ptr,
                                                            le[nxt].ptr, counters.ptr + 1, next_index.ptr);
        k_ct_next_cl<<<ct_grid(N), CT_BLOCK, 0, s>>>(L, N, next_index.ptr, cl_next.ptr);
        if ((e = cudaGetLastError())) return fail(e);
        unsigned cnt[4];
        if ((e = cudaMemcpyAsync(cnt, counters.ptr, sizeof(cnt), cudaMemcpyDeviceToHost, s)) ||
            (e = cudaStreamSynchronize(s)))
            return fail(e);
        if (cnt[3] != 0) { err = "device cluster tree: a partition chain did not end or the order broke"; return false; }
        if (cnt[0] > 0) {
            // median fallback on the host (AABB_LongestAxisSplit.hpp:205-247): nth_element of
            // the centres along the axis, then the cluster's range reordered by it
            h_fb.resize(cnt[0]);
            h_ord.resize(N);
            if ((e = cudaMemcpyAsync(h_fb.data(), fb.ptr, sizeof(int4) * cnt[0], cudaMemcpyDeviceToHost, s)) ||
                (e = cudaMemcpyAsync(h_ord.data(), ord_new.ptr, ord_new.bytes(), cudaMemcpyDeviceToHost, s)) ||
                (e = cudaStreamSynchronize(s)))
                return fail(e);
            if (lperm.size() < static_cast<size_t>(N)) {
                lperm.resize(N);
                linv.resize(N);
                score.resize(N);
            }
            for (const int4& f : h_fb) {
                const int b = f.x, en = f.y, dir = f.z, mid = b + (en - b) / 2;
                if (b < 0 || en > N || b >= en || dir < 0 || dir > 2) { err = "device cluster tree: bad fallback range"; return false; }
                for (int i = b; i < en; ++i)
                    if (h_ord[i] < 0 || h_ord[i] >= N) { err = "device cluster tree: broken order"; return false; }
                for (int i = b; i < en; ++i) {
                    score[i] = hcen[3 * static_cast<size_t>(h_ord[i]) + dir];
                    lperm[i] = i;
                }
                const double* sc = score.data();
                std::nth_element(lperm.begin() + b, lperm.begin() + mid, lperm.begin() + en,
                                 [sc](int x, int y) { return sc[x] < sc[y]; });
                // position i receives the primitive at position lperm[i]
                for (int i = b; i < en; ++i) linv[i] = h_ord[lperm[i]];
                for (int i = b; i < en; ++i) h_ord[i] = linv[i];
            }
            if ((e = cudaMemcpyAsync(ord_new.ptr, h_ord.data(), ord_new.bytes(), cudaMemcpyHostToDevice, s)))
                return fail(e);
        }
        std::swap(ord.ptr, ord_new.ptr);
        std::swap(cl.ptr, cl_next.ptr);
        k_ct_boxes<<<ct_grid(32ll * 2 * n_level), CT_BLOCK, 0, s>>>(2 * n_level, N, kids.ptr, Cb.ptr, Ce.ptr, ord.ptr,
                                                                   plo.ptr, phi.ptr, C_box.ptr, counters.ptr + 3);
        if ((e = cudaGetLastError())) return fail(e);
        n_level = static_cast<int>(cnt[1]);
        cur = nxt;
    }
    HostTree T;
    T.dom = dom;
    T.size = size;
    T.nV = nV;
    T.N = N;
    T.NC = NC;
    T.perm.resize(N);
    T.leaf_of.resize(N);
    T.C_begin.resize(NC); T.C_end.resize(NC); T.C_left.resize(NC); T.C_right.resize(NC);
    T.C_parent.resize(NC); T.C_depth.resize(NC);
    T.C_box.resize(7 * static_cast<size_t>(NC));
    const int ps = 1 + 3 + 3 * size;
    DevBuf<double> d_P;
    if ((e = d_P.alloc(static_cast<size_t>(ps) * N))) return fail(e);
    k_ct_serialize<<<ct_grid(N), CT_BLOCK, 0, s>>>(size, N, d_V.ptr, d_S.ptr, ord.ptr, cen.ptr, rad2.ptr, d_P.ptr,
                                                   counters.ptr + 3);
    P_out.resize(static_cast<size_t>(ps) * N);
    unsigned final_error = 0;
    if ((e = cudaGetLastError()) ||
        (e = cudaMemcpyAsync(T.perm.data(), ord.ptr, ord.bytes(), cudaMemcpyDeviceToHost, s)) ||
        (e = cudaMemcpyAsync(T.leaf_of.data(), leaf.ptr, leaf.bytes(), cudaMemcpyDeviceToHost, s)) ||
        (e = cudaMemcpyAsync(T.C_begin.data(), Cb.ptr, Cb.bytes(), cudaMemcpyDeviceToHost, s)) ||
        (e = cudaMemcpyAsync(T.C_end.data(), Ce.ptr, Ce.bytes(), cudaMemcpyDeviceToHost, s)) ||
        (e = cudaMemcpyAsync(T.C_left.data(), Cl.ptr, Cl.bytes(), cudaMemcpyDeviceToHost, s)) ||
        (e = cudaMemcpyAsync(T.C_right.data(), Cr.ptr, Cr.bytes(), cudaMemcpyDeviceToHost, s)) ||
        (e = cudaMemcpyAsync(T.C_parent.data(), Cp.ptr, Cp.bytes(), cudaMemcpyDeviceToHost, s)) ||
        (e = cudaMemcpyAsync(T.C_depth.data(), Cd.ptr, Cd.bytes(), cudaMemcpyDeviceToHost, s)) ||
        (e = cudaMemcpyAsync(T.C_box.data(), C_box.ptr, C_box.bytes(), cudaMemcpyDeviceToHost, s)) ||
        (e = cudaMemcpyAsync(P_out.data(), d_P.ptr, d_P.bytes(), cudaMemcpyDeviceToHost, s)) ||
        (e = cudaMemcpyAsync(&final_error, counters.ptr + 3, sizeof(unsigned), cudaMemcpyDeviceToHost, s)) ||
        (e = cudaStreamSynchronize(s)))
        return fail(e);
    if (final_error != 0) { err = "device cluster tree: the final order is not a permutation"; return false; }
    {
        // every primitive exactly once (a broken order falls back to the host build)
        std::vector<char> seen(N, 0);
        for (int i = 0; i < N; ++i) {
            const int j = T.perm[i];
            if (j < 0 || j >= N || seen[j]) { err = "device cluster tree: the final order is not a permutation"; return false; }
            seen[j] = 1;
        }
    }
    T.depth = 0;
    for (int C = 0; C < NC; ++C) T.depth = std::max(T.depth, T.C_depth[C]);
    T.inv_perm.assign(N, 0);
    for (int i = 0; i < N; ++i) T.inv_perm[T.perm[i]] = i;
    T_out = std::move(T);
    return true;
}

}  // namespace rpb
