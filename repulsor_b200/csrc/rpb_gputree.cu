// Block cluster tree on the B200: the dual traversal of the cluster tree that classifies
// every block pair as far field (admissible cluster pair), near field, very near or
// intersecting (src/ClusterTreePairTraversor/Traverse_DepthFirst.hpp:52-258 with
// src/BlockClusterTree/BlockSplit_Kernel.hpp:164-251), and the full symmetric CSR patterns
// (src/BlockClusterTree.hpp:306-326). The cluster tree itself (the longest-axis splits
// with their in-place swaps) stays on the host.
//
// The traversal runs breadth first: one launch per level of block pairs, one thread per
// pair, children and results appended through atomic counters. The decisions come from
// host/bct_rules.hpp, the same code the host builder runs, and this file is compiled
// without fused multiply-adds, so the pair sets equal the host builder's bit for bit
// (the order of discovery differs; the CSR rows are sorted). Rows and columns are then
// sorted on the device (CUB radix sort of 64-bit (row, column) keys).
#include <cub/cub.cuh>

#include <algorithm>
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

}  // namespace rpb
