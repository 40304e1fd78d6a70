// Block cluster tree decisions shared by the host builder (tree_builder.cpp) and the GPU
// traversal (rpb_gputree.cu, compiled without fused multiply-adds), so that both classify
// every block pair identically (bit-identical pair lists):
//  * exact squared distances of segments and triangles (the reference's GJK distance on
//    polytopes, src/GJK.hpp:1162-1183, restated in closed form)
//  * the far-field MAC on cluster boxes (src/BlockClusterTree/BlockSplit_Kernel.hpp:164-251):
//    max(r_i^2, r_j^2) < theta_far^2 * dist(box_i, box_j)^2
//  * the leaf classification into near / very near / intersecting
//    (src/BlockClusterTree/BlockSplit_Kernel.hpp:181-251, AdaptivitySettings::theta)
#pragma once

#include <cmath>

#ifdef __CUDACC__
#define RPB_HD __host__ __device__ inline
#else
#define RPB_HD inline
#endif

namespace rpb {
namespace bct {

constexpr double kMaxDouble = 1.7976931348623157e308;
constexpr double kEpsDouble = 2.220446049250313e-16;

RPB_HD double dmin(double a, double b) { return b < a ? b : a; }             // std::min
RPB_HD double dmax(double a, double b) { return a < b ? b : a; }             // std::max
RPB_HD double clamp01(double x) { return x < 0.0 ? 0.0 : (1.0 < x ? 1.0 : x); }  // std::clamp(x, 0, 1)
RPB_HD double dot3(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

RPB_HD double segseg2(const double* a0, const double* a1, const double* b0, const double* b1)
{
    double u[3], v[3], w[3];
    for (int k = 0; k < 3; ++k) { u[k] = a1[k] - a0[k]; v[k] = b1[k] - b0[k]; w[k] = a0[k] - b0[k]; }
    const double A = dot3(u, u), B = dot3(u, v), C = dot3(v, v), D = dot3(u, w), E = dot3(v, w);
    auto eval = [&](double s, double t) {
        double d2 = 0;
        for (int k = 0; k < 3; ++k) { const double d = w[k] + s * u[k] - t * v[k]; d2 += d * d; }
        return d2;
    };
    double best = kMaxDouble;
    // interior critical point
    const double den = A * C - B * B;
    if (den > 0) {
        const double s = (B * E - C * D) / den, t = (A * E - B * D) / den;
        if (s >= 0 && s <= 1 && t >= 0 && t <= 1) best = eval(s, t);
    }
    // boundary: s in {0,1} with optimal t, t in {0,1} with optimal s
    for (int e = 0; e < 2; ++e) {
        const double s = e;
        const double t = C > 0 ? clamp01((B * s + E) / C) : 0.0;
        best = dmin(best, eval(s, t));
        const double t2 = e;
        const double s2 = A > 0 ? clamp01((B * t2 - D) / A) : 0.0;
        best = dmin(best, eval(s2, t2));
    }
    return best;
}

RPB_HD double pointtri2(const double* p, const double* a, const double* b, const double* c)
{
    // projection onto the plane; inside test by barycentric coordinates, else edges
    double e0[3], e1[3], d[3];
    for (int k = 0; k < 3; ++k) { e0[k] = b[k] - a[k]; e1[k] = c[k] - a[k]; d[k] = p[k] - a[k]; }
    const double a00 = dot3(e0, e0), a01 = dot3(e0, e1), a11 = dot3(e1, e1);
    const double b0 = dot3(e0, d), b1 = dot3(e1, d);
    const double det = a00 * a11 - a01 * a01;
    if (det > 0) {
        const double s = (a11 * b0 - a01 * b1) / det, t = (a00 * b1 - a01 * b0) / det;
        if (s >= 0 && t >= 0 && s + t <= 1) {
            double d2 = 0;
            for (int k = 0; k < 3; ++k) { const double x = d[k] - s * e0[k] - t * e1[k]; d2 += x * x; }
            return d2;
        }
    }
    return dmin(dmin(segseg2(p, p, a, b), segseg2(p, p, b, c)), segseg2(p, p, c, a));
}

RPB_HD bool segtri_hit(const double* p, const double* q, const double* a, const double* b, const double* c)
{
    double e0[3], e1[3], dir[3], n[3];
    for (int k = 0; k < 3; ++k) { e0[k] = b[k] - a[k]; e1[k] = c[k] - a[k]; dir[k] = q[k] - p[k]; }
    n[0] = e0[1] * e1[2] - e0[2] * e1[1];
    n[1] = e0[2] * e1[0] - e0[0] * e1[2];
    n[2] = e0[0] * e1[1] - e0[1] * e1[0];
    const double den = dot3(n, dir);
    if (den == 0) return false;
    double ap[3];
    for (int k = 0; k < 3; ++k) ap[k] = a[k] - p[k];
    const double t = dot3(n, ap) / den;
    if (t < 0 || t > 1) return false;
    double x[3];
    for (int k = 0; k < 3; ++k) x[k] = p[k] + t * dir[k] - a[k];
    const double a00 = dot3(e0, e0), a01 = dot3(e0, e1), a11 = dot3(e1, e1);
    const double b0 = dot3(e0, x), b1 = dot3(e1, x);
    const double det = a00 * a11 - a01 * a01;
    if (det <= 0) return false;
    const double s = (a11 * b0 - a01 * b1) / det, u = (a00 * b1 - a01 * b0) / det;
    return s >= 0 && u >= 0 && s + u <= 1;
}

RPB_HD double tritri2(const double* A, const double* B)
{
    for (int e = 0; e < 3; ++e) {
        const int f = (e + 1) % 3;
        if (segtri_hit(A + 3 * e, A + 3 * f, B, B + 3, B + 6)) return 0.0;
        if (segtri_hit(B + 3 * e, B + 3 * f, A, A + 3, A + 6)) return 0.0;
    }
    double best = kMaxDouble;
    for (int v = 0; v < 3; ++v) {
        best = dmin(best, pointtri2(A + 3 * v, B, B + 3, B + 6));
        best = dmin(best, pointtri2(B + 3 * v, A, A + 3, A + 6));
    }
    for (int e = 0; e < 3; ++e)
        for (int f = 0; f < 3; ++f)
            best = dmin(best, segseg2(A + 3 * e, A + 3 * ((e + 1) % 3), B + 3 * f, B + 3 * ((f + 1) % 3)));
    return best;
}

// Far-field MAC of two cluster boxes [r2, centre(3), half(3)].
RPB_HD bool boxes_admissible(const double* a, const double* b, double far_t2)
{
    double d2 = 0;
    for (int k = 0; k < 3; ++k) {
        const double lo = dmax(a[1 + k] - a[4 + k], b[1 + k] - b[4 + k]);
        const double hi = dmin(a[1 + k] + a[4 + k], b[1 + k] + b[4 + k]);
        const double x = dmax(0.0, lo - hi);
        d2 += x * x;
    }
    return dmax(a[0], b[0]) < far_t2 * d2;
}

// Leaf pair of serialized polytopes [r2, centre(3), hull] that share no vertex:
// 0 near field, 1 very near (subdivided quadrature), 2 intersecting.
RPB_HD int classify_leaf(int dom, const double* A, const double* B, double near_t2)
{
    const double tol = dmax(A[0], B[0]);
    // cheap separation certificate from the bounding balls
    double cc = 0;
    for (int k = 0; k < 3; ++k) { const double d = A[1 + k] - B[1 + k]; cc += d * d; }
    using std::sqrt;
    const double lb = sqrt(cc) - sqrt(A[0]) - sqrt(B[0]);
    if (lb > 0 && near_t2 * lb * lb > tol) return 0;
    const double d2 = (dom == 1) ? segseg2(A + 4, A + 7, B + 4, B + 7) : tritri2(A + 4, B + 4);
    if (near_t2 * d2 > tol) return 0;
    const double tol_i = kEpsDouble * dmin(A[0], B[0]);
    return (near_t2 * d2 <= tol_i) ? 2 : 1;
}

}  // namespace bct
}  // namespace rpb
