// Exact squared distances between segments / triangles (FP64), used by the
// very-near quadrature's separation test (the GJK multipole acceptance criterion
// of src/GJK.hpp:1162-1172 for polytopes).
#pragma once

#include <cuda_runtime.h>

namespace rpb {

__host__ __device__ inline double gdot(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

__host__ __device__ inline double gclamp01(double x) { return x < 0.0 ? 0.0 : (x > 1.0 ? 1.0 : x); }

__host__ __device__ inline double seg_seg_d2(const double* a0, const double* a1, const double* b0, const double* b1)
{
    double u[3], v[3], w[3];
    for (int k = 0; k < 3; ++k) { u[k] = a1[k] - a0[k]; v[k] = b1[k] - b0[k]; w[k] = a0[k] - b0[k]; }
    const double A = gdot(u, u), B = gdot(u, v), C = gdot(v, v), D = gdot(u, w), E = gdot(v, w);
    double best = 1.0e300;
    auto ev = [&](double s, double t) {
        double d2 = 0;
        for (int k = 0; k < 3; ++k) { const double d = w[k] + s * u[k] - t * v[k]; d2 += d * d; }
        return d2;
    };
    const double den = A * C - B * B;
    if (den > 0) {
        const double s = (B * E - C * D) / den, t = (A * E - B * D) / den;
        if (s >= 0 && s <= 1 && t >= 0 && t <= 1) best = ev(s, t);
    }
    for (int e = 0; e < 2; ++e) {
        const double s = e;
        const double t = C > 0 ? gclamp01((B * s + E) / C) : 0.0;
        const double d1 = ev(s, t);
        best = d1 < best ? d1 : best;
        const double t2 = e;
        const double s2 = A > 0 ? gclamp01((B * t2 - D) / A) : 0.0;
        const double d2 = ev(s2, t2);
        best = d2 < best ? d2 : best;
    }
    return best;
}

__host__ __device__ inline double point_tri_d2(const double* p, const double* a, const double* b, const double* c)
{
    double e0[3], e1[3], d[3];
    for (int k = 0; k < 3; ++k) { e0[k] = b[k] - a[k]; e1[k] = c[k] - a[k]; d[k] = p[k] - a[k]; }
    const double a00 = gdot(e0, e0), a01 = gdot(e0, e1), a11 = gdot(e1, e1);
    const double b0 = gdot(e0, d), b1 = gdot(e1, d);
    const double det = a00 * a11 - a01 * a01;
    if (det > 0) {
        const double s = (a11 * b0 - a01 * b1) / det, t = (a00 * b1 - a01 * b0) / det;
        if (s >= 0 && t >= 0 && s + t <= 1) {
            double d2 = 0;
            for (int k = 0; k < 3; ++k) { const double x = d[k] - s * e0[k] - t * e1[k]; d2 += x * x; }
            return d2;
        }
    }
    double best = seg_seg_d2(p, p, a, b);
    double t2 = seg_seg_d2(p, p, b, c);
    best = t2 < best ? t2 : best;
    t2 = seg_seg_d2(p, p, c, a);
    return t2 < best ? t2 : best;
}

__host__ __device__ inline bool seg_tri_hit(const double* p, const double* q, const double* a, const double* b,
                                            const double* c)
{
    double e0[3], e1[3], dir[3], n[3];
    for (int k = 0; k < 3; ++k) { e0[k] = b[k] - a[k]; e1[k] = c[k] - a[k]; dir[k] = q[k] - p[k]; }
    n[0] = e0[1] * e1[2] - e0[2] * e1[1];
    n[1] = e0[2] * e1[0] - e0[0] * e1[2];
    n[2] = e0[0] * e1[1] - e0[1] * e1[0];
    const double den = gdot(n, dir);
    if (den == 0) return false;
    double ap[3];
    for (int k = 0; k < 3; ++k) ap[k] = a[k] - p[k];
    const double t = gdot(n, ap) / den;
    if (t < 0 || t > 1) return false;
    double x[3];
    for (int k = 0; k < 3; ++k) x[k] = p[k] + t * dir[k] - a[k];
    const double a00 = gdot(e0, e0), a01 = gdot(e0, e1), a11 = gdot(e1, e1);
    const double b0 = gdot(e0, x), b1 = gdot(e1, x);
    const double det = a00 * a11 - a01 * a01;
    if (det <= 0) return false;
    const double s = (a11 * b0 - a01 * b1) / det, u = (a00 * b1 - a01 * b0) / det;
    return s >= 0 && u >= 0 && s + u <= 1;
}

__host__ __device__ inline double tri_tri_d2(const double* A, const double* B)
{
    for (int e = 0; e < 3; ++e) {
        const int f = (e + 1) % 3;
        if (seg_tri_hit(A + 3 * e, A + 3 * f, B, B + 3, B + 6)) return 0.0;
        if (seg_tri_hit(B + 3 * e, B + 3 * f, A, A + 3, A + 6)) return 0.0;
    }
    double best = 1.0e300;
    for (int v = 0; v < 3; ++v) {
        double t = point_tri_d2(A + 3 * v, B, B + 3, B + 6);
        best = t < best ? t : best;
        t = point_tri_d2(B + 3 * v, A, A + 3, A + 6);
        best = t < best ? t : best;
    }
    for (int e = 0; e < 3; ++e)
        for (int f = 0; f < 3; ++f) {
            const double t = seg_seg_d2(A + 3 * e, A + 3 * ((e + 1) % 3), B + 3 * f, B + 3 * ((f + 1) % 3));
            best = t < best ? t : best;
        }
    return best;
}

}  // namespace rpb
