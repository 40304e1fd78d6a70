// Device-side data layouts and helpers shared by the B200 kernels.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace rpb {

constexpr int WARP = 32;

// Programmatic dependent launch (sm_90+). A kernel launched with launch_pdl may start while
// its predecessor in the stream still runs: it reads only data that no kernel writes
// (patterns, offsets, plans) before pdl_wait(), which returns once the predecessor has
// completed and its writes are visible; pdl_launch_dependents() then lets the next
// kernel of the stream start its own prologue. Without the launch attribute both are
// no-ops.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_launch_dependents() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

template <typename... KArgs, typename... Args>
inline cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t stream,
                              Args... args)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
}

// Pair data of a primitive: barycentre and unit normal (triangles) or unit tangent
// (edges), weight a (all FP64) and diameter. The normal projector is P = n n^T
// (triangles) or I - t t^T (edges); keeping n/t in FP64 lets v^T P v be formed
// without the FP32 rounding of P, whose error relative to v^T P v grows like
// eps / (kappa r)^2 for nearby pairs on smooth surfaces. 64 bytes.
struct __align__(16) PrimDatum {
    double c[3];
    double n[3];
    double a;
    float diam;
    float pad;
};
static_assert(sizeof(PrimDatum) == 64, "PrimDatum must be 64 bytes");

// Pair data of a cluster: centre of mass (FP64), averaged projector (packed upper
// triangle (0,0),(0,1),(0,2),(1,1),(1,2),(2,2)) in FP32 — far pairs project in FP32 —,
// and the weight. 64 bytes: four 16-byte loads per gather.
struct __align__(16) ClusterDatum {
    double c[3];
    float P[6];
    double a;
    float pad[2];
};
static_assert(sizeof(ClusterDatum) == 64, "ClusterDatum must be 64 bytes");

// Tangent-point exponents of one evaluation. q = numerator, p = denominator.
struct TPExp {
    double q, p;
    double s_exp_metric;   // -(2(s-1)+n)/2, s = (p-n)/q  (TP0_Kernel_FF.hpp:72-73)
    int qh, ph;            // q/2, p/2 when integral, else -1
};

template <typename T>
__device__ __forceinline__ T load_datum(const T* __restrict__ base, int i)
{
    static_assert(sizeof(T) % 16 == 0, "datum size");
    constexpr int Q = sizeof(T) / 16;
    const float4* p = reinterpret_cast<const float4*>(base + i);
    T d;
    float4* o = reinterpret_cast<float4*>(&d);
#pragma unroll
    for (int k = 0; k < Q; ++k) o[k] = __ldg(p + k);
    return d;
}

template <typename T>
__device__ __forceinline__ void store_datum(T* base, int i, const T& d)
{
    constexpr int Q = sizeof(T) / 16;
    float4* dst = reinterpret_cast<float4*>(base + i);
    const float4* src = reinterpret_cast<const float4*>(&d);
#pragma unroll
    for (int k = 0; k < Q; ++k) __stcg(dst + k, src[k]);
}

// Error-free transformation of a sum (Knuth's TwoSum).
__device__ __forceinline__ void two_sum(float a, float b, float& s, float& e)
{
    s = a + b;
    const float bp = s - a;
    e = (a - (s - bp)) + (b - bp);
}

// Compensated warp butterfly: returns the row sum (hi + lo) of `x` in every lane.
__device__ __forceinline__ double warp_sum_compensated(float x)
{
    float hi = x, lo = 0.0f;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        const float oh = __shfl_xor_sync(0xffffffffu, hi, off);
        const float ol = __shfl_xor_sync(0xffffffffu, lo, off);
        float s, e;
        two_sum(hi, oh, s, e);
        hi = s;
        lo = lo + ol + e;
    }
    return static_cast<double>(hi) + static_cast<double>(lo);
}

__device__ __forceinline__ double warp_sum_f64(double x)
{
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) x += __shfl_xor_sync(0xffffffffu, x, off);
    return x;
}

template <typename T>
__device__ __forceinline__ T ipow_pos(T x, int k)
{
    T r = T(1);
    while (k > 0) {
        if (k & 1) r *= x;
        x *= x;
        k >>= 1;
    }
    return r;
}

__device__ __forceinline__ float  dev_pow(float x, float y) { return exp2f(y * __log2f(x)); }
__device__ __forceinline__ double dev_pow(double x, double y) { return pow(x, y); }
__device__ __forceinline__ float  dev_rcp(float x) { return __fdividef(1.0f, x); }   // MUFU reciprocal, ~2 ulp
__device__ __forceinline__ double dev_rcp(double x) { return 1.0 / x; }

}  // namespace rpb
