// Host stand-in for <cuda_runtime.h>, used ONLY to compile the reference's
// own Kernels/*.cu bodies with g++ so they can run on the CPU as a checker
// (oracle/_ref) and as the timed CPU baseline. Test infrastructure, never
// part of the shipped library.
//
// Two builds:
//   default            : float arithmetic (the reference's own precision)
//   -DISA_REF_FP64     : every `float` token in the kernels becomes `double`
//                        and the f-suffixed math calls map to their double
//                        versions, giving an FP64 run of the same kernel text.
//
// Texture fetches follow the documented CUDA rules (CUDA C Programming Guide,
// "Texture Fetching"): normalized coordinates are scaled by the extent,
// linear filtering samples at xB = x*N - 0.5 with i = floor(xB) and
// alpha = frac(xB) (exact here; hardware keeps 8 fractional bits), clamp
// addressing clamps the texel index, mirror addressing reflects it with the
// edge texel repeated (period 2N).
#pragma once
#include <cmath>
#include <cfloat>
#include <cstdio>
#include <cstdint>
#include <cstddef>

using std::isnan;
using std::isfinite;

#ifdef ISA_REF_FP64
#define float double
#define sinf sin
#define cosf cos
#define expf exp
#define sqrtf sqrt
#define powf pow
#define roundf round
#define fminf fmin
#define fmaxf fmax
#define fabsf fabs
#define floorf floor
#define ceilf ceil
#define atan2f atan2
#endif

struct float2 { float x, y; };
struct float3 { float x, y, z; };
struct float4 { float x, y, z, w; };
struct int2 { int x, y; };

static inline float2 make_float2(float x, float y) { float2 r; r.x = x; r.y = y; return r; }
static inline float3 make_float3(float x, float y, float z) { float3 r; r.x = x; r.y = y; r.z = z; return r; }
static inline float4 make_float4(float x, float y, float z, float w) { float4 r; r.x = x; r.y = y; r.z = z; r.w = w; return r; }

static inline int min(int a, int b) { return a < b ? a : b; }
static inline int max(int a, int b) { return a > b ? a : b; }

#define __global__
#define __device__
#define __host__
#define __constant__
#define __forceinline__ inline
#define __shared__ thread_local
static inline void __syncthreads() {}

typedef unsigned long long cudaTextureObject_t;

// Host-side texture description that a cudaTextureObject_t points to.
enum isa_ref_addr { ISA_REF_CLAMP = 0, ISA_REF_MIRROR = 1 };
enum isa_ref_filter { ISA_REF_POINT = 0, ISA_REF_LINEAR = 1 };
struct isa_ref_tex {
    const void* data;   // base of a pitched image of `float` (real) elements
    int width, height;  // in texels
    size_t pitch;       // bytes per row
    int channels;       // 1, 2 or 4
    int addr;           // isa_ref_addr
    int filter;         // isa_ref_filter
};

static inline int isa_ref_wrap(int i, int n, int addr) {
    if (addr == ISA_REF_CLAMP) return i < 0 ? 0 : (i >= n ? n - 1 : i);
    int p = 2 * n;
    int j = i % p;
    if (j < 0) j += p;
    return j >= n ? p - 1 - j : j;
}

static inline const float* isa_ref_texel(const isa_ref_tex* t, int i, int j) {
    i = isa_ref_wrap(i, t->width, t->addr);
    j = isa_ref_wrap(j, t->height, t->addr);
    return (const float*)((const char*)t->data + (size_t)j * t->pitch) + (size_t)i * t->channels;
}

static inline void isa_ref_fetch(const isa_ref_tex* t, float u, float v, float* out) {
    float x = u * t->width;
    float y = v * t->height;
    if (t->filter == ISA_REF_POINT) {
        const float* p = isa_ref_texel(t, (int)std::floor(x), (int)std::floor(y));
        for (int c = 0; c < t->channels; c++) out[c] = p[c];
        return;
    }
    float xb = x - 0.5f, yb = y - 0.5f;
    float fx = std::floor(xb), fy = std::floor(yb);
    int i = (int)fx, j = (int)fy;
    float a = xb - fx, b = yb - fy;
    const float* p00 = isa_ref_texel(t, i, j);
    const float* p10 = isa_ref_texel(t, i + 1, j);
    const float* p01 = isa_ref_texel(t, i, j + 1);
    const float* p11 = isa_ref_texel(t, i + 1, j + 1);
    // texels with zero weight are skipped (a non-finite neighbour does not leak)
    for (int c = 0; c < t->channels; c++) {
        float v = 0;
        if (a != 1 && b != 1) v += (1 - a) * (1 - b) * p00[c];
        if (a != 0 && b != 1) v += a * (1 - b) * p10[c];
        if (a != 1 && b != 0) v += (1 - a) * b * p01[c];
        if (a != 0 && b != 0) v += a * b * p11[c];
        out[c] = v;
    }
}

template <class T> static inline T tex2D(cudaTextureObject_t obj, float u, float v);
template <> inline float tex2D<float>(cudaTextureObject_t obj, float u, float v) {
    float r[4]; isa_ref_fetch((const isa_ref_tex*)obj, u, v, r); return r[0];
}
template <> inline float2 tex2D<float2>(cudaTextureObject_t obj, float u, float v) {
    float r[4]; isa_ref_fetch((const isa_ref_tex*)obj, u, v, r); return make_float2(r[0], r[1]);
}
template <> inline float4 tex2D<float4>(cudaTextureObject_t obj, float u, float v) {
    float r[4]; isa_ref_fetch((const isa_ref_tex*)obj, u, v, r); return make_float4(r[0], r[1], r[2], r[3]);
}
