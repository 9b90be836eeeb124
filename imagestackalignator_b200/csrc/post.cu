// Colour and tone post-processing of the merged image in one pass: the NPP
// chain of the controller's SaveAs16BitTiff (ImageStackAlignatorController.cs
// :2197-2260) and ProcessColorsAndShow (:2262-2320), which in the reference
// is eight full-image passes (two ThresholdLTGT, two ColorTwist, LUTCubic,
// two MulC, GammasRGB) plus the conversion.
//
// Per pixel, in FP32 with every operation rounded on its own (no fused
// multiply-add, so that an FP32 restatement on the host reproduces it):
//   v = ThresholdLTGT(v, 0 -> 0, CameraWhite -> CameraWhite)
//   v = twist1 * v                         (ColorTwist: m0 r + m1 g + m2 b + m3)
//   v = ThresholdLTGT(v, 0 -> 0, 1 -> 1)
//   v = LUT(v) per channel                 (cubic through the 4 nearest levels, Horner in v - x[k])
//   v = twist2 * v
//   v = v * 2^Exposure
//   v = GammasRGB(v)                       (NaN -> 0, clamp [0, 1], sRGB curve; kernel.cu:290-332)
//   out = Convert(v * 65535 | 255, round to nearest even, saturate)
// The ROI (the raw file's crop) is applied by reading only the crop.
#include "isa_internal.cuh"

namespace {

__device__ __forceinline__ float thr_ltgt(float v, float hi)
{
    // nppiThreshold_LTValGTVal: below 0 -> 0, above hi -> hi, otherwise (and NaN) unchanged
    return v < 0.f ? 0.f : (v > hi ? hi : v);
}

__device__ __forceinline__ float twist_row(const float* m, float r, float g, float b)
{
    return __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(m[0], r), __fmul_rn(m[1], g)), __fmul_rn(m[2], b)), m[3]);
}

// applysRGBGamma (kernel.cu:290-301) after GammasRGB's NaN and clamp steps (:317-327)
__device__ __forceinline__ float gamma_srgb(float v)
{
    if (isnan(v)) v = 0.f;
    v = fmaxf(fminf(v, 1.0f), 0.0f);
    return v <= 0.0031308f ? 12.92f * v : (1.0f + 0.055f) * powf(v, 1.0f / 2.4f) - 0.055f;
}

struct LutView {
    const float* x;
    const float4* c;
    int n, uniform;
};

// Largest k in [0, n - 2] with x[k] <= v (0 below the first level or for NaN).
__device__ __forceinline__ int lut_segment(const LutView& L, float v)
{
    int k;
    if (L.uniform) {
        // levels within half a step of i / (n - 1): a guess from the value, then exact steps against the stored levels
        k = (int)__fmul_rz(v, (float)(L.n - 1));
        k = min(max(k, 0), L.n - 2);
        while (k > 0 && v < L.x[k]) k--;
        while (k < L.n - 2 && v >= L.x[k + 1]) k++;
    } else {
        int lo = 0, hi = L.n - 2;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (v >= L.x[mid]) lo = mid;
            else hi = mid - 1;
        }
        k = lo;
    }
    return k;
}

// The cubic through the four nearest levels, as per-segment coefficients in
// t = v - x[k] (computed on the host in FP64), evaluated by Horner's rule.
__device__ __forceinline__ float lut_cubic(const LutView& L, float v)
{
    const int k = lut_segment(L, v);
    const float4 c = L.c[k];
    const float t = __fsub_rn(v, L.x[k]);
    return __fadd_rn(__fmul_rn(__fadd_rn(__fmul_rn(__fadd_rn(__fmul_rn(c.w, t), c.z), t), c.y), t), c.x);
}

constexpr int PP_NT = 256, PP_PX = 4;  // threads per CTA, consecutive pixels per thread

// A persistent grid: each CTA copies the LUT into shared memory once (the
// kernel-parameter copy is read with per-thread addresses, which the
// constant cache serialises) and then walks rows y = blockIdx.x, + gridDim.x, ...
template <int FMT>
__global__ void __launch_bounds__(PP_NT) k_postprocess(const float* __restrict__ img, size_t pitch, const __grid_constant__ isa_post_args A,
                                                       void* __restrict__ out, size_t out_pitch)
{
    __shared__ float sx[ISA_MAX_LUT];
    __shared__ float4 sc[ISA_MAX_LUT - 1];
    for (int i = threadIdx.x; i < A.nlut; i += PP_NT) {
        sx[i] = A.lut_x[i];
        if (i < A.nlut - 1) sc[i] = make_float4(A.lut_c[i][0], A.lut_c[i][1], A.lut_c[i][2], A.lut_c[i][3]);
    }
    __syncthreads();
    const LutView L{sx, sc, A.nlut, A.uniform};
    constexpr float full = FMT == ISA_POST_RGB16 ? 65535.f : 255.f;
    constexpr unsigned cap = FMT == ISA_POST_RGB16 ? 65535u : 255u;
    for (int y = blockIdx.x; y < A.crop_h; y += gridDim.x) {
        const float* prow = isa::row_ptr(img, pitch, A.crop_y + y) + 3 * A.crop_x;
        for (int x0 = PP_PX * threadIdx.x; x0 < A.crop_w; x0 += PP_PX * PP_NT) {
            const int np = min(PP_PX, A.crop_w - x0);
            float v[PP_PX][3];
            // all loads first (12 independent loads in flight per thread)
#pragma unroll
            for (int q = 0; q < PP_PX; q++)
#pragma unroll
                for (int c = 0; c < 3; c++) v[q][c] = q < np ? __ldg(prow + 3 * (x0 + q) + c) : 0.f;
            unsigned o[PP_PX][3];
#pragma unroll
            for (int q = 0; q < PP_PX; q++) {
                const float r = thr_ltgt(v[q][0], A.wb[0]), g = thr_ltgt(v[q][1], A.wb[1]), b = thr_ltgt(v[q][2], A.wb[2]);
                const float r1 = lut_cubic(L, thr_ltgt(twist_row(A.t1, r, g, b), 1.f));
                const float g1 = lut_cubic(L, thr_ltgt(twist_row(A.t1 + 4, r, g, b), 1.f));
                const float b1 = lut_cubic(L, thr_ltgt(twist_row(A.t1 + 8, r, g, b), 1.f));
                const float r2 = __fmul_rn(twist_row(A.t2, r1, g1, b1), A.amp);
                const float g2 = __fmul_rn(twist_row(A.t2 + 4, r1, g1, b1), A.amp);
                const float b2 = __fmul_rn(twist_row(A.t2 + 8, r1, g1, b1), A.amp);
                // cvt.rni: round to nearest even, negative and NaN -> 0
                o[q][0] = min(__float2uint_rn(__fmul_rn(gamma_srgb(r2), full)), cap);
                o[q][1] = min(__float2uint_rn(__fmul_rn(gamma_srgb(g2), full)), cap);
                o[q][2] = min(__float2uint_rn(__fmul_rn(gamma_srgb(b2), full)), cap);
            }
            if (FMT == ISA_POST_RGB16) {
                uint16_t* d = isa::row_ptr((uint16_t*)out, out_pitch, y) + 3 * x0;
                if (np == PP_PX && ((uintptr_t)d & 7) == 0) {
                    // 4 pixels = 12 samples = three 8-byte stores
                    uint2* d8 = (uint2*)d;
                    d8[0] = make_uint2(o[0][0] | (o[0][1] << 16), o[0][2] | (o[1][0] << 16));
                    d8[1] = make_uint2(o[1][1] | (o[1][2] << 16), o[2][0] | (o[2][1] << 16));
                    d8[2] = make_uint2(o[2][2] | (o[3][0] << 16), o[3][1] | (o[3][2] << 16));
                } else {
                    for (int q = 0; q < np; q++)
                        for (int c = 0; c < 3; c++) d[3 * q + c] = (uint16_t)o[q][c];
                }
            } else {
                uchar4* d = isa::row_ptr((uchar4*)out, out_pitch, y) + x0;
                if (np == PP_PX && ((uintptr_t)d & 15) == 0) {
                    uint4 w;
                    w.x = o[0][2] | (o[0][1] << 8) | (o[0][0] << 16) | 0xff000000u;
                    w.y = o[1][2] | (o[1][1] << 8) | (o[1][0] << 16) | 0xff000000u;
                    w.z = o[2][2] | (o[2][1] << 8) | (o[2][0] << 16) | 0xff000000u;
                    w.w = o[3][2] | (o[3][1] << 8) | (o[3][0] << 16) | 0xff000000u;
                    *(uint4*)d = w;
                } else {
                    for (int q = 0; q < np; q++) d[q] = make_uchar4((unsigned char)o[q][2], (unsigned char)o[q][1], (unsigned char)o[q][0], 255);
                }
            }
        }
    }
}

}  // namespace

cudaError_t isa_launch_postprocess(const float* img, size_t pitch, const isa_post_args& a, int format, void* out, size_t out_pitch,
                                   cudaStream_t st)
{
    if (a.crop_w <= 0 || a.crop_h <= 0) return cudaSuccess;
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    // 8 CTAs of 256 threads per SM (shared memory 10 KB each)
    const int g = std::min(a.crop_h, 8 * sms);
    if (format == ISA_POST_RGB16) k_postprocess<ISA_POST_RGB16><<<g, PP_NT, 0, st>>>(img, pitch, a, out, out_pitch);
    else k_postprocess<ISA_POST_BGRA8><<<g, PP_NT, 0, st>>>(img, pitch, a, out, out_pitch);
    return cudaGetLastError();
}
