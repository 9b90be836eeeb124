// Kernel parameters (structure tensor -> anisotropic kernel, kernel.cu:601-700),
// kernel-weighted Bayer accumulation (accumulateImages / accumulateImagesSuperRes,
// DeBayerKernels.cu:290-468) generalised to a merge scale s, and the final
// normalisation (ApplyWeighting, kernel.cu:336-391).
//
// Accumulation geometry: output pixel (x, y) samples the kernel parameters
// (clamp) and the flow (mirror) bilinearly at input position
// ((x + 0.5 + ox) / s, (y + 0.5 + oy) / s); the shift is round(s * flow);
// tap (px, py) reads the raw sample floor((x + px + sx + ox) / s) clamped to
// the crop, the certainty of the unshifted tap's half-resolution pixel and
// adds to the channel of the sample's CFA colour. s = 1 / origin 0 / whole
// frame is accumulateImages; s = 2 / origin (W/2, H/2) / central crop is
// accumulateImagesSuperRes.
//
// k_accumulate takes a list of frames and keeps the running sums in
// registers: with one frame and accumulate_into = 1 it is the reference's
// per-frame read-modify-write pass; with all frames it reads each frame's
// inputs once and writes the sums once. The 25 tap weights depend only on
// the kernel parameters, so they are computed once per output pixel.
#include "isa_internal.cuh"

namespace {

__global__ void k_structure_tensor(const float* __restrict__ img, size_t pitch, int W, int H, float* __restrict__ st3, size_t st_pitch)
{
    int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= W || y >= H) return;
    auto at = [&](int xx, int yy) { return __ldg(isa::row_ptr(img, pitch, isa::mirror(yy, H)) + isa::mirror(xx, W)); };
    // ComputeDerivatives2Kernel (opticalFlow.cu:151-185) then ComputeStructureTensor (kernel.cu:601-625)
    float dx = (at(x + 2, y) - at(x + 1, y) * 8.0f + at(x - 1, y) * 8.0f - at(x - 2, y)) / 12.0f;
    float dy = (at(x, y + 2) - at(x, y + 1) * 8.0f + at(x, y - 1) * 8.0f - at(x, y - 2)) / 12.0f;
    float* o = isa::row_ptr(st3, st_pitch, y) + 3 * x;
    o[0] = dx * dx;
    o[1] = dy * dy;
    o[2] = dx * dy;
}

// ComputeKernelParam (kernel.cu:628-700) evaluated in FP64: the FP32 form
// loses the determinant to cancellation where the kernel is strongly
// anisotropic. Output channels 0..2 = (b22, b11, -b12) / det; a 4th channel,
// when present, is 0 (the reference's float4 copy, controller :1865-1876).
__global__ void k_kernel_param(const float* __restrict__ st3, size_t st_pitch, int W, int H, float* __restrict__ out, size_t out_pitch, int oc,
                               float Dth, float Dtr, float kDetail, float kDenoise, float kStretch, float kShrink)
{
    int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= W || y >= H) return;
    const float* g = isa::row_ptr(st3, st_pitch, y) + 3 * x;
    double a11 = g[0], a22 = g[1], a12 = g[2];
    double hlp = sqrt((a22 - a11) * (a22 - a11) + 4.0 * a12 * a12);
    double c = 2.0 * a12, s = a22 - a11 + hlp;
    double nrm = sqrt(c * c + s * s);
    if (nrm > 0) { c /= nrm; s /= nrm; } else { c = 1; s = 0; }
    double l1 = (a11 + a22 + hlp) / 2.0, l2 = (a11 + a22 - hlp) / 2.0;
    double A = 1 + sqrt((l1 - l2) * (l1 - l2) / ((l1 + l2) * (l1 + l2)));
    double D = 1 - sqrt(l1) / (double)Dtr + (double)Dth;
    D = fmax(fmin(1.0, D), 0.0);
    double kd = kDetail;
    double k1 = (1.0 - D) * (kd * (double)kStretch * A) + D * kd * (double)kDenoise;
    double k2 = (1.0 - D) * (kd / (double)kShrink * A) + D * kd * (double)kDenoise;
    k1 *= k1;
    k2 *= k2;
    double x2 = c, y2 = s, x1 = s, y1 = -c;
    double b11 = k1 * x1 * x1 + x2 * x2 * k2;
    double b12 = k1 * x1 * y1 + x2 * y2 * k2;
    double b22 = k1 * y1 * y1 + y2 * y2 * k2;
    double det = b11 * b22 - b12 * b12 + (double)0.0000000001f;
    float* o = isa::row_ptr(out, out_pitch, y) + oc * x;
    o[0] = (float)(b22 / det);
    o[1] = (float)(b11 / det);
    o[2] = (float)(-b12 / det);
    if (oc == 4) o[3] = 0.f;
}

struct F3 { float v[3]; };

__device__ __forceinline__ int floor_div_s(int v, const isa_accum_geom& g)
{
    if (g.s_int == 1) return v;
    if (g.s_int == 2) return v >> 1;  // arithmetic shift: floor for negatives
    if (g.s_int > 0) { int q = v / g.s_int; return (v % g.s_int != 0 && v < 0) ? q - 1 : q; }
    return (int)floorf((float)v / g.s);
}

template <int KC>
__device__ __forceinline__ void kparam_sample(const float* kp, size_t pitch, int W, int H, float xb, float yb, float k[3])
{
    float fx = floorf(xb), fy = floorf(yb);
    int i = (int)fx, j = (int)fy;
    float a = xb - fx, b = yb - fy;
    if (a == 0.f && b == 0.f) {  // exact texel (s = 1)
        const float* p = isa::row_ptr(kp, pitch, isa::clampi(j, 0, H - 1)) + KC * isa::clampi(i, 0, W - 1);
        k[0] = __ldg(p); k[1] = __ldg(p + 1); k[2] = __ldg(p + 2);
        return;
    }
    int i0 = isa::clampi(i, 0, W - 1), i1 = isa::clampi(i + 1, 0, W - 1), j0 = isa::clampi(j, 0, H - 1), j1 = isa::clampi(j + 1, 0, H - 1);
    const float* r0 = isa::row_ptr(kp, pitch, j0);
    const float* r1 = isa::row_ptr(kp, pitch, j1);
#pragma unroll
    for (int c = 0; c < 3; c++)
        k[c] = isa::lerp2(__ldg(r0 + KC * i0 + c), __ldg(r0 + KC * i1 + c), __ldg(r1 + KC * i0 + c), __ldg(r1 + KC * i1 + c), a, b);
}

__device__ __forceinline__ float2 flow_sample(const float2* fl, size_t pitch, int W, int H, float xb, float yb)
{
    float fx = floorf(xb), fy = floorf(yb);
    int i = (int)fx, j = (int)fy;
    float a = xb - fx, b = yb - fy;
    if (a == 0.f && b == 0.f) return __ldg(isa::row_ptr(fl, pitch, isa::mirror(j, H)) + isa::mirror(i, W));
    int i0 = isa::mirror(i, W), i1 = isa::mirror(i + 1, W), j0 = isa::mirror(j, H), j1 = isa::mirror(j + 1, H);
    const float2* r0 = isa::row_ptr(fl, pitch, j0);
    const float2* r1 = isa::row_ptr(fl, pitch, j1);
    float2 p00 = __ldg(r0 + i0), p10 = __ldg(r0 + i1), p01 = __ldg(r1 + i0), p11 = __ldg(r1 + i1);
    return make_float2(isa::lerp2(p00.x, p10.x, p01.x, p11.x, a, b), isa::lerp2(p00.y, p10.y, p01.y, p11.y, a, b));
}

// BIL (sample mode BILINEAR): each frame contributes at the four integer
// shifts around s * flow with the bilinear weights of its fractional part
// (the certainty of a tap is scaled by the corner's weight); corners of
// weight zero are skipped, so at integer flow the sums are ROUND's.
template <int KC, bool BIL>
__global__ void __launch_bounds__(256) k_accumulate(isa_accum_geom g, unsigned cfa, const isa_frame_in* __restrict__ frames, int nframes,
                                                   isa_frame_in single, size_t raw_pitch, size_t flow_pitch, size_t mask_pitch, const float* __restrict__ kparam,
                                                   size_t kp_pitch, F3 white, F3 black, float* __restrict__ acc, float* __restrict__ wsum,
                                                   size_t out_pitch, int accumulate_into)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = g.yb0 + blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= g.Wo || y >= g.yb1) return;
    float* ap = isa::row_ptr(acc, out_pitch, y) + 3 * x;
    float* wp = isa::row_ptr(wsum, out_pitch, y) + 3 * x;
    if (x < 1 || y < 1 || x >= g.Wo - 1 || y >= g.Ho - 1) {
        if (!accumulate_into) { ap[0] = ap[1] = ap[2] = 0.f; wp[0] = wp[1] = wp[2] = 0.f; }
        return;
    }
    float a[3] = {0.f, 0.f, 0.f}, w[3] = {0.f, 0.f, 0.f};
    if (accumulate_into) {
        a[0] = ap[0]; a[1] = ap[1]; a[2] = ap[2];
        w[0] = wp[0]; w[1] = wp[1]; w[2] = wp[2];
    }
    const float xb = ((float)x + 0.5f + (float)g.ox) / g.s - 0.5f;
    const float yb = ((float)y + 0.5f + (float)g.oy) / g.s - 0.5f;
    float k[3];
    kparam_sample<KC>(kparam, kp_pitch, g.W, g.H, xb, yb, k);
    float wt[25];
#pragma unroll
    for (int py = -2; py <= 2; py++)
#pragma unroll
        for (int px = -2; px <= 2; px++) {
            float q = px * px * k[0] + 2 * px * py * k[2] + py * py * k[1];
            float v = expf(-0.5f * q);
            if (!isfinite(v)) v = px * py == 0 ? 1.f : 0.f;
            wt[(py + 2) * 5 + px + 2] = v;
        }
    // unshifted taps (mask rows/columns) do not depend on the frame
    int ux[5], uy[5];
#pragma unroll
    for (int d = 0; d < 5; d++) {
        ux[d] = isa::clampi(floor_div_s(x + d - 2 + g.ox, g), g.cx0, g.cx1) >> 1;
        uy[d] = isa::clampi(floor_div_s(y + d - 2 + g.oy, g), g.cy0, g.cy1) >> 1;
    }
    for (int f = 0; f < nframes; f++) {
        const isa_frame_in fr = frames ? frames[f] : single;
        int sx0 = 0, sy0 = 0;
        float bx = 0.f, by = 0.f;
        if (fr.flow) {
            float2 fl = flow_sample(fr.flow, flow_pitch, g.W, g.H, xb, yb);
            if constexpr (BIL) {
                const float hx = fl.x * g.s, hy = fl.y * g.s;
                const float fx = floorf(hx), fy = floorf(hy);
                sx0 = (int)fx; sy0 = (int)fy;
                bx = hx - fx; by = hy - fy;
            } else {
                sx0 = (int)roundf(fl.x * g.s);
                sy0 = (int)roundf(fl.y * g.s);
            }
        }
        if constexpr (BIL) {
            // the four corners' taps fall on 6 x 6 output-grid positions: their source rows, columns and CFA
            // colours once; each tap's mask cell (the unshifted tap's) is shared by the corners
            const float wk[4] = {(1.f - bx) * (1.f - by), bx * (1.f - by), (1.f - bx) * by, bx * by};
            int qxs[6];
            const uint16_t* rrs[6];
            int qys[6];
#pragma unroll
            for (int d = 0; d < 6; d++) {
                qxs[d] = isa::clampi(floor_div_s(x + d - 2 + sx0 + g.ox, g), g.cx0, g.cx1);
                qys[d] = isa::clampi(floor_div_s(y + d - 2 + sy0 + g.oy, g), g.cy0, g.cy1);
                rrs[d] = isa::row_ptr(fr.raw, raw_pitch, qys[d]);
            }
#pragma unroll
            for (int py = 0; py < 5; py++) {
                const float4* mr = fr.mask ? isa::row_ptr(fr.mask, mask_pitch, uy[py]) : nullptr;
#pragma unroll
                for (int px = 0; px < 5; px++) {
                    float4 m = make_float4(1.f, 1.f, 1.f, 1.f);
                    if (mr) m = __ldg(mr + ux[px]);
                    const float ww = wt[py * 5 + px];
#pragma unroll
                    for (int corner = 0; corner < 4; corner++) {
                        if (wk[corner] == 0.f) continue;
                        const int dx = corner & 1, dy = corner >> 1;
                        const int qx = qxs[px + dx], qy = qys[py + dy];
                        const int c = isa::cfa_at(cfa, qx, qy);
                        if (c > 2) continue;
                        float raw = (float)__ldg(rrs[py + dy] + qx);
                        raw = (raw - black.v[c]) / white.v[c];
                        float cert = c == 0 ? m.x : (c == 1 ? m.y : m.z);
                        if (!isfinite(cert)) cert = 0.f;
                        cert *= wk[corner];
                        a[c] += raw * ww * cert;
                        w[c] += ww * cert;
                    }
                }
            }
        } else {
#pragma unroll
            for (int py = 0; py < 5; py++) {
                const int qy = isa::clampi(floor_div_s(y + py - 2 + sy0 + g.oy, g), g.cy0, g.cy1);
                const uint16_t* rr = isa::row_ptr(fr.raw, raw_pitch, qy);
                const float4* mr = fr.mask ? isa::row_ptr(fr.mask, mask_pitch, uy[py]) : nullptr;
#pragma unroll
                for (int px = 0; px < 5; px++) {
                    const int qx = isa::clampi(floor_div_s(x + px - 2 + sx0 + g.ox, g), g.cx0, g.cx1);
                    const int c = isa::cfa_at(cfa, qx, qy);
                    if (c > 2) continue;
                    float raw = (float)__ldg(rr + qx);
                    raw = (raw - black.v[c]) / white.v[c];
                    float cert = 1.f;
                    if (mr) {
                        float4 m = __ldg(mr + ux[px]);
                        cert = c == 0 ? m.x : (c == 1 ? m.y : m.z);
                        if (!isfinite(cert)) cert = 0.f;
                    }
                    const float ww = wt[py * 5 + px];
                    a[c] += raw * ww * cert;
                    w[c] += ww * cert;
                }
            }
        }
    }
    ap[0] = a[0]; ap[1] = a[1]; ap[2] = a[2];
    wp[0] = w[0]; wp[1] = w[1]; wp[2] = w[2];
}

__global__ void k_apply_weighting(float* img, size_t img_pitch, const float* __restrict__ acc, const float* __restrict__ wsum, size_t pitch,
                                  int W, int H, float thr)
{
    int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= W || y >= H) return;
    float* o = isa::row_ptr(img, img_pitch, y) + 3 * x;
    const float* a = isa::row_ptr(acc, pitch, y) + 3 * x;
    const float* w = isa::row_ptr(wsum, pitch, y) + 3 * x;
    for (int c = 0; c < 3; c++) {
        float v = a[c], ww = w[c];
        if (ww < thr) { v += o[c]; ww += 1; }
        o[c] = ww != 0 ? v / ww : 0.f;
    }
}

// ---- adjoint of the merge for an L2 loss --------------------------------------
// L = sum over output pixels and channels of (out - target)^2 with
// out_c = acc_c / wsum_c (ApplyWeighting with threshold 0). With
// g_c = 2 (out_c - target_c) and h_c = g_c / wsum_c, a tap t of frame f with
// normalised sample v, certainty c and weight w contributes
//   dL/dw_t += c h_c (v - out_c),   dL/dcert += w h_c (v - out_c),
// the weights w_t = exp(-q_t / 2) of the kernel parameters k give
// dL/dk = sum_t dL/dw_t dw_t/dk, and the bilinear lookup of k scatters it to
// the kernel-parameter image. Certainty gradients are scattered to the
// frame's mask cell (atomic adds; their order is not fixed). loss may be null
// (a launch over some of the frames of a merge whose loss another adds).
//
// BIL: a frame's contribution is sum_k beta_k T_k over the four integer
// shifts k around s * flow, beta the bilinear weights of its fractional part
// (bx, by). With D_k = dL/dbeta_k = sum over k's taps of w c h_c (v - out_c),
// dL/dbx = (1 - by)(D_1 - D_0) + by (D_3 - D_2) and
// dL/dby = (1 - bx)(D_2 - D_0) + bx (D_3 - D_1); times s, they go to the
// four flow texels of the bilinear (mirror) flow lookup in gflow (atomic
// adds). A corner of weight zero still gives its D (the one-sided
// derivative) but nothing to the kernel-parameter and mask gradients.
__device__ __forceinline__ void flow_scatter(float2* gflow, size_t pitch, int W, int H, float xb, float yb, float gx, float gy)
{
    const float fx = floorf(xb), fy = floorf(yb);
    const int i = (int)fx, j = (int)fy;
    const float a = xb - fx, b = yb - fy;
    const int i0 = isa::mirror(i, W), i1 = isa::mirror(i + 1, W), j0 = isa::mirror(j, H), j1 = isa::mirror(j + 1, H);
    const float w[4] = {(1.f - a) * (1.f - b), a * (1.f - b), (1.f - a) * b, a * b};
    const int xs[4] = {i0, i1, i0, i1}, ys[4] = {j0, j0, j1, j1};
#pragma unroll
    for (int k = 0; k < 4; k++) {
        if (w[k] == 0.f) continue;
        float* d = (float*)(isa::row_ptr(gflow, pitch, ys[k]) + xs[k]);
        atomicAdd(d, w[k] * gx);
        atomicAdd(d + 1, w[k] * gy);
    }
}

template <int KC, bool BIL>
__global__ void __launch_bounds__(256, 2) k_accumulate_bwd(isa_accum_geom g, unsigned cfa, const isa_frame_in* __restrict__ frames, int nframes,
                                                       size_t raw_pitch, size_t flow_pitch, size_t mask_pitch, const float* __restrict__ kparam,
                                                       size_t kp_pitch, F3 white, F3 black, const float* __restrict__ out, size_t out_pitch,
                                                       const float* __restrict__ wsum, size_t ws_pitch, const float* __restrict__ target,
                                                       size_t tg_pitch, const float* __restrict__ weight, size_t wt_pitch, float* __restrict__ gkp,
                                                       float4* __restrict__ gmask, size_t gmask_stride, double* __restrict__ loss,
                                                       float2* __restrict__ gflow)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    double lsum = 0.0;
    if (x < g.Wo && y < g.Ho) {
        const float* op = isa::row_ptr(out, out_pitch, y) + 3 * x;
        const float* wp = isa::row_ptr(wsum, ws_pitch, y) + 3 * x;
        const float* tp = isa::row_ptr(target, tg_pitch, y) + 3 * x;
        const float om = weight ? isa::row_ptr(weight, wt_pitch, y)[x] : 1.f;
        float o[3], h[3];
#pragma unroll
        for (int c = 0; c < 3; c++) {
            o[c] = op[c];
            const float d = o[c] - tp[c];
            lsum += (double)om * d * d;
            h[c] = wp[c] != 0.f ? 2.f * om * d / wp[c] : 0.f;
        }
        if (x >= 1 && y >= 1 && x < g.Wo - 1 && y < g.Ho - 1 && (h[0] != 0.f || h[1] != 0.f || h[2] != 0.f)) {
            const float xb = ((float)x + 0.5f + (float)g.ox) / g.s - 0.5f;
            const float yb = ((float)y + 0.5f + (float)g.oy) / g.s - 0.5f;
            float k[3];
            kparam_sample<KC>(kparam, kp_pitch, g.W, g.H, xb, yb, k);
            float wt[25], G[25];
            bool live[25];
#pragma unroll
            for (int py = -2; py <= 2; py++)
#pragma unroll
                for (int px = -2; px <= 2; px++) {
                    const int t = (py + 2) * 5 + px + 2;
                    float q = px * px * k[0] + 2 * px * py * k[2] + py * py * k[1];
                    float v = expf(-0.5f * q);
                    live[t] = isfinite(v);  // the fallback weight does not depend on k
                    if (!live[t]) v = px * py == 0 ? 1.f : 0.f;
                    wt[t] = v;
                    G[t] = 0.f;
                }
            int ux[5], uy[5];
#pragma unroll
            for (int d = 0; d < 5; d++) {
                ux[d] = isa::clampi(floor_div_s(x + d - 2 + g.ox, g), g.cx0, g.cx1) >> 1;
                uy[d] = isa::clampi(floor_div_s(y + d - 2 + g.oy, g), g.cy0, g.cy1) >> 1;
            }
            for (int f = 0; f < nframes; f++) {
                const isa_frame_in fr = frames[f];
                int sx0 = 0, sy0 = 0;
                float bx = 0.f, by = 0.f;
                if (fr.flow) {
                    float2 fl = flow_sample(fr.flow, flow_pitch, g.W, g.H, xb, yb);
                    if constexpr (BIL) {
                        const float hx = fl.x * g.s, hy = fl.y * g.s;
                        const float fx = floorf(hx), fy = floorf(hy);
                        sx0 = (int)fx; sy0 = (int)fy;
                        bx = hx - fx; by = hy - fy;
                    } else {
                        sx0 = (int)roundf(fl.x * g.s);
                        sy0 = (int)roundf(fl.y * g.s);
                    }
                }
                float4* gm = gmask + (size_t)f * gmask_stride;
                float D[4] = {0.f, 0.f, 0.f, 0.f};
                if constexpr (BIL) {
                    // taps outer, corners inner (as the forward): the 6 x 6 positions once, the tap's mask cell and
                    // its gradient (per channel, summed over the corners) once per tap
                    const float wk[4] = {(1.f - bx) * (1.f - by), bx * (1.f - by), (1.f - bx) * by, bx * by};
                    const bool need_d = fr.flow != nullptr;
                    int qxs[6], qys[6];
                    const uint16_t* rrs[6];
#pragma unroll
                    for (int d = 0; d < 6; d++) {
                        qxs[d] = isa::clampi(floor_div_s(x + d - 2 + sx0 + g.ox, g), g.cx0, g.cx1);
                        qys[d] = isa::clampi(floor_div_s(y + d - 2 + sy0 + g.oy, g), g.cy0, g.cy1);
                        rrs[d] = isa::row_ptr(fr.raw, raw_pitch, qys[d]);
                    }
#pragma unroll
                    for (int py = 0; py < 5; py++) {
                        const float4* mr = fr.mask ? isa::row_ptr(fr.mask, mask_pitch, uy[py]) : nullptr;
#pragma unroll
                        for (int px = 0; px < 5; px++) {
                            float4 m = make_float4(1.f, 1.f, 1.f, 1.f);
                            if (mr) m = __ldg(mr + ux[px]);
                            const float ww = wt[py * 5 + px];
                            float gc[3] = {0.f, 0.f, 0.f}, Gt = 0.f;
#pragma unroll
                            for (int corner = 0; corner < 4; corner++) {
                                if (wk[corner] == 0.f && !need_d) continue;
                                const int dx = corner & 1, dy = corner >> 1;
                                const int qx = qxs[px + dx], qy = qys[py + dy];
                                const int c = isa::cfa_at(cfa, qx, qy);
                                if (c > 2) continue;
                                float raw = (float)__ldg(rrs[py + dy] + qx);
                                raw = (raw - black.v[c]) / white.v[c];
                                const float hc = c == 0 ? h[0] : (c == 1 ? h[1] : h[2]);
                                const float oc = c == 0 ? o[0] : (c == 1 ? o[1] : o[2]);
                                const float r = hc * (raw - oc);
                                float cert = c == 0 ? m.x : (c == 1 ? m.y : m.z);
                                if (!isfinite(cert)) cert = 0.f;
                                else if (c == 0) gc[0] += ww * r * wk[corner];
                                else if (c == 1) gc[1] += ww * r * wk[corner];
                                else gc[2] += ww * r * wk[corner];
                                D[corner] += ww * cert * r;
                                Gt += cert * r * wk[corner];
                            }
                            G[py * 5 + px] += Gt;
                            if (mr) {
                                float* dst = (float*)(isa::row_ptr(gm, mask_pitch, uy[py]) + ux[px]);
#pragma unroll
                                for (int c = 0; c < 3; c++)
                                    if (gc[c] != 0.f) atomicAdd(dst + c, gc[c]);
                            }
                        }
                    }
                } else {
#pragma unroll
                    for (int py = 0; py < 5; py++) {
                        const int qy = isa::clampi(floor_div_s(y + py - 2 + sy0 + g.oy, g), g.cy0, g.cy1);
                        const uint16_t* rr = isa::row_ptr(fr.raw, raw_pitch, qy);
                        const float4* mr = fr.mask ? isa::row_ptr(fr.mask, mask_pitch, uy[py]) : nullptr;
#pragma unroll
                        for (int px = 0; px < 5; px++) {
                            const int qx = isa::clampi(floor_div_s(x + px - 2 + sx0 + g.ox, g), g.cx0, g.cx1);
                            const int c = isa::cfa_at(cfa, qx, qy);
                            if (c > 2) continue;
                            float raw = (float)__ldg(rr + qx);
                            raw = (raw - black.v[c]) / white.v[c];
                            const float hc = c == 0 ? h[0] : (c == 1 ? h[1] : h[2]);
                            const float oc = c == 0 ? o[0] : (c == 1 ? o[1] : o[2]);
                            const float r = hc * (raw - oc);
                            float cert = 1.f;
                            if (mr) {
                                const float4 m = __ldg(mr + ux[px]);
                                cert = c == 0 ? m.x : (c == 1 ? m.y : m.z);
                                if (!isfinite(cert)) cert = 0.f;
                                else {
                                    float* dst = (float*)(isa::row_ptr(gm, mask_pitch, uy[py]) + ux[px]) + c;
                                    atomicAdd(dst, wt[py * 5 + px] * r);
                                }
                            }
                            G[py * 5 + px] += cert * r;
                        }
                    }
                }
                if (BIL && fr.flow && gflow) {
                    const float dbx = (1.f - by) * (D[1] - D[0]) + by * (D[3] - D[2]);
                    const float dby = (1.f - bx) * (D[2] - D[0]) + bx * (D[3] - D[1]);
                    flow_scatter(gflow, flow_pitch, g.W, g.H, xb, yb, dbx * g.s, dby * g.s);
                }
            }
            // dL/dk, then the transpose of the bilinear lookup (clamp addressing, zero weights skipped as in lerp2)
            float gk[3] = {0.f, 0.f, 0.f};
#pragma unroll
            for (int py = -2; py <= 2; py++)
#pragma unroll
                for (int px = -2; px <= 2; px++) {
                    const int t = (py + 2) * 5 + px + 2;
                    if (!live[t]) continue;
                    const float gw = G[t] * wt[t];
                    gk[0] += -0.5f * (float)(px * px) * gw;
                    gk[1] += -0.5f * (float)(py * py) * gw;
                    gk[2] += -(float)(px * py) * gw;
                }
            const float fx = floorf(xb), fy = floorf(yb);
            const int i = (int)fx, j = (int)fy;
            const float a = xb - fx, b = yb - fy;
            const int i0 = isa::clampi(i, 0, g.W - 1), i1 = isa::clampi(i + 1, 0, g.W - 1), j0 = isa::clampi(j, 0, g.H - 1), j1 = isa::clampi(j + 1, 0, g.H - 1);
            const float w00 = (1.f - a) * (1.f - b), w10 = a * (1.f - b), w01 = (1.f - a) * b, w11 = a * b;
#pragma unroll
            for (int c = 0; c < 3; c++) {
                atomicAdd(gkp + ((size_t)j0 * g.W + i0) * 3 + c, w00 * gk[c]);
                if (a != 0.f) atomicAdd(gkp + ((size_t)j0 * g.W + i1) * 3 + c, w10 * gk[c]);
                if (b != 0.f) atomicAdd(gkp + ((size_t)j1 * g.W + i0) * 3 + c, w01 * gk[c]);
                if (a != 0.f && b != 0.f) atomicAdd(gkp + ((size_t)j1 * g.W + i1) * 3 + c, w11 * gk[c]);
            }
        }
    }
    // block sum of the loss, one atomic per block
    for (int o = 16; o > 0; o >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
    __shared__ double sl[8];
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    if ((tid & 31) == 0) sl[tid >> 5] = lsum;
    __syncthreads();
    if (tid == 0 && loss) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x * blockDim.y) / 32; w++) t += sl[w];
        atomicAdd(loss, t);
    }
}

// dL/d(kDetail, kDenoise, Dth, Dtr, kStretch, kShrink) from dL/dkparam: the
// chain rule through k_kernel_param's FP64 arithmetic, summed over pixels.
__global__ void __launch_bounds__(256) k_kparam_bwd(const float* __restrict__ st3, size_t st_pitch, int W, int H, const float* __restrict__ gkp,
                                                   float Dth, float Dtr, float kDetail, float kDenoise, float kStretch, float kShrink,
                                                   double* __restrict__ grad)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    double gp[6] = {0, 0, 0, 0, 0, 0};
    if (x < W && y < H) {
        const float* gk = gkp + ((size_t)y * W + x) * 3;
        const double g0 = gk[0], g1 = gk[1], g2 = gk[2];
        if (g0 != 0.0 || g1 != 0.0 || g2 != 0.0) {
            const float* gs = isa::row_ptr(st3, st_pitch, y) + 3 * x;
            double a11 = gs[0], a22 = gs[1], a12 = gs[2];
            double hlp = sqrt((a22 - a11) * (a22 - a11) + 4.0 * a12 * a12);
            double c = 2.0 * a12, s = a22 - a11 + hlp;
            double nrm = sqrt(c * c + s * s);
            if (nrm > 0) { c /= nrm; s /= nrm; } else { c = 1; s = 0; }
            double l1 = (a11 + a22 + hlp) / 2.0, l2 = (a11 + a22 - hlp) / 2.0;
            double A = 1 + sqrt((l1 - l2) * (l1 - l2) / ((l1 + l2) * (l1 + l2)));
            double Draw = 1 - sqrt(l1) / (double)Dtr + (double)Dth;
            double D = fmax(fmin(1.0, Draw), 0.0);
            const double kd = kDetail, kst = kStretch, ksh = kShrink, kdn = kDenoise;
            double u1 = (1.0 - D) * (kd * kst * A) + D * kd * kdn;
            double u2 = (1.0 - D) * (kd / ksh * A) + D * kd * kdn;
            double k1 = u1 * u1, k2 = u2 * u2;
            double x2 = c, y2 = s, x1 = s, y1 = -c;
            double b11 = k1 * x1 * x1 + x2 * x2 * k2;
            double b12 = k1 * x1 * y1 + x2 * y2 * k2;
            double b22 = k1 * y1 * y1 + y2 * y2 * k2;
            double det = b11 * b22 - b12 * b12 + (double)0.0000000001f;
            double id = 1.0 / det, id2 = id * id;
            // out0 = b22/det, out1 = b11/det, out2 = -b12/det; d(det) = b22 db11 + b11 db22 - 2 b12 db12
            double gb11 = g0 * (-b22 * b22 * id2) + g1 * (id - b11 * b22 * id2) + g2 * (b12 * b22 * id2);
            double gb22 = g0 * (id - b22 * b11 * id2) + g1 * (-b11 * b11 * id2) + g2 * (b12 * b11 * id2);
            double gb12 = g0 * (2.0 * b22 * b12 * id2) + g1 * (2.0 * b11 * b12 * id2) + g2 * (-id - 2.0 * b12 * b12 * id2);
            double gk1 = gb11 * x1 * x1 + gb12 * x1 * y1 + gb22 * y1 * y1;
            double gk2 = gb11 * x2 * x2 + gb12 * x2 * y2 + gb22 * y2 * y2;
            double gu1 = 2.0 * u1 * gk1, gu2 = 2.0 * u2 * gk2;
            gp[0] = gu1 * ((1.0 - D) * kst * A + D * kdn) + gu2 * ((1.0 - D) * A / ksh + D * kdn);
            gp[1] = (gu1 + gu2) * D * kd;
            gp[4] = gu1 * (1.0 - D) * kd * A;
            gp[5] = gu2 * (-(1.0 - D) * kd * A / (ksh * ksh));
            if (Draw > 0.0 && Draw < 1.0) {
                double gD = gu1 * (-kd * kst * A + kd * kdn) + gu2 * (-kd * A / ksh + kd * kdn);
                gp[2] = gD;
                gp[3] = gD * sqrt(l1) / ((double)Dtr * (double)Dtr);
            }
        }
    }
    __shared__ double sg[8][6];
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
#pragma unroll
    for (int q = 0; q < 6; q++) {
        double v = gp[q];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if ((tid & 31) == 0) sg[tid >> 5][q] = v;
    }
    __syncthreads();
    if (tid < 6) {
        double t = 0.0;
        for (int w = 0; w < 8; w++) t += sg[w][tid];
        atomicAdd(grad + tid, t);
    }
}

inline dim3 grid2(int w, int h, dim3 b) { return dim3((w + b.x - 1) / b.x, (h + b.y - 1) / b.y); }

}  // namespace

cudaError_t isa_launch_structure_tensor(const float* img, size_t pitch, int W, int H, float* st3, size_t st_pitch, cudaStream_t st)
{
    dim3 b(32, 8);
    k_structure_tensor<<<grid2(W, H, b), b, 0, st>>>(img, pitch, W, H, st3, st_pitch);
    return cudaGetLastError();
}

cudaError_t isa_launch_kernel_param(const float* st3, size_t st_pitch, int W, int H, float* out, size_t out_pitch, int out_channels, float Dth,
                                    float Dtr, float kDetail, float kDenoise, float kStretch, float kShrink, cudaStream_t st)
{
    if (out_channels != 3 && out_channels != 4) return cudaErrorInvalidValue;
    dim3 b(32, 8);
    k_kernel_param<<<grid2(W, H, b), b, 0, st>>>(st3, st_pitch, W, H, out, out_pitch, out_channels, Dth, Dtr, kDetail, kDenoise, kStretch,
                                                 kShrink);
    return cudaGetLastError();
}

cudaError_t isa_launch_accumulate(const isa_accum_geom& g, unsigned cfa, const isa_frame_in* frames, int nframes, const isa_frame_in* single,
                                  size_t raw_pitch,
                                  size_t flow_pitch, size_t mask_pitch, const float* kparam, size_t kparam_pitch, int kparam_channels,
                                  const float* white, const float* black, float* acc, float* wsum, size_t out_pitch, int accumulate_into,
                                  cudaStream_t st)
{
    if (!g.bilinear && g.s_int == 2 && kparam_channels == 4 && isa_accumulate_x2_supported(cfa))
        return isa_launch_accumulate_x2(g, cfa, frames, nframes, single, raw_pitch, flow_pitch, mask_pitch, kparam, kparam_pitch, white, black, acc,
                                        wsum, out_pitch, accumulate_into, st);
    F3 wh, bl;
    for (int c = 0; c < 3; c++) { wh.v[c] = white[c]; bl.v[c] = black[c]; }
    isa_frame_in one = single ? *single : isa_frame_in{nullptr, nullptr, nullptr};
    if (g.yb0 < 0 || g.yb1 > g.Ho || g.yb1 <= g.yb0) return cudaErrorInvalidValue;
    dim3 b(g.bx > 0 ? g.bx : 32, g.by > 0 ? g.by : 8), grd = grid2(g.Wo, g.yb1 - g.yb0, b);
    if (b.x * b.y > 256) return cudaErrorInvalidValue;
    if (kparam_channels == 4 && g.bilinear)
        k_accumulate<4, true><<<grd, b, 0, st>>>(g, cfa, frames, nframes, one, raw_pitch, flow_pitch, mask_pitch, kparam, kparam_pitch, wh, bl, acc,
                                                 wsum, out_pitch, accumulate_into);
    else if (kparam_channels == 4)
        k_accumulate<4, false><<<grd, b, 0, st>>>(g, cfa, frames, nframes, one, raw_pitch, flow_pitch, mask_pitch, kparam, kparam_pitch, wh, bl, acc,
                                                  wsum, out_pitch, accumulate_into);
    else if (kparam_channels == 3 && g.bilinear)
        k_accumulate<3, true><<<grd, b, 0, st>>>(g, cfa, frames, nframes, one, raw_pitch, flow_pitch, mask_pitch, kparam, kparam_pitch, wh, bl, acc,
                                                 wsum, out_pitch, accumulate_into);
    else if (kparam_channels == 3)
        k_accumulate<3, false><<<grd, b, 0, st>>>(g, cfa, frames, nframes, one, raw_pitch, flow_pitch, mask_pitch, kparam, kparam_pitch, wh, bl, acc,
                                                  wsum, out_pitch, accumulate_into);
    else
        return cudaErrorInvalidValue;
    return cudaGetLastError();
}

cudaError_t isa_launch_apply_weighting(float* img, size_t img_pitch, const float* acc, const float* wsum, size_t pitch, int W, int H, float thr,
                                       cudaStream_t st)
{
    dim3 b(32, 8);
    k_apply_weighting<<<grid2(W, H, b), b, 0, st>>>(img, img_pitch, acc, wsum, pitch, W, H, thr);
    return cudaGetLastError();
}

cudaError_t isa_launch_accumulate_bwd(const isa_accum_geom& g, unsigned cfa, const isa_frame_in* frames, int nframes, size_t raw_pitch,
                                      size_t flow_pitch, size_t mask_pitch, const float* kparam, size_t kparam_pitch, const float* white,
                                      const float* black, const float* out, size_t out_pitch, const float* wsum, size_t ws_pitch, const float* target,
                                      size_t tg_pitch, const float* weight, size_t wt_pitch, float* gkp, float4* gmask, size_t gmask_stride, double* loss,
                                      float2* gflow, cudaStream_t st)
{
    F3 wh, bl;
    for (int c = 0; c < 3; c++) { wh.v[c] = white[c]; bl.v[c] = black[c]; }
    dim3 b(32, 8), grd = grid2(g.Wo, g.Ho, b);
    if (g.bilinear)
        k_accumulate_bwd<4, true><<<grd, b, 0, st>>>(g, cfa, frames, nframes, raw_pitch, flow_pitch, mask_pitch, kparam, kparam_pitch, wh, bl, out,
                                                     out_pitch, wsum, ws_pitch, target, tg_pitch, weight, wt_pitch, gkp, gmask, gmask_stride, loss,
                                                     gflow);
    else
        k_accumulate_bwd<4, false><<<grd, b, 0, st>>>(g, cfa, frames, nframes, raw_pitch, flow_pitch, mask_pitch, kparam, kparam_pitch, wh, bl, out,
                                                      out_pitch, wsum, ws_pitch, target, tg_pitch, weight, wt_pitch, gkp, gmask, gmask_stride, loss,
                                                      nullptr);
    return cudaGetLastError();
}

cudaError_t isa_launch_kparam_bwd(const float* st3, size_t st_pitch, int W, int H, const float* gkp, float Dth, float Dtr, float kDetail,
                                  float kDenoise, float kStretch, float kShrink, double* grad6, cudaStream_t st)
{
    dim3 b(32, 8);
    k_kparam_bwd<<<grid2(W, H, b), b, 0, st>>>(st3, st_pitch, W, H, gkp, Dth, Dtr, kDetail, kDenoise, kStretch, kShrink, grad6);
    return cudaGetLastError();
}
