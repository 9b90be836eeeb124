// Robustness mask (ComputeRobustnessMask, RobustnessModell.cu:29-157) and its
// 5x5 erosion (NPP ErodeBorder, ImageStackAlignatorController.cs:1976).
//
// The flow is read as the reference's linear/mirror texture does at a
// half-resolution pixel's normalized position: for a full-resolution flow
// this is the mean of the 2x2 block under the half-res pixel. The running
// max/min of the reference compares each of the 25 taps with the centre
// only (RobustnessModell.cu:52-60), so M depends on the centre and the
// (+2, +2) tap alone; that is what is evaluated here, with identical result.
#include "isa_internal.cuh"

namespace {

__device__ __forceinline__ float2 flow_sample(const float2* flow, size_t pitch, int Wf, int Hf, int Wh, int Hh, int qx, int qy)
{
    float xb = ((float)qx + 0.5f) / (float)Wh * Wf - 0.5f, yb = ((float)qy + 0.5f) / (float)Hh * Hf - 0.5f;
    float fx = floorf(xb), fy = floorf(yb);
    int i = (int)fx, j = (int)fy;
    float a = xb - fx, b = yb - fy;
    int i0 = isa::mirror(i, Wf), i1 = isa::mirror(i + 1, Wf), j0 = isa::mirror(j, Hf), j1 = isa::mirror(j + 1, Hf);
    const float2* r0 = isa::row_ptr(flow, pitch, j0);
    const float2* r1 = isa::row_ptr(flow, pitch, j1);
    float2 p00 = __ldg(r0 + i0), p10 = __ldg(r0 + i1), p01 = __ldg(r1 + i0), p11 = __ldg(r1 + i1);
    return make_float2(isa::lerp2(p00.x, p10.x, p01.x, p11.x, a, b), isa::lerp2(p00.y, p10.y, p01.y, p11.y, a, b));
}

// Mask value of interior half-res pixel (x, y); ref/mov are float3 images.
__device__ float4 mask_at(const float* __restrict__ ref3, const float* __restrict__ mov3, size_t img_pitch, int Wh, int Hh,
                          const float2* __restrict__ flow, size_t flow_pitch, int Wf, int Hf, float alpha, float beta, float thr_m,
                          float s_lit, float t_lit, int x, int y)
{
    float2 sf = flow_sample(flow, flow_pitch, Wf, Hf, Wh, Hh, x, y);
    float2 sl = flow_sample(flow, flow_pitch, Wf, Hf, Wh, Hh, x + 2, y + 2);
    float mxx = fmaxf(sl.x, sf.x), mxy = fmaxf(sl.y, sf.y);
    float mnx = fminf(sl.x, sf.x), mny = fminf(sl.y, sf.y);
    int shx = (int)roundf(sf.x * 0.5f), shy = (int)roundf(sf.y * 0.5f);
    float mr[3] = {0.f, 0.f, 0.f}, mm[3] = {0.f, 0.f, 0.f}, pr[9][3];
    for (int j = -1; j <= 1; j++)
        for (int i = -1; i <= 1; i++) {
            const float* p = isa::row_ptr(ref3, img_pitch, y + j) + 3 * (x + i);
            int qy = isa::clampi(y + shy + j, 0, Hh - 1), qx = isa::clampi(x + shx + i, 0, Wh - 1);
            const float* q = isa::row_ptr(mov3, img_pitch, qy) + 3 * qx;
            int k = (j + 1) * 3 + i + 1;
            for (int c = 0; c < 3; c++) {
                pr[k][c] = __ldg(p + c);
                mr[c] += pr[k][c];
                mm[c] += __ldg(q + c);
            }
        }
    for (int c = 0; c < 3; c++) { mr[c] /= 9.0f; mm[c] /= 9.0f; }
    float md = fabsf(mr[0] - mm[0]) + fabsf(mr[1] - mm[1]) + fabsf(mr[2] - mm[2]);
    md /= 3.0f;
    mxx *= 0.5f * md; mxy *= 0.5f * md; mnx *= 0.5f * md; mny *= 0.5f * md;
    float M = sqrtf((mxx - mnx) * (mxx - mnx) + (mxy - mny) * (mxy - mny));
    float sd[3] = {0.f, 0.f, 0.f};
    for (int k = 0; k < 9; k++)
        for (int c = 0; c < 3; c++) sd[c] += (pr[k][c] - mr[c]) * (pr[k][c] - mr[c]);
    float sgain = M > thr_m ? 0.f : s_lit;
    float out[3];
    for (int c = 0; c < 3; c++) {
        float sr = sqrtf(sd[c] / 9.0f);
        float smd = sqrtf(alpha * mr[c] + beta);
        if (c == 1) smd /= sqrtf(2.0f);
        float dist = fabsf(mr[c] - mm[c]);
        float sig = fmaxf(smd, sr);
        dist = dist * (sr * sr / (sr * sr + smd * smd));
        out[c] = fmaxf(fminf(sgain * expf(-dist * dist / (sig * sig)) - t_lit, 1.0f), 0.0f);
    }
    return make_float4(out[0], out[1], out[2], M);
}

__global__ void k_robustness(const float* __restrict__ ref3, const float* __restrict__ mov3, size_t img_pitch, float4* __restrict__ mask,
                             size_t mask_pitch, int Wh, int Hh, const float2* __restrict__ flow, size_t flow_pitch, int Wf, int Hf,
                             float alpha, float beta, float thr_m, float s, float t)
{
    int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= Wh - 1 || y >= Hh - 1 || x < 1 || y < 1) return;
    isa::row_ptr(mask, mask_pitch, y)[x] =
        mask_at(ref3, mov3, img_pitch, Wh, Hh, flow, flow_pitch, Wf, Hf, alpha, beta, thr_m, s, t, x, y);
}

__global__ void k_erode(const float4* __restrict__ in, size_t in_pitch, float4* __restrict__ out, size_t out_pitch, int W, int H, int size)
{
    int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= W || y >= H) return;
    int a = size / 2;
    float4 m = make_float4(INFINITY, INFINITY, INFINITY, INFINITY);
    for (int j = 0; j < size; j++) {
        const float4* r = isa::row_ptr(in, in_pitch, isa::clampi(y + j - a, 0, H - 1));
        for (int i = 0; i < size; i++) {
            float4 v = __ldg(r + isa::clampi(x + i - a, 0, W - 1));
            m.x = fminf(m.x, v.x); m.y = fminf(m.y, v.y); m.z = fminf(m.z, v.z); m.w = fminf(m.w, v.w);
        }
    }
    isa::row_ptr(out, out_pitch, y)[x] = m;
}

// Fused mask + erosion for one frame: the mask over the output tile plus an
// (erode/2) halo is computed into shared memory (border pixels keep the
// reference's initial value 1, controller :1891), then the min filter with
// replicate border is taken. ref3 / mov3: half-res RGB of deBayersSubSample3.
constexpr int RB_TX = 32, RB_TY = 8, RB_MAXA = 4;

__global__ void __launch_bounds__(256) k_robustness_erode(const float* __restrict__ ref3, const float* __restrict__ mov3, size_t img_pitch,
                                                         int Wh, int Hh, const float2* __restrict__ flow, size_t flow_pitch, int Wf,
                                                         int Hf, float alpha, float beta, float thr_m, float s, float t, int size,
                                                         float4* __restrict__ out, size_t out_pitch)
{
    __shared__ float4 sm[(RB_TY + 2 * RB_MAXA) * (RB_TX + 2 * RB_MAXA)];
    const int a = size / 2;
    const int SW = RB_TX + 2 * a, SH = RB_TY + 2 * a;
    const int x0 = blockIdx.x * RB_TX, y0 = blockIdx.y * RB_TY;
    const int tid = threadIdx.y * blockDim.x + threadIdx.x, nt = blockDim.x * blockDim.y;
    for (int i = tid; i < SW * SH; i += nt) {
        int sy = i / SW, sx = i - sy * SW;
        int qx = isa::clampi(x0 + sx - a, 0, Wh - 1), qy = isa::clampi(y0 + sy - a, 0, Hh - 1);
        float4 v = make_float4(1.f, 1.f, 1.f, 1.f);
        if (qx >= 1 && qx < Wh - 1 && qy >= 1 && qy < Hh - 1)
            v = mask_at(ref3, mov3, img_pitch, Wh, Hh, flow, flow_pitch, Wf, Hf, alpha, beta, thr_m, s, t, qx, qy);
        sm[i] = v;
    }
    __syncthreads();
    int x = x0 + threadIdx.x, y = y0 + threadIdx.y;
    if (x >= Wh || y >= Hh) return;
    float4 m = make_float4(INFINITY, INFINITY, INFINITY, INFINITY);
    for (int j = 0; j < size; j++)
        for (int i = 0; i < size; i++) {
            float4 v = sm[(threadIdx.y + j) * SW + threadIdx.x + i];
            m.x = fminf(m.x, v.x); m.y = fminf(m.y, v.y); m.z = fminf(m.z, v.z); m.w = fminf(m.w, v.w);
        }
    isa::row_ptr(out, out_pitch, y)[x] = m;
}

// ---- pipeline form: statistics that do not depend on the moved frame are
// computed once per burst, the moved image's 3x3 means once per frame, and
// the mask itself reads them; every value is produced by the same arithmetic
// in the same order as mask_at, so the masks are identical.

// 3x3 means and standard deviations of the reference (interior pixels).
__global__ void k_ref_stats(const float* __restrict__ ref3, size_t img_pitch, int Wh, int Hh, float4* __restrict__ mr_out,
                            float4* __restrict__ sr_out, size_t sp)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= Wh - 1 || y >= Hh - 1 || x < 1 || y < 1) return;
    float mr[3] = {0.f, 0.f, 0.f}, pr[9][3];
    for (int j = -1; j <= 1; j++)
        for (int i = -1; i <= 1; i++) {
            const float* p = isa::row_ptr(ref3, img_pitch, y + j) + 3 * (x + i);
            const int k = (j + 1) * 3 + i + 1;
            for (int c = 0; c < 3; c++) {
                pr[k][c] = __ldg(p + c);
                mr[c] += pr[k][c];
            }
        }
    for (int c = 0; c < 3; c++) mr[c] /= 9.0f;
    float sd[3] = {0.f, 0.f, 0.f};
    for (int k = 0; k < 9; k++)
        for (int c = 0; c < 3; c++) sd[c] += (pr[k][c] - mr[c]) * (pr[k][c] - mr[c]);
    isa::row_ptr(mr_out, sp, y)[x] = make_float4(mr[0], mr[1], mr[2], 0.f);
    isa::row_ptr(sr_out, sp, y)[x] = make_float4(sqrtf(sd[0] / 9.0f), sqrtf(sd[1] / 9.0f), sqrtf(sd[2] / 9.0f), 0.f);
}

// 3x3 means of the moved image with the reference's per-tap clamping, at
// every centre inside the image.
__global__ void k_box3(const float* __restrict__ mov3, size_t img_pitch, int Wh, int Hh, float4* __restrict__ box, size_t sp)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= Wh || y >= Hh) return;
    float mm[3] = {0.f, 0.f, 0.f};
    for (int j = -1; j <= 1; j++)
        for (int i = -1; i <= 1; i++) {
            const float* q = isa::row_ptr(mov3, img_pitch, isa::clampi(y + j, 0, Hh - 1)) + 3 * isa::clampi(x + i, 0, Wh - 1);
            for (int c = 0; c < 3; c++) mm[c] += __ldg(q + c);
        }
    isa::row_ptr(box, sp, y)[x] = make_float4(mm[0] / 9.0f, mm[1] / 9.0f, mm[2] / 9.0f, 0.f);
}

struct RobustTabs {
    const float4* mr;
    const float4* sr;
    const float4* box;
    size_t sp;
};

// mask_at with the reference statistics and the moved 3x3 means looked up;
// a shifted centre outside the image (whose clamped taps differ from the
// clamped centre's) is summed directly. The terms the adjoint needs are
// returned too: the three exponentials E_c and the gain sg (s, or 0 where
// M exceeds the threshold), so that mask_c = clamp(sg E_c - t, 0, 1).
struct MaskTerms { float m[3]; float M; float E[3]; float sg; };

// 3x3 mean of the moving half-res image around (cx, cy): the table entry, or
// (a centre outside the image) the clamped taps summed directly.
__device__ __forceinline__ void moved_mean(const RobustTabs& tb, const float* __restrict__ mov3, size_t img_pitch, int Wh, int Hh, int cx, int cy,
                                           float mm[3])
{
    if ((unsigned)cx < (unsigned)Wh && (unsigned)cy < (unsigned)Hh) {
        const float4 b4 = __ldg(isa::row_ptr(tb.box, tb.sp, cy) + cx);
        mm[0] = b4.x; mm[1] = b4.y; mm[2] = b4.z;
    } else {
        mm[0] = mm[1] = mm[2] = 0.f;
        for (int j = -1; j <= 1; j++)
            for (int i = -1; i <= 1; i++) {
                const float* q = isa::row_ptr(mov3, img_pitch, isa::clampi(cy + j, 0, Hh - 1)) + 3 * isa::clampi(cx + i, 0, Wh - 1);
                for (int c = 0; c < 3; c++) mm[c] += __ldg(q + c);
            }
        for (int c = 0; c < 3; c++) mm[c] /= 9.0f;
    }
}

// Offset of the moved 3x3 mean for the flow sample sf at a half-res pixel:
// ROUND, round(sf / 2); BIL (sample mode BILINEAR), floor(sf / 2) and the
// fractional part (bx, by) that blends the four means around it.
template <bool BIL>
__device__ __forceinline__ void moved_offset(float2 sf, int& shx, int& shy, float& bx, float& by)
{
    if constexpr (BIL) {
        const float hx = sf.x * 0.5f, hy = sf.y * 0.5f;
        const float fx = floorf(hx), fy = floorf(hy);
        shx = (int)fx; shy = (int)fy;
        bx = hx - fx; by = hy - fy;
    } else {
        shx = (int)roundf(sf.x * 0.5f); shy = (int)roundf(sf.y * 0.5f);
        bx = by = 0.f;
    }
}

template <bool BIL>
__device__ __forceinline__ MaskTerms mask_terms(const RobustTabs& tb, const float* __restrict__ mov3, size_t img_pitch, int Wh, int Hh,
                                                const float2* __restrict__ flow, size_t flow_pitch, int Wf, int Hf, float alpha, float beta,
                                                float thr_m, float s_lit, float t_lit, int x, int y)
{
    float2 sf = flow_sample(flow, flow_pitch, Wf, Hf, Wh, Hh, x, y);
    float2 sl = flow_sample(flow, flow_pitch, Wf, Hf, Wh, Hh, x + 2, y + 2);
    float mxx = fmaxf(sl.x, sf.x), mxy = fmaxf(sl.y, sf.y);
    float mnx = fminf(sl.x, sf.x), mny = fminf(sl.y, sf.y);
    int shx, shy;
    float bx, by;
    moved_offset<BIL>(sf, shx, shy, bx, by);
    const float4 r4 = __ldg(isa::row_ptr(tb.mr, tb.sp, y) + x), s4 = __ldg(isa::row_ptr(tb.sr, tb.sp, y) + x);
    const float mr[3] = {r4.x, r4.y, r4.z}, sr3[3] = {s4.x, s4.y, s4.z};
    float mm[3];
    moved_mean(tb, mov3, img_pitch, Wh, Hh, x + shx, y + shy, mm);
    if constexpr (BIL) {
        const float w0 = (1.f - bx) * (1.f - by);
#pragma unroll
        for (int c = 0; c < 3; c++) mm[c] *= w0;
#pragma unroll
        for (int k = 1; k < 4; k++) {
            const float wk = ((k & 1) ? bx : 1.f - bx) * ((k >> 1) ? by : 1.f - by);
            if (wk == 0.f) continue;
            float mk[3];
            moved_mean(tb, mov3, img_pitch, Wh, Hh, x + shx + (k & 1), y + shy + (k >> 1), mk);
#pragma unroll
            for (int c = 0; c < 3; c++) mm[c] += wk * mk[c];
        }
    }
    float md = fabsf(mr[0] - mm[0]) + fabsf(mr[1] - mm[1]) + fabsf(mr[2] - mm[2]);
    md /= 3.0f;
    mxx *= 0.5f * md; mxy *= 0.5f * md; mnx *= 0.5f * md; mny *= 0.5f * md;
    MaskTerms r;
    r.M = sqrtf((mxx - mnx) * (mxx - mnx) + (mxy - mny) * (mxy - mny));
    r.sg = r.M > thr_m ? 0.f : s_lit;
#pragma unroll
    for (int c = 0; c < 3; c++) {
        float sr = sr3[c];
        float smd = sqrtf(alpha * mr[c] + beta);
        if (c == 1) smd /= sqrtf(2.0f);
        float dist = fabsf(mr[c] - mm[c]);
        float sig = fmaxf(smd, sr);
        dist = dist * (sr * sr / (sr * sr + smd * smd));
        r.E[c] = expf(-dist * dist / (sig * sig));
        r.m[c] = fmaxf(fminf(r.sg * r.E[c] - t_lit, 1.0f), 0.0f);
    }
    return r;
}

template <bool BIL>
__device__ __forceinline__ float4 mask_fast(const RobustTabs& tb, const float* __restrict__ mov3, size_t img_pitch, int Wh, int Hh,
                                            const float2* __restrict__ flow, size_t flow_pitch, int Wf, int Hf, float alpha, float beta, float thr_m,
                                            float s_lit, float t_lit, int x, int y)
{
    const MaskTerms r = mask_terms<BIL>(tb, mov3, img_pitch, Wh, Hh, flow, flow_pitch, Wf, Hf, alpha, beta, thr_m, s_lit, t_lit, x, y);
    return make_float4(r.m[0], r.m[1], r.m[2], r.M);
}

// Adjoint support: the un-eroded mask of every half-res pixel (border 1, as
// in the forward) and its exponentials and gain (zero on the border, whose
// value does not depend on s and t).
template <bool BIL>
__global__ void k_mask_store(RobustTabs tb, const float* __restrict__ mov3, size_t img_pitch, int Wh, int Hh, const float2* __restrict__ flow,
                             size_t flow_pitch, int Wf, int Hf, float alpha, float beta, float thr_m, float s, float t, float4* __restrict__ m_out,
                             float4* __restrict__ aux_out, size_t sp)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= Wh || y >= Hh) return;
    float4 m = make_float4(1.f, 1.f, 1.f, 1.f), aux = make_float4(0.f, 0.f, 0.f, 0.f);
    if (x >= 1 && x < Wh - 1 && y >= 1 && y < Hh - 1) {
        const MaskTerms r = mask_terms<BIL>(tb, mov3, img_pitch, Wh, Hh, flow, flow_pitch, Wf, Hf, alpha, beta, thr_m, s, t, x, y);
        m = make_float4(r.m[0], r.m[1], r.m[2], r.M);
        aux = make_float4(r.E[0], r.E[1], r.E[2], r.sg);
    }
    isa::row_ptr(m_out, sp, y)[x] = m;
    isa::row_ptr(aux_out, sp, y)[x] = aux;
}

// Mask over a 32 x 32 output tile plus the erosion halo in shared memory
// (border pixels 1, replicate addressing as k_robustness_erode), then the
// separable min filter: rows, then columns.
constexpr int RF_T = 32;

template <bool BIL>
__global__ void __launch_bounds__(256) k_robustness_erode_fast(RobustTabs tb, const float* __restrict__ mov3, size_t img_pitch, int Wh, int Hh,
                                                              const float2* __restrict__ flow, size_t flow_pitch, int Wf, int Hf, float alpha,
                                                              float beta, float thr_m, float s, float t, int size, float4* __restrict__ out,
                                                              size_t out_pitch)
{
    __shared__ float4 sm[(RF_T + 2 * RB_MAXA) * (RF_T + 2 * RB_MAXA)];
    __shared__ float4 hm[(RF_T + 2 * RB_MAXA) * RF_T];
    const int a = size / 2;
    const int SW = RF_T + 2 * a, SH = RF_T + 2 * a;
    const int x0 = blockIdx.x * RF_T, y0 = blockIdx.y * RF_T;
    const int tid = threadIdx.x;
    for (int i = tid; i < SW * SH; i += 256) {
        const int sy = i / SW, sx = i - sy * SW;
        const int qx = isa::clampi(x0 + sx - a, 0, Wh - 1), qy = isa::clampi(y0 + sy - a, 0, Hh - 1);
        float4 v = make_float4(1.f, 1.f, 1.f, 1.f);
        if (qx >= 1 && qx < Wh - 1 && qy >= 1 && qy < Hh - 1)
            v = mask_fast<BIL>(tb, mov3, img_pitch, Wh, Hh, flow, flow_pitch, Wf, Hf, alpha, beta, thr_m, s, t, qx, qy);
        sm[i] = v;
    }
    __syncthreads();
    for (int i = tid; i < SH * RF_T; i += 256) {
        const int sy = i / RF_T, x = i - sy * RF_T;
        float4 m = sm[sy * SW + x];
        for (int k = 1; k < size; k++) {
            const float4 v = sm[sy * SW + x + k];
            m.x = fminf(m.x, v.x); m.y = fminf(m.y, v.y); m.z = fminf(m.z, v.z); m.w = fminf(m.w, v.w);
        }
        hm[sy * RF_T + x] = m;
    }
    __syncthreads();
    for (int i = tid; i < RF_T * RF_T; i += 256) {
        const int ly = i / RF_T, lx = i - ly * RF_T;
        const int x = x0 + lx, y = y0 + ly;
        if (x >= Wh || y >= Hh) continue;
        float4 m = hm[ly * RF_T + lx];
        for (int k = 1; k < size; k++) {
            const float4 v = hm[(ly + k) * RF_T + lx];
            m.x = fminf(m.x, v.x); m.y = fminf(m.y, v.y); m.z = fminf(m.z, v.z); m.w = fminf(m.w, v.w);
        }
        isa::row_ptr(out, out_pitch, y)[x] = m;
    }
}

// Adjoint of the 5x5 erosion: each eroded value's gradient goes to the
// first pixel of its window (row-major, replicate border) holding the
// minimum, per channel.
__global__ void k_erode_route(const float4* __restrict__ m, const float4* __restrict__ g_eroded, size_t sp, int Wh, int Hh, int size,
                              float4* __restrict__ g_mask)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= Wh || y >= Hh) return;
    const float4 ge = isa::row_ptr(g_eroded, sp, y)[x];
    const float gc[3] = {ge.x, ge.y, ge.z};
    const int a = size / 2;
#pragma unroll
    for (int c = 0; c < 3; c++) {
        if (gc[c] == 0.f) continue;
        float best = INFINITY;
        int bx = x, by = y;
        for (int j = 0; j < size; j++) {
            const int yy = isa::clampi(y + j - a, 0, Hh - 1);
            for (int i = 0; i < size; i++) {
                const int xx = isa::clampi(x + i - a, 0, Wh - 1);
                const float4 v = __ldg(isa::row_ptr(m, sp, yy) + xx);
                const float vc = c == 0 ? v.x : (c == 1 ? v.y : v.z);
                if (vc < best) { best = vc; bx = xx; by = yy; }
            }
        }
        atomicAdd((float*)(isa::row_ptr(g_mask, sp, by) + bx) + c, gc[c]);
    }
}

// dL/ds and dL/dt from the un-eroded mask's gradient: mask_c = clamp(sg E_c - t, 0, 1).
__global__ void __launch_bounds__(256) k_mask_param_bwd(const float4* __restrict__ m, const float4* __restrict__ aux, const float4* __restrict__ g_mask,
                                                       size_t sp, int Wh, int Hh, float t_lit, double* __restrict__ grad2)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    double gs = 0.0, gt = 0.0;
    if (x >= 1 && x < Wh - 1 && y >= 1 && y < Hh - 1) {
        const float4 gm = __ldg(isa::row_ptr(g_mask, sp, y) + x);
        const float4 ax = __ldg(isa::row_ptr(aux, sp, y) + x);
        const float g[3] = {gm.x, gm.y, gm.z}, E[3] = {ax.x, ax.y, ax.z};
#pragma unroll
        for (int c = 0; c < 3; c++) {
            const float raw = ax.w * E[c] - t_lit;
            if (g[c] != 0.f && raw > 0.f && raw < 1.f) {
                if (ax.w != 0.f) gs += (double)g[c] * E[c];
                gt -= (double)g[c];
            }
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        gs += __shfl_xor_sync(0xffffffffu, gs, o);
        gt += __shfl_xor_sync(0xffffffffu, gt, o);
    }
    __shared__ double sh[8][2];
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    if ((tid & 31) == 0) { sh[tid >> 5][0] = gs; sh[tid >> 5][1] = gt; }
    __syncthreads();
    if (tid < 2) {
        double t = 0.0;
        for (int w = 0; w < 8; w++) t += sh[w][tid];
        atomicAdd(grad2 + tid, t);
    }
}

// dL/dflow of the mask in sample mode BILINEAR, from the un-eroded mask's
// gradient g_mask: mask_c = clamp(sg E_c - t, 0, 1), E_c = exp(-dist_c^2 /
// sig_c^2), dist_c = |mr_c - mm_c| k_c with k_c = sr_c^2 / (sr_c^2 + smd_c^2),
// and mm_c the blend of the four moved 3x3 means B_k around sf / 2 (sf the
// flow sample of the half-res pixel):
//   dmm/dbx = (1 - by)(B_1 - B_0) + by (B_3 - B_2),
//   dmm/dby = (1 - bx)(B_2 - B_0) + bx (B_3 - B_1),
// and d(sf / 2)/dsf = 1/2. The flow also enters M, which only switches sg at
// a threshold (zero derivative almost everywhere). The gradient of sf goes to
// the four full-res flow texels of its bilinear (mirror) lookup (atomic adds).
__global__ void __launch_bounds__(256) k_mask_flow_bwd(RobustTabs tb, const float* __restrict__ mov3, size_t img_pitch, int Wh, int Hh,
                                                      const float2* __restrict__ flow, size_t flow_pitch, int Wf, int Hf, float alpha, float beta,
                                                      float t_lit, const float4* __restrict__ aux, const float4* __restrict__ g_mask,
                                                      float2* __restrict__ gflow)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x < 1 || x >= Wh - 1 || y < 1 || y >= Hh - 1) return;
    const float4 gm = __ldg(isa::row_ptr(g_mask, tb.sp, y) + x);
    const float4 ax = __ldg(isa::row_ptr(aux, tb.sp, y) + x);
    if (ax.w == 0.f || (gm.x == 0.f && gm.y == 0.f && gm.z == 0.f)) return;
    const float2 sf = flow_sample(flow, flow_pitch, Wf, Hf, Wh, Hh, x, y);
    int shx, shy;
    float bx, by;
    moved_offset<true>(sf, shx, shy, bx, by);
    float B[4][3];
#pragma unroll
    for (int k = 0; k < 4; k++) moved_mean(tb, mov3, img_pitch, Wh, Hh, x + shx + (k & 1), y + shy + (k >> 1), B[k]);
    float mm[3];
    const float w0 = (1.f - bx) * (1.f - by);
#pragma unroll
    for (int c = 0; c < 3; c++) mm[c] = B[0][c] * w0;
#pragma unroll
    for (int k = 1; k < 4; k++) {
        const float wk = ((k & 1) ? bx : 1.f - bx) * ((k >> 1) ? by : 1.f - by);
        if (wk == 0.f) continue;
#pragma unroll
        for (int c = 0; c < 3; c++) mm[c] += wk * B[k][c];
    }
    const float4 r4 = __ldg(isa::row_ptr(tb.mr, tb.sp, y) + x), s4 = __ldg(isa::row_ptr(tb.sr, tb.sp, y) + x);
    const float mr[3] = {r4.x, r4.y, r4.z}, sr3[3] = {s4.x, s4.y, s4.z}, g[3] = {gm.x, gm.y, gm.z}, E[3] = {ax.x, ax.y, ax.z};
    float ghx = 0.f, ghy = 0.f;
#pragma unroll
    for (int c = 0; c < 3; c++) {
        const float raw = ax.w * E[c] - t_lit;
        if (g[c] == 0.f || !(raw > 0.f && raw < 1.f)) continue;
        const float sr = sr3[c];
        float smd = sqrtf(alpha * mr[c] + beta);
        if (c == 1) smd /= sqrtf(2.0f);
        const float sig = fmaxf(smd, sr);
        const float kc = sr * sr / (sr * sr + smd * smd);
        const float dist = fabsf(mr[c] - mm[c]) * kc;
        const float sgn = mm[c] > mr[c] ? 1.f : (mm[c] < mr[c] ? -1.f : 0.f);
        const float gmm = g[c] * ax.w * E[c] * (-2.f * dist / (sig * sig)) * kc * sgn;
        ghx += gmm * ((1.f - by) * (B[1][c] - B[0][c]) + by * (B[3][c] - B[2][c]));
        ghy += gmm * ((1.f - bx) * (B[2][c] - B[0][c]) + bx * (B[3][c] - B[1][c]));
    }
    // the transpose of flow_sample at the half-res pixel
    const float xb = ((float)x + 0.5f) / (float)Wh * Wf - 0.5f, yb = ((float)y + 0.5f) / (float)Hh * Hf - 0.5f;
    const float fx = floorf(xb), fy = floorf(yb);
    const int i = (int)fx, j = (int)fy;
    const float a = xb - fx, b = yb - fy;
    const int i0 = isa::mirror(i, Wf), i1 = isa::mirror(i + 1, Wf), j0 = isa::mirror(j, Hf), j1 = isa::mirror(j + 1, Hf);
    const float w[4] = {(1.f - a) * (1.f - b), a * (1.f - b), (1.f - a) * b, a * b};
    const int xs[4] = {i0, i1, i0, i1}, ys[4] = {j0, j0, j1, j1};
#pragma unroll
    for (int k = 0; k < 4; k++) {
        if (w[k] == 0.f) continue;
        float* d = (float*)(isa::row_ptr(gflow, flow_pitch, ys[k]) + xs[k]);
        atomicAdd(d, w[k] * 0.5f * ghx);
        atomicAdd(d + 1, w[k] * 0.5f * ghy);
    }
}

inline dim3 grid2(int w, int h, dim3 b) { return dim3((w + b.x - 1) / b.x, (h + b.y - 1) / b.y); }

}  // namespace

cudaError_t isa_launch_robustness(const float* ref3, const float* mov3, size_t img_pitch, float4* mask, size_t mask_pitch, int Wh, int Hh,
                                  const float2* flow, size_t flow_pitch, int Wf, int Hf, float alpha, float beta, float thr_m, float s,
                                  float t, cudaStream_t st)
{
    dim3 b(32, 8);
    k_robustness<<<grid2(Wh, Hh, b), b, 0, st>>>(ref3, mov3, img_pitch, mask, mask_pitch, Wh, Hh, flow, flow_pitch, Wf, Hf, alpha, beta,
                                                 thr_m, s, t);
    return cudaGetLastError();
}

cudaError_t isa_launch_erode(const float4* in, size_t in_pitch, float4* out, size_t out_pitch, int W, int H, int size, cudaStream_t st)
{
    dim3 b(32, 8);
    k_erode<<<grid2(W, H, b), b, 0, st>>>(in, in_pitch, out, out_pitch, W, H, size);
    return cudaGetLastError();
}

// Fused mask + erosion from half-res RGB images.
cudaError_t isa_launch_robustness_erode(const float* ref3, const float* mov3, size_t img_pitch, int Wh, int Hh, const float2* flow,
                                        size_t flow_pitch, int Wf, int Hf, float alpha, float beta, float thr_m, float s, float t, int size,
                                        float4* out, size_t out_pitch, cudaStream_t st)
{
    if (size < 1 || size / 2 > RB_MAXA) return cudaErrorInvalidValue;
    dim3 b(RB_TX, RB_TY);
    k_robustness_erode<<<grid2(Wh, Hh, b), b, 0, st>>>(ref3, mov3, img_pitch, Wh, Hh, flow, flow_pitch, Wf, Hf, alpha, beta, thr_m, s, t, size,
                                                       out, out_pitch);
    return cudaGetLastError();
}

cudaError_t isa_launch_ref_stats(const float* ref3, size_t img_pitch, int Wh, int Hh, float4* mr, float4* sr, size_t sp, cudaStream_t st)
{
    dim3 b(32, 8);
    k_ref_stats<<<grid2(Wh, Hh, b), b, 0, st>>>(ref3, img_pitch, Wh, Hh, mr, sr, sp);
    return cudaGetLastError();
}

cudaError_t isa_launch_box3(const float* mov3, size_t img_pitch, int Wh, int Hh, float4* box, size_t sp, cudaStream_t st)
{
    dim3 b(32, 8);
    k_box3<<<grid2(Wh, Hh, b), b, 0, st>>>(mov3, img_pitch, Wh, Hh, box, sp);
    return cudaGetLastError();
}

cudaError_t isa_launch_robustness_erode_tabs(const float4* mr, const float4* sr, const float4* box, size_t sp, const float* mov3, size_t img_pitch,
                                             int Wh, int Hh, const float2* flow, size_t flow_pitch, int Wf, int Hf, float alpha, float beta,
                                             float thr_m, float s, float t, int size, float4* out, size_t out_pitch, int bil, cudaStream_t st)
{
    if (size < 1 || size / 2 > RB_MAXA) return cudaErrorInvalidValue;
    RobustTabs tb{mr, sr, box, sp};
    dim3 g((Wh + RF_T - 1) / RF_T, (Hh + RF_T - 1) / RF_T);
    if (bil)
        k_robustness_erode_fast<true><<<g, 256, 0, st>>>(tb, mov3, img_pitch, Wh, Hh, flow, flow_pitch, Wf, Hf, alpha, beta, thr_m, s, t, size, out,
                                                         out_pitch);
    else
        k_robustness_erode_fast<false><<<g, 256, 0, st>>>(tb, mov3, img_pitch, Wh, Hh, flow, flow_pitch, Wf, Hf, alpha, beta, thr_m, s, t, size, out,
                                                          out_pitch);
    return cudaGetLastError();
}

cudaError_t isa_launch_mask_store(const float4* mr, const float4* sr, const float4* box, size_t sp, const float* mov3, size_t img_pitch, int Wh,
                                  int Hh, const float2* flow, size_t flow_pitch, int Wf, int Hf, float alpha, float beta, float thr_m, float s,
                                  float t, float4* m_out, float4* aux_out, int bil, cudaStream_t st)
{
    RobustTabs tb{mr, sr, box, sp};
    dim3 b(32, 8);
    if (bil)
        k_mask_store<true><<<grid2(Wh, Hh, b), b, 0, st>>>(tb, mov3, img_pitch, Wh, Hh, flow, flow_pitch, Wf, Hf, alpha, beta, thr_m, s, t, m_out,
                                                           aux_out, sp);
    else
        k_mask_store<false><<<grid2(Wh, Hh, b), b, 0, st>>>(tb, mov3, img_pitch, Wh, Hh, flow, flow_pitch, Wf, Hf, alpha, beta, thr_m, s, t, m_out,
                                                            aux_out, sp);
    return cudaGetLastError();
}

cudaError_t isa_launch_mask_flow_bwd(const float4* mr, const float4* sr, const float4* box, size_t sp, const float* mov3, size_t img_pitch, int Wh,
                                     int Hh, const float2* flow, size_t flow_pitch, int Wf, int Hf, float alpha, float beta, float t,
                                     const float4* aux, const float4* g_mask, float2* gflow, cudaStream_t st)
{
    RobustTabs tb{mr, sr, box, sp};
    dim3 b(32, 8);
    k_mask_flow_bwd<<<grid2(Wh, Hh, b), b, 0, st>>>(tb, mov3, img_pitch, Wh, Hh, flow, flow_pitch, Wf, Hf, alpha, beta, t, aux, g_mask, gflow);
    return cudaGetLastError();
}

cudaError_t isa_launch_erode_route(const float4* m, const float4* g_eroded, size_t sp, int Wh, int Hh, int size, float4* g_mask, cudaStream_t st)
{
    dim3 b(32, 8);
    k_erode_route<<<grid2(Wh, Hh, b), b, 0, st>>>(m, g_eroded, sp, Wh, Hh, size, g_mask);
    return cudaGetLastError();
}

cudaError_t isa_launch_mask_param_bwd(const float4* m, const float4* aux, const float4* g_mask, size_t sp, int Wh, int Hh, float t, double* grad2,
                                      cudaStream_t st)
{
    dim3 b(32, 8);
    k_mask_param_bwd<<<grid2(Wh, Hh, b), b, 0, st>>>(m, aux, g_mask, sp, Wh, Hh, t, grad2);
    return cudaGetLastError();
}
