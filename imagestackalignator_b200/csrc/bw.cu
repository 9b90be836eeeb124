// Tracking-image preparation and demosaic kernels.
//
// k_demosaic_gray fuses, for one output tile, what the reference runs as
// NPP Convert + Set(0) + deBayerGreenKernel + deBayerRedBlueKernel + NPP Div
// (ImageStackAlignatorController.cs:1268-1311, DeBayerKernels.cu:55-231)
// and, for tracking images, GammasRGB (kernel.cu:290-332) + NPP ColorToGray
// (controller :2404-2408). The raw tile with a 3-pixel halo is staged in
// shared memory as linear values, the green plane is built over a 1-pixel
// halo, then red/blue by colour differences.
#include "isa_internal.cuh"

namespace {

constexpr int DM_TX = 58, DM_TY = 16;                // output tile (58 + 6 = 32 pixel pairs of halo'd tile)
constexpr int DM_LW = DM_TX + 6, DM_LH = DM_TY + 6;  // linear tile (halo 3)
constexpr int DM_GW = DM_TX + 2, DM_GH = DM_TY + 2;  // green tile (halo 1)

struct Color3 { float v[3]; };

__device__ __forceinline__ float srgb_gamma(float v) {
    return v <= 0.0031308f ? 12.92f * v : (1.0f + 0.055f) * powf(v, 1.0f / 2.4f) - 0.055f;
}

// The same curve with the power evaluated as exp2(log2(v) / 2.4) (hardware
// log2 approximation; relative error about 3e-7 on [0.0031308, 1]).
__device__ __forceinline__ float srgb_gamma_fast(float v) {
    return v <= 0.0031308f ? 12.92f * v : (1.0f + 0.055f) * exp2f(__log2f(v) * (1.0f / 2.4f)) - 0.055f;
}

// Thread (tx, ty) of a (32, 8) block works on pixel pairs (2 tx, 2 tx + 1)
// of a row: the column parity of each pixel of the pair is a compile-time
// constant and the row parity is the same for the whole warp, so the CFA
// colour, and with it every branch below, is uniform across the warp.
__global__ void __launch_bounds__(256) k_demosaic_gray(const uint16_t* __restrict__ raw, size_t raw_pitch, int W, int H, unsigned cfa,
                                                      Color3 black, Color3 scale, Color3 rdivisor, Color3 gw, int gamma_gray,
                                                      float* __restrict__ gray, size_t gray_pitch, float* __restrict__ rgb,
                                                      size_t rgb_pitch, bool vec_gray, bool vec_rgb)
{
    __shared__ float lin[DM_LH][DM_LW];
    __shared__ float grn[DM_GH][DM_GW];
    const int x0 = blockIdx.x * DM_TX, y0 = blockIdx.y * DM_TY;  // x0, y0 even
    const int tx = threadIdx.x, ty = threadIdx.y;
    // 1. black-subtracted, white-balanced linear values with a 3-pixel halo
    for (int ly = ty; ly < DM_LH; ly += 8) {
        const int gy = y0 + ly - 3;
        const bool yin = gy >= 0 && gy < H;
        const uint16_t* rr = isa::row_ptr(raw, raw_pitch, yin ? gy : 0);
        // colours of the two columns of a pair on this row (odd, then even image column)
        float bl[2], sc[2];
#pragma unroll
        for (int k = 0; k < 2; k++) {
            const int c = isa::cfa_at(cfa, k + 1, gy);
            bl[k] = c == 0 ? black.v[0] : (c == 1 ? black.v[1] : black.v[2]);
            sc[k] = c == 0 ? scale.v[0] : (c == 1 ? scale.v[1] : scale.v[2]);
        }
        for (int pi = tx; pi < DM_LW / 2; pi += 32) {
#pragma unroll
            for (int k = 0; k < 2; k++) {
                const int lx = 2 * pi + k, gx = x0 + lx - 3;
                float v = 0.f;
                if (yin && gx >= 0 && gx < W) v = ((float)__ldg(rr + gx) - bl[k]) * sc[k];
                lin[ly][lx] = v;
            }
        }
    }
    __syncthreads();
    // 2. green plane (Wu-Zhang gradient-weighted interpolation) with a 1-pixel halo
    for (int ly = ty; ly < DM_GH; ly += 8) {
        const int gy = y0 + ly - 1;
        for (int pi = tx; pi < DM_GW / 2; pi += 32) {
#pragma unroll
            for (int k = 0; k < 2; k++) {
                const int lx = 2 * pi + k, gx = x0 + lx - 1;
                float g = 0.f;
                if (gx >= 2 && gx < W - 2 && gy >= 2 && gy < H - 2) {
                    const int c = isa::cfa_at(cfa, gx, gy);
                    const int cx = lx + 2, cy = ly + 2;  // position in lin
                    if (c == 1) {
                        g = lin[cy][cx];
                    } else if (c == 0 || c == 2) {
                        const float p = lin[cy][cx];
                        const float xm2 = lin[cy][cx - 2], xm1 = lin[cy][cx - 1], xp1 = lin[cy][cx + 1], xp2 = lin[cy][cx + 2];
                        const float ym2 = lin[cy - 2][cx], ym1 = lin[cy - 1][cx], yp1 = lin[cy + 1][cx], yp2 = lin[cy + 2][cx];
                        const float gradX = 0.5f * fabsf(xp1 - xm1), gradY = 0.5f * fabsf(yp1 - ym1);
                        const float lapX = 0.25f * fabsf(2.0f * p - xm2 - xp2), lapY = 0.25f * fabsf(2.0f * p - ym2 - yp2);
                        const float ipX = 0.125f * (-xm2 + 4.0f * xm1 + 2.0f * p + 4.0f * xp1 - xp2);
                        const float ipY = 0.125f * (-ym2 + 4.0f * ym1 + 2.0f * p + 4.0f * yp1 - yp2);
                        const float w = __fdividef(gradY + lapY, gradX + gradY + lapX + lapY + 0.000000001f);
                        g = w * ipX + (1.0f - w) * ipY;
                    }
                }
                grn[ly][lx] = g;
            }
        }
    }
    __syncthreads();
    // 3. red and blue by colour differences, removal of the white balance, output
    if (tx >= DM_TX / 2) return;
    for (int ly = ty; ly < DM_TY; ly += 8) {
        const int gy = y0 + ly;
        if (gy >= H) break;
        float o[2][3];
#pragma unroll
        for (int k = 0; k < 2; k++) {
            const int lx = 2 * tx + k, gx = x0 + lx;
            float r = 0.f, g = 0.f, b = 0.f;
            if (gx >= 2 && gx < W - 2 && gy >= 2 && gy < H - 2) {
                const int c = isa::cfa_at(cfa, gx, gy);
                const int nx = isa::cfa_at(cfa, gx + 1, gy);
                const int cx = lx + 3, cy = ly + 3;  // lin
                const int kx = lx + 1, ky = ly + 1;  // grn
                g = grn[ky][kx];
                if (c == 1) {
                    const float hsum = (lin[cy][cx - 1] - grn[ky][kx - 1]) + (lin[cy][cx + 1] - grn[ky][kx + 1]);
                    const float vsum = (lin[cy - 1][cx] - grn[ky - 1][kx]) + (lin[cy + 1][cx] - grn[ky + 1][kx]);
                    const float h = g + 0.5f * hsum, v = g + 0.5f * vsum;
                    if (nx == 0) { r = h; b = v; } else { b = h; r = v; }
                } else if (c == 0 || c == 2) {
                    const float own = lin[cy][cx];
                    const float other = g + 0.25f * ((lin[cy - 1][cx - 1] - grn[ky - 1][kx - 1]) + (lin[cy - 1][cx + 1] - grn[ky - 1][kx + 1]) +
                                                     (lin[cy + 1][cx + 1] - grn[ky + 1][kx + 1]) + (lin[cy + 1][cx - 1] - grn[ky + 1][kx - 1]));
                    if (c == 0) { r = own; b = other; } else { b = own; r = other; }
                }
            }
            o[k][0] = r * rdivisor.v[0];
            o[k][1] = g * rdivisor.v[1];
            o[k][2] = b * rdivisor.v[2];
        }
        const int gx0 = x0 + 2 * tx;
        if (gx0 >= W) continue;  // W is even: both pixels of the pair are inside or outside together
        if (rgb) {
            float* op = isa::row_ptr(rgb, rgb_pitch, gy) + 3 * gx0;
            if (vec_rgb) {
                ((float2*)op)[0] = make_float2(o[0][0], o[0][1]);
                ((float2*)op)[1] = make_float2(o[0][2], o[1][0]);
                ((float2*)op)[2] = make_float2(o[1][1], o[1][2]);
            } else {
#pragma unroll
                for (int k = 0; k < 6; k++) op[k] = o[k / 3][k % 3];
            }
        }
        if (gray) {
            float q[2];
#pragma unroll
            for (int k = 0; k < 2; k++) {
                float r = o[k][0], g = o[k][1], b = o[k][2];
                if (gamma_gray) {
                    r = isnan(r) ? 0.f : r; g = isnan(g) ? 0.f : g; b = isnan(b) ? 0.f : b;
                    r = srgb_gamma_fast(fmaxf(fminf(r, 1.0f), 0.0f));
                    g = srgb_gamma_fast(fmaxf(fminf(g, 1.0f), 0.0f));
                    b = srgb_gamma_fast(fmaxf(fminf(b, 1.0f), 0.0f));
                }
                q[k] = gw.v[0] * r + gw.v[1] * g + gw.v[2] * b;
            }
            float* gp = isa::row_ptr(gray, gray_pitch, gy) + gx0;
            if (vec_gray) *(float2*)gp = make_float2(q[0], q[1]);
            else { gp[0] = q[0]; gp[1] = q[1]; }
        }
    }
}

// GammasRGB (kernel.cu:303-332) on an RGB image.
__global__ void k_gamma(float* rgb, size_t pitch, int W, int H)
{
    int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= W || y >= H) return;
    float* p = isa::row_ptr(rgb, pitch, y) + 3 * x;
    for (int c = 0; c < 3; c++) {
        float v = p[c];
        if (isnan(v)) v = 0.f;
        p[c] = srgb_gamma(fmaxf(fminf(v, 1.0f), 0.0f));
    }
}

// fourierFilter (kernel.cu:704-779) on a batch of half spectra; post_scale
// folds in the 1/(W*H) of the inverse transform (PreAlignment.cs:277).
__global__ void k_fourier_filter(float2* spec, size_t pitch, size_t batch_stride, int W, int H, float lp, float hp, float lps, float hps,
                                 int clear_axis, float post_scale)
{
    int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= W / 2 + 1 || y >= H) return;
    float fil = isa::fourier_mask(x, y, W, H, lp, hp, lps, hps, clear_axis);
    fil *= post_scale;
    float2* p = (float2*)((char*)spec + blockIdx.z * batch_stride + (size_t)y * pitch) + x;
    float2 v = *p;
    v.x *= fil;
    v.y *= fil;
    *p = v;
}

struct Taps { float t[100]; int n; };

// One pass of NPP FilterGaussBorder (separable, replicate border).
template <bool VERT>
__global__ void k_gauss_pass(const float* __restrict__ in, size_t in_pitch, float* __restrict__ out, size_t out_pitch, int W, int H, int C,
                             Taps taps, int clamp_in)
{
    int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= W * C || y >= H) return;
    int px = x / C, c = x - px * C;
    int c0 = taps.n / 2;
    float s = 0.f;
    for (int k = 0; k < taps.n; k++) {
        int sx = VERT ? px : isa::clampi(px + k - c0, 0, W - 1);
        int sy = VERT ? isa::clampi(y + k - c0, 0, H - 1) : y;
        float v = isa::row_ptr(in, in_pitch, sy)[sx * C + c];
        if (clamp_in) v = v < 0.f ? 0.f : (v > 1.f ? 1.f : v);
        s = fmaf(taps.t[k], v, s);
    }
    isa::row_ptr(out, out_pitch, y)[x] = s;
}

// Both passes of the separable Gauss in one launch for one channel and
// radius R <= 4: the input tile with an R halo (replicate border, optional
// clamp to [0, 1]) and the horizontally filtered rows live in shared memory.
// The arithmetic and its order are those of the two k_gauss_pass launches,
// so the result is the same; HBM traffic is one read and one write.
constexpr int G2_TX = 128, G2_TY = 32;

template <int R>
__global__ void __launch_bounds__(256) k_gauss2d(const float* __restrict__ in, size_t in_pitch, float* __restrict__ out, size_t out_pitch, int W,
                                                 int H, Taps taps, int clamp_in)
{
    constexpr int SW = G2_TX + 2 * R, SH = G2_TY + 2 * R, NT = 2 * R + 1;
    __shared__ float s_in[SH][SW];
    __shared__ float s_h[SH][G2_TX];
    const int x0 = blockIdx.x * G2_TX, y0 = blockIdx.y * G2_TY;
    const int tid = threadIdx.x;
    float t[NT];
#pragma unroll
    for (int k = 0; k < NT; k++) t[k] = taps.t[k];
    // all loads of a thread are issued before its stores (compile-time trip counts)
    constexpr int RY = (SH + 7) / 8, RX = (SW + 31) / 32;
    float v[RY][RX];
    const int lane = tid & 31, wy = tid >> 5;
    int cx[RX];
#pragma unroll
    for (int k = 0; k < RX; k++) cx[k] = isa::clampi(x0 - R + lane + 32 * k, 0, W - 1);
#pragma unroll
    for (int j = 0; j < RY; j++) {
        const int yy = wy + 8 * j;
        if (yy < SH) {
            const float* row = isa::row_ptr(in, in_pitch, isa::clampi(y0 - R + yy, 0, H - 1));
#pragma unroll
            for (int k = 0; k < RX; k++)
                if (lane + 32 * k < SW) v[j][k] = __ldg(row + cx[k]);
        }
    }
#pragma unroll
    for (int j = 0; j < RY; j++) {
        const int yy = wy + 8 * j;
        if (yy < SH) {
#pragma unroll
            for (int k = 0; k < RX; k++)
                if (lane + 32 * k < SW) {
                    float q = v[j][k];
                    if (clamp_in) q = q < 0.f ? 0.f : (q > 1.f ? 1.f : q);
                    s_in[yy][lane + 32 * k] = q;
                }
        }
    }
    __syncthreads();
    for (int yy = tid >> 5; yy < SH; yy += 8)
        for (int xx = tid & 31; xx < G2_TX; xx += 32) {
            float s = 0.f;
#pragma unroll
            for (int k = 0; k < NT; k++) s = fmaf(t[k], s_in[yy][xx + k], s);
            s_h[yy][xx] = s;
        }
    __syncthreads();
    for (int yy = tid >> 5; yy < G2_TY; yy += 8) {
        const int y = y0 + yy;
        if (y >= H) break;
        float* orow = isa::row_ptr(out, out_pitch, y);
        for (int xx = tid & 31; xx < G2_TX; xx += 32) {
            const int x = x0 + xx;
            if (x >= W) break;
            float s = 0.f;
#pragma unroll
            for (int k = 0; k < NT; k++) s = fmaf(t[k], s_h[yy + k][xx], s);
            orow[x] = s;
        }
    }
}

// NPP ResizeSqrPixel super-sampling by an integer factor: block mean.
__global__ void k_resize_box(const float* __restrict__ in, size_t in_pitch, int L, float* __restrict__ out, size_t out_pitch, int Wo, int Ho)
{
    int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= Wo || y >= Ho) return;
    float s = 0.f;
    for (int j = 0; j < L; j++) {
        const float* r = isa::row_ptr(in, in_pitch, y * L + j) + x * L;
        for (int i = 0; i < L; i++) s += r[i];
    }
    isa::row_ptr(out, out_pitch, y)[x] = s / (float)(L * L);
}

// The 2x, 4x and 8x box means of one image from a single read: a thread owns
// an 8 x 8 block and sums each output's L x L pixels in the order of
// k_resize_box (rows, then columns, from 0), so the values are identical.
__global__ void k_pyramid248(const float* __restrict__ in, size_t in_pitch, int W, int H, float* __restrict__ o2, size_t p2, float* __restrict__ o4,
                             size_t p4, float* __restrict__ o8, size_t p8)
{
    const int bx = blockIdx.x * blockDim.x + threadIdx.x, by = blockIdx.y * blockDim.y + threadIdx.y;
    const int x0 = 8 * bx, y0 = 8 * by;
    if (x0 >= W - 1 || y0 >= H - 1) return;  // no 2x2 output starts here
    float v[8][8];
    const bool full = x0 + 8 <= W && y0 + 8 <= H && ((((uintptr_t)in) | in_pitch) & 15) == 0;
#pragma unroll
    for (int j = 0; j < 8; j++) {
        const float* r = isa::row_ptr(in, in_pitch, min(y0 + j, H - 1)) + x0;
        if (full) {
            const float4 a = __ldg((const float4*)r), b = __ldg((const float4*)r + 1);
            v[j][0] = a.x; v[j][1] = a.y; v[j][2] = a.z; v[j][3] = a.w; v[j][4] = b.x; v[j][5] = b.y; v[j][6] = b.z; v[j][7] = b.w;
        } else {
#pragma unroll
            for (int i = 0; i < 8; i++) v[j][i] = x0 + i < W ? __ldg(r + i) : 0.f;
        }
    }
    const int W2 = W / 2, H2 = H / 2, W4 = W / 4, H4 = H / 4, W8 = W / 8, H8 = H / 8;
#pragma unroll
    for (int qy = 0; qy < 4; qy++)
#pragma unroll
        for (int qx = 0; qx < 4; qx++) {
            const int x = 4 * bx + qx, y = 4 * by + qy;
            if (x < W2 && y < H2) {
                float s = 0.f;
#pragma unroll
                for (int j = 0; j < 2; j++)
#pragma unroll
                    for (int i = 0; i < 2; i++) s += v[2 * qy + j][2 * qx + i];
                isa::row_ptr(o2, p2, y)[x] = s / 4.0f;
            }
        }
#pragma unroll
    for (int qy = 0; qy < 2; qy++)
#pragma unroll
        for (int qx = 0; qx < 2; qx++) {
            const int x = 2 * bx + qx, y = 2 * by + qy;
            if (x < W4 && y < H4) {
                float s = 0.f;
#pragma unroll
                for (int j = 0; j < 4; j++)
#pragma unroll
                    for (int i = 0; i < 4; i++) s += v[4 * qy + j][4 * qx + i];
                isa::row_ptr(o4, p4, y)[x] = s / 16.0f;
            }
        }
    if (bx < W8 && by < H8) {
        float s = 0.f;
#pragma unroll
        for (int j = 0; j < 8; j++)
#pragma unroll
            for (int i = 0; i < 8; i++) s += v[j][i];
        isa::row_ptr(o8, p8, by)[bx] = s / 64.0f;
    }
}

// deBayersSubSample3 (DeBayerKernels.cu:244-283).
__global__ void k_subsample(const uint16_t* __restrict__ raw, size_t raw_pitch, int Wh, int Hh, unsigned cfa, float max_val,
                            float* __restrict__ out, size_t out_pitch)
{
    int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= Wh || y >= Hh) return;
    float f = 1.0f / max_val;
    float p[3] = {0.f, 0.f, 0.f};
    for (int ix = 0; ix < 2; ix++)
        for (int iy = 0; iy < 2; iy++) {
            int c = isa::cfa_at(cfa, ix, iy);
            float v = (float)isa::row_ptr(raw, raw_pitch, 2 * y + iy)[2 * x + ix];
            if (c == 1) p[1] += v * f * 0.5f;
            else if (c == 0) p[0] = v * f;
            else if (c == 2) p[2] = v * f;
        }
    float* o = isa::row_ptr(out, out_pitch, y) + 3 * x;
    o[0] = p[0]; o[1] = p[1]; o[2] = p[2];
}

inline dim3 grid2(int w, int h, dim3 b) { return dim3((w + b.x - 1) / b.x, (h + b.y - 1) / b.y); }

}  // namespace

cudaError_t isa_launch_demosaic_gray(const uint16_t* raw, size_t raw_pitch, int W, int H, unsigned cfa, const float* black,
                                     const float* scale, const float* divisor, const float* gray_w, int gamma_gray,
                                     float* gray, size_t gray_pitch, float* rgb, size_t rgb_pitch, cudaStream_t st)
{
    Color3 b, s, d, g;
    for (int c = 0; c < 3; c++) { b.v[c] = black[c]; s.v[c] = scale[c]; d.v[c] = (float)(1.0 / (double)divisor[c]); g.v[c] = gray_w ? gray_w[c] : 0.f; }
    if (W & 1) return cudaErrorInvalidValue;
    // pixel pairs are stored as float2 where rows are 8-byte aligned
    const bool vg = !((gray_pitch & 7) || ((uintptr_t)gray & 7)), vr = !((rgb_pitch & 7) || ((uintptr_t)rgb & 7));
    dim3 blk(32, 8), grd((W + DM_TX - 1) / DM_TX, (H + DM_TY - 1) / DM_TY);
    k_demosaic_gray<<<grd, blk, 0, st>>>(raw, raw_pitch, W, H, cfa, b, s, d, g, gamma_gray, gray, gray_pitch, rgb, rgb_pitch, vg, vr);
    return cudaGetLastError();
}

cudaError_t isa_launch_gamma(float* rgb, size_t pitch, int W, int H, cudaStream_t st)
{
    dim3 b(32, 8);
    k_gamma<<<grid2(W, H, b), b, 0, st>>>(rgb, pitch, W, H);
    return cudaGetLastError();
}

cudaError_t isa_launch_fourier_filter(float2* spec, size_t pitch, int W, int H, int batch, size_t batch_stride, float lp, float hp,
                                      float lps, float hps, int clear_axis, float post_scale, cudaStream_t st)
{
    dim3 b(32, 8);
    dim3 g = grid2(W / 2 + 1, H, b);
    g.z = batch;
    k_fourier_filter<<<g, b, 0, st>>>(spec, pitch, batch_stride, W, H, lp, hp, lps, hps, clear_axis, post_scale);
    return cudaGetLastError();
}

cudaError_t isa_launch_gauss(const float* in, size_t in_pitch, float* out, size_t out_pitch, float* tmp, size_t tmp_pitch, int W, int H,
                             int C, const float* taps, int ntaps, int clamp01_input, cudaStream_t st)
{
    if (ntaps < 1 || ntaps > 99) return cudaErrorInvalidValue;
    Taps t;
    t.n = ntaps;
    for (int i = 0; i < ntaps; i++) t.t[i] = taps[i];
    if (C == 1 && in != out && (ntaps & 1) && ntaps <= 9) {
        dim3 g((W + G2_TX - 1) / G2_TX, (H + G2_TY - 1) / G2_TY);
        switch (ntaps / 2) {
        case 0: k_gauss2d<0><<<g, 256, 0, st>>>(in, in_pitch, out, out_pitch, W, H, t, clamp01_input); break;
        case 1: k_gauss2d<1><<<g, 256, 0, st>>>(in, in_pitch, out, out_pitch, W, H, t, clamp01_input); break;
        case 2: k_gauss2d<2><<<g, 256, 0, st>>>(in, in_pitch, out, out_pitch, W, H, t, clamp01_input); break;
        case 3: k_gauss2d<3><<<g, 256, 0, st>>>(in, in_pitch, out, out_pitch, W, H, t, clamp01_input); break;
        default: k_gauss2d<4><<<g, 256, 0, st>>>(in, in_pitch, out, out_pitch, W, H, t, clamp01_input); break;
        }
        return cudaGetLastError();
    }
    dim3 b(64, 4);
    k_gauss_pass<false><<<grid2(W * C, H, b), b, 0, st>>>(in, in_pitch, tmp, tmp_pitch, W, H, C, t, clamp01_input);
    k_gauss_pass<true><<<grid2(W * C, H, b), b, 0, st>>>(tmp, tmp_pitch, out, out_pitch, W, H, C, t, 0);
    return cudaGetLastError();
}

cudaError_t isa_launch_resize_box(const float* in, size_t in_pitch, int W, int H, int L, float* out, size_t out_pitch, cudaStream_t st)
{
    int Wo = W / L, Ho = H / L;
    dim3 b(32, 8);
    k_resize_box<<<grid2(Wo, Ho, b), b, 0, st>>>(in, in_pitch, L, out, out_pitch, Wo, Ho);
    return cudaGetLastError();
}

cudaError_t isa_launch_subsample(const uint16_t* raw, size_t raw_pitch, int W, int H, unsigned cfa, float max_val, float* out,
                                 size_t out_pitch, cudaStream_t st)
{
    dim3 b(32, 8);
    k_subsample<<<grid2(W / 2, H / 2, b), b, 0, st>>>(raw, raw_pitch, W / 2, H / 2, cfa, max_val, out, out_pitch);
    return cudaGetLastError();
}

cudaError_t isa_launch_pyramid248(const float* in, size_t in_pitch, int W, int H, float* o2, size_t p2, float* o4, size_t p4, float* o8, size_t p8,
                                  cudaStream_t st)
{
    dim3 b(32, 8);
    k_pyramid248<<<grid2((W + 7) / 8, (H + 7) / 8, b), b, 0, st>>>(in, in_pitch, W, H, o2, p2, o4, p4, o8, p8);
    return cudaGetLastError();
}
