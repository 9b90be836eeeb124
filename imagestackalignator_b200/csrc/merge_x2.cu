// Kernel-weighted Bayer accumulation at merge scale 2 (the reference's
// accumulateImagesSuperRes, DeBayerKernels.cu:379-468, and its whole-frame
// generalisation), restructured for issue efficiency.
//
// At s = 2 the 5 x 5 taps of an output pixel read only a 3 x 3 block of
// source samples: tap px reads column ((Xs + px) >> 1) with Xs = X + sx, so
// relative to k0 = (Xs - 2) >> 1 the tap -> column map is 0 0 1 1 2 for even
// Xs and 0 1 1 2 2 for odd Xs (same for rows). Per frame the kernel loads the
// 3 x 3 samples and the <= 2 x 2 half-resolution mask cells once, then runs a
// tap loop specialised on the parity of (Xs, Ys), so every tap's source
// sample and CFA parity class are compile-time registers. Sums are kept per
// parity class relative to (k0, j0) and folded into colours once per frame:
//   acc_c += (sum w cert raw - black_c sum w cert) / white_c,  wsum_c += sum w cert
// which equals the reference's per-tap sum of (raw - black_c) / white_c * w * cert.
// Output pixels whose 3 x 3 block or mask window reaches the crop border take
// the per-tap path with the reference's clamps.
//
// Threads: a warp covers 32 output pixels of one row with stride 2, so the
// parity of X is uniform in the warp and the parity of Xs changes only where
// round(2 * flow) changes between neighbouring pixels.
#include "isa_internal.cuh"

namespace {

struct C3 { float v[3]; };

template <int P>
__device__ __forceinline__ constexpr int cell_of(int p) { return P ? (p + 3) >> 1 : (p + 2) >> 1; }

__device__ __forceinline__ float comp(const float4& m, int ch) { return ch == 0 ? m.x : (ch == 1 ? m.y : m.z); }

__device__ __forceinline__ float4 sanitize(float4 m)
{
    m.x = isfinite(m.x) ? m.x : 0.f;
    m.y = isfinite(m.y) ? m.y : 0.f;
    m.z = isfinite(m.z) ? m.z : 0.f;
    return m;
}

__device__ __forceinline__ float2 flow_at(const float2* fl, size_t pitch, int W, int H, float xb, float yb)
{
    float fx = floorf(xb), fy = floorf(yb);
    int i = (int)fx, j = (int)fy;
    float a = xb - fx, b = yb - fy;
    int i0 = isa::mirror(i, W), i1 = isa::mirror(i + 1, W), j0 = isa::mirror(j, H), j1 = isa::mirror(j + 1, H);
    const float2* r0 = isa::row_ptr(fl, pitch, j0);
    const float2* r1 = isa::row_ptr(fl, pitch, j1);
    float2 p00 = __ldg(r0 + i0), p10 = __ldg(r0 + i1), p01 = __ldg(r1 + i0), p11 = __ldg(r1 + i1);
    return make_float2(isa::lerp2(p00.x, p10.x, p01.x, p11.x, a, b), isa::lerp2(p00.y, p10.y, p01.y, p11.y, a, b));
}

// One frame's taps for the interior case; PX, PY = parity of Xs, Ys.
// v: 3 x 3 source samples (raw, not normalised); MC[dr][dc][r]: mask
// certainty of mask cell (dr, dc) for relative parity class r.
template <int PX, int PY>
__device__ __forceinline__ void frame_taps(const float (&w)[25], const float (&v)[3][3], const float (&MC)[2][2][4], unsigned mrow, unsigned mcol,
                                           float (&Ar)[4], float (&Wr)[4])
{
#pragma unroll
    for (int py = -2; py <= 2; py++) {
        const int j = cell_of<PY>(py);
        const int dr = (mrow >> (py + 2)) & 1;
        // the two classes of this row (column parity 0 / 1), both mask columns
        float c00 = dr ? MC[1][0][(j & 1) * 2] : MC[0][0][(j & 1) * 2];
        float c01 = dr ? MC[1][1][(j & 1) * 2] : MC[0][1][(j & 1) * 2];
        float c10 = dr ? MC[1][0][(j & 1) * 2 + 1] : MC[0][0][(j & 1) * 2 + 1];
        float c11 = dr ? MC[1][1][(j & 1) * 2 + 1] : MC[0][1][(j & 1) * 2 + 1];
#pragma unroll
        for (int px = -2; px <= 2; px++) {
            const int i = cell_of<PX>(px);
            const int r = (j & 1) * 2 + (i & 1);
            const int dc = (mcol >> (px + 2)) & 1;
            const float cert = (i & 1) ? (dc ? c11 : c10) : (dc ? c01 : c00);
            const float wc = w[(py + 2) * 5 + px + 2] * cert;
            Wr[r] += wc;
            Ar[r] = fmaf(wc, v[j][i], Ar[r]);
        }
    }
}

__global__ void __launch_bounds__(256, 2) k_accumulate_x2(isa_accum_geom g, unsigned cfa, const isa_frame_in* __restrict__ frames, int nframes,
                                                     isa_frame_in single, size_t raw_pitch, size_t flow_pitch, size_t mask_pitch,
                                                     const float4* __restrict__ kparam, size_t kp_pitch, C3 white, C3 black,
                                                     float* __restrict__ acc, float* __restrict__ wsum, size_t out_pitch, int accumulate_into)
{
    const int lane = threadIdx.x, wy = threadIdx.y;
    const int x = blockIdx.x * 64 + 2 * lane + (wy & 1);
    const int y = blockIdx.y * 4 + (wy >> 1);
    if (x >= g.Wo || y >= g.Ho) return;
    float* ap = isa::row_ptr(acc, out_pitch, y) + 3 * x;
    float* wp = isa::row_ptr(wsum, out_pitch, y) + 3 * x;
    if (x < 1 || y < 1 || x >= g.Wo - 1 || y >= g.Ho - 1) {
        if (!accumulate_into) { ap[0] = ap[1] = ap[2] = 0.f; wp[0] = wp[1] = wp[2] = 0.f; }
        return;
    }
    float a[3] = {0.f, 0.f, 0.f}, ws[3] = {0.f, 0.f, 0.f};
    if (accumulate_into) {
        a[0] = ap[0]; a[1] = ap[1]; a[2] = ap[2];
        ws[0] = wp[0]; ws[1] = wp[1]; ws[2] = wp[2];
    }
    const int X = x + g.ox, Y = y + g.oy;
    const float xb = ((float)x + 0.5f + (float)g.ox) / 2.0f - 0.5f;
    const float yb = ((float)y + 0.5f + (float)g.oy) / 2.0f - 0.5f;
    // kernel parameters: bilinear, clamp addressing
    float k0p, k1p, k2p;
    {
        float fx = floorf(xb), fy = floorf(yb);
        int i = (int)fx, j = (int)fy;
        float ax = xb - fx, by = yb - fy;
        int i0 = isa::clampi(i, 0, g.W - 1), i1 = isa::clampi(i + 1, 0, g.W - 1), j0 = isa::clampi(j, 0, g.H - 1), j1 = isa::clampi(j + 1, 0, g.H - 1);
        float4 p00 = __ldg(isa::row_ptr(kparam, kp_pitch, j0) + i0), p10 = __ldg(isa::row_ptr(kparam, kp_pitch, j0) + i1);
        float4 p01 = __ldg(isa::row_ptr(kparam, kp_pitch, j1) + i0), p11 = __ldg(isa::row_ptr(kparam, kp_pitch, j1) + i1);
        k0p = isa::lerp2(p00.x, p10.x, p01.x, p11.x, ax, by);
        k1p = isa::lerp2(p00.y, p10.y, p01.y, p11.y, ax, by);
        k2p = isa::lerp2(p00.z, p10.z, p01.z, p11.z, ax, by);
    }
    float w[25];
#pragma unroll
    for (int py = -2; py <= 2; py++)
#pragma unroll
        for (int px = -2; px <= 2; px++) {
            float q = px * px * k0p + 2 * px * py * k2p + py * py * k1p;
            float vv = expf(-0.5f * q);
            if (!isfinite(vv)) vv = px * py == 0 ? 1.f : 0.f;
            w[(py + 2) * 5 + px + 2] = vv;
        }
    // unshifted taps -> half-resolution mask cells (frame independent)
    const int ux0 = isa::clampi((X - 2) >> 1, g.cx0, g.cx1) >> 1, uy0 = isa::clampi((Y - 2) >> 1, g.cy0, g.cy1) >> 1;
    unsigned mcol = 0, mrow = 0;
    bool mask_interior = ((X - 2) >> 1) >= g.cx0 && ((X + 2) >> 1) <= g.cx1 && ((Y - 2) >> 1) >= g.cy0 && ((Y + 2) >> 1) <= g.cy1;
#pragma unroll
    for (int d = 0; d < 5; d++) {
        mcol |= (unsigned)((isa::clampi((X + d - 2) >> 1, g.cx0, g.cx1) >> 1) - ux0) << d;
        mrow |= (unsigned)((isa::clampi((Y + d - 2) >> 1, g.cy0, g.cy1) >> 1) - uy0) << d;
    }
    const int ux1 = ux0 + ((mcol >> 4) & 1), uy1 = uy0 + ((mrow >> 4) & 1);
    for (int f = 0; f < nframes; f++) {
        const isa_frame_in fr = frames ? frames[f] : single;
        int sx = 0, sy = 0;
        if (fr.flow) {
            float2 fl = flow_at(fr.flow, flow_pitch, g.W, g.H, xb, yb);
            sx = (int)roundf(fl.x * 2.0f);
            sy = (int)roundf(fl.y * 2.0f);
        }
        const int Xs = X + sx, Ys = Y + sy;
        const int k0 = (Xs - 2) >> 1, j0 = (Ys - 2) >> 1;
        float Aa[4] = {0.f, 0.f, 0.f, 0.f}, Wa[4] = {0.f, 0.f, 0.f, 0.f};  // per absolute parity class
        if (mask_interior && k0 >= g.cx0 && k0 + 2 <= g.cx1 && j0 >= g.cy0 && j0 + 2 <= g.cy1) {
            float v[3][3];
#pragma unroll
            for (int j = 0; j < 3; j++) {
                const uint16_t* rr = isa::row_ptr(fr.raw, raw_pitch, j0 + j) + k0;
                v[j][0] = (float)__ldg(rr);
                v[j][1] = (float)__ldg(rr + 1);
                v[j][2] = (float)__ldg(rr + 2);
            }
            float4 M[2][2];
            if (fr.mask) {
                const float4* m0 = isa::row_ptr(fr.mask, mask_pitch, uy0);
                const float4* m1 = isa::row_ptr(fr.mask, mask_pitch, uy1);
                M[0][0] = sanitize(__ldg(m0 + ux0)); M[0][1] = sanitize(__ldg(m0 + ux1));
                M[1][0] = sanitize(__ldg(m1 + ux0)); M[1][1] = sanitize(__ldg(m1 + ux1));
            } else {
                M[0][0] = M[0][1] = M[1][0] = M[1][1] = make_float4(1.f, 1.f, 1.f, 1.f);
            }
            // channel of each relative parity class (class r = row parity * 2 + column parity, relative to k0, j0)
            int ch[4];
#pragma unroll
            for (int r = 0; r < 4; r++) ch[r] = isa::cfa_at(cfa, k0 + (r & 1), j0 + (r >> 1));
            float MC[2][2][4];
#pragma unroll
            for (int dr = 0; dr < 2; dr++)
#pragma unroll
                for (int dc = 0; dc < 2; dc++)
#pragma unroll
                    for (int r = 0; r < 4; r++) MC[dr][dc][r] = comp(M[dr][dc], ch[r]);
            float Ar[4] = {0.f, 0.f, 0.f, 0.f}, Wr[4] = {0.f, 0.f, 0.f, 0.f};
            switch ((Xs & 1) | ((Ys & 1) << 1)) {
            case 0: frame_taps<0, 0>(w, v, MC, mrow, mcol, Ar, Wr); break;
            case 1: frame_taps<1, 0>(w, v, MC, mrow, mcol, Ar, Wr); break;
            case 2: frame_taps<0, 1>(w, v, MC, mrow, mcol, Ar, Wr); break;
            default: frame_taps<1, 1>(w, v, MC, mrow, mcol, Ar, Wr); break;
            }
            // relative -> absolute class: absolute = relative ^ ((j0 & 1) * 2 + (k0 & 1))
            const bool fx_ = k0 & 1, fy_ = j0 & 1;
            float A1[4], W1[4];
            A1[0] = fx_ ? Ar[1] : Ar[0]; A1[1] = fx_ ? Ar[0] : Ar[1]; A1[2] = fx_ ? Ar[3] : Ar[2]; A1[3] = fx_ ? Ar[2] : Ar[3];
            W1[0] = fx_ ? Wr[1] : Wr[0]; W1[1] = fx_ ? Wr[0] : Wr[1]; W1[2] = fx_ ? Wr[3] : Wr[2]; W1[3] = fx_ ? Wr[2] : Wr[3];
            Aa[0] = fy_ ? A1[2] : A1[0]; Aa[1] = fy_ ? A1[3] : A1[1]; Aa[2] = fy_ ? A1[0] : A1[2]; Aa[3] = fy_ ? A1[1] : A1[3];
            Wa[0] = fy_ ? W1[2] : W1[0]; Wa[1] = fy_ ? W1[3] : W1[1]; Wa[2] = fy_ ? W1[0] : W1[2]; Wa[3] = fy_ ? W1[1] : W1[3];
        } else {
            // border: per-tap reference arithmetic with the crop clamps
#pragma unroll 1
            for (int py = -2; py <= 2; py++) {
                const int qy = isa::clampi((Ys + py) >> 1, g.cy0, g.cy1);
                const int uy = isa::clampi((Y + py) >> 1, g.cy0, g.cy1) >> 1;
                const uint16_t* rr = isa::row_ptr(fr.raw, raw_pitch, qy);
                const float4* mr = fr.mask ? isa::row_ptr(fr.mask, mask_pitch, uy) : nullptr;
#pragma unroll 1
                for (int px = -2; px <= 2; px++) {
                    const int qx = isa::clampi((Xs + px) >> 1, g.cx0, g.cx1);
                    const int ux = isa::clampi((X + px) >> 1, g.cx0, g.cx1) >> 1;
                    const int cls = ((qy & 1) << 1) | (qx & 1);
                    const int c = isa::cfa_at(cfa, qx, qy);
                    float cert = 1.f;
                    if (mr) {
                        cert = comp(__ldg(mr + ux), c);
                        if (!isfinite(cert)) cert = 0.f;
                    }
                    // the weight is recomputed here: indexing w[] with loop
                    // counters would move the array out of registers
                    float wv = expf(-0.5f * (px * px * k0p + 2 * px * py * k2p + py * py * k1p));
                    if (!isfinite(wv)) wv = px * py == 0 ? 1.f : 0.f;
                    const float wc = wv * cert;
                    const float raw = (float)__ldg(rr + qx);
#pragma unroll
                    for (int k = 0; k < 4; k++)
                        if (k == cls) { Wa[k] += wc; Aa[k] = fmaf(wc, raw, Aa[k]); }
                }
            }
        }
        // classes -> colours, normalised as the reference does per tap
        float Ac[3] = {0.f, 0.f, 0.f}, Wc[3] = {0.f, 0.f, 0.f};
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const int c = isa::cfa_at(cfa, k & 1, k >> 1);
#pragma unroll
            for (int cc = 0; cc < 3; cc++)
                if (cc == c) { Ac[cc] += Aa[k]; Wc[cc] += Wa[k]; }
        }
#pragma unroll
        for (int cc = 0; cc < 3; cc++) {
            a[cc] += (Ac[cc] - black.v[cc] * Wc[cc]) / white.v[cc];
            ws[cc] += Wc[cc];
        }
    }
    ap[0] = a[0]; ap[1] = a[1]; ap[2] = a[2];
    wp[0] = ws[0]; wp[1] = ws[1]; wp[2] = ws[2];
}

}  // namespace

cudaError_t isa_launch_accumulate_x2(const isa_accum_geom& g, unsigned cfa, const isa_frame_in* frames, int nframes, const isa_frame_in* single,
                                     size_t raw_pitch, size_t flow_pitch, size_t mask_pitch, const float* kparam, size_t kparam_pitch,
                                     const float* white, const float* black, float* acc, float* wsum, size_t out_pitch, int accumulate_into,
                                     cudaStream_t st)
{
    C3 wh, bl;
    for (int c = 0; c < 3; c++) { wh.v[c] = white[c]; bl.v[c] = black[c]; }
    isa_frame_in one = single ? *single : isa_frame_in{nullptr, nullptr, nullptr};
    dim3 b(32, 8), grd((g.Wo + 63) / 64, (g.Ho + 3) / 4);
    k_accumulate_x2<<<grd, b, 0, st>>>(g, cfa, frames, nframes, one, raw_pitch, flow_pitch, mask_pitch, (const float4*)kparam, kparam_pitch, wh,
                                       bl, acc, wsum, out_pitch, accumulate_into);
    return cudaGetLastError();
}
