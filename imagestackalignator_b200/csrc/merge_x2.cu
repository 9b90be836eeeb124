// Kernel-weighted Bayer accumulation at merge scale 2 (the reference's
// accumulateImagesSuperRes, DeBayerKernels.cu:379-468, and its whole-frame
// generalisation), restructured so that no lane of a warp diverges from the
// others on the interior path.
//
// Geometry at s = 2. Output pixel (X, Y) (origin included) with shift
// (sx, sy) = round(2 * flow) reads, for its 5 x 5 taps, source samples
// q = (Xs + p) >> 1 with Xs = X + sx: a 3 x 3 block of cells starting at
// k0 = (Xs - 2) >> 1, j0 = (Ys - 2) >> 1. Tap p -> cell is 0 0 1 1 2 when
// Xs is even and 0 1 1 2 2 when it is odd (rows alike). The certainty of a
// tap comes from the half-resolution mask cell of the UNSHIFTED tap,
// (X + p) >> 2, so which of the two mask columns a tap reads depends only on
// X mod 4 (and rows on Y mod 4).
//
// Work layout. A CTA of 8 warps covers output columns bx*128 + 4*lane + ph
// and rows by*32 + 4*warp + rph, so X mod 4 and Y mod 4 are the same for
// every thread of the CTA: the tap -> mask-quadrant pattern is a template
// parameter (16 instantiations, chosen per CTA). The parity of (Xs, Ys)
// still varies from pixel to pixel; it is applied with selects, never with
// branches:
//   per tap row, the five weighted taps fold into three cell weights, the
//   taps -1 and +1 going to one of two cells by the column parity;
//   the five rows fold into three cell rows the same way by the row parity;
//   the 3 x 3 cell weights multiply the 3 x 3 samples into the four
//   relative CFA classes, which map to R, G, B through two bits per frame.
// Per frame and channel: acc_c += (sum w cert raw - black_c sum w cert) /
// white_c, wsum_c += sum w cert: the reference's per-tap
// (raw - black_c) / white_c * w * cert summed over the taps of the frame.
// Pixels whose 3 x 3 block or mask window reaches the crop border take a
// per-tap path with the reference's clamps.
#include "isa_internal.cuh"

namespace {

struct C3 { float v[3]; };

// Bayer description: green where (row parity ^ column parity) == g0, red on
// rows with parity ry.
struct Bayer { int g0, ry; };

// Mask column (0/1, relative to (X - 2) >> 2) of tap p for X mod 4 == M.
__host__ __device__ constexpr int quad_of(int M, int p) { return ((M + p + 4) >> 2) - ((M + 2) >> 2); }

__device__ __forceinline__ float comp(const float4& m, int ch) { return ch == 0 ? m.x : (ch == 1 ? m.y : m.z); }

__device__ __forceinline__ float4 sanitize(float4 m)
{
    m.x = isfinite(m.x) ? m.x : 0.f;
    m.y = isfinite(m.y) ? m.y : 0.f;
    m.z = isfinite(m.z) ? m.z : 0.f;
    return m;
}

// Certainties of the four relative CFA classes (class r = row parity * 2 +
// column parity, relative to (k0, j0)) in mask cell m. hG: relative class 0
// is green; fr: non-green cells on relative row 0 are red.
__device__ __forceinline__ void class_certs(const float4& m, bool hG, bool fr, float (&c)[4])
{
    const float rb0 = fr ? m.x : m.z, rb1 = fr ? m.z : m.x;
    c[0] = hG ? m.y : rb0;
    c[1] = hG ? rb0 : m.y;
    c[2] = hG ? rb1 : m.y;
    c[3] = hG ? m.y : rb1;
}

// One tap row: weights w[0..4] (taps -2..2), certainties cc[mask column][cell
// column parity] of the row, column parity PX of Xs -> cell weights R0..R2.
template <int XM>
__device__ __forceinline__ void row_cells(float w0, float w1, float w2, float w3, float w4, const float (&cc)[2][2], bool PX, float& R0, float& R1,
                                          float& R2)
{
    constexpr int d0 = quad_of(XM, -2), d1 = quad_of(XM, -1), d2 = quad_of(XM, 0), d3 = quad_of(XM, 1), d4 = quad_of(XM, 2);
    const float t0 = w0 * cc[d0][0];
    const float t2 = w2 * cc[d2][1];
    const float t4 = w4 * cc[d4][0];
    const float tm = w1 * (PX ? cc[d1][1] : cc[d1][0]);  // tap -1: cell PX
    const float tp = w3 * (PX ? cc[d3][0] : cc[d3][1]);  // tap +1: cell 1 + PX
    R0 = PX ? t0 : t0 + tm;
    R1 = t2 + (PX ? tm : tp);
    R2 = PX ? t4 + tp : t4;
}

// Row certainties for a tap row in mask row DR whose cell row has parity rp.
template <int DR>
__device__ __forceinline__ void row_certs(const float (&cq)[2][2][4], bool rp, float (&cc)[2][2])
{
#pragma unroll
    for (int dc = 0; dc < 2; dc++)
#pragma unroll
        for (int cp = 0; cp < 2; cp++) cc[dc][cp] = rp ? cq[DR][dc][2 + cp] : cq[DR][dc][cp];
}

struct X2Args {
    isa_accum_geom g;
    unsigned cfa;
    Bayer bayer;
    const isa_frame_in* frames;
    int nframes;
    isa_frame_in single;
    size_t raw_pitch, flow_pitch, mask_pitch;
    const float4* kparam;
    size_t kp_pitch;
    C3 rwhite, black;
    float* acc;
    float* wsum;
    size_t out_pitch;
    int accumulate_into;
};

template <int XM, int YM, bool SANE>
__device__ __forceinline__ void pixel_x2(const X2Args& A, int x, int y)
{
    const isa_accum_geom& g = A.g;
    float* ap = isa::row_ptr(A.acc, A.out_pitch, y) + 3 * x;
    float* wp = isa::row_ptr(A.wsum, A.out_pitch, y) + 3 * x;
    if (x < 1 || y < 1 || x >= g.Wo - 1 || y >= g.Ho - 1) {
        if (!A.accumulate_into) { ap[0] = ap[1] = ap[2] = 0.f; wp[0] = wp[1] = wp[2] = 0.f; }
        return;
    }
    float a[3] = {0.f, 0.f, 0.f}, ws[3] = {0.f, 0.f, 0.f};
    if (A.accumulate_into) {
        a[0] = ap[0]; a[1] = ap[1]; a[2] = ap[2];
        ws[0] = wp[0]; ws[1] = wp[1]; ws[2] = wp[2];
    }
    const int X = x + g.ox, Y = y + g.oy;
    const float xb = ((float)x + 0.5f + (float)g.ox) / 2.0f - 0.5f;
    const float yb = ((float)y + 0.5f + (float)g.oy) / 2.0f - 0.5f;
    const float fxb = floorf(xb), fyb = floorf(yb);
    const int ib = (int)fxb, jb = (int)fyb;
    const float ax = xb - fxb, by = yb - fyb;
    // kernel parameters: bilinear, clamp addressing
    float k0p, k1p, k2p;
    {
        const int i0 = isa::clampi(ib, 0, g.W - 1), i1 = isa::clampi(ib + 1, 0, g.W - 1);
        const int j0 = isa::clampi(jb, 0, g.H - 1), j1 = isa::clampi(jb + 1, 0, g.H - 1);
        const float4 p00 = __ldg(isa::row_ptr(A.kparam, A.kp_pitch, j0) + i0), p10 = __ldg(isa::row_ptr(A.kparam, A.kp_pitch, j0) + i1);
        const float4 p01 = __ldg(isa::row_ptr(A.kparam, A.kp_pitch, j1) + i0), p11 = __ldg(isa::row_ptr(A.kparam, A.kp_pitch, j1) + i1);
        k0p = isa::lerp2(p00.x, p10.x, p01.x, p11.x, ax, by);
        k1p = isa::lerp2(p00.y, p10.y, p01.y, p11.y, ax, by);
        k2p = isa::lerp2(p00.z, p10.z, p01.z, p11.z, ax, by);
    }
    float w[5][5];
#pragma unroll
    for (int py = -2; py <= 2; py++)
#pragma unroll
        for (int px = -2; px <= 2; px++) {
            float q = px * px * k0p + 2 * px * py * k2p + py * py * k1p;
            float vv = expf(-0.5f * q);
            if (!isfinite(vv)) vv = px * py == 0 ? 1.f : 0.f;
            w[py + 2][px + 2] = vv;
        }
    // flow: bilinear, mirror addressing (same position for every frame)
    const int fi0 = isa::mirror(ib, g.W), fi1 = isa::mirror(ib + 1, g.W);
    const size_t fr0 = (size_t)isa::mirror(jb, g.H) * A.flow_pitch, fr1 = (size_t)isa::mirror(jb + 1, g.H) * A.flow_pitch;
    // interior: the unshifted taps' mask cells are (X - 2) >> 2 + {0, 1}, rows alike,
    // and the shifted 3 x 3 block [k0, k0 + 2] x [j0, j0 + 2] lies inside the crop:
    // k0 = (X + sx - 2) >> 1 in [cx0, cx1 - 2]  <=>  sx in [2 cx0 + 2 - X, 2 cx1 - 1 - X]
    const bool mask_interior = ((X - 2) >> 1) >= g.cx0 && ((X + 2) >> 1) <= g.cx1 && ((Y - 2) >> 1) >= g.cy0 && ((Y + 2) >> 1) <= g.cy1;
    const int sxlo = mask_interior ? 2 * g.cx0 + 2 - X : (1 << 29), sylo = 2 * g.cy0 + 2 - Y;
    const unsigned sxspan = mask_interior ? (unsigned)(2 * g.cx1 - 1 - X - sxlo) : 0u, syspan = (unsigned)(2 * g.cy1 - 1 - Y - sylo);
    const int ux0 = (X - 2) >> 2, uy0 = (Y - 2) >> 2;
    const size_t moff = (size_t)uy0 * A.mask_pitch + (size_t)ux0 * sizeof(float4);
    for (int f = 0; f < A.nframes; f++) {
        const isa_frame_in fr = A.frames ? A.frames[f] : A.single;
        int sx = 0, sy = 0;
        if (fr.flow) {
            const char* fb = (const char*)fr.flow;
            const float2 p00 = __ldg((const float2*)(fb + fr0) + fi0), p10 = __ldg((const float2*)(fb + fr0) + fi1);
            const float2 p01 = __ldg((const float2*)(fb + fr1) + fi0), p11 = __ldg((const float2*)(fb + fr1) + fi1);
            sx = (int)roundf(isa::lerp2(p00.x, p10.x, p01.x, p11.x, ax, by) * 2.0f);
            sy = (int)roundf(isa::lerp2(p00.y, p10.y, p01.y, p11.y, ax, by) * 2.0f);
        }
        const int Xs = X + sx, Ys = Y + sy;
        const int k0 = (Xs - 2) >> 1, j0 = (Ys - 2) >> 1;
        float Ac[3] = {0.f, 0.f, 0.f}, Wc[3] = {0.f, 0.f, 0.f};
        if ((unsigned)(sx - sxlo) <= sxspan && (unsigned)(sy - sylo) <= syspan) {
            float v[3][3];
#pragma unroll
            for (int j = 0; j < 3; j++) {
                const uint16_t* rr = isa::row_ptr(fr.raw, A.raw_pitch, j0 + j) + k0;
                v[j][0] = (float)__ldg(rr);
                v[j][1] = (float)__ldg(rr + 1);
                v[j][2] = (float)__ldg(rr + 2);
            }
            const bool fx = k0 & 1, fy = j0 & 1;
            const bool hG = (int)(fx ^ fy) == A.bayer.g0, frr = (int)fy == A.bayer.ry;
            float cq[2][2][4];
            if (fr.mask) {
                const float4* m0 = (const float4*)((const char*)fr.mask + moff);
                const float4* m1 = (const float4*)((const char*)fr.mask + moff + A.mask_pitch);
                float4 M00 = __ldg(m0), M01 = __ldg(m0 + 1), M10 = __ldg(m1), M11 = __ldg(m1 + 1);
                if (!SANE) { M00 = sanitize(M00); M01 = sanitize(M01); M10 = sanitize(M10); M11 = sanitize(M11); }
                class_certs(M00, hG, frr, cq[0][0]);
                class_certs(M01, hG, frr, cq[0][1]);
                class_certs(M10, hG, frr, cq[1][0]);
                class_certs(M11, hG, frr, cq[1][1]);
            } else {
#pragma unroll
                for (int i = 0; i < 16; i++) (&cq[0][0][0])[i] = 1.f;
            }
            const bool PX = Xs & 1, PY = Ys & 1;
            // tap rows -> cell weights per row (rows -1 and +1 have cell-row parity PY and !PY)
            float Rm2[3], Rm1[3], R0[3], Rp1[3], Rp2[3];
            {
                float cc[2][2];
                row_certs<quad_of(YM, -2)>(cq, false, cc);
                row_cells<XM>(w[0][0], w[0][1], w[0][2], w[0][3], w[0][4], cc, PX, Rm2[0], Rm2[1], Rm2[2]);
                row_certs<quad_of(YM, -1)>(cq, PY, cc);
                row_cells<XM>(w[1][0], w[1][1], w[1][2], w[1][3], w[1][4], cc, PX, Rm1[0], Rm1[1], Rm1[2]);
                row_certs<quad_of(YM, 0)>(cq, true, cc);
                row_cells<XM>(w[2][0], w[2][1], w[2][2], w[2][3], w[2][4], cc, PX, R0[0], R0[1], R0[2]);
                row_certs<quad_of(YM, 1)>(cq, !PY, cc);
                row_cells<XM>(w[3][0], w[3][1], w[3][2], w[3][3], w[3][4], cc, PX, Rp1[0], Rp1[1], Rp1[2]);
                row_certs<quad_of(YM, 2)>(cq, false, cc);
                row_cells<XM>(w[4][0], w[4][1], w[4][2], w[4][3], w[4][4], cc, PX, Rp2[0], Rp2[1], Rp2[2]);
            }
            float Wcell[3][3];
#pragma unroll
            for (int i = 0; i < 3; i++) {
                Wcell[0][i] = PY ? Rm2[i] : Rm2[i] + Rm1[i];
                Wcell[1][i] = R0[i] + (PY ? Rm1[i] : Rp1[i]);
                Wcell[2][i] = PY ? Rp2[i] + Rp1[i] : Rp2[i];
            }
            // relative classes
            const float A0 = Wcell[0][0] * v[0][0] + Wcell[0][2] * v[0][2] + Wcell[2][0] * v[2][0] + Wcell[2][2] * v[2][2];
            const float A1 = Wcell[0][1] * v[0][1] + Wcell[2][1] * v[2][1];
            const float A2 = Wcell[1][0] * v[1][0] + Wcell[1][2] * v[1][2];
            const float A3 = Wcell[1][1] * v[1][1];
            const float W0 = Wcell[0][0] + Wcell[0][2] + Wcell[2][0] + Wcell[2][2];
            const float W1 = Wcell[0][1] + Wcell[2][1];
            const float W2 = Wcell[1][0] + Wcell[1][2];
            const float W3 = Wcell[1][1];
            // relative classes -> R, G, B
            const float NA0 = hG ? A1 : A0, NA1 = hG ? A2 : A3, NW0 = hG ? W1 : W0, NW1 = hG ? W2 : W3;
            Ac[1] = hG ? A0 + A3 : A1 + A2;
            Wc[1] = hG ? W0 + W3 : W1 + W2;
            Ac[0] = frr ? NA0 : NA1;
            Ac[2] = frr ? NA1 : NA0;
            Wc[0] = frr ? NW0 : NW1;
            Wc[2] = frr ? NW1 : NW0;
        } else {
            // border: per-tap reference arithmetic with the crop clamps
#pragma unroll 1
            for (int py = -2; py <= 2; py++) {
                const int qy = isa::clampi((Ys + py) >> 1, g.cy0, g.cy1);
                const int uy = isa::clampi((Y + py) >> 1, g.cy0, g.cy1) >> 1;
                const uint16_t* rr = isa::row_ptr(fr.raw, A.raw_pitch, qy);
                const float4* mr = fr.mask ? isa::row_ptr(fr.mask, A.mask_pitch, uy) : nullptr;
#pragma unroll 1
                for (int px = -2; px <= 2; px++) {
                    const int qx = isa::clampi((Xs + px) >> 1, g.cx0, g.cx1);
                    const int ux = isa::clampi((X + px) >> 1, g.cx0, g.cx1) >> 1;
                    const int c = isa::cfa_at(A.cfa, qx, qy);
                    float cert = 1.f;
                    if (mr) {
                        cert = comp(__ldg(mr + ux), c);
                        if (!isfinite(cert)) cert = 0.f;
                    }
                    // the weight is recomputed here: indexing w[][] with loop
                    // counters would move the array out of registers
                    float wv = expf(-0.5f * (px * px * k0p + 2 * px * py * k2p + py * py * k1p));
                    if (!isfinite(wv)) wv = px * py == 0 ? 1.f : 0.f;
                    const float wc = wv * cert;
                    const float raw = (float)__ldg(rr + qx);
#pragma unroll
                    for (int k = 0; k < 3; k++)
                        if (k == c) { Wc[k] += wc; Ac[k] = fmaf(wc, raw, Ac[k]); }
                }
            }
        }
#pragma unroll
        for (int cc = 0; cc < 3; cc++) {
            a[cc] += (Ac[cc] - A.black.v[cc] * Wc[cc]) * A.rwhite.v[cc];
            ws[cc] += Wc[cc];
        }
    }
    ap[0] = a[0]; ap[1] = a[1]; ap[2] = a[2];
    wp[0] = ws[0]; wp[1] = ws[1]; wp[2] = ws[2];
}

template <bool SANE>
__global__ void __launch_bounds__(256, SANE ? 3 : 2) k_accumulate_x2(const X2Args A)
{
    const int ph = blockIdx.x & 3, rph = blockIdx.y & 3;
    const int x = (blockIdx.x >> 2) * 128 + 4 * threadIdx.x + ph;
    const int y = A.g.yb0 + (blockIdx.y >> 2) * 32 + 4 * threadIdx.y + rph;
    if (x >= A.g.Wo || y >= A.g.yb1) return;
    // X mod 4 and Y mod 4 are the same for the whole CTA
    switch (((ph + A.g.ox) & 3) | (((rph + A.g.oy) & 3) << 2)) {
#define ISA_X2_CASE(k) \
    case k: pixel_x2<((k) & 3), ((k) >> 2), SANE>(A, x, y); break;
        ISA_X2_CASE(0) ISA_X2_CASE(1) ISA_X2_CASE(2) ISA_X2_CASE(3) ISA_X2_CASE(4) ISA_X2_CASE(5) ISA_X2_CASE(6) ISA_X2_CASE(7)
        ISA_X2_CASE(8) ISA_X2_CASE(9) ISA_X2_CASE(10) ISA_X2_CASE(11) ISA_X2_CASE(12) ISA_X2_CASE(13) ISA_X2_CASE(14) ISA_X2_CASE(15)
#undef ISA_X2_CASE
    }
}

// The CFA is a Bayer pattern: codes 0/1/2 only, the two greens on one
// diagonal, red and blue on the other.
bool bayer_of(unsigned cfa, Bayer& b)
{
    int c[4];
    for (int i = 0; i < 4; i++) c[i] = (cfa >> (2 * i)) & 3;  // index = row parity * 2 + column parity
    if (c[1] == 1 && c[2] == 1 && c[0] != 1 && c[3] != 1 && c[0] != c[3]) {
        b.g0 = 1;
        b.ry = c[0] == 0 ? 0 : 1;
        return (c[0] == 0 || c[0] == 2) && (c[3] == 0 || c[3] == 2);
    }
    if (c[0] == 1 && c[3] == 1 && c[1] != 1 && c[2] != 1 && c[1] != c[2]) {
        b.g0 = 0;
        b.ry = c[1] == 0 ? 0 : 1;
        return (c[1] == 0 || c[1] == 2) && (c[2] == 0 || c[2] == 2);
    }
    return false;
}

}  // namespace

bool isa_accumulate_x2_supported(unsigned cfa)
{
    Bayer b;
    return bayer_of(cfa, b);
}

cudaError_t isa_launch_accumulate_x2(const isa_accum_geom& g, unsigned cfa, const isa_frame_in* frames, int nframes, const isa_frame_in* single,
                                     size_t raw_pitch, size_t flow_pitch, size_t mask_pitch, const float* kparam, size_t kparam_pitch,
                                     const float* white, const float* black, float* acc, float* wsum, size_t out_pitch, int accumulate_into,
                                     cudaStream_t st)
{
    X2Args A;
    if (!bayer_of(cfa, A.bayer)) return cudaErrorInvalidValue;
    A.g = g;
    A.cfa = cfa;
    A.frames = frames;
    A.nframes = nframes;
    A.single = single ? *single : isa_frame_in{nullptr, nullptr, nullptr};
    A.raw_pitch = raw_pitch; A.flow_pitch = flow_pitch; A.mask_pitch = mask_pitch;
    A.kparam = (const float4*)kparam; A.kp_pitch = kparam_pitch;
    for (int c = 0; c < 3; c++) { A.rwhite.v[c] = (float)(1.0 / (double)white[c]); A.black.v[c] = black[c]; }
    A.acc = acc; A.wsum = wsum; A.out_pitch = out_pitch; A.accumulate_into = accumulate_into;
    if (g.yb0 % 32 || g.yb0 < 0 || g.yb1 > g.Ho || g.yb1 <= g.yb0) return cudaErrorInvalidValue;
    dim3 b(32, 8), grd(((g.Wo + 127) / 128) * 4, ((g.yb1 - g.yb0 + 31) / 32) * 4);
    if (g.masks_finite)
        k_accumulate_x2<true><<<grd, b, 0, st>>>(A);
    else
        k_accumulate_x2<false><<<grd, b, 0, st>>>(A);
    return cudaGetLastError();
}
