// Lucas-Kanade refinement (OpticalFlow.LucasKanade, PEFStudioDX/OpticalFlow.cs:147-164;
// kernels opticalFlow.cu:28-325).
//
// Texture reads of the reference are replaced by explicit arithmetic with the
// same addressing: flow field from the tile grid = linear/clamp sample
// (opticalFlow.cu:48-94), warp = linear/mirror sample of the image at
// x + flow(x) (opticalFlow.cu:28-45), derivatives = five-tap differences with
// mirror addressing (opticalFlow.cu:97-185). Sample positions are split into
// the integer pixel and the sub-pixel flow part so that FP32 keeps full
// sub-pixel precision far from the origin.
//
// k_lk_stream fuses one reference iteration (warp, Set(0) x3, derivatives,
// lucasKanadeOptim) for a vertical strip of the image, walking down it row by
// row: FP32 gradient products, FP64 sliding window sums, and the 2x2
// pseudo-inverse in FP64.
#include "isa_internal.cuh"

#include <algorithm>
#include <type_traits>

namespace {

__device__ __forceinline__ float bilinear_mirror(const float* img, size_t pitch, int W, int H, int px, int py, float fx, float fy)
{
    float flx = floorf(fx), fly = floorf(fy);
    int ix = px + (int)flx, iy = py + (int)fly;
    float a = fx - flx, b = fy - fly;
    int x0 = isa::mirror(ix, W), x1 = isa::mirror(ix + 1, W), y0 = isa::mirror(iy, H), y1 = isa::mirror(iy + 1, H);
    const float* r0 = isa::row_ptr(img, pitch, y0);
    const float* r1 = isa::row_ptr(img, pitch, y1);
    float p00 = __ldg(r0 + x0), p10 = __ldg(r0 + x1), p01 = __ldg(r1 + x0), p11 = __ldg(r1 + x1);
    return isa::lerp2(p00, p10, p01, p11, a, b);
}

// lucasKanadeOptim's pseudo-inverse (opticalFlow.cu:229-290) in FP64 and the
// flow update u = M (sxt, syt). For a well-conditioned matrix
// (lambda2 > 1e-3 lambda1) the angle/singular-value construction of the
// reference equals the closed-form inverse to ~1e-10 relative; below that the
// reference's own construction is evaluated (lk_svd). The pixel is
// left unchanged where sigma1 < minDet (the reference tests
// min(sigma1, sigma1)).
__device__ __forceinline__ float2 lk_apply(float2 f, double m0, double m1, double m2, double m3, double sxt, double syt)
{
    double u = m0 * sxt + m1 * syt, v = m2 * sxt + m3 * syt;
    if (isnan(u)) u = 0;
    if (isnan(v)) v = 0;
    return make_float2((float)((double)f.x + u), (float)((double)f.y + v));
}

// The ill-conditioned branch: the reference's angle/singular-value
// construction of the pseudo-inverse. Out of line: it is rarely taken, and
// inlined at every solve it would multiply the code of the per-pixel
// kernels. ok = false where sigma1 < minDet (no update).
struct LkM {
    double m0, m1, m2, m3;
    bool ok;
};

__device__ __noinline__ LkM lk_svd(double a, double b, double d, double min_det)
{
    LkM r{0.0, 0.0, 0.0, 0.0, false};
    const double c = b;
    double th = 0.5 * atan2(2 * a * c + 2 * b * d, a * a + b * b - c * c - d * d);
    double ct = cos(th), st = sin(th);
    double S1 = a * a + b * b + c * c + d * d;
    double S2 = sqrt((a * a + b * b - c * c - d * d) * (a * a + b * b - c * c - d * d) + 4 * (a * c + b * d) * (a * c + b * d));
    double s1 = sqrt((S1 + S2) / 2), s2 = sqrt((S1 - S2) / 2);
    if (s1 < min_det) return r;
    s1 = s1 != 0 ? 1 / s1 : 0;
    s2 = s2 != 0 ? 1 / s2 : 0;
    double ep = 0.5 * atan2(2 * a * b + 2 * c * d, a * a - b * b + c * c - d * d);
    double ce = cos(ep), se = sin(ep);
    double q11 = (a * ct + c * st) * ce + (b * ct + d * st) * se;
    double q22 = (a * st - c * ct) * se + (-b * st + d * ct) * ce;
    q11 = q11 > 0 ? 1 : (q11 < 0 ? -1 : 0);
    q22 = q22 > 0 ? 1 : (q22 < 0 ? -1 : 0);
    double V0 = q11 * ce, V1 = -q22 * se, V2 = q11 * se, V3 = q22 * ce;
    double m0 = s1 * ct, m1 = s1 * st, m2 = s2 * -st, m3 = s2 * ct;
    r.m0 = V0 * m0 + V1 * m2;
    r.m1 = V0 * m1 + V1 * m3;
    r.m2 = V2 * m0 + V3 * m2;
    r.m3 = V2 * m1 + V3 * m3;
    r.ok = true;
    return r;
}

// The pseudo-inverse M of the window matrix [a b; b d], as the forward
// chooses it; false where the reference leaves the pixel unchanged.
__device__ __forceinline__ bool lk_matrix(double a, double b, double d, double min_det, double& m0, double& m1, double& m2, double& m3)
{
    // the largest eigenvalue only steers two threshold tests, so a float
    // square root is enough (the reference compares sigma1 with minDet and
    // the branch point is a conditioning bound)
    double hd = 0.5 * (a - d);
    double l1 = 0.5 * (a + d) + (double)sqrtf((float)(hd * hd + b * b));
    double det = a * d - b * b;
    if (det > 1e-3 * l1 * l1) {
        if (l1 < min_det) return false;
        double inv = 1.0 / det;
        m0 = d * inv; m1 = -b * inv; m2 = -b * inv; m3 = a * inv;
        return true;
    }
    const LkM r = lk_svd(a, b, d, min_det);
    m0 = r.m0; m1 = r.m1; m2 = r.m2; m3 = r.m3;
    return r.ok;
}

__device__ __forceinline__ float2 lk_update(float2 f, double a, double b, double d, double sxt, double syt, double min_det)
{
    double m0, m1, m2, m3;
    if (!lk_matrix(a, b, d, min_det, m0, m1, m2, m3)) return f;
    return lk_apply(f, m0, m1, m2, m3, sxt, syt);
}

// Adjoint of lk_update at one pixel for the upstream gradient g of the
// updated flow: with delta = M c (c = (sxt, syt)) and gamma = M^T g, the
// window sums get dL/dsxx = -gamma_x delta_x, dL/dsxy = -(gamma_x delta_y +
// gamma_y delta_x), dL/dsyy = -gamma_y delta_y, dL/dsxt = gamma_x,
// dL/dsyt = gamma_y (d(M c) = -M dM M c). A component the forward sets to 0
// (NaN) passes no gradient; a pixel it leaves unchanged gets zeros.
__device__ __forceinline__ void lk_coeffs(float2 g, double a, double b, double d, double sxt, double syt, double min_det, float co[5])
{
    co[0] = co[1] = co[2] = co[3] = co[4] = 0.f;
    double m0, m1, m2, m3;
    if (!lk_matrix(a, b, d, min_det, m0, m1, m2, m3)) return;
    double u = m0 * sxt + m1 * syt, v = m2 * sxt + m3 * syt;
    const double gx = isnan(u) ? 0.0 : (double)g.x, gy = isnan(v) ? 0.0 : (double)g.y;
    if (isnan(u)) u = 0;
    if (isnan(v)) v = 0;
    const double c0 = m0 * gx + m2 * gy, c1 = m1 * gx + m3 * gy;
    co[0] = (float)(-c0 * u);
    co[1] = (float)(-(c0 * v + c1 * u));
    co[2] = (float)(-c1 * v);
    co[3] = (float)c0;
    co[4] = (float)c1;
}

// c, s: cosine and sine of the pre-alignment rotation (uniform, computed once
// on the host). Each thread writes FF_PX consecutive pixels of a row.
constexpr int FF_PX = 4;

__global__ void k_flow_from_tiles(const float2* __restrict__ tiles, size_t tile_pitch, int tcx, int tcy, int W, int H, float bx, float by,
                                  float c, float s, float2* __restrict__ flow, size_t flow_pitch)
{
    const int xq = (blockIdx.x * blockDim.x + threadIdx.x) * FF_PX, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (xq >= W || y >= H) return;
    const float pcy = (float)(y - H / 2);
    const float yb = ((float)y + 0.5f) / (float)H * tcy - 0.5f;
    const float fly = floorf(yb);
    const int j = (int)fly;
    const float b = yb - fly;
    const int j0 = isa::clampi(j, 0, tcy - 1), j1 = isa::clampi(j + 1, 0, tcy - 1);
    const float2* r0 = isa::row_ptr(tiles, tile_pitch, j0);
    const float2* r1 = isa::row_ptr(tiles, tile_pitch, j1);
    const float fx0 = c * -bx - s * -by, fy0 = s * -bx + c * -by;
    float2 res[FF_PX];
#pragma unroll
    for (int q = 0; q < FF_PX; q++) {
        const int x = min(xq + q, W - 1);
        float fx = fx0, fy = fy0;
        const float pcx = (float)(x - W / 2);
        fx += c * pcx - s * pcy - pcx;
        fy += s * pcx + c * pcy - pcy;
        const float xb = ((float)x + 0.5f) / (float)W * tcx - 0.5f;
        const float flx = floorf(xb);
        const int i = (int)flx;
        const float a = xb - flx;
        const int i0 = isa::clampi(i, 0, tcx - 1), i1 = isa::clampi(i + 1, 0, tcx - 1);
        const float2 p00 = __ldg(r0 + i0), p10 = __ldg(r0 + i1), p01 = __ldg(r1 + i0), p11 = __ldg(r1 + i1);
        fx += isa::lerp2(p00.x, p10.x, p01.x, p11.x, a, b);
        fy += isa::lerp2(p00.y, p10.y, p01.y, p11.y, a, b);
        res[q] = make_float2(fx, fy);
    }
    float2* o = isa::row_ptr(flow, flow_pitch, y) + xq;
    if (xq + FF_PX <= W && ((uintptr_t)o & 15) == 0) {
        ((float4*)o)[0] = make_float4(res[0].x, res[0].y, res[1].x, res[1].y);
        ((float4*)o)[1] = make_float4(res[2].x, res[2].y, res[3].x, res[3].y);
    } else {
        for (int q = 0; q < FF_PX && xq + q < W; q++) o[q] = res[q];
    }
}

__global__ void k_warp(const float* __restrict__ img, size_t img_pitch, int W, int H, const float2* __restrict__ flow, size_t flow_pitch,
                       float* __restrict__ out, size_t out_pitch)
{
    int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= W || y >= H) return;
    float2 f = isa::row_ptr(flow, flow_pitch, y)[x];
    isa::row_ptr(out, out_pitch, y)[x] = bilinear_mirror(img, img_pitch, W, H, x, y, f.x, f.y);
}

__device__ __forceinline__ float at_m(const float* img, size_t pitch, int W, int H, int x, int y)
{
    return __ldg(isa::row_ptr(img, pitch, isa::mirror(y, H)) + isa::mirror(x, W));
}

__global__ void k_derivatives(const float* __restrict__ src, const float* __restrict__ tgt, size_t pitch, int W, int H, float* ix, float* iy,
                              float* it, size_t out_pitch)
{
    int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= W || y >= H) return;
    float t0 = (at_m(src, pitch, W, H, x + 2, y) - at_m(src, pitch, W, H, x + 1, y) * 8.0f + at_m(src, pitch, W, H, x - 1, y) * 8.0f -
                at_m(src, pitch, W, H, x - 2, y)) / 12.0f;
    float t1 = (at_m(tgt, pitch, W, H, x + 2, y) - at_m(tgt, pitch, W, H, x + 1, y) * 8.0f + at_m(tgt, pitch, W, H, x - 1, y) * 8.0f -
                at_m(tgt, pitch, W, H, x - 2, y)) / 12.0f;
    isa::row_ptr(ix, out_pitch, y)[x] = (t0 + t1) * 0.5f;
    isa::row_ptr(it, out_pitch, y)[x] = at_m(src, pitch, W, H, x, y) - at_m(tgt, pitch, W, H, x, y);
    t0 = (at_m(src, pitch, W, H, x, y + 2) - at_m(src, pitch, W, H, x, y + 1) * 8.0f + at_m(src, pitch, W, H, x, y - 1) * 8.0f -
          at_m(src, pitch, W, H, x, y - 2)) / 12.0f;
    t1 = (at_m(tgt, pitch, W, H, x, y + 2) - at_m(tgt, pitch, W, H, x, y + 1) * 8.0f + at_m(tgt, pitch, W, H, x, y - 1) * 8.0f -
          at_m(tgt, pitch, W, H, x, y - 2)) / 12.0f;
    isa::row_ptr(iy, out_pitch, y)[x] = (t0 + t1) * 0.5f;
}

__global__ void k_derivatives2(const float* __restrict__ img, size_t pitch, int W, int H, float* ix, float* iy, size_t out_pitch)
{
    int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= W || y >= H) return;
    isa::row_ptr(ix, out_pitch, y)[x] = (at_m(img, pitch, W, H, x + 2, y) - at_m(img, pitch, W, H, x + 1, y) * 8.0f +
                                         at_m(img, pitch, W, H, x - 1, y) * 8.0f - at_m(img, pitch, W, H, x - 2, y)) / 12.0f;
    isa::row_ptr(iy, out_pitch, y)[x] = (at_m(img, pitch, W, H, x, y + 2) - at_m(img, pitch, W, H, x, y + 1) * 8.0f +
                                         at_m(img, pitch, W, H, x, y - 1) * 8.0f - at_m(img, pitch, W, H, x, y - 2)) / 12.0f;
}

// lucasKanadeOptim over precomputed derivative images (the reference's
// separate-kernel form): FP32 products, FP64 window sums and solve.
__global__ void k_lk_sums(float2* flow, size_t flow_pitch, const float* __restrict__ ix, const float* __restrict__ iy,
                          const float* __restrict__ it, size_t pitch, int W, int H, int h, float min_det)
{
    int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x < h || x >= W - h || y < h || y >= H - h) return;
    double sxx = 0, sxy = 0, syy = 0, sxt = 0, syt = 0;
    for (int j = -h; j <= h; j++) {
        const float* rx = isa::row_ptr(ix, pitch, y + j);
        const float* ry = isa::row_ptr(iy, pitch, y + j);
        const float* rt = isa::row_ptr(it, pitch, y + j);
        for (int i = -h; i <= h; i++) {
            float dx = rx[x + i], dy = ry[x + i], dt = rt[x + i];
            sxx += dx * dx; sxy += dx * dy; syy += dy * dy; sxt += dx * dt; syt += dy * dt;
        }
    }
    float2* fp = isa::row_ptr(flow, flow_pitch, y) + x;
    *fp = lk_update(*fp, sxx, sxy, syy, sxt, syt, min_det);
}

// Streaming form of one reference iteration (warp, Set(0) x3, derivatives,
// lucasKanadeOptim). A CTA of LKS_NT threads owns a vertical strip of LKS_NT
// columns (SW = LKS_NT - 2R output columns, R = h + 2) and `sh` output rows:
// thread t owns image column x0 - R + t (mirrored at the border) and walks
// down the strip two rows per step:
//   1. the warped source and the reference of the two rows go into a ring of
//      six rows of (warped, reference) pairs in shared memory; the global
//      loads of the next two rows are issued one step ahead (bilinear
//      samples) and two steps ahead (flow);
//   2. after a barrier, five-tap derivatives at the two centre rows (own
//      column and neighbours from the ring), FP32 products, and per-column
//      vertical window sums in FP64 registers (the product leaving the
//      window comes from a shared ring of the last 2h + 1 product rows that
//      only its own thread touches);
//   3. after a second barrier, the row window sums of the two output rows
//      (2h + 1 columns, two pixels per thread, FP64) and the 2x2 solve.
// The FP64 sums hold the FP32 products exactly enough that the order of
// summation does not matter at FP32 output precision. Threads at the strip's
// edges (t < 2, t >= LKS_NT - 2) compute products from padding; their column
// sums are never read.
constexpr int LKS_NT = 128, LKS_PX = 2;

template <int H>
struct LkStream {
    static constexpr int R = H + 2, SW = LKS_NT - 2 * R, WIN = 2 * H + 1;
    static constexpr int PX = LKS_PX, NSEG = (SW + PX - 1) / PX;  // row-sum phase: PX output pixels per thread, NSEG threads per row
    static_assert(SW > 0 && SW % 2 == 0 && PX % 2 == 0 && 2 * NSEG <= LKS_NT, "two output rows of PX-pixel segments per step");
    static_assert(SW - 2 + WIN + PX <= LKS_NT, "the last segment's window stays inside its row of column sums");
    static constexpr int EPAD = 2;  // float2 either side of the pair ring: the edge threads' taps stay in shared memory
    static constexpr size_t OFF_P4 = (size_t)(6 * LKS_NT + 2 * EPAD) * 8;           // [WIN][NT] float4: products 0-3
    static constexpr size_t OFF_P1 = OFF_P4 + (size_t)WIN * LKS_NT * 16;            // [WIN][NT] float: product 4
    static constexpr size_t OFF_C = (OFF_P1 + (size_t)WIN * LKS_NT * 4 + 15) / 16 * 16;  // [2][5][NT] double: column sums
    static constexpr size_t TOTAL = OFF_C + (size_t)2 * 5 * LKS_NT * 8;
};

// Bilinear source samples of one row (mirror addressing) and the reference texel.
struct LkTaps {
    float s00, s10, s01, s11, a, b, r;
};

// ADJ: the adjoint-coefficient form. The same window sums at the flow
// flow_in; instead of the update, each pixel writes lk_coeffs of the
// upstream gradient gin (float2, rows at flow_pitch) to five float planes
// (aout, rows at a_pitch, planes a_plane bytes apart): dL/d(sxx, sxy, syy,
// sxt, syt), zero where the forward leaves the pixel unchanged.
template <int H, bool ADJ>
__global__ void __launch_bounds__(LKS_NT, 512 / LKS_NT) k_lk_stream(const float2* __restrict__ flow_in, float2* __restrict__ flow_out, size_t flow_pitch,
                                                         const float* __restrict__ src, const float* __restrict__ ref, size_t img_pitch, int W,
                                                         int Himg, int sh, float min_det, const float2* __restrict__ gin, float* __restrict__ aout,
                                                         size_t a_pitch, size_t a_plane)
{
    using L = LkStream<H>;
    constexpr int R = L::R, SW = L::SW, WIN = L::WIN, NT = LKS_NT, NSEG = L::NSEG, PX = L::PX;
    extern __shared__ __align__(16) unsigned char smem[];
    float2* E = (float2*)smem + L::EPAD;              // [6][NT] (warped source, reference), three two-row slots
    float4* P4 = (float4*)(smem + L::OFF_P4);
    float* P1 = (float*)(smem + L::OFF_P1);
    double* Cs = (double*)(smem + L::OFF_C);
    const int t = threadIdx.x;
    const int x0 = blockIdx.x * SW, y0 = blockIdx.y * sh;
    const int nout = min(sh, Himg - y0);
    const int nsteps = (nout + 2 * R + 1) / 2;  // rows 0 .. 2 nsteps - 1 of the strip (one extra, mirrored, when nout is odd)
    const int col = isa::mirror(x0 - R + t, W);
    const float* refc = ref + col;
    const float2* flc = flow_in + col;
    const auto erow = [&](int e) { return isa::mirror(y0 - R + e, Himg); };
    const auto flow_at = [&](int e) { return __ldg(isa::row_ptr(flc, flow_pitch, erow(e))); };
    const auto sample = [&](int e, float2 f, LkTaps& q) {
        const int row = erow(e);
        const float flx = floorf(f.x), fly = floorf(f.y);
        const int ix = col + (int)flx, iy = row + (int)fly;
        q.a = f.x - flx;
        q.b = f.y - fly;
        if ((unsigned)ix < (unsigned)(W - 1) && (unsigned)iy < (unsigned)(Himg - 1)) {
            const float* p0 = isa::row_ptr(src, img_pitch, iy) + ix;
            const float* p1 = isa::row_ptr(p0, img_pitch, 1);
            q.s00 = __ldg(p0); q.s10 = __ldg(p0 + 1); q.s01 = __ldg(p1); q.s11 = __ldg(p1 + 1);
        } else {
            const int xa = isa::mirror(ix, W), xb = isa::mirror(ix + 1, W);
            const float* r0 = isa::row_ptr(src, img_pitch, isa::mirror(iy, Himg));
            const float* r1 = isa::row_ptr(src, img_pitch, isa::mirror(iy + 1, Himg));
            q.s00 = __ldg(r0 + xa); q.s10 = __ldg(r0 + xb); q.s01 = __ldg(r1 + xa); q.s11 = __ldg(r1 + xb);
        }
        q.r = __ldg(isa::row_ptr(refc, img_pitch, row));
    };
    LkTaps qa, qb;
    sample(0, flow_at(0), qa);
    sample(1, flow_at(1), qb);
    float2 fa = flow_at(2), fb = flow_at(3);
    // the product ring starts at zero: the first 2h + 1 rows subtract nothing
#pragma unroll 1
    for (int k = 0; k < WIN; k++) {
        P4[k * NT + t] = make_float4(0.f, 0.f, 0.f, 0.f);
        P1[k * NT + t] = 0.f;
    }
    double cs[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    int pw = 0;                                 // product ring slot of the next product row
    int sn = 0, s2 = 2 * NT, s1 = 4 * NT;       // pair slots: rows 2s, 2s+1 / 2s-4, 2s-3 / 2s-2, 2s-1
    // row-sum phase: thread t < 2 NSEG sums output row (t / NSEG) of the step at columns j0 .. j0 + PX - 1
    const int rr = t / NSEG, j0 = PX * (t - rr * NSEG);
    const bool summer = t < 2 * NSEG;

    // one product row: the centre row's pairs at c (neighbours in the ring) and above/below it in the own column
    const auto product_row = [&](const float2* c, float2 vm2, float2 vm1, float2 vp1, float2 vp2) {
        const float2 cm2 = c[-2], cm1 = c[-1], c0 = c[0], cp1 = c[1], cp2 = c[2];
        // five-tap derivatives averaged over both images: ((8 (c[-1] - c[1]) + c[2] - c[-2]) / 12 of each) / 2
        const float gx = (cp2.x - cm2.x) + (cp2.y - cm2.y) + 8.0f * ((cm1.x - cp1.x) + (cm1.y - cp1.y));
        const float gy = (vp2.x - vm2.x) + (vp2.y - vm2.y) + 8.0f * ((vm1.x - vp1.x) + (vm1.y - vp1.y));
        const float dx = gx * (1.0f / 24.0f), dy = gy * (1.0f / 24.0f);
        const float dt = c0.x - c0.y;
        const float p0 = dx * dx, p1 = dx * dy, p2 = dy * dy, p3 = dx * dt, p4 = dy * dt;
        const float4 o4 = P4[pw * NT + t];
        const float o1 = P1[pw * NT + t];
        cs[0] += (double)p0 - (double)o4.x;
        cs[1] += (double)p1 - (double)o4.y;
        cs[2] += (double)p2 - (double)o4.z;
        cs[3] += (double)p3 - (double)o4.w;
        cs[4] += (double)p4 - (double)o1;
        P4[pw * NT + t] = make_float4(p0, p1, p2, p3);
        P1[pw * NT + t] = p4;
        pw = pw + 1 == WIN ? 0 : pw + 1;
    };
    // one step: rows 2s, 2s+1 into the ring, then (DER) product rows of centres 2s-2, 2s-1, then (OUT) output rows 2s-4-2h, 2s-3-2h
    const auto step = [&](int s, auto der, auto out) {
        float2* en = E + sn;
        en[t] = make_float2(isa::lerp2(qa.s00, qa.s10, qa.s01, qa.s11, qa.a, qa.b), qa.r);
        en[NT + t] = make_float2(isa::lerp2(qb.s00, qb.s10, qb.s01, qb.s11, qb.a, qb.b), qb.r);
        sample(2 * s + 2, fa, qa);
        sample(2 * s + 3, fb, qb);
        fa = flow_at(2 * s + 4);
        fb = flow_at(2 * s + 5);
        __syncthreads();
        if constexpr (decltype(der)::value) {
            const float2* e2 = E + s2 + t;  // rows 2s-4, 2s-3
            const float2* e1 = E + s1 + t;  // rows 2s-2, 2s-1 (the centres)
            const float2 v0 = e2[0], v1 = e2[NT], v4 = en[t], v5 = en[NT + t];
            const float2 v2 = e1[0], v3 = e1[NT];
            product_row(e1, v0, v1, v3, v4);
            if constexpr (decltype(out)::value) {
#pragma unroll
                for (int ch = 0; ch < 5; ch++) Cs[ch * NT + t] = cs[ch];
            }
            product_row(e1 + NT, v1, v2, v4, v5);
            if constexpr (decltype(out)::value) {
#pragma unroll
                for (int ch = 0; ch < 5; ch++) Cs[(5 + ch) * NT + t] = cs[ch];
                __syncthreads();
                const int y = y0 + 2 * s - 4 - 2 * H + rr;  // output row
                const int x = x0 + j0;
                if (summer && y < y0 + nout && x < W) {
                    const float2* irow = isa::row_ptr(ADJ ? gin : flow_in, flow_pitch, y) + x;
                    float2 fin[PX];
#pragma unroll
                    for (int k = 0; k < PX; k++) fin[k] = j0 + k < SW && x + k < W ? __ldg(irow + k) : make_float2(0.f, 0.f);
                    // window sums of pixel j0 (2h + 1 columns from j0 + 2), then sliding by one column per pixel
                    const double* cr = Cs + rr * 5 * NT + j0 + 2;
                    double v[PX][5];
#pragma unroll
                    for (int ch = 0; ch < 5; ch++) {
                        const double* c = cr + ch * NT;
                        double sum = 0.0;
#pragma unroll
                        for (int d = 0; d < WIN; d++) sum += c[d];
                        v[0][ch] = sum;
#pragma unroll
                        for (int k = 1; k < PX; k++) v[k][ch] = sum = sum + (c[WIN + k - 1] - c[k - 1]);
                    }
                    const bool yin = y >= H && y < Himg - H;
                    if constexpr (ADJ) {
                        float* arow = isa::row_ptr(aout, a_pitch, y) + x;
#pragma unroll
                        for (int k = 0; k < PX; k++) {
                            const int xk = x + k;
                            if (j0 + k < SW && xk < W) {
                                float co[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
                                if (yin && xk >= H && xk < W - H) lk_coeffs(fin[k], v[k][0], v[k][1], v[k][2], v[k][3], v[k][4], min_det, co);
#pragma unroll
                                for (int ch = 0; ch < 5; ch++) ((float*)((char*)arow + ch * a_plane))[k] = co[ch];
                            }
                        }
                    } else {
                        float2* orow = isa::row_ptr(flow_out, flow_pitch, y) + x;
#pragma unroll
                        for (int k = 0; k < PX; k++) {
                            const int xk = x + k;
                            if (j0 + k < SW && xk < W)
                                orow[k] = yin && xk >= H && xk < W - H ? lk_update(fin[k], v[k][0], v[k][1], v[k][2], v[k][3], v[k][4], min_det) : fin[k];
                        }
                    }
                }
            } else {
                __syncthreads();  // the next step overwrites rows 2s-4, 2s-3
            }
        }
        const int tmp = s2;
        s2 = s1;
        s1 = sn;
        sn = tmp;
    };
    using T_ = std::true_type;
    using F_ = std::false_type;
    int s = 0;
#pragma unroll 1
    for (; s < 2; s++) step(s, F_{}, F_{});
#pragma unroll 1
    for (; s < R; s++) step(s, T_{}, F_{});
#pragma unroll 1
    for (; s < nsteps; s++) step(s, T_{}, T_{});
}

// Strip height: the grid of (column strips x row strips) CTAs should fill
// whole waves of the CTAs resident on the device; a CTA's time grows with its
// rows plus the 2R halo rows.
template <int H>
int lk_strip_rows(int W, int Himg)
{
    using L = LkStream<H>;
    static int slots_by_dev[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 64;
    int slots = slots_by_dev[dev];
    if (slots <= 0) {
        int nsm = 0, occ = 0;
        if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_lk_stream<H, false>, LKS_NT, L::TOTAL) != cudaSuccess || nsm * occ <= 0)
            return 64;
        slots = slots_by_dev[dev] = nsm * occ;
    }
    const long nx = (W + L::SW - 1) / L::SW;
    int best = 64;
    long best_cost = -1;
    for (int sh = 32; sh <= 192; sh += 2) {
        const long ny = (Himg + sh - 1) / sh;
        const long waves = (nx * ny + slots - 1) / slots;
        const long cost = waves * (std::min(sh, Himg) + 2 * L::R);
        if (best_cost < 0 || cost < best_cost) { best_cost = cost; best = sh; }
    }
    return best;
}

template <int H>
cudaError_t launch_lk(const float2* flow_in, float2* flow_out, size_t flow_pitch, const float* src, const float* ref, size_t img_pitch, int W, int Himg,
                      float min_det, const float2* gin, float* aout, size_t a_pitch, size_t a_plane, cudaStream_t st, int strip_rows = 0)
{
    using L = LkStream<H>;
    const bool adj = aout != nullptr;
    cudaError_t e = cudaFuncSetAttribute(adj ? k_lk_stream<H, true> : k_lk_stream<H, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)L::TOTAL);
    if (e != cudaSuccess) return e;
    const int sh = strip_rows > 0 ? strip_rows : lk_strip_rows<H>(W, Himg);
    dim3 g((W + L::SW - 1) / L::SW, (Himg + sh - 1) / sh);
    if (adj)
        k_lk_stream<H, true><<<g, LKS_NT, L::TOTAL, st>>>(flow_in, nullptr, flow_pitch, src, ref, img_pitch, W, Himg, sh, min_det, gin, aout, a_pitch,
                                                          a_plane);
    else
        k_lk_stream<H, false><<<g, LKS_NT, L::TOTAL, st>>>(flow_in, flow_out, flow_pitch, src, ref, img_pitch, W, Himg, sh, min_det, nullptr, nullptr, 0,
                                                           0);
    return cudaGetLastError();
}

// ---- adjoint of one LK iteration --------------------------------------------
// f_out(p) = f_in(p) + M(p) c(p) where M, c come from the (2h+1)^2 window
// sums of the products of dx, dy, dt at q, which are five-tap derivatives
// (mirror addressing) of the warped source w(q) = src(q + f_in(q)) and the
// reference. Given g = dL/df_out: k_lk_stream<h, true> writes the window
// sums' gradients a(p); k_box5 sums them over the window around each q
// (A(q)); k_lk_adj_deriv turns A into gradients of dx, dy, dt at q;
// k_lk_adj_flow applies the transposed derivative taps to get dL/dw and,
// through the bilinear warp, dL/df_in = g + dL/dw grad(w).

// Sum of five float planes over the (2h+1)^2 window around each pixel, zero
// outside the frame. CTA tile BX_TX x BX_TY plus the halo in shared memory:
// row sums, then column sums.
constexpr int BX_TX = 32, BX_TY = 16;

__global__ void __launch_bounds__(256) k_box5(const float* __restrict__ a, size_t pitch, size_t plane, int W, int Himg, int h, float* __restrict__ out)
{
    extern __shared__ float bsm[];
    const int SWp = BX_TX + 2 * h, SHp = BX_TY + 2 * h, win = 2 * h + 1;
    float* t0 = bsm;
    float* t1 = bsm + SWp * SHp;
    const int x0 = blockIdx.x * BX_TX, y0 = blockIdx.y * BX_TY, tid = threadIdx.x;
    for (int ch = 0; ch < 5; ch++) {
        const float* ap = (const float*)((const char*)a + ch * plane);
        float* op = (float*)((char*)out + ch * plane);
        for (int i = tid; i < SWp * SHp; i += 256) {
            const int sy = i / SWp, sx = i - sy * SWp;
            const int gx = x0 + sx - h, gy = y0 + sy - h;
            t0[i] = (unsigned)gx < (unsigned)W && (unsigned)gy < (unsigned)Himg ? __ldg(isa::row_ptr(ap, pitch, gy) + gx) : 0.f;
        }
        __syncthreads();
        for (int i = tid; i < SHp * BX_TX; i += 256) {
            const int sy = i / BX_TX, x = i - sy * BX_TX;
            float v = 0.f;
            for (int k = 0; k < win; k++) v += t0[sy * SWp + x + k];
            t1[i] = v;
        }
        __syncthreads();
        for (int i = tid; i < BX_TY * BX_TX; i += 256) {
            const int ly = i / BX_TX, lx = i - ly * BX_TX;
            const int x = x0 + lx, y = y0 + ly;
            if (x >= W || y >= Himg) continue;
            float v = 0.f;
            for (int k = 0; k < win; k++) v += t1[(ly + k) * BX_TX + lx];
            isa::row_ptr(op, pitch, y)[x] = v;
        }
        __syncthreads();
    }
}

// dL/d(dx, dy, dt) at q from the window-summed gradients A(q) of the
// products (dx^2, dx dy, dy^2, dx dt, dy dt); dx, dy, dt recomputed from the
// warped source w and the reference as the forward computes them.
__global__ void k_lk_adj_deriv(const float* __restrict__ w, size_t w_pitch, const float* __restrict__ ref, size_t r_pitch, int W, int Himg,
                               const float* __restrict__ A, size_t pitch, size_t plane, float* __restrict__ gd)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= W || y >= Himg) return;
    const auto wv = [&](int xx, int yy) { return __ldg(isa::row_ptr(w, w_pitch, isa::mirror(yy, Himg)) + isa::mirror(xx, W)); };
    const auto rv = [&](int xx, int yy) { return __ldg(isa::row_ptr(ref, r_pitch, isa::mirror(yy, Himg)) + isa::mirror(xx, W)); };
    const float gx = (wv(x + 2, y) - wv(x - 2, y)) + (rv(x + 2, y) - rv(x - 2, y)) + 8.0f * ((wv(x - 1, y) - wv(x + 1, y)) + (rv(x - 1, y) - rv(x + 1, y)));
    const float gy = (wv(x, y + 2) - wv(x, y - 2)) + (rv(x, y + 2) - rv(x, y - 2)) + 8.0f * ((wv(x, y - 1) - wv(x, y + 1)) + (rv(x, y - 1) - rv(x, y + 1)));
    const float dx = gx * (1.0f / 24.0f), dy = gy * (1.0f / 24.0f), dt = wv(x, y) - rv(x, y);
    float a[5];
#pragma unroll
    for (int ch = 0; ch < 5; ch++) a[ch] = __ldg(isa::row_ptr((const float*)((const char*)A + ch * plane), pitch, y) + x);
    isa::row_ptr(gd, pitch, y)[x] = 2.f * dx * a[0] + dy * a[1] + dt * a[3];
    isa::row_ptr((float*)((char*)gd + plane), pitch, y)[x] = dx * a[1] + 2.f * dy * a[2] + dt * a[4];
    isa::row_ptr((float*)((char*)gd + 2 * plane), pitch, y)[x] = dx * a[3] + dy * a[4];
}

// dL/dw(x) = dL/ddt(x) + the transposed five-tap filters of dL/ddx and
// dL/ddy: w(x) enters 24 dx(q) with coefficient c_k wherever
// mirror(q + k) = x (c_2 = 1, c_-2 = -1, c_-1 = 8, c_1 = -8), which happens
// only for q within 2 of x. Then dL/df_in(x) = g(x) + dL/dw(x) times the
// gradient of the bilinear (mirror) sample of src at x + f_in(x).
__global__ void k_lk_adj_flow(const float* __restrict__ gd, size_t pitch, size_t plane, const float* __restrict__ src, size_t s_pitch,
                              const float2* __restrict__ f, const float2* __restrict__ gout, float2* __restrict__ gin, size_t fpitch, int W, int Himg)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= W || y >= Himg) return;
    const float* gdx = gd;
    const float* gdy = (const float*)((const char*)gd + plane);
    const float* gdt = (const float*)((const char*)gd + 2 * plane);
    const int ks[4] = {2, -2, -1, 1};
    const float cs[4] = {1.f / 24.f, -1.f / 24.f, 8.f / 24.f, -8.f / 24.f};
    float gw = __ldg(isa::row_ptr(gdt, pitch, y) + x);
#pragma unroll
    for (int dq = -2; dq <= 2; dq++) {
        const int qx = x + dq, qy = y + dq;
        if ((unsigned)qx < (unsigned)W) {
            const float g = __ldg(isa::row_ptr(gdx, pitch, y) + qx);
#pragma unroll
            for (int t = 0; t < 4; t++)
                if (isa::mirror(qx + ks[t], W) == x) gw += cs[t] * g;
        }
        if ((unsigned)qy < (unsigned)Himg) {
            const float g = __ldg(isa::row_ptr(gdy, pitch, qy) + x);
#pragma unroll
            for (int t = 0; t < 4; t++)
                if (isa::mirror(qy + ks[t], Himg) == y) gw += cs[t] * g;
        }
    }
    const float2 fl = __ldg(isa::row_ptr(f, fpitch, y) + x);
    const float flx = floorf(fl.x), fly = floorf(fl.y);
    const int ix = x + (int)flx, iy = y + (int)fly;
    const float a = fl.x - flx, b = fl.y - fly;
    const int xa = isa::mirror(ix, W), xb = isa::mirror(ix + 1, W);
    const float* r0 = isa::row_ptr(src, s_pitch, isa::mirror(iy, Himg));
    const float* r1 = isa::row_ptr(src, s_pitch, isa::mirror(iy + 1, Himg));
    const float s00 = __ldg(r0 + xa), s10 = __ldg(r0 + xb), s01 = __ldg(r1 + xa), s11 = __ldg(r1 + xb);
    const float dwx = (1.f - b) * (s10 - s00) + b * (s11 - s01);
    const float dwy = (1.f - a) * (s01 - s00) + a * (s11 - s10);
    const float2 go = __ldg(isa::row_ptr(gout, fpitch, y) + x);
    isa::row_ptr(gin, fpitch, y)[x] = make_float2(go.x + gw * dwx, go.y + gw * dwy);
}

// Transpose of the tile term of k_flow_from_tiles: one warp per tile (i, j)
// sums weight x g over the pixels whose bilinear (clamp) lookup reads the
// tile, with the forward's own sample positions and weights.
__global__ void k_tiles_bwd(const float2* __restrict__ g, size_t fpitch, int W, int H, int tcx, int tcy, float2* __restrict__ gt, size_t tpitch)
{
    const int wid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (wid >= tcx * tcy) return;
    const int i = wid % tcx, j = wid / tcx;
    const int ylo = j == 0 ? 0 : max(0, (int)floorf((j - 0.5f) * H / tcy - 0.5f) - 1);
    const int yhi = j == tcy - 1 ? H - 1 : min(H - 1, (int)ceilf((j + 1.5f) * H / tcy - 0.5f) + 1);
    const int xlo = i == 0 ? 0 : max(0, (int)floorf((i - 0.5f) * W / tcx - 0.5f) - 1);
    const int xhi = i == tcx - 1 ? W - 1 : min(W - 1, (int)ceilf((i + 1.5f) * W / tcx - 0.5f) + 1);
    float sx = 0.f, sy = 0.f;
    for (int y = ylo; y <= yhi; y++) {
        const float yb = ((float)y + 0.5f) / (float)H * tcy - 0.5f;
        const float fly = floorf(yb);
        const int jj = (int)fly;
        const float b = yb - fly;
        const int j0 = isa::clampi(jj, 0, tcy - 1), j1 = isa::clampi(jj + 1, 0, tcy - 1);
        const float wy = (j0 == j ? 1.f - b : 0.f) + (j1 == j ? b : 0.f);
        if (wy == 0.f) continue;
        const float2* gr = isa::row_ptr(g, fpitch, y);
        for (int x = xlo + lane; x <= xhi; x += 32) {
            const float xb = ((float)x + 0.5f) / (float)W * tcx - 0.5f;
            const float flx = floorf(xb);
            const int ii = (int)flx;
            const float a = xb - flx;
            const int i0 = isa::clampi(ii, 0, tcx - 1), i1 = isa::clampi(ii + 1, 0, tcx - 1);
            const float wx = (i0 == i ? 1.f - a : 0.f) + (i1 == i ? a : 0.f);
            if (wx == 0.f) continue;
            const float2 v = __ldg(gr + x);
            sx += wx * wy * v.x;
            sy += wx * wy * v.y;
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        sx += __shfl_xor_sync(0xffffffffu, sx, o);
        sy += __shfl_xor_sync(0xffffffffu, sy, o);
    }
    if (lane == 0) isa::row_ptr(gt, tpitch, j)[i] = make_float2(sx, sy);
}

inline dim3 grid2(int w, int h, dim3 b) { return dim3((w + b.x - 1) / b.x, (h + b.y - 1) / b.y); }

}  // namespace

cudaError_t isa_launch_flow_from_tiles(const float2* tiles, size_t tile_pitch, int tcx, int tcy, int W, int H, float bx, float by, float rot,
                                       float2* flow, size_t flow_pitch, cudaStream_t st)
{
    dim3 b(32, 8);
    const float c = rot == 0.f ? 1.f : (float)cos((double)rot), s = rot == 0.f ? 0.f : (float)sin((double)rot);
    k_flow_from_tiles<<<grid2((W + FF_PX - 1) / FF_PX, H, b), b, 0, st>>>(tiles, tile_pitch, tcx, tcy, W, H, bx, by, c, s, flow, flow_pitch);
    return cudaGetLastError();
}

cudaError_t isa_launch_warp(const float* img, size_t img_pitch, int W, int H, const float2* flow, size_t flow_pitch, float* out,
                            size_t out_pitch, cudaStream_t st)
{
    dim3 b(32, 8);
    k_warp<<<grid2(W, H, b), b, 0, st>>>(img, img_pitch, W, H, flow, flow_pitch, out, out_pitch);
    return cudaGetLastError();
}

cudaError_t isa_launch_derivatives(const float* src, const float* tgt, size_t pitch, int W, int H, float* ix, float* iy, float* it,
                                   size_t out_pitch, cudaStream_t st)
{
    dim3 b(32, 8);
    k_derivatives<<<grid2(W, H, b), b, 0, st>>>(src, tgt, pitch, W, H, ix, iy, it, out_pitch);
    return cudaGetLastError();
}

cudaError_t isa_launch_derivatives2(const float* img, size_t pitch, int W, int H, float* ix, float* iy, size_t out_pitch, cudaStream_t st)
{
    dim3 b(32, 8);
    k_derivatives2<<<grid2(W, H, b), b, 0, st>>>(img, pitch, W, H, ix, iy, out_pitch);
    return cudaGetLastError();
}

cudaError_t isa_launch_lk_sums(float2* flow, size_t flow_pitch, const float* ix, const float* iy, const float* it, size_t pitch, int W, int H,
                               int half, float min_det, cudaStream_t st)
{
    dim3 b(32, 8);
    k_lk_sums<<<grid2(W, H, b), b, 0, st>>>(flow, flow_pitch, ix, iy, it, pitch, W, H, half, min_det);
    return cudaGetLastError();
}

cudaError_t isa_launch_lk_iteration(const float2* flow_in, float2* flow_out, size_t flow_pitch, const float* src, const float* ref,
                                    size_t img_pitch, int W, int H, int half, float min_det, cudaStream_t st, int strip_rows)
{
    switch (half) {
#define ISA_LK_CASE(h) case h: return launch_lk<h>(flow_in, flow_out, flow_pitch, src, ref, img_pitch, W, H, min_det, nullptr, nullptr, 0, 0, st, strip_rows);
    ISA_LK_CASE(0) ISA_LK_CASE(1) ISA_LK_CASE(2) ISA_LK_CASE(3) ISA_LK_CASE(4) ISA_LK_CASE(5) ISA_LK_CASE(6) ISA_LK_CASE(7) ISA_LK_CASE(8)
    ISA_LK_CASE(9) ISA_LK_CASE(10) ISA_LK_CASE(11) ISA_LK_CASE(12) ISA_LK_CASE(13) ISA_LK_CASE(14) ISA_LK_CASE(15)
#undef ISA_LK_CASE
    }
    return cudaErrorInvalidValue;
}

cudaError_t isa_launch_lk_adjoint(const float2* f, const float2* gout, float2* gin, size_t fpitch, const float* src, const float* ref, size_t img_pitch,
                                  int W, int H, int half, float min_det, float* wplane, float* a5, float* A5, float* gd3, cudaStream_t st)
{
    if (half < 0 || half > 15) return cudaErrorInvalidValue;
    const size_t sp = (size_t)W * 4, plane = sp * H;
    cudaError_t e = isa_launch_warp(src, img_pitch, W, H, f, fpitch, wplane, sp, st);
    if (e != cudaSuccess) return e;
    switch (half) {
#define ISA_LK_CASE(h) case h: e = launch_lk<h>(f, nullptr, fpitch, src, ref, img_pitch, W, H, min_det, gout, a5, sp, plane, st); break;
    ISA_LK_CASE(0) ISA_LK_CASE(1) ISA_LK_CASE(2) ISA_LK_CASE(3) ISA_LK_CASE(4) ISA_LK_CASE(5) ISA_LK_CASE(6) ISA_LK_CASE(7) ISA_LK_CASE(8)
    ISA_LK_CASE(9) ISA_LK_CASE(10) ISA_LK_CASE(11) ISA_LK_CASE(12) ISA_LK_CASE(13) ISA_LK_CASE(14) ISA_LK_CASE(15)
#undef ISA_LK_CASE
    }
    if (e != cudaSuccess) return e;
    const size_t bsmem = (size_t)((BX_TX + 2 * half) * (BX_TY + 2 * half) + (BX_TY + 2 * half) * BX_TX) * sizeof(float);
    k_box5<<<dim3((W + BX_TX - 1) / BX_TX, (H + BX_TY - 1) / BX_TY), 256, bsmem, st>>>(a5, sp, plane, W, H, half, A5);
    dim3 b(32, 8);
    k_lk_adj_deriv<<<grid2(W, H, b), b, 0, st>>>(wplane, sp, ref, img_pitch, W, H, A5, sp, plane, gd3);
    k_lk_adj_flow<<<grid2(W, H, b), b, 0, st>>>(gd3, sp, plane, src, img_pitch, f, gout, gin, fpitch, W, H);
    return cudaGetLastError();
}

cudaError_t isa_launch_tiles_bwd(const float2* g, size_t fpitch, int W, int H, int tcx, int tcy, float2* gt, size_t tpitch, cudaStream_t st)
{
    const long warps = (long)tcx * tcy;
    k_tiles_bwd<<<(unsigned)((warps * 32 + 255) / 256), 256, 0, st>>>(g, fpitch, W, H, tcx, tcy, gt, tpitch);
    return cudaGetLastError();
}
