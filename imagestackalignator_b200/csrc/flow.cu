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
// k_lk_iteration fuses one reference iteration (warp, Set(0) x3, derivatives,
// lucasKanadeOptim) for a 32 x 16 tile: warped and reference images over the
// tile plus a (h + 2) halo in shared memory, FP32 gradient products over the
// h halo, exact FP64 sliding window sums, and the 2x2 pseudo-inverse in FP64.
#include "isa_internal.cuh"

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

// lucasKanadeOptim's pseudo-inverse (opticalFlow.cu:229-290) in FP64. For a
// well-conditioned matrix (lambda2 > 1e-3 lambda1) the angle/singular-value
// construction of the reference equals the closed-form inverse to ~1e-10
// relative; below that the reference's own construction is evaluated.
// Returns false where the reference leaves the pixel unchanged
// (sigma1 < minDet; the reference tests min(sigma1, sigma1)).
__device__ __forceinline__ bool lk_pinv(double a, double b, double d, double min_det, double (&M)[4])
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
        M[0] = d * inv; M[1] = -b * inv; M[2] = -b * inv; M[3] = a * inv;
        return true;
    }
    const double c = b;
    double th = 0.5 * atan2(2 * a * c + 2 * b * d, a * a + b * b - c * c - d * d);
    double ct = cos(th), st = sin(th);
    double S1 = a * a + b * b + c * c + d * d;
    double S2 = sqrt((a * a + b * b - c * c - d * d) * (a * a + b * b - c * c - d * d) + 4 * (a * c + b * d) * (a * c + b * d));
    double s1 = sqrt((S1 + S2) / 2), s2 = sqrt((S1 - S2) / 2);
    if (s1 < min_det) return false;
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
    M[0] = V0 * m0 + V1 * m2;
    M[1] = V0 * m1 + V1 * m3;
    M[2] = V2 * m0 + V3 * m2;
    M[3] = V2 * m1 + V3 * m3;
    return true;
}

__device__ __forceinline__ float2 lk_update(float2 f, double sxx, double sxy, double syy, double sxt, double syt, double min_det)
{
    double M[4];
    if (!lk_pinv(sxx, sxy, syy, min_det, M)) return f;
    double u = M[0] * sxt + M[1] * syt, v = M[2] * sxt + M[3] * syt;
    if (isnan(u)) u = 0;
    if (isnan(v)) v = 0;
    return make_float2((float)((double)f.x + u), (float)((double)f.y + v));
}

__global__ void k_flow_from_tiles(const float2* __restrict__ tiles, size_t tile_pitch, int tcx, int tcy, int W, int H, float bx, float by,
                                  float rot, float2* __restrict__ flow, size_t flow_pitch)
{
    int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= W || y >= H) return;
    float c = cosf(rot), s = sinf(rot);
    float fx = c * -bx - s * -by;
    float fy = s * -bx + c * -by;
    float pcx = (float)(x - W / 2), pcy = (float)(y - H / 2);
    fx += c * pcx - s * pcy - pcx;
    fy += s * pcx + c * pcy - pcy;
    float xb = ((float)x + 0.5f) / (float)W * tcx - 0.5f, yb = ((float)y + 0.5f) / (float)H * tcy - 0.5f;
    float flx = floorf(xb), fly = floorf(yb);
    int i = (int)flx, j = (int)fly;
    float a = xb - flx, b = yb - fly;
    int i0 = isa::clampi(i, 0, tcx - 1), i1 = isa::clampi(i + 1, 0, tcx - 1), j0 = isa::clampi(j, 0, tcy - 1), j1 = isa::clampi(j + 1, 0, tcy - 1);
    const float2* r0 = isa::row_ptr(tiles, tile_pitch, j0);
    const float2* r1 = isa::row_ptr(tiles, tile_pitch, j1);
    float2 p00 = r0[i0], p10 = r0[i1], p01 = r1[i0], p11 = r1[i1];
    fx += isa::lerp2(p00.x, p10.x, p01.x, p11.x, a, b);
    fy += isa::lerp2(p00.y, p10.y, p01.y, p11.y, a, b);
    isa::row_ptr(flow, flow_pitch, y)[x] = make_float2(fx, fy);
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

constexpr int LK_TW = 32, LK_TH = 16;

// Tile geometry for half window H: warped/reference images over the tile
// plus an (H + 2) halo (E), gradient products over the tile plus an H halo
// (G), per-column vertical window sums of the products for the tile rows,
// stored with one leading slot per row for the in-place prefix sum (V).
template <int H>
struct LkDims {
    static constexpr int R = H + 2, EW = LK_TW + 2 * R, EH = LK_TH + 2 * R;
    static constexpr int GW = LK_TW + 2 * H, GH = LK_TH + 2 * H, GN = GW * GH, WIN = 2 * H + 1;
    static constexpr int VS = GW + 1;
    static constexpr size_t E_BYTES = (size_t)EW * EH * 4;
    static constexpr size_t P_BYTES = (size_t)5 * GN * 4;
    static constexpr size_t OFF_R = E_BYTES, OFF_P = 2 * E_BYTES, OFF_V = (OFF_P + P_BYTES + 15) / 16 * 16;
    static constexpr size_t TOTAL = OFF_V + (size_t)5 * LK_TH * VS * 8;
};

// One reference iteration (warp, Set(0) x3, derivatives, lucasKanadeOptim)
// for a 32 x 16 tile, blockDim (32, 8). Window sums: FP32 products summed in
// FP64, first down each column with a sliding window (exact: FP64 holds the
// sum of a few FP32 values), then along each row through a prefix sum.
template <int H>
__global__ void __launch_bounds__(256) k_lk_iteration(const float2* __restrict__ flow_in, float2* __restrict__ flow_out, size_t flow_pitch,
                                                     const float* __restrict__ src, const float* __restrict__ ref, size_t img_pitch, int W,
                                                     int Himg, float min_det)
{
    using D = LkDims<H>;
    extern __shared__ __align__(16) unsigned char smem[];
    float* Ew = (float*)smem;
    float* Er = (float*)(smem + D::OFF_R);
    float* P = (float*)(smem + D::OFF_P);
    double* V = (double*)(smem + D::OFF_V);
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * 32 + tx;
    const int x0 = blockIdx.x * LK_TW, y0 = blockIdx.y * LK_TH;
    // 1. warped source and reference, mirrored at the image border
    for (int ey = ty; ey < D::EH; ey += 8) {
        const int my = isa::mirror(y0 - D::R + ey, Himg);
        const float2* frow = isa::row_ptr(flow_in, flow_pitch, my);
        const float* rrow = isa::row_ptr(ref, img_pitch, my);
        for (int ex = tx; ex < D::EW; ex += 32) {
            const int mx = isa::mirror(x0 - D::R + ex, W);
            const float2 f = __ldg(frow + mx);
            Ew[ey * D::EW + ex] = bilinear_mirror(src, img_pitch, W, Himg, mx, my, f.x, f.y);
            Er[ey * D::EW + ex] = __ldg(rrow + mx);
        }
    }
    __syncthreads();
    // 2. derivatives (five-tap, averaged over both images) and products
    for (int gy = ty; gy < D::GH; gy += 8)
        for (int gx = tx; gx < D::GW; gx += 32) {
            const int e = (gy + 2) * D::EW + gx + 2;
            float t0 = (Ew[e + 2] - Ew[e + 1] * 8.0f + Ew[e - 1] * 8.0f - Ew[e - 2]) / 12.0f;
            float t1 = (Er[e + 2] - Er[e + 1] * 8.0f + Er[e - 1] * 8.0f - Er[e - 2]) / 12.0f;
            const float dx = (t0 + t1) * 0.5f;
            t0 = (Ew[e + 2 * D::EW] - Ew[e + D::EW] * 8.0f + Ew[e - D::EW] * 8.0f - Ew[e - 2 * D::EW]) / 12.0f;
            t1 = (Er[e + 2 * D::EW] - Er[e + D::EW] * 8.0f + Er[e - D::EW] * 8.0f - Er[e - 2 * D::EW]) / 12.0f;
            const float dy = (t0 + t1) * 0.5f;
            const float dt = Ew[e] - Er[e];
            const int g = gy * D::GW + gx;
            P[g] = dx * dx;
            P[D::GN + g] = dx * dy;
            P[2 * D::GN + g] = dy * dy;
            P[3 * D::GN + g] = dx * dt;
            P[4 * D::GN + g] = dy * dt;
        }
    __syncthreads();
    // 3. vertical sliding sums per (channel, column)
    for (int job = tid; job < 5 * D::GW; job += 256) {
        const int ch = job / D::GW, gx = job - ch * D::GW;
        const float* col = P + ch * D::GN + gx;
        double* out = V + (size_t)ch * LK_TH * D::VS + 1 + gx;
        double sum = 0;
#pragma unroll
        for (int k = 0; k < D::WIN; k++) sum += (double)col[k * D::GW];
        out[0] = sum;
#pragma unroll 4
        for (int y = 1; y < LK_TH; y++) {
            sum += (double)col[(y + D::WIN - 1) * D::GW] - (double)col[(y - 1) * D::GW];
            out[y * D::VS] = sum;
        }
    }
    __syncthreads();
    // 4. prefix sums along each row (slot 0 holds 0)
    if (tid < 5 * LK_TH) {
        double* row = V + (size_t)tid * D::VS;
        double acc = 0;
        row[0] = 0;
        for (int k = 1; k < D::VS; k++) {
            acc += row[k];
            row[k] = acc;
        }
    }
    __syncthreads();
    // 5. window sums = prefix differences; 2x2 solve; update
    for (int ly = ty; ly < LK_TH; ly += 8) {
        const int x = x0 + tx, y = y0 + ly;
        if (x >= W || y >= Himg) continue;
        float2 f = __ldg(isa::row_ptr(flow_in, flow_pitch, y) + x);
        if (x >= H && x < W - H && y >= H && y < Himg - H) {
            double v[5];
#pragma unroll
            for (int ch = 0; ch < 5; ch++) {
                const double* row = V + (size_t)(ch * LK_TH + ly) * D::VS;
                v[ch] = row[tx + D::WIN] - row[tx];
            }
            f = lk_update(f, v[0], v[1], v[2], v[3], v[4], min_det);
        }
        isa::row_ptr(flow_out, flow_pitch, y)[x] = f;
    }
}

template <int H>
cudaError_t launch_lk(const float2* flow_in, float2* flow_out, size_t flow_pitch, const float* src, const float* ref, size_t img_pitch, int W, int Himg,
                      float min_det, cudaStream_t st)
{
    using D = LkDims<H>;
    cudaError_t e = cudaFuncSetAttribute(k_lk_iteration<H>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)D::TOTAL);
    if (e != cudaSuccess) return e;
    dim3 g((W + LK_TW - 1) / LK_TW, (Himg + LK_TH - 1) / LK_TH);
    k_lk_iteration<H><<<g, dim3(32, 8), D::TOTAL, st>>>(flow_in, flow_out, flow_pitch, src, ref, img_pitch, W, Himg, min_det);
    return cudaGetLastError();
}

inline dim3 grid2(int w, int h, dim3 b) { return dim3((w + b.x - 1) / b.x, (h + b.y - 1) / b.y); }

}  // namespace

cudaError_t isa_launch_flow_from_tiles(const float2* tiles, size_t tile_pitch, int tcx, int tcy, int W, int H, float bx, float by, float rot,
                                       float2* flow, size_t flow_pitch, cudaStream_t st)
{
    dim3 b(32, 8);
    k_flow_from_tiles<<<grid2(W, H, b), b, 0, st>>>(tiles, tile_pitch, tcx, tcy, W, H, bx, by, rot, flow, flow_pitch);
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
                                    size_t img_pitch, int W, int H, int half, float min_det, cudaStream_t st)
{
    switch (half) {
#define ISA_LK_CASE(h) case h: return launch_lk<h>(flow_in, flow_out, flow_pitch, src, ref, img_pitch, W, H, min_det, st);
    ISA_LK_CASE(0) ISA_LK_CASE(1) ISA_LK_CASE(2) ISA_LK_CASE(3) ISA_LK_CASE(4) ISA_LK_CASE(5) ISA_LK_CASE(6) ISA_LK_CASE(7) ISA_LK_CASE(8)
    ISA_LK_CASE(9) ISA_LK_CASE(10) ISA_LK_CASE(11) ISA_LK_CASE(12) ISA_LK_CASE(13) ISA_LK_CASE(14) ISA_LK_CASE(15)
#undef ISA_LK_CASE
    }
    return cudaErrorInvalidValue;
}
