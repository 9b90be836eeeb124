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
// lucasKanadeOptim). A CTA of LKS_NT threads owns a vertical strip: thread t
// owns image column x0 - R + t (R = h + 2, mirrored at the border) and walks
// down the strip one row at a time:
//   1. the warped source and the reference at (column, row) go into a
//      six-row ring in shared memory (one row more than the derivatives
//      read, so a slot is rewritten only after the next row's barrier and
//      the step needs no barrier at its end); the global loads for the next
//      rows are issued one and two rows ahead (flow, then the bilinear
//      samples);
//   2. five-tap derivatives at the ring's centre row (neighbouring columns
//      from shared memory), FP32 products, and per-column vertical window
//      sums in FP64 registers (the product leaving the window comes from a
//      per-thread ring of the last 2h + 1 rows);
//   3. every two output rows, the row window sums (sliding FP64 sums over
//      2h + 1 columns, two pixels per thread) and the 2x2 solve.
// The FP64 sums hold the FP32 products exactly enough that the order of
// summation does not matter at FP32 output precision.
constexpr int LKS_NT = 128, LKS_SH = 64;

template <int H>
struct LkStream {
    static constexpr int R = H + 2, SW = LKS_NT - 2 * R, WIN = 2 * H + 1;
    static constexpr int NSEG = (SW + 1) / 2;
    static constexpr size_t E_BYTES = (size_t)2 * 6 * LKS_NT * 4;
    static constexpr size_t P_BYTES = (size_t)WIN * 5 * LKS_NT * 4;
    static constexpr size_t OFF_P = E_BYTES, OFF_C = (OFF_P + P_BYTES + 15) / 16 * 16;
    static constexpr size_t TOTAL = OFF_C + (size_t)2 * 5 * LKS_NT * 8;
};

template <int H>
__global__ void __launch_bounds__(LKS_NT) k_lk_stream(const float2* __restrict__ flow_in, float2* __restrict__ flow_out, size_t flow_pitch,
                                                      const float* __restrict__ src, const float* __restrict__ ref, size_t img_pitch, int W,
                                                      int Himg, float min_det)
{
    using L = LkStream<H>;
    constexpr int R = L::R, SW = L::SW, WIN = L::WIN, NT = LKS_NT;
    extern __shared__ __align__(16) unsigned char smem[];
    float* Ew = (float*)smem;            // [6][NT]
    float* Er = Ew + 6 * NT;              // [6][NT]
    float* Pr = (float*)(smem + L::OFF_P);    // [WIN][5][NT]
    double* Cs = (double*)(smem + L::OFF_C);  // [2][5][NT]
    const int t = threadIdx.x;
    const int x0 = blockIdx.x * SW, y0 = blockIdx.y * LKS_SH;
    const int nout = min(LKS_SH, Himg - y0);
    const int nE = nout + 2 * R;
    const int col = isa::mirror(x0 - R + t, W);
    // pipeline: flow two rows ahead, bilinear samples one row ahead
    float2 fnext;
    float s00, s10, s01, s11, sa, sb, sref;
    const auto erow = [&](int e) { return isa::mirror(y0 - R + e, Himg); };
    const auto issue_samples = [&](int row, float2 f) {
        const float flx = floorf(f.x), fly = floorf(f.y);
        const int ix = col + (int)flx, iy = row + (int)fly;
        sa = f.x - flx;
        sb = f.y - fly;
        const int xa = isa::mirror(ix, W), xb = isa::mirror(ix + 1, W);
        const float* r0 = isa::row_ptr(src, img_pitch, isa::mirror(iy, Himg));
        const float* r1 = isa::row_ptr(src, img_pitch, isa::mirror(iy + 1, Himg));
        s00 = __ldg(r0 + xa); s10 = __ldg(r0 + xb); s01 = __ldg(r1 + xa); s11 = __ldg(r1 + xb);
        sref = __ldg(isa::row_ptr(ref, img_pitch, row) + col);
    };
    issue_samples(erow(0), __ldg(isa::row_ptr(flow_in, flow_pitch, erow(0)) + col));
    if (nE > 1) fnext = __ldg(isa::row_ptr(flow_in, flow_pitch, erow(1)) + col);
    double cs[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    // ring slots of rows e, e-1, e-2, e-3, e-4 (mod 5) and of the product row (mod WIN), advanced incrementally
    int r0 = 0, r1 = 5, r2 = 4, r3 = 3, r4 = 2, pw = 0;
    for (int e = 0; e < nE; e++) {
        Ew[r0 * NT + t] = isa::lerp2(s00, s10, s01, s11, sa, sb);
        Er[r0 * NT + t] = sref;
        if (e + 1 < nE) {
            issue_samples(erow(e + 1), fnext);
            if (e + 2 < nE) fnext = __ldg(isa::row_ptr(flow_in, flow_pitch, erow(e + 2)) + col);
        }
        __syncthreads();
        if (e >= 4) {
            const int gi = e - 4;  // product row: image row y0 - h + gi
            if (t >= 2 && t < NT - 2) {
                // five-tap derivatives averaged over both images: ((8 (c[-1] - c[1]) + c[2] - c[-2]) / 12 of each) / 2
                const float* ew = Ew + r2 * NT + t;
                const float* er = Er + r2 * NT + t;
                const float gx = (ew[2] - ew[-2]) + (er[2] - er[-2]) + 8.0f * ((ew[-1] - ew[1]) + (er[-1] - er[1]));
                const float gy = (Ew[r0 * NT + t] - Ew[r4 * NT + t]) + (Er[r0 * NT + t] - Er[r4 * NT + t]) +
                                 8.0f * ((Ew[r3 * NT + t] - Ew[r1 * NT + t]) + (Er[r3 * NT + t] - Er[r1 * NT + t]));
                const float dx = gx * (1.0f / 24.0f), dy = gy * (1.0f / 24.0f);
                const float dt = ew[0] - er[0];
                const float p[5] = {dx * dx, dx * dy, dy * dy, dx * dt, dy * dt};
                float* pr = Pr + pw * 5 * NT + t;
#pragma unroll
                for (int ch = 0; ch < 5; ch++) {
                    const float old = gi >= WIN ? pr[ch * NT] : 0.f;
                    cs[ch] += (double)p[ch] - (double)old;
                    pr[ch * NT] = p[ch];
                }
            }
            pw = pw + 1 == WIN ? 0 : pw + 1;
            if (gi >= 2 * H) {
                const int o = gi - 2 * H;  // output row y0 + o
                if (t >= 2 && t < NT - 2) {
#pragma unroll
                    for (int ch = 0; ch < 5; ch++) Cs[((o & 1) * 5 + ch) * NT + t] = cs[ch];
                }
                if ((o & 1) || o == nout - 1) {
                    __syncthreads();
                    const int rlo = o & ~1, nr = o - rlo + 1;
                    if (t < nr * L::NSEG) {
                        const int r = rlo + t / L::NSEG, j0 = 2 * (t % L::NSEG);
                        const double* cr = Cs + (r & 1) * 5 * NT + j0 + 2;
                        double v0[5], v1[5];
#pragma unroll
                        for (int ch = 0; ch < 5; ch++) {
                            const double* c = cr + ch * NT;
                            double s = 0.0;
#pragma unroll
                            for (int d = 0; d < WIN; d++) s += c[d];
                            v0[ch] = s;
                            v1[ch] = s + (c[WIN] - c[0]);
                        }
                        const int y = y0 + r;
                        const bool yin = y >= H && y < Himg - H;
                        float2* orow = isa::row_ptr(flow_out, flow_pitch, y);
                        const float2* irow = isa::row_ptr(flow_in, flow_pitch, y);
                        int x = x0 + j0;
                        if (j0 < SW && x < W) {
                            float2 f = __ldg(irow + x);
                            if (yin && x >= H && x < W - H) f = lk_update(f, v0[0], v0[1], v0[2], v0[3], v0[4], min_det);
                            orow[x] = f;
                        }
                        x++;
                        if (j0 + 1 < SW && x < W) {
                            float2 f = __ldg(irow + x);
                            if (yin && x >= H && x < W - H) f = lk_update(f, v1[0], v1[1], v1[2], v1[3], v1[4], min_det);
                            orow[x] = f;
                        }
                    }
                }
            }
        }
        r4 = r3; r3 = r2; r2 = r1; r1 = r0; r0 = r0 + 1 == 6 ? 0 : r0 + 1;
    }
}

template <int H>
cudaError_t launch_lk(const float2* flow_in, float2* flow_out, size_t flow_pitch, const float* src, const float* ref, size_t img_pitch, int W, int Himg,
                      float min_det, cudaStream_t st)
{
    using L = LkStream<H>;
    cudaError_t e = cudaFuncSetAttribute(k_lk_stream<H>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L::TOTAL);
    if (e != cudaSuccess) return e;
    dim3 g((W + L::SW - 1) / L::SW, (Himg + LKS_SH - 1) / LKS_SH);
    k_lk_stream<H><<<g, LKS_NT, L::TOTAL, st>>>(flow_in, flow_out, flow_pitch, src, ref, img_pitch, W, Himg, min_det);
    return cudaGetLastError();
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
