// Pyramid tile alignment (PatchTracker.Track, PEFStudioDX/PatchTracker.cs:317-360)
// and the multi-pair least-squares solve (ShiftCollection.MinimizeCUBLAS,
// PEFStudioDX/ShiftCollection.cs:738-822).
//
// k_track: one CTA per (frame pair, tile). The reference template tile (T x T,
// kernel.cu:175-228) and the search block (B x B, B = T + 2S, kernel.cu:234-288)
// are staged in shared memory; the L2 map D(s) = sum (r - t(s))^2 for
// s in [-S, S]^2 is computed directly (the reference's FFT cross-correlation,
// squaredSum and box filters, kernel.cu:29-171, compute the same quantity as
// sum r^2 + sum t^2 - 2 CC). One thread per (template row, shift row), rows
// reduced with warp shuffles; warp 0 then does findMinimum (kernel.cu:422-546)
// and preShift += result (:355-358).
#include "isa_internal.cuh"
#include <float.h>
#include <algorithm>

namespace {

__constant__ float c_fit[5][9] = {
    {0.25f, -0.5f, 0.25f, 0.5f, -1.0f, 0.5f, 0.25f, -0.5f, 0.25f},       // d2/dx2
    {0.25f, 0.5f, 0.25f, -0.5f, -1.0f, -0.5f, 0.25f, 0.5f, 0.25f},       // d2/dy2
    {0.25f, 0.f, -0.25f, 0.f, 0.f, 0.f, -0.25f, 0.f, 0.25f},             // d2/dxdy
    {-0.125f, 0.f, 0.125f, -0.25f, 0.f, 0.25f, -0.125f, 0.f, 0.125f},   // d/dx
    {-0.125f, -0.25f, -0.125f, 0.f, 0.f, 0.f, 0.125f, 0.25f, 0.125f}};  // d/dy

__device__ __forceinline__ void tile_offset(int tx, int ty, int T, int Wl, int Hl, float bx, float by, float rot, float addx, float addy,
                                            int& ox, int& oy)
{
    float sf = 0.f, cf = 1.f;  // sinf(0) and cosf(0) are exact
    if (rot != 0.f) { sf = sinf(rot); cf = cosf(rot); }
    float sx = addx, sy = addy;
    sx += cf * -bx - sf * -by;
    sy += sf * -bx + cf * -by;
    float pcx = (float)(tx * T + T / 2 - Wl / 2), pcy = (float)(ty * T + T / 2 - Hl / 2);
    sx += cf * pcx - sf * pcy - pcx;
    sy += sf * pcx + cf * pcy - pcy;
    ox = (int)roundf(sx);
    oy = (int)roundf(sy);
}

// Shared-memory layout of k_track, in floats. The template is stored as
// interleaved row pairs (rows 2i and 2i + 1 side by side), so one 64-bit
// load gives a thread both of its template rows.
template <int T, int S>
struct TrackDims {
    static_assert(T % 2 == 0 && T <= 64 && 32 % (T / 2 > 32 ? 32 : T / 2) == 0, "tile size");
    static constexpr int B = T + 2 * S, D = 2 * S + 1;
    static constexpr int HP = T / 2;        // template row pairs = lanes summed per shift row
    static constexpr int TP2 = T + 1;       // row-pair stride in float2: odd, so 64-bit column reads are conflict-free
    static constexpr int BP = B + 1;        // odd stride: conflict-free column reads
    static constexpr int NI = HP * D;       // (row pair, shift row) items
    static constexpr int NT = (NI + 31) / 32 * 32;
    static constexpr int OFF_TPL = 0, OFF_BLK = OFF_TPL + HP * TP2 * 2, OFF_MAP = OFF_BLK + B * BP;
    static constexpr int TOTAL = OFF_MAP + D * D;
    static constexpr size_t BYTES = (size_t)TOTAL * sizeof(float);
};

// Thread (row pair, sy) streams template rows 2i, 2i + 1 against block rows
// 2i + sy, 2i + 1 + sy with a D-wide register window of float2 pairs,
// accumulating (r - t)^2 for both rows and the D column shifts with packed
// FP32x2 arithmetic (each lane of a pair rounds exactly as the scalar
// operation would); the rows are then summed across lanes with shuffles in
// a fixed order (deterministic), and warp 0 finds the first minimum.
template <int T, int S>
__global__ void __launch_bounds__(TrackDims<T, S>::NT) k_track(const float* const* __restrict__ frames, size_t pitch, int Wl, int Hl, int tcx,
                                                               int tcy, const isa_pair_desc* __restrict__ pairs, float2* __restrict__ grids,
                                                               size_t grid_pitch, size_t grid_stride, float threshold, float* __restrict__ scores,
                                                               int* __restrict__ argmin_out, int* __restrict__ offsets_out)
{
    using L = TrackDims<T, S>;
    constexpr int B = L::B, D = L::D, TP2 = L::TP2, BP = L::BP, HP = L::HP;
    extern __shared__ __align__(16) float smf[];
    float* tpl = smf + L::OFF_TPL;
    float* blk = smf + L::OFF_BLK;
    float* map = smf + L::OFF_MAP;
    const int p = blockIdx.x;
    const int tile = blockIdx.y;
    const int ty = tile / tcx, tx = tile - ty * tcx;
    const isa_pair_desc pd = pairs[p];
    float2* gline = (float2*)((char*)grids + (size_t)pd.grid * grid_stride + (size_t)ty * grid_pitch);
    const float* imr = frames[pd.ref];
    const float* imt = frames[pd.trk];
    int oxr, oyr, oxt, oyt;
    tile_offset(tx, ty, T, Wl, Hl, pd.base_ref_x, pd.base_ref_y, pd.rot_ref, 0.f, 0.f, oxr, oyr);
    float2 pre = gline[tx];
    tile_offset(tx, ty, T, Wl, Hl, pd.base_trk_x, pd.base_trk_y, pd.rot_trk, pre.x, pre.y, oxt, oyt);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    constexpr int NW = L::NT / 32;
    // stage the template and the search block, one row per warp iteration; all loads of a warp are
    // issued before any store, so their latencies overlap
    constexpr int TX = (T + 31) / 32, BX = (B + 31) / 32;
    constexpr int TR = (T + NW - 1) / NW, BR = (B + NW - 1) / NW;
    float vt[TR][TX], vb[BR][BX];
    const int xr0 = tx * T + S + oxr, yr0 = ty * T + S + oyr, xt0 = tx * T + oxt, yt0 = ty * T + oyt;
    if (xr0 >= 0 && xr0 + T <= Wl && yr0 >= 0 && yr0 + T <= Hl && xt0 >= 0 && xt0 + B <= Wl && yt0 >= 0 && yt0 + B <= Hl) {
        // both regions inside the level image: no clamping, rows a fixed stride apart
        const char* pr = (const char*)(imr + xr0 + lane) + (size_t)(yr0 + warp) * pitch;
        const char* pt = (const char*)(imt + xt0 + lane) + (size_t)(yt0 + warp) * pitch;
        const size_t step = (size_t)NW * pitch;
#pragma unroll
        for (int i = 0; i < TR; i++)
            if (warp + i * NW < T) {
#pragma unroll
                for (int k = 0; k < TX; k++)
                    if (lane + 32 * k < T) vt[i][k] = __ldg((const float*)(pr + i * step) + 32 * k);
            }
#pragma unroll
        for (int i = 0; i < BR; i++)
            if (warp + i * NW < B) {
#pragma unroll
                for (int k = 0; k < BX; k++)
                    if (lane + 32 * k < B) vb[i][k] = __ldg((const float*)(pt + i * step) + 32 * k);
            }
    } else {
        // clamped columns once per lane, clamped rows per iteration (replicate border)
        int cr[TX], ct[BX];
#pragma unroll
        for (int k = 0; k < TX; k++) cr[k] = isa::clampi(xr0 + lane + 32 * k, 0, Wl - 1);
#pragma unroll
        for (int k = 0; k < BX; k++) ct[k] = isa::clampi(xt0 + lane + 32 * k, 0, Wl - 1);
#pragma unroll
        for (int i = 0; i < TR; i++) {
            const int y = warp + i * NW;
            if (y < T) {
                const float* row = isa::row_ptr(imr, pitch, isa::clampi(yr0 + y, 0, Hl - 1));
#pragma unroll
                for (int k = 0; k < TX; k++)
                    if (lane + 32 * k < T) vt[i][k] = __ldg(row + cr[k]);
            }
        }
#pragma unroll
        for (int i = 0; i < BR; i++) {
            const int y = warp + i * NW;
            if (y < B) {
                const float* row = isa::row_ptr(imt, pitch, isa::clampi(yt0 + y, 0, Hl - 1));
#pragma unroll
                for (int k = 0; k < BX; k++)
                    if (lane + 32 * k < B) vb[i][k] = __ldg(row + ct[k]);
            }
        }
    }
#pragma unroll
    for (int i = 0; i < TR; i++) {
        const int y = warp + i * NW;
        if (y < T) {
            float* dst = tpl + (y >> 1) * TP2 * 2 + (y & 1);
#pragma unroll
            for (int k = 0; k < TX; k++)
                if (lane + 32 * k < T) dst[2 * (lane + 32 * k)] = vt[i][k];
        }
    }
#pragma unroll
    for (int i = 0; i < BR; i++) {
        const int y = warp + i * NW;
        if (y < B) {
#pragma unroll
            for (int k = 0; k < BX; k++)
                if (lane + 32 * k < B) blk[y * BP + lane + 32 * k] = vb[i][k];
        }
    }
    __syncthreads();
    const int yp = tid % HP, sy = tid / HP;
    float2 acc[D];
#pragma unroll
    for (int k = 0; k < D; k++) acc[k] = make_float2(0.f, 0.f);
    if (tid < L::NI) {
        const float2* tr = (const float2*)tpl + yp * TP2;
        const float* b0 = blk + (2 * yp + sy) * BP;
        const float* b1 = b0 + BP;
        const float2 m1 = make_float2(-1.f, -1.f);
        float2 win[D];
#pragma unroll
        for (int k = 0; k < D - 1; k++) win[k] = make_float2(b0[k], b1[k]);
#pragma unroll
        for (int x = 0; x < T; x++) {
            win[D - 1] = make_float2(b0[x + D - 1], b1[x + D - 1]);
            const float2 r = tr[x];
#pragma unroll
            for (int k = 0; k < D; k++) {
                const float2 d = __ffma2_rn(win[k], m1, r);  // r - t, exactly rounded
                acc[k] = __ffma2_rn(d, d, acc[k]);
            }
#pragma unroll
            for (int k = 0; k < D - 1; k++) win[k] = win[k + 1];
        }
    }
    float sum[D];
#pragma unroll
    for (int k = 0; k < D; k++) sum[k] = acc[k].x + acc[k].y;
#pragma unroll
    for (int o = HP / 2; o > 0; o >>= 1)
#pragma unroll
        for (int k = 0; k < D; k++) sum[k] += __shfl_xor_sync(0xffffffffu, sum[k], o);
    if (tid < L::NI && yp == 0) {
#pragma unroll
        for (int k = 0; k < D; k++) map[sy * D + k] = sum[k];
    }
    __syncthreads();
    if (warp == 0) {
        // map = sum of the partials; first strict minimum and maximum over the map
        float mn = FLT_MAX, mx = -FLT_MAX;
        int mi = 0x7fffffff;
        for (int i = lane; i < D * D; i += 32) {
            const float v = map[i];
            mx = fmaxf(mx, v);
            if (v < mn) { mn = v; mi = i; }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const float omn = __shfl_xor_sync(0xffffffffu, mn, o), omx = __shfl_xor_sync(0xffffffffu, mx, o);
            const int omi = __shfl_xor_sync(0xffffffffu, mi, o);
            if (omn < mn || (omn == mn && omi < mi)) { mn = omn; mi = omi; }
            mx = fmaxf(mx, omx);
        }
        __syncwarp();
        if (lane == 0) {
            if (mi == 0x7fffffff) mi = -1;
            size_t tix = (size_t)p * tcx * tcy + tile;
            if (argmin_out) argmin_out[tix] = mi;
            if (offsets_out) { offsets_out[2 * tix] = oxt; offsets_out[2 * tix + 1] = oyt; }
            float cx = 0.f, cy = 0.f;
            if (mi >= 0) {
                int iy = mi / D, ix = mi - iy * D;
                cy = (float)iy;
                cx = (float)ix;
                if (ix < 1 || iy < 1 || ix >= 2 * S || iy >= 2 * S) {
                    cx = 0.f; cy = 0.f;
                } else {
                    float a11 = 0.f, a22 = 0.f, a12 = 0.f, b1 = 0.f, b2 = 0.f;
#pragma unroll
                    for (int k = 0; k < 9; k++) {
                        float v = map[(iy + k / 3 - 1) * D + ix + k % 3 - 1];
                        a11 += c_fit[0][k] * v; a22 += c_fit[1][k] * v; a12 += c_fit[2][k] * v;
                        b1 += c_fit[3][k] * v; b2 += c_fit[4][k] * v;
                    }
                    a11 = fmaxf(a11, 0.0f);
                    a22 = fmaxf(a22, 0.0f);
                    float det = a11 * a22 - a12 * a12;
                    if (det < 0) { a12 = 0; det = a11 * a22; }
                    if (det != 0) {
                        float mux = (a22 * b1 - a12 * b2) / det, muy = (a11 * b2 - a12 * b1) / det;
                        if (fabsf(mux) > 1) mux = 0;
                        if (fabsf(muy) > 1) muy = 0;
                        cx -= mux; cy -= muy;
                    }
                    cx -= S; cy -= S;
                }
            }
            if (threshold + mn > mx) { cx = 0.f; cy = 0.f; }
            pre.x += cx;
            pre.y += cy;
            gline[tx] = pre;
        }
        if (scores) {
            __syncwarp();
            const size_t tix = (size_t)p * tcx * tcy + tile;
            for (int i = lane; i < D * D; i += 32) scores[tix * D * D + i] = map[i];
        }
    }
}

template <int T, int S>
cudaError_t launch_track_ts(const float* const* frames, size_t pitch, int Wl, int Hl, int tcx, int tcy, const isa_pair_desc* pairs,
                            int npairs, float2* grids, size_t grid_pitch, size_t grid_stride, float thr, float* scores, int* argmin,
                            int* offsets, cudaStream_t st)
{
    using L = TrackDims<T, S>;
    if (L::BYTES > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(k_track<T, S>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L::BYTES);
        if (e != cudaSuccess) return e;
    }
    dim3 g(npairs, tcx * tcy);
    k_track<T, S><<<g, L::NT, L::BYTES, st>>>(frames, pitch, Wl, Hl, tcx, tcy, pairs, grids, grid_pitch, grid_stride, thr, scores, argmin, offsets);
    return cudaGetLastError();
}

// UpSampleShifts (kernel.cu:552-598) for a batch of pair grids.
__global__ void k_upsample(const float2* __restrict__ in, size_t in_pitch, size_t in_stride, float2* __restrict__ out, size_t out_pitch,
                           size_t out_stride, int oldLevel, int newLevel, int ocx, int ocy, int ncx, int ncy, int oldT, int newT)
{
    int nx = blockIdx.x * blockDim.x + threadIdx.x, ny = blockIdx.y * blockDim.y + threadIdx.y;
    if (nx >= ncx || ny >= ncy) return;
    const char* ib = (const char*)in + blockIdx.z * in_stride;
    float factor = (float)oldLevel * oldT / (float)(newLevel * newT);
    float ox = nx / factor, oy = ny / factor;
    int x0 = (int)floorf(ox), x1 = (int)ceilf(ox), y0 = (int)floorf(oy), y1 = (int)ceilf(oy);
    x0 = min(x0, ocx - 1); x1 = min(x1, ocx - 1); y0 = min(y0, ocy - 1); y1 = min(y1, ocy - 1);
    const float2* r0 = (const float2*)(ib + (size_t)y0 * in_pitch);
    const float2* r1 = (const float2*)(ib + (size_t)y1 * in_pitch);
    float2 v00 = r0[x0], v10 = r0[x1], v01 = r1[x0], v11 = r1[x1];
    float wx = 1.0f - (x1 - ox), wy = 1.0f - (y1 - oy);
    float t0 = v00.x + (v10.x - v00.x) * wx, t1 = v01.x + (v11.x - v01.x) * wx;
    float2 o;
    o.x = t0 + (t1 - t0) * wy;
    t0 = v00.y + (v10.y - v00.y) * wx;
    t1 = v01.y + (v11.y - v01.y) * wx;
    o.y = t0 + (t1 - t0) * wy;
    o.x *= oldLevel / (float)newLevel;
    o.y *= oldLevel / (float)newLevel;
    ((float2*)((char*)out + blockIdx.z * out_stride + (size_t)ny * out_pitch))[nx] = o;
}

// Per-tile least squares with outlier removal, one warp per tile (no block
// barriers). Rows of the incidence matrix are intervals [a, b) of the
// one-to-one shifts with a common sign (true for every tracking strategy of
// ShiftCollection.CreateShiftMatrix), so N = A^T A is updated in place when a
// row is removed, and A x is a difference of prefix sums. Each round solves
// [N | A^T b] in FP64 by Gauss-Jordan with partial pivoting: lane r owns row
// r of the augmented matrix (odd row stride: conflict-free 64-bit access).
struct SolveLayout {
    int n1, m, as;          // unknowns, rows, augmented row stride (odd)
    int off_aug, off_rhs, off_xs, off_p;  // in doubles, after N
    int nd;                 // doubles per warp
    size_t bytes;           // per warp (doubles + b floats + active bytes, 16-aligned)
};

__host__ __device__ inline SolveLayout solve_layout(int m, int n1)
{
    SolveLayout L;
    L.n1 = n1; L.m = m; L.as = (n1 + 2) | 1;
    L.off_aug = n1 * n1;
    L.off_rhs = L.off_aug + n1 * L.as;
    L.off_xs = L.off_rhs + 2 * n1;
    L.off_p = L.off_xs + 2 * n1;
    L.nd = L.off_p + 2 * (n1 + 1);
    L.bytes = ((size_t)L.nd * 8 + (size_t)2 * m * 4 + (size_t)m + 15) / 16 * 16;
    return L;
}

__global__ void k_solve(const int* __restrict__ row_a, const int* __restrict__ row_b, const int* __restrict__ row_sign,
                        const double* __restrict__ N0, int m, int n1, float2* __restrict__ grids, size_t grid_pitch, size_t grid_stride,
                        const int* __restrict__ row_grid, int tcx, int tcy, float2* __restrict__ x_out, int* __restrict__ status)
{
    extern __shared__ __align__(16) unsigned char smem_s[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int tile = blockIdx.x * (blockDim.x >> 5) + warp;
    if (tile >= tcx * tcy) return;  // the whole warp leaves; only warp-level synchronisation below
    const SolveLayout L = solve_layout(m, n1);
    double* N = (double*)(smem_s + (size_t)warp * L.bytes);
    double* aug = N + L.off_aug;
    double* rhs = N + L.off_rhs;
    double* xs = N + L.off_xs;
    double* P = N + L.off_p;
    float* b = (float*)(N + L.nd);
    unsigned char* active = (unsigned char*)(b + 2 * m);
    const int AS = L.as, na = n1 + 2;
    const int ty = tile / tcx, tx = tile - ty * tcx;
    for (int i = lane; i < n1 * n1; i += 32) N[i] = N0[i];
    for (int k = lane; k < m; k += 32) {
        const float2 v = ((const float2*)((const char*)grids + (size_t)row_grid[k] * grid_stride + (size_t)ty * grid_pitch))[tx];
        b[2 * k] = v.x; b[2 * k + 1] = v.y;
        active[k] = 1;
    }
    for (int i = lane; i < 2 * n1; i += 32) xs[i] = 0.0;
    __syncwarp();
    // rhs = A^T b
    for (int i = lane; i < n1; i += 32) {
        double sx = 0, sy = 0;
        for (int k = 0; k < m; k++)
            if (__ldg(row_a + k) <= i && i < __ldg(row_b + k)) {
                const double sg = __ldg(row_sign + k);
                sx += sg * (double)b[2 * k]; sy += sg * (double)b[2 * k + 1];
            }
        rhs[2 * i] = sx; rhs[2 * i + 1] = sy;
    }
    int st = -1;
    for (int round_ = 0; round_ < 10; round_++) {
        __syncwarp();
        for (int i = lane; i < n1 * n1; i += 32) { const int r = i / n1, c = i - r * n1; aug[r * AS + c] = N[i]; }
        double sc = 0;
        for (int i = lane; i < n1; i += 32) {
            aug[i * AS + n1] = rhs[2 * i]; aug[i * AS + n1 + 1] = rhs[2 * i + 1];
            sc = fmax(sc, fabs(N[i * n1 + i]));
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) sc = fmax(sc, __shfl_xor_sync(0xffffffffu, sc, o));
        const double tol = 1e-12 * (sc > 0 ? sc : 1.0);
        __syncwarp();
        // Gauss-Jordan with partial pivoting (first largest |pivot|)
        bool singular = false;
        for (int c = 0; c < n1; c++) {
            double bv = -2.0;
            int br = 0x7fffffff;
            for (int r = c + lane; r < n1; r += 32) {
                // the first largest |pivot| scanning down from row c; a NaN
                // is never chosen, except a NaN in row c, which nothing beats
                double v = fabs(aug[r * AS + c]);
                if (!(v >= 0)) v = r == c ? INFINITY : -1.0;
                if (v > bv) { bv = v; br = r; }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const double ov = __shfl_xor_sync(0xffffffffu, bv, o);
                const int orr = __shfl_xor_sync(0xffffffffu, br, o);
                if (ov > bv || (ov == bv && orr < br)) { bv = ov; br = orr; }
            }
            const int pr = br;
            const double piv = aug[pr * AS + c];
            if (!(fabs(piv) > tol)) { singular = true; break; }
            __syncwarp();
            if (pr != c)
                for (int j = lane; j < na; j += 32) {
                    const double t = aug[c * AS + j];
                    aug[c * AS + j] = aug[pr * AS + j];
                    aug[pr * AS + j] = t;
                }
            __syncwarp();
            for (int j = c + 1 + lane; j < na; j += 32) aug[c * AS + j] /= piv;
            if (lane == 0) aug[c * AS + c] = 1.0;
            __syncwarp();
            for (int r = lane; r < n1; r += 32) {
                if (r == c) continue;
                double* row = aug + r * AS;
                const double f = row[c];
                const double* prow = aug + c * AS;
                for (int j = c; j < na; j++) row[j] -= f * prow[j];
            }
            __syncwarp();
        }
        if (singular) { st = -3; break; }  // keep the previous solution
        for (int i = lane; i < n1; i += 32) { xs[2 * i] = aug[i * AS + n1]; xs[2 * i + 1] = aug[i * AS + n1 + 1]; }
        __syncwarp();
        if (lane == 0) {
            P[0] = 0; P[1] = 0;
            for (int i = 0; i < n1; i++) { P[2 * (i + 1)] = P[2 * i] + xs[2 * i]; P[2 * (i + 1) + 1] = P[2 * i + 1] + xs[2 * i + 1]; }
        }
        __syncwarp();
        // largest squared residual above 1; residuals within a relative 1e-9
        // of it count as ties and the lowest row wins (order independent)
        double best = 1.0;
        for (int k = lane; k < m; k += 32) {
            if (!active[k]) continue;
            const int ra = __ldg(row_a + k), rb = __ldg(row_b + k);
            const double sg = __ldg(row_sign + k);
            const double dx = b[2 * k] - sg * (P[2 * rb] - P[2 * ra]), dy = b[2 * k + 1] - sg * (P[2 * rb + 1] - P[2 * ra + 1]);
            best = fmax(best, dx * dx + dy * dy);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) best = fmax(best, __shfl_xor_sync(0xffffffffu, best, o));
        int bi = 0x7fffffff;
        if (best > 1.0) {
            const double thr = best * (1 - 1e-9);
            for (int k = lane; k < m; k += 32) {
                if (!active[k]) continue;
                const int ra = __ldg(row_a + k), rb = __ldg(row_b + k);
                const double sg = __ldg(row_sign + k);
                const double dx = b[2 * k] - sg * (P[2 * rb] - P[2 * ra]), dy = b[2 * k + 1] - sg * (P[2 * rb + 1] - P[2 * ra + 1]);
                const double d = dx * dx + dy * dy;
                if (d >= thr && d > 1.0) { bi = k; break; }
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) bi = min(bi, __shfl_xor_sync(0xffffffffu, bi, o));
        const int k = bi == 0x7fffffff ? -1 : bi;
        st = k;
        if (k < 0) break;
        const int a = __ldg(row_a + k), e = __ldg(row_b + k);
        const double sg = __ldg(row_sign + k);
        const double bx = b[2 * k], by = b[2 * k + 1];
        __syncwarp();
        const int w = e - a;
        for (int i = lane; i < w * w; i += 32) {
            const int r = a + i / w, c = a + i % w;
            N[r * n1 + c] -= 1.0;
        }
        for (int i = a + lane; i < e; i += 32) { rhs[2 * i] -= sg * bx; rhs[2 * i + 1] -= sg * by; }
        if (lane == 0) { b[2 * k] = 0.f; b[2 * k + 1] = 0.f; active[k] = 0; }
    }
    __syncwarp();
    if (lane == 0) {
        status[tile] = st;
        P[0] = 0; P[1] = 0;
        for (int i = 0; i < n1; i++) { P[2 * (i + 1)] = P[2 * i] + xs[2 * i]; P[2 * (i + 1) + 1] = P[2 * i + 1] + xs[2 * i + 1]; }
    }
    for (int i = lane; i < n1; i += 32) x_out[(size_t)tile * n1 + i] = make_float2((float)xs[2 * i], (float)xs[2 * i + 1]);
    __syncwarp();
    for (int k = lane; k < m; k += 32) {
        const int ra = __ldg(row_a + k), rb = __ldg(row_b + k);
        const double sg = __ldg(row_sign + k);
        const double px = sg * (P[2 * rb] - P[2 * ra]), py = sg * (P[2 * rb + 1] - P[2 * ra + 1]);
        ((float2*)((char*)grids + (size_t)row_grid[k] * grid_stride + (size_t)ty * grid_pitch))[tx] = make_float2((float)px, (float)py);
    }
}

// getOptimalShifts (ShiftMinimizerKernels.cu:179-218).
__global__ void k_optimal(const float2* __restrict__ x, int n1, int tcx, int tcy, int ref, int trk, float2* __restrict__ out, size_t out_pitch)
{
    int tx = blockIdx.x * blockDim.x + threadIdx.x, ty = blockIdx.y * blockDim.y + threadIdx.y;
    if (tx >= tcx || ty >= tcy) return;
    const float2* r = x + (size_t)(tx + ty * tcx) * n1;
    float2 s = make_float2(0.f, 0.f);
    if (ref < trk) for (int i = ref; i < trk; i++) { s.x += r[i].x; s.y += r[i].y; }
    else if (trk < ref) for (int i = trk; i < ref; i++) { s.x -= r[i].x; s.y -= r[i].y; }
    ((float2*)((char*)out + (size_t)ty * out_pitch))[tx] = s;
}

}  // namespace

#define ISA_TRACK_CASE(TT, SS) \
    if (T == TT && S == SS) return launch_track_ts<TT, SS>(frames, img_pitch, Wl, Hl, tcx, tcy, pairs, npairs, grids, grid_pitch, grid_stride, threshold, scores, argmin, offsets, st);

cudaError_t isa_launch_track(const float* const* frames, size_t img_pitch, int Wl, int Hl, int T, int S, int tcx, int tcy,
                             const isa_pair_desc* pairs, int npairs, float2* grids, size_t grid_pitch, size_t grid_stride, float threshold,
                             float* scores, int* argmin, int* offsets, cudaStream_t st)
{
    if (npairs <= 0 || tcx <= 0 || tcy <= 0) return cudaSuccess;
    ISA_TRACK_CASE(32, 1) ISA_TRACK_CASE(32, 2) ISA_TRACK_CASE(32, 3) ISA_TRACK_CASE(32, 4)
    ISA_TRACK_CASE(32, 5) ISA_TRACK_CASE(32, 6)
    ISA_TRACK_CASE(16, 1) ISA_TRACK_CASE(16, 2) ISA_TRACK_CASE(16, 4) ISA_TRACK_CASE(16, 8)
    ISA_TRACK_CASE(64, 2)
    ISA_TRACK_CASE(8, 2) ISA_TRACK_CASE(8, 4)
    return cudaErrorInvalidValue;
}

cudaError_t isa_launch_upsample(const float2* in, size_t in_pitch, size_t in_stride, float2* out, size_t out_pitch, size_t out_stride,
                                int ngrids, int oldLevel, int newLevel, int ocx, int ocy, int ncx, int ncy, int oldT, int newT,
                                cudaStream_t st)
{
    if (ngrids <= 0) return cudaSuccess;
    dim3 b(16, 16), g((ncx + 15) / 16, (ncy + 15) / 16, ngrids);
    k_upsample<<<g, b, 0, st>>>(in, in_pitch, in_stride, out, out_pitch, out_stride, oldLevel, newLevel, ocx, ocy, ncx, ncy, oldT, newT);
    return cudaGetLastError();
}

size_t isa_solve_smem(int m, int n1) { return solve_layout(m, n1).bytes; }

// Loads the solver's device code on the current device (CUDA loads modules
// lazily, at first use, and loading allocates the module's globals).
cudaError_t isa_solve_prepare()
{
    cudaFuncAttributes a;
    return cudaFuncGetAttributes(&a, k_solve);
}

cudaError_t isa_launch_solve(const int* row_a, const int* row_b, const int* row_sign, const double* N0, int m, int n1, float2* grids,
                             size_t grid_pitch, size_t grid_stride, const int* row_grid, int tcx, int tcy, float2* x_out, int* status,
                             cudaStream_t st)
{
    const size_t per_warp = isa_solve_smem(m, n1);
    if (per_warp > 227 * 1024) return cudaErrorInvalidValue;
    const int wpc = (int)std::max<size_t>(1, std::min<size_t>(4, (200 * 1024) / per_warp));
    const size_t smem = per_warp * wpc;
    cudaError_t e = cudaFuncSetAttribute(k_solve, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const int ntiles = tcx * tcy;
    k_solve<<<(ntiles + wpc - 1) / wpc, 32 * wpc, smem, st>>>(row_a, row_b, row_sign, N0, m, n1, grids, grid_pitch, grid_stride, row_grid, tcx, tcy,
                                                          x_out, status);
    return cudaGetLastError();
}

cudaError_t isa_launch_optimal(const float2* x, int n1, int tcx, int tcy, int ref, int trk, float2* out, size_t out_pitch, cudaStream_t st)
{
    dim3 b(32, 8), g((tcx + 31) / 32, (tcy + 7) / 8);
    k_optimal<<<g, b, 0, st>>>(x, n1, tcx, tcy, ref, trk, out, out_pitch);
    return cudaGetLastError();
}
