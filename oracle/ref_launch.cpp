// ref_launch.cpp -- host launcher for the reference's own Kernels/*.cu bodies
// compiled with g++ (see oracle/Makefile). TEST INFRASTRUCTURE: the checker
// that pins oracle/isa_oracle.c and the timed CPU baseline; never shipped.
//
// Each ref_* function mirrors one C# wrapper's RunSafe: the same block shape
// and grid rounding (ManagedCuda SetComputeSize = ceil(size / block)), the
// same argument order and the same texture modes, with images passed as
// contiguous (pitch = width * element size) host arrays. The grid is walked
// with OpenMP over blocks and the kernel body is called once per CUDA thread.
// Kernels that synchronise threads through shared memory
// (boxFilterWithBorderX/Y, kernel.cu:59-128) cannot run one thread at a time;
// their effect (a T-wide sliding sum of squares) is restated in ref_tile_scores.
#include <omp.h>
#include <vector>
#include <cstring>
#include <cstdlib>
#include <utility>
#include "cuda_runtime.h"  // after the standard headers: the FP64 build redefines `float`
#include "device_launch_parameters.h"

thread_local uint3 blockIdx;
thread_local uint3 threadIdx;
thread_local uint3 blockDim;
thread_local uint3 gridDim;

extern "C" {
// storage the kernels declare extern (DeBayerKernels.cu:41; dynamic shared
// memory of kernel.cu:70/107 and RobustnessModell.cu:46)
int c_cfaPattern[2][2];
thread_local float shared[4 * 128];
thread_local float3 pixelsRef[8 * 8 * 9];

// reference kernel prototypes (Kernels/*.cu)
void deBayerGreenKernel(const int, const int, const float*, int, float3*, int, float3, float3);
void deBayerRedBlueKernel(const int, const int, const float*, int, float3*, int, float3, float3);
void deBayersSubSample3(unsigned short*, float3*, float, int, int, int);
void accumulateImages(unsigned short*, float3*, float3*, const float4*, const float3*, const float2*, float3, float3, int, int, int, int, int);
void accumulateImagesSuperRes(unsigned short*, float3*, float3*, const float4*, cudaTextureObject_t, cudaTextureObject_t, float3, float3, int, int, int, int, int, int);
void ComputeRobustnessMask(const float3*, const float3*, float4*, cudaTextureObject_t, int, int, int, int, float, float, float);
void WarpingKernel(int, int, int, cudaTextureObject_t, float*, cudaTextureObject_t);
void CreateFlowFieldFromTiles(float2*, cudaTextureObject_t, int, int, int, int, int, int, float2, float);
void ComputeDerivativesKernel(int, int, int, float*, float*, float*, cudaTextureObject_t, cudaTextureObject_t);
void ComputeDerivatives2Kernel(int, int, int, float*, float*, cudaTextureObject_t);
void lucasKanadeOptim(float2*, const float*, const float*, const float*, int, int, int, int, int, float);
void squaredSum(const float*, float*, int, int, int);
void normalizedCC(const float*, const float*, const float*, float*, int, int, int);
void convertToTilesOverlapBorder(const float*, float*, int, int, int, int, int, int, int, float2, float);
void convertToTilesOverlapPreShift(const float*, float*, const float2*, int, int, int, int, int, int, int, int, float2, float);
void GammasRGB(float3*, int, int, int);
void ApplyWeighting(float3*, const float3*, const float3*, int, int, int, float);
void findMinimum(const float*, float2*, int, int, int, int, float);
void UpSampleShifts(const float2*, float2*, int, int, int, int, int, int, int, int, int, int);
void ComputeStructureTensor(const float*, const float*, float3*, int, int, int, int);
void ComputeKernelParam(float3*, int, int, int, float, float, float, float, float, float);
void fourierFilter(float2*, size_t, int, int, float, float, float, float, int);
void checkForOutliers(float2*, const float*, float*, int*, int*, int, int, int);
void getOptimalShifts(float2*, const float2*, int, int, int, int, int, int);
void conjugateComplexMulKernel(const float2*, float2*, int);
}

typedef float real;  // `float` is `double` in the -DISA_REF_FP64 build

static unsigned cdiv(unsigned a, unsigned b) { return (a + b - 1) / b; }

template <class F>
static void run_grid(dim3 block, unsigned sx, unsigned sy, unsigned sz, F&& body)
{
    dim3 grid{cdiv(sx, block.x), cdiv(sy, block.y), cdiv(sz, block.z)};
    long total = (long)grid.x * grid.y * grid.z;
#pragma omp parallel for schedule(dynamic, 4)
    for (long b = 0; b < total; b++) {
        blockDim = block;
        gridDim = grid;
        blockIdx.x = (unsigned)(b % grid.x);
        blockIdx.y = (unsigned)((b / grid.x) % grid.y);
        blockIdx.z = (unsigned)(b / ((long)grid.x * grid.y));
        for (unsigned tz = 0; tz < block.z; tz++)
            for (unsigned ty = 0; ty < block.y; ty++)
                for (unsigned tx = 0; tx < block.x; tx++) {
                    threadIdx.x = tx; threadIdx.y = ty; threadIdx.z = tz;
                    body();
                }
    }
}

static isa_ref_tex make_tex(const void* data, int w, int h, int ch, int addr, int filter)
{
    isa_ref_tex t;
    t.data = data; t.width = w; t.height = h; t.pitch = (size_t)w * ch * sizeof(real);
    t.channels = ch; t.addr = addr; t.filter = filter;
    return t;
}
#define TEXOBJ(t) ((cudaTextureObject_t)(uintptr_t)&(t))

static float3 f3(const real* v) { return make_float3(v[0], v[1], v[2]); }
static float2 f2(const real* v) { return make_float2(v[0], v[1]); }

extern "C" {

int ref_real_size(void) { return (int)sizeof(real); }
void ref_set_threads(int n) { if (n > 0) omp_set_num_threads(n); }

void ref_set_cfa(const int* cfa)
{
    c_cfaPattern[0][0] = cfa[0]; c_cfaPattern[0][1] = cfa[1];
    c_cfaPattern[1][0] = cfa[2]; c_cfaPattern[1][1] = cfa[3];
}

// DeBayerFullRes (controller :1268-1311) with the reference kernels;
// DeBayerKernels.cs:36-44 / 72-80 launch 32x16 over the input.
void ref_debayer_full(const uint16_t* raw, int W, int H, const int* cfa, const real* black, const real* scale,
                      const real* divisor, real* rgb)
{
    ref_set_cfa(cfa);
    std::vector<real> in((size_t)W * H);
    for (size_t i = 0; i < in.size(); i++) in[i] = raw[i];
    std::memset(rgb, 0, (size_t)W * H * 3 * sizeof(real));
    float3 bp = f3(black), sc = f3(scale);
    int sin = W * (int)sizeof(real), sout = W * 3 * (int)sizeof(real);
    run_grid(dim3{32, 16, 1}, W, H, 1, [&] { deBayerGreenKernel(W, H, in.data(), sin, (float3*)rgb, sout, bp, sc); });
    run_grid(dim3{32, 16, 1}, W, H, 1, [&] { deBayerRedBlueKernel(W, H, in.data(), sin, (float3*)rgb, sout, bp, sc); });
    for (size_t i = 0; i < (size_t)W * H; i++)
        for (int c = 0; c < 3; c++) rgb[i * 3 + c] /= divisor[c];
}

void ref_gamma_srgb(real* rgb, int W, int H)
{
    run_grid(dim3{16, 16, 1}, W, H, 1, [&] { GammasRGB((float3*)rgb, W, H, W * 3 * (int)sizeof(real)); });
}

// fourierFilter coefficients: run the kernel on a spectrum of ones.
void ref_fourier_filter_mask(int W, int H, real lp, real hp, real lps, real hps, int clearAxis, real* mask)
{
    int Wc = W / 2 + 1;
    std::vector<float2> spec((size_t)Wc * H, make_float2(1, 1));
    run_grid(dim3{32, 32, 1}, Wc, H, 1, [&] {
        fourierFilter(spec.data(), (size_t)Wc * sizeof(float2), W, H, lp, hp, lps, hps, clearAxis);
    });
    for (size_t i = 0; i < spec.size(); i++) mask[i] = spec[i].x;
}

// conjugateComplexMulKernel.RunSafe (BasicKernels.cs:65-81): b = conj(a) * b
// elementwise, block 128 (PreAlignment.cs:200 passes the reference spectrum
// as a and the rotated frame's as b).
void ref_conj_mul(const real* a, real* b, int n)
{
    run_grid(dim3{128, 1, 1}, (unsigned)n, 1, 1, [&] { conjugateComplexMulKernel((const float2*)a, (float2*)b, n); });
}

// PatchTracker.Track (PatchTracker.cs:317-360) for one pair. Tiles are cut
// by the reference kernels (BasicKernels.cs:33-61: block 24x1x8); the cuFFT
// cross-correlation is computed directly into the fft-shifted layout that
// normalizedCC reads; the box filters are restated; squaredSum, normalizedCC
// and findMinimum are the reference kernels; preShift += result.
void ref_track_pair(const real* imgTrack, const real* imgRef, int Wl, int Hl, int T, int S, int tcx, int tcy,
                    real* preShift, const real* baseRef, real rotRef, const real* baseTrk, real rotTrk,
                    real threshold, real* scores)
{
    int B = T + 2 * S, D = 2 * S + 1, nt = tcx * tcy;
    size_t tb = (size_t)B * B;
    std::vector<real> tpl(tb * nt), blk(tb * nt), cc(tb * nt, 0), box(tb * nt, 0), sq(nt), map((size_t)nt * D * D);
    std::vector<float2> patch(nt);
    int pitch = Wl * (int)sizeof(real);
    float2 bR = f2(baseRef), bT = f2(baseTrk);
    run_grid(dim3{24, 1, 8}, B, B, nt, [&] {
        convertToTilesOverlapBorder(imgRef, tpl.data(), Wl, Hl, pitch, S, T, tcx, tcy, bR, rotRef);
    });
    run_grid(dim3{24, 1, 8}, B, B, nt, [&] {
        convertToTilesOverlapPreShift(imgTrack, blk.data(), (const float2*)preShift, tcx * 2 * (int)sizeof(real), Wl, Hl,
                                      pitch, S, T, tcx, tcy, bT, rotTrk);
    });
#pragma omp parallel for schedule(dynamic, 4)
    for (int t = 0; t < nt; t++) {
        const real* a = &tpl[t * tb];
        const real* b = &blk[t * tb];
        real* c = &cc[t * tb];
        for (int sy = -S; sy <= S; sy++)
            for (int sx = -S; sx <= S; sx++) {
                real s = 0;
                for (int y = S; y < S + T; y++)
                    for (int x = S; x < S + T; x++) s += a[y * B + x] * b[(y + sy) * B + x + sx];
                int fx = sx < 0 ? B + sx : sx, fy = sy < 0 ? B + sy : sy;
                c[fy * B + fx] = s;
            }
        // boxFilterWithBorderX then Y (kernel.cu:59-128) restated
        std::vector<real> bx(tb, 0);
        for (int y = 0; y < B; y++)
            for (int x = T / 2; x <= 2 * S + T / 2; x++) {
                real s = 0;
                for (int k = -T / 2; k < T / 2; k++) s += b[y * B + x + k] * b[y * B + x + k];
                bx[y * B + x] = s;
            }
        real* o = &box[t * tb];
        for (int y = T / 2; y <= 2 * S + T / 2; y++)
            for (int x = 0; x < B; x++) {
                real s = 0;
                for (int k = -T / 2; k < T / 2; k++) s += bx[(y + k) * B + x];
                o[y * B + x] = s;
            }
    }
    run_grid(dim3{128, 1, 1}, nt, 1, 1, [&] { squaredSum(tpl.data(), sq.data(), S, T, nt); });
    dim3 nb = D > 8 ? dim3{8, 8, 4} : dim3{(unsigned)D, (unsigned)D, 4};
    run_grid(nb, D, D, nt, [&] { normalizedCC(cc.data(), sq.data(), box.data(), map.data(), S, T, nt); });
    run_grid(dim3{128, 1, 1}, nt, 1, 1, [&] {
        findMinimum(map.data(), patch.data(), tcx * (int)sizeof(float2), S, nt, tcx, threshold);
    });
    for (int t = 0; t < nt; t++) { preShift[t * 2] += patch[t].x; preShift[t * 2 + 1] += patch[t].y; }
    if (scores) std::memcpy(scores, map.data(), map.size() * sizeof(real));
}

void ref_upsample_shifts(const real* in, real* out, int oldLevel, int newLevel, int ocx, int ocy, int ncx, int ncy, int oldT, int newT)
{
    run_grid(dim3{16, 16, 1}, ncx, ncy, 1, [&] {
        UpSampleShifts((const float2*)in, (float2*)out, ocx * (int)sizeof(float2), ncx * (int)sizeof(float2), oldLevel, newLevel,
                       ocx, ocy, ncx, ncy, oldT, newT);
    });
}

void ref_optimal_shifts(const real* x, int n1, int tcx, int tcy, int ref, int trk, real* out)
{
    run_grid(dim3{32, 8, 1}, tcx, tcy, 1, [&] {
        getOptimalShifts((float2*)out, (const float2*)x, n1 + 1, tcx, tcy, tcx * (int)sizeof(float2), ref, trk);
    });
}

// ShiftCollection.MinimizeCUBLAS (ShiftCollection.cs:738-822): the batched
// cuBLAS products and the batched matrix inverse are restated (plain loops,
// Gauss-Jordan); checkForOutliers is the reference kernel on the same
// column-major layouts. A: m x n1 row-major incidence matrix.
void ref_solve_shifts(const real* Arow, int m, int n1, int tiles, real* meas, real* x, int* status)
{
    std::vector<real> A((size_t)tiles * m * n1), Asafe((size_t)m * n1);
    for (int k = 0; k < m; k++)
        for (int j = 0; j < n1; j++) Asafe[(size_t)j * m + k] = Arow[(size_t)k * n1 + j];  // column-major, ld m
    for (int t = 0; t < tiles; t++) std::memcpy(&A[(size_t)t * m * n1], Asafe.data(), Asafe.size() * sizeof(real));
    std::vector<real> optT((size_t)tiles * m * 2), oneT((size_t)tiles * n1 * 2);
    std::vector<int> st(tiles, 0), info(tiles, 0);
    for (int round_ = 0; round_ < 10; round_++) {
#pragma omp parallel for schedule(dynamic, 8)
        for (int t = 0; t < tiles; t++) {
            const real* a = &A[(size_t)t * m * n1];
            std::vector<real> N((size_t)n1 * n1), Ni((size_t)n1 * n1, 0);
            for (int i = 0; i < n1; i++)
                for (int j = 0; j < n1; j++) {
                    real s = 0;
                    for (int k = 0; k < m; k++) s += a[(size_t)i * m + k] * a[(size_t)j * m + k];
                    N[(size_t)j * n1 + i] = s;
                }
            for (int i = 0; i < n1; i++) Ni[(size_t)i * n1 + i] = 1;
            int bad = 0;
            for (int c = 0; c < n1 && !bad; c++) {
                int p = c;
                for (int r = c + 1; r < n1; r++) if (std::fabs(N[(size_t)c * n1 + r]) > std::fabs(N[(size_t)c * n1 + p])) p = r;
                real d = N[(size_t)c * n1 + p];
                if (d == 0) { bad = 1; break; }
                for (int k = 0; k < n1; k++) {
                    std::swap(N[(size_t)k * n1 + c], N[(size_t)k * n1 + p]);
                    std::swap(Ni[(size_t)k * n1 + c], Ni[(size_t)k * n1 + p]);
                }
                for (int k = 0; k < n1; k++) { N[(size_t)k * n1 + c] /= d; Ni[(size_t)k * n1 + c] /= d; }
                for (int r = 0; r < n1; r++) {
                    if (r == c) continue;
                    real f = N[(size_t)c * n1 + r];
                    for (int k = 0; k < n1; k++) { N[(size_t)k * n1 + r] -= f * N[(size_t)k * n1 + c]; Ni[(size_t)k * n1 + r] -= f * Ni[(size_t)k * n1 + c]; }
                }
            }
            info[t] = bad;
            // solved = Ni * A^T (n1 x m); oneToOne = solved * meas (n1 x 2); opt = A * oneToOne (m x 2)
            real* one = &oneT[(size_t)t * n1 * 2];
            const real* b = meas + (size_t)t * m * 2;
            for (int i = 0; i < n1; i++)
                for (int c = 0; c < 2; c++) {
                    real s = 0;
                    for (int k = 0; k < m; k++) {
                        real sv = 0;
                        for (int j = 0; j < n1; j++) sv += Ni[(size_t)j * n1 + i] * a[(size_t)j * m + k];
                        s += sv * b[k * 2 + c];
                    }
                    one[(size_t)c * n1 + i] = s;
                }
            real* opt = &optT[(size_t)t * m * 2];
            for (int k = 0; k < m; k++)
                for (int c = 0; c < 2; c++) {
                    real s = 0;
                    for (int j = 0; j < n1; j++) s += a[(size_t)j * m + k] * one[(size_t)c * n1 + j];
                    opt[(size_t)c * m + k] = s;
                }
        }
        run_grid(dim3{128, 1, 1}, tiles, 1, 1, [&] {
            checkForOutliers((float2*)meas, optT.data(), A.data(), st.data(), info.data(), tiles, n1 + 1, m);
        });
        int sum = 0;
        for (int t = 0; t < tiles; t++) sum += st[t];
        if (sum == -tiles) break;
    }
    for (int t = 0; t < tiles; t++) {
        status[t] = st[t];
        const real* one = &oneT[(size_t)t * n1 * 2];
        for (int i = 0; i < n1; i++) { x[((size_t)t * n1 + i) * 2] = one[i]; x[((size_t)t * n1 + i) * 2 + 1] = one[n1 + i]; }
        for (int k = 0; k < m; k++)
            for (int c = 0; c < 2; c++) {
                real s = 0;
                for (int j = 0; j < n1; j++) s += Asafe[(size_t)j * m + k] * one[(size_t)c * n1 + j];
                meas[((size_t)t * m + k) * 2 + c] = s;
            }
    }
}

// OpticalFlowKernels.cs:73-82: block 32x6, tile-grid texture linear/clamp.
void ref_flow_from_tiles(const real* tiles, int tcx, int tcy, int W, int H, const real* base, real rot, int T, real* flow)
{
    isa_ref_tex t = make_tex(tiles, tcx, tcy, 2, ISA_REF_CLAMP, ISA_REF_LINEAR);
    float2 b = f2(base);
    run_grid(dim3{32, 6, 1}, W, H, 1, [&] {
        CreateFlowFieldFromTiles((float2*)flow, TEXOBJ(t), T, tcx, tcy, W, H, W * 2 * (int)sizeof(real), b, rot);
    });
}

// OpticalFlowKernels.cs:44-55: image linear/mirror, flow point/clamp.
void ref_warp(const real* img, int W, int H, const real* flow, real* out)
{
    isa_ref_tex ti = make_tex(img, W, H, 1, ISA_REF_MIRROR, ISA_REF_LINEAR);
    isa_ref_tex tf = make_tex(flow, W, H, 2, ISA_REF_CLAMP, ISA_REF_POINT);
    run_grid(dim3{32, 6, 1}, W, H, 1, [&] { WarpingKernel(W, H, W * (int)sizeof(real), TEXOBJ(tf), out, TEXOBJ(ti)); });
}

void ref_derivatives(const real* src, const real* tgt, int W, int H, real* Ix, real* Iy, real* It)
{
    isa_ref_tex ts = make_tex(src, W, H, 1, ISA_REF_MIRROR, ISA_REF_LINEAR);
    isa_ref_tex tt = make_tex(tgt, W, H, 1, ISA_REF_MIRROR, ISA_REF_LINEAR);
    run_grid(dim3{32, 6, 1}, W, H, 1, [&] { ComputeDerivativesKernel(W, H, W * (int)sizeof(real), Ix, Iy, It, TEXOBJ(ts), TEXOBJ(tt)); });
}

void ref_derivatives2(const real* img, int W, int H, real* Ix, real* Iy)
{
    isa_ref_tex ts = make_tex(img, W, H, 1, ISA_REF_MIRROR, ISA_REF_LINEAR);
    run_grid(dim3{32, 6, 1}, W, H, 1, [&] { ComputeDerivatives2Kernel(W, H, W * (int)sizeof(real), Ix, Iy, TEXOBJ(ts)); });
}

// OpticalFlowKernels.cs:167-172: block 32x16.
void ref_lucas_kanade(real* flow, const real* Ix, const real* Iy, const real* It, int W, int H, int h, real minDet)
{
    run_grid(dim3{32, 16, 1}, W, H, 1, [&] {
        lucasKanadeOptim((float2*)flow, Ix, Iy, It, W * 2 * (int)sizeof(real), W * (int)sizeof(real), W, H, h, minDet);
    });
}

void ref_debayer_subsample(const uint16_t* raw, int W, int H, const int* cfa, real maxVal, real* out)
{
    ref_set_cfa(cfa);
    int Wh = W / 2, Hh = H / 2;
    run_grid(dim3{16, 16, 1}, Wh, Hh, 1, [&] {
        deBayersSubSample3((unsigned short*)raw, (float3*)out, maxVal, Wh, Hh, Wh * 3 * (int)sizeof(real));
    });
}

// RobustnessModellKernel.cs:51-61: block 8x8, flow texture linear/mirror.
// The reference kernel hard-codes s = 1.5 and t = 0.12.
void ref_robustness_mask(const real* ref, const real* mov, int Wh, int Hh, const real* flow, int Wf, int Hf,
                         real alpha, real beta, real thresholdM, real* mask)
{
    isa_ref_tex tf = make_tex(flow, Wf, Hf, 2, ISA_REF_MIRROR, ISA_REF_LINEAR);
    run_grid(dim3{8, 8, 1}, Wh, Hh, 1, [&] {
        ComputeRobustnessMask((const float3*)ref, (const float3*)mov, (float4*)mask, TEXOBJ(tf), Wh, Hh, Wh * 3 * (int)sizeof(real),
                              Wh * 4 * (int)sizeof(real), alpha, beta, thresholdM);
    });
}

void ref_structure_tensor(const real* dx, const real* dy, int W, int H, real* out)
{
    run_grid(dim3{24, 8, 1}, W, H, 1, [&] { ComputeStructureTensor(dx, dy, (float3*)out, W, H, W * (int)sizeof(real), W * 3 * (int)sizeof(real)); });
}

void ref_kernel_param(real* st, int W, int H, real Dth, real Dtr, real kDetail, real kDenoise, real kStretch, real kShrink)
{
    run_grid(dim3{24, 8, 1}, W, H, 1, [&] {
        ComputeKernelParam((float3*)st, W, H, W * 3 * (int)sizeof(real), Dth, Dtr, kDetail, kDenoise, kStretch, kShrink);
    });
}

// accumulateImages (DeBayerKernels.cs:136-160): block 16x16 over the output
// (output size = input size in the reference).
void ref_accumulate(const uint16_t* raw, int W, int H, const int* cfa, real* acc, real* wsum, const real* mask,
                    const real* kparam3, const real* flow, const real* white, const real* black)
{
    ref_set_cfa(cfa);
    run_grid(dim3{16, 16, 1}, W, H, 1, [&] {
        accumulateImages((unsigned short*)raw, (float3*)acc, (float3*)wsum, (const float4*)mask, (const float3*)kparam3,
                         (const float2*)flow, f3(white), f3(black), W, H, W * 3 * (int)sizeof(real),
                         (W / 2) * 4 * (int)sizeof(real), W * 2 * (int)sizeof(real));
    });
}

// accumulateImagesSuperRes (DeBayerKernels.cs:179-211): kernel texture
// linear/clamp over float4 parameters, flow texture linear/mirror.
void ref_accumulate_superres(const uint16_t* raw, int W, int H, const int* cfa, real* acc, real* wsum, const real* mask,
                             const real* kparam4, const real* flow, const real* white, const real* black)
{
    ref_set_cfa(cfa);
    isa_ref_tex tk = make_tex(kparam4, W, H, 4, ISA_REF_CLAMP, ISA_REF_LINEAR);
    isa_ref_tex tf = make_tex(flow, W, H, 2, ISA_REF_MIRROR, ISA_REF_LINEAR);
    run_grid(dim3{16, 16, 1}, W, H, 1, [&] {
        accumulateImagesSuperRes((unsigned short*)raw, (float3*)acc, (float3*)wsum, (const float4*)mask, TEXOBJ(tk), TEXOBJ(tf),
                                 f3(white), f3(black), W, H, W * 3 * (int)sizeof(real), (W / 2) * 4 * (int)sizeof(real),
                                 W * 4 * (int)sizeof(real), W * 2 * (int)sizeof(real));
    });
}

void ref_apply_weighting(real* img, const real* acc, const real* wsum, int W, int H, real thr)
{
    run_grid(dim3{16, 16, 1}, W, H, 1, [&] {
        ApplyWeighting((float3*)img, (const float3*)acc, (const float3*)wsum, W, H, W * 3 * (int)sizeof(real), thr);
    });
}

}  // extern "C"
