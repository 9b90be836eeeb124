// Global pre-alignment kernels (PreAlignment.ScanAngles,
// PEFStudioDX/PreAlignment.cs:176-261): cubic rotation of a tracking image
// about its centre (the reference's NPP WarpAffine with InterpolationMode
// Cubic after Set(0)), the conjugate spectrum product of the cross-correlation
// (conjugateComplexMulKernel, kernel.cu:395-411) and the position of the
// maximum of the correlation surface (NPP MaxIndex).
//
// Rotation: destination pixel p samples the source at R(angle) (p - c) + c,
// c = (W/2, H/2), with R the matrix inverse of the reference's
// Matrix3x3.Rotation (Matrix.cs:81-91) about the centre (RotAroundCenter,
// Matrix.cs:93-99), pixel centres at integer coordinates. Destination pixels
// whose source position lies outside [0, W-1] x [0, H-1] keep 0. The cubic
// kernel is Keys' cubic convolution with a = -0.5 over a 4 x 4 neighbourhood
// (taps clamped to the image).
#include "isa_internal.cuh"

namespace {

__device__ __forceinline__ float keys_cubic(float t)
{
    t = fabsf(t);
    const float a = -0.5f;
    if (t <= 1.f) return ((a + 2.f) * t - (a + 3.f)) * t * t + 1.f;
    if (t < 2.f) return ((a * t - 5.f * a) * t + 8.f * a) * t - 4.f * a;
    return 0.f;
}

__global__ void k_rotate_cubic(const float* __restrict__ src, size_t pitch, int W, int H, double ca, double sa, float* __restrict__ dst,
                               size_t dst_pitch)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= W || y >= H) return;
    const double cx = W / 2.0, cy = H / 2.0;
    const double dx = x - cx, dy = y - cy;
    const double sx = ca * dx - sa * dy + cx, sy = sa * dx + ca * dy + cy;
    float v = 0.f;
    if (sx >= 0.0 && sx <= W - 1.0 && sy >= 0.0 && sy <= H - 1.0) {
        const double fx = floor(sx), fy = floor(sy);
        const int x0 = (int)fx, y0 = (int)fy;
        const float ax = (float)(sx - fx), ay = (float)(sy - fy);
        float wx[4], wy[4];
#pragma unroll
        for (int k = 0; k < 4; k++) {
            wx[k] = keys_cubic(ax - (float)(k - 1));
            wy[k] = keys_cubic(ay - (float)(k - 1));
        }
        v = 0.f;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const float* row = isa::row_ptr(src, pitch, isa::clampi(y0 - 1 + j, 0, H - 1));
            float r = 0.f;
#pragma unroll
            for (int i = 0; i < 4; i++) r = fmaf(wx[i], __ldg(row + isa::clampi(x0 - 1 + i, 0, W - 1)), r);
            v = fmaf(wy[j], r, v);
        }
    }
    isa::row_ptr(dst, dst_pitch, y)[x] = v;
}

// b = conj(a) * b (conjugateComplexMulKernel, kernel.cu:395-411)
__global__ void k_conj_mul(const float2* __restrict__ a, float2* __restrict__ b, size_t n)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float2 va = a[i];
    va.y = -va.y;
    const float2 vb = b[i];
    float2 r;
    r.x = va.x * vb.x - va.y * vb.y;
    r.y = va.x * vb.y + va.y * vb.x;
    b[i] = r;
}

struct ValIdx { float v; int i; };

// larger value wins; equal values: the lower row-major index (the first maximum)
__device__ __forceinline__ void vi_max(float& v, int& i, float ov, int oi)
{
    if (ov > v || (ov == v && oi < i)) { v = ov; i = oi; }
}

constexpr int AM_THREADS = 256;

__device__ __forceinline__ void block_argmax(float& v, int& i)
{
    __shared__ float sv[AM_THREADS / 32];
    __shared__ int si[AM_THREADS / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) vi_max(v, i, __shfl_xor_sync(0xffffffffu, v, o), __shfl_xor_sync(0xffffffffu, i, o));
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) { sv[warp] = v; si[warp] = i; }
    __syncthreads();
    if (warp == 0) {
        v = lane < AM_THREADS / 32 ? sv[lane] : -INFINITY;
        i = lane < AM_THREADS / 32 ? si[lane] : 0x7fffffff;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) vi_max(v, i, __shfl_xor_sync(0xffffffffu, v, o), __shfl_xor_sync(0xffffffffu, i, o));
    }
}

__global__ void __launch_bounds__(AM_THREADS) k_argmax_partial(const float* __restrict__ img, int n, ValIdx* __restrict__ part)
{
    float v = -INFINITY;
    int i = 0x7fffffff;
    for (int k = blockIdx.x * AM_THREADS + threadIdx.x; k < n; k += gridDim.x * AM_THREADS) vi_max(v, i, __ldg(img + k), k);
    block_argmax(v, i);
    if (threadIdx.x == 0) part[blockIdx.x] = ValIdx{v, i};
}

__global__ void __launch_bounds__(AM_THREADS) k_argmax_final(const ValIdx* __restrict__ part, int nparts, ValIdx* __restrict__ out)
{
    float v = -INFINITY;
    int i = 0x7fffffff;
    for (int k = threadIdx.x; k < nparts; k += AM_THREADS) vi_max(v, i, part[k].v, part[k].i);
    block_argmax(v, i);
    if (threadIdx.x == 0) *out = ValIdx{v, i};
}

}  // namespace

cudaError_t isa_launch_rotate_cubic(const float* src, size_t pitch, int W, int H, double angle_deg, float* dst, size_t dst_pitch, cudaStream_t st)
{
    const double r = angle_deg / 180.0 * M_PI;
    dim3 b(32, 8), g((W + 31) / 32, (H + 7) / 8);
    k_rotate_cubic<<<g, b, 0, st>>>(src, pitch, W, H, cos(r), sin(r), dst, dst_pitch);
    return cudaGetLastError();
}

cudaError_t isa_launch_conj_mul(const float2* a, float2* b, size_t n, cudaStream_t st)
{
    k_conj_mul<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(a, b, n);
    return cudaGetLastError();
}

size_t isa_argmax_scratch_bytes() { return (size_t)1024 * sizeof(ValIdx); }

// out: one (float value, int index) pair; scratch: isa_argmax_scratch_bytes()
cudaError_t isa_launch_argmax(const float* img, int n, void* scratch, void* out, cudaStream_t st)
{
    const int nb = std::min(1024, std::max(1, (n + AM_THREADS * 8 - 1) / (AM_THREADS * 8)));
    k_argmax_partial<<<nb, AM_THREADS, 0, st>>>(img, n, (ValIdx*)scratch);
    k_argmax_final<<<1, AM_THREADS, 0, st>>>((const ValIdx*)scratch, nb, (ValIdx*)out);
    return cudaGetLastError();
}
