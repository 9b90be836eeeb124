// Shared device helpers and launch declarations of the burst-merge library.
// Layouts follow the reference's NPP images: row-major, pitch in bytes,
// channels interleaved (float2 flow, float3 RGB, float4 masks/kernels).
#pragma once
#include <cuda_runtime.h>
#include "isa.h"
#include <stdint.h>
#include <math.h>
#include <algorithm>

#define ISA_DEV __device__ __forceinline__

namespace isa {

// ---- pitched access ------------------------------------------------------
template <class T>
ISA_DEV T* row_ptr(T* base, size_t pitch, int y) { return (T*)((char*)base + (size_t)y * pitch); }
template <class T>
ISA_DEV const T* row_ptr(const T* base, size_t pitch, int y) { return (const T*)((const char*)base + (size_t)y * pitch); }

ISA_DEV int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// Mirror addressing of a CUDA texture: reflect the texel index with the
// edge texel repeated (period 2n).
ISA_DEV int mirror(int i, int n) {
    if ((unsigned)i < (unsigned)n) return i;
    int p = 2 * n;
    int j = i % p;
    if (j < 0) j += p;
    return j >= n ? p - 1 - j : j;
}

// Bilinear blend with the weights (1-a)(1-b), a(1-b), (1-a)b, ab, a and b in
// [0, 1). Texels whose weight is zero do not contribute, so a non-finite
// neighbour does not leak into an exact-texel sample.
ISA_DEV float lerp2(float p00, float p10, float p01, float p11, float a, float b) {
    float v = (1.f - a) * (1.f - b) * p00;
    if (a != 0.f) v += a * (1.f - b) * p10;
    if (b != 0.f) v += (1.f - a) * b * p01;
    if (a != 0.f && b != 0.f) v += a * b * p11;
    return v;
}

// CFA code at (x, y): cfa packed as 4 x 2 bits, (y&1)*2 + (x&1) selects.
ISA_DEV int cfa_at(unsigned cfa, int x, int y) { return (cfa >> ((((y & 1) << 1) | (x & 1)) * 2)) & 3; }

// fourierFilter's coefficient (kernel.cu:704-779) of half-spectrum bin (x, y) of a W x H transform.
ISA_DEV float fourier_mask(int x, int y, int W, int H, float lp, float hp, float lps, float hps, int clear_axis)
{
    float mx = (float)x, my = (float)y;
    if (my > H * 0.5f) my = (H - my) * -1.0f;
    mx /= W;
    my /= H;
    float dist = sqrtf(mx * mx + my * my);
    float fil = 0;
    lp = lp - lps;
    hp = hp + hps;
    if (lp > 0) { if (dist <= lp) fil = 1; }
    else { if (dist <= 1.0f) fil = 1; }
    if (lps > 0) {
        float f2 = (-fil + 1.0f) * expf(-((dist - lp) * (dist - lp) / (2 * lps * lps)));
        if (f2 > 0.001f) fil = f2;
    }
    if (lps > 0 && lp == 0 && hp == 0 && hps == 0) fil = expf(-((dist - lp) * (dist - lp) / (2 * lps * lps)));
    if (hp > 0) {
        float f2 = dist >= hp ? 1.0f : 0.0f;
        fil *= f2;
        if (hps > 0) {
            float f3 = (-f2 + 1.0f) * expf(-((dist - hp) * (dist - hp) / (2 * hps * hps)));
            if (f3 > 0.001f) fil = f3;
        }
    }
    if (x < clear_axis || fabsf(my) * H < clear_axis) fil = 0;
    return fil;
}

}  // namespace isa

// ---- launchers implemented in the .cu files (host side) -------------------
// fft.cu: mixed-radix transforms in shared memory (plan = radices of the stages)
constexpr int ISA_FFT_MAX_STAGES = 24;
// radix[s]: the stage's radix; ns[s]: the product of the radices before it; mns[s]: 2^32 / ns + 1 (division by ns
// as a multiply-high, exact for the sizes used: numerator and divisor below 2^15)
struct isa_fft_plan { int n, nst; int radix[ISA_FFT_MAX_STAGES]; int ns[ISA_FFT_MAX_STAGES]; unsigned mns[ISA_FFT_MAX_STAGES]; };
struct isa_fft_filter { float lp, hp, lps, hps; int clear_axis; float post_scale; };
enum { ISA_FFT_COLS_FWD = 0, ISA_FFT_COLS_FILTER = 1, ISA_FFT_COLS_XCORR = 2 };
bool isa_fft_plan_make(int n, isa_fft_plan& p);
void isa_fft_twiddles(int n, float2* out);  // e^{-2 pi i k / n}, k < n, from double precision
int isa_fft_cols_per_cta(int H);            // 0: H too long for one column in shared memory
cudaError_t isa_launch_fft_rows_r2c(const float* in, size_t in_pitch, float2* spec, size_t spec_pitch, int W, int H, const isa_fft_plan& pn,
                                    const float2* tw_n, const float2* tw_w, cudaStream_t st);
// bins k >= kfrom are multiplied by kscale before the inverse (kfrom > W / 2: none)
cudaError_t isa_launch_fft_rows_c2r(const float2* spec, size_t spec_pitch, float* out, size_t out_pitch, int W, int H, const isa_fft_plan& pn,
                                    const float2* tw_n, const float2* tw_w, int clamp01, int kfrom, float kscale, cudaStream_t st);
// columns [0, ncols) of the half spectrum
cudaError_t isa_launch_fft_cols(float2* spec, size_t spec_pitch, int W, int H, int ncols, const isa_fft_plan& ph, const float2* tw_h, int mode,
                                const isa_fft_filter& f, const float2* ref, size_t ref_pitch, cudaStream_t st);
// the first bin column from which the filter is 1 at every row (W / 2 + 1: none)
int isa_fft_filter_columns(int W, const isa_fft_filter& f);

struct isa_pair_desc {
    int ref, trk;          // frame indices
    int grid;              // index of this pair's shift grid
    float base_ref_x, base_ref_y, rot_ref;
    float base_trk_x, base_trk_y, rot_trk;
};

// bw.cu
cudaError_t isa_launch_demosaic_gray(const uint16_t* raw, size_t raw_pitch, int W, int H, unsigned cfa, const float* black,
                                     const float* scale, const float* divisor, const float* gray_w, int gamma_gray,
                                     float* gray, size_t gray_pitch, float* rgb, size_t rgb_pitch, cudaStream_t st);
cudaError_t isa_launch_gamma(float* rgb, size_t pitch, int W, int H, cudaStream_t st);
cudaError_t isa_launch_fourier_filter(float2* spec, size_t pitch, int W, int H, int batch, size_t batch_stride, float lp, float hp,
                                      float lps, float hps, int clear_axis, float post_scale, cudaStream_t st);
cudaError_t isa_launch_gauss(const float* in, size_t in_pitch, float* out, size_t out_pitch, float* tmp, size_t tmp_pitch, int W,
                             int H, int C, const float* taps, int ntaps, int clamp01_input, cudaStream_t st);
cudaError_t isa_launch_resize_box(const float* in, size_t in_pitch, int W, int H, int L, float* out, size_t out_pitch,
                                  cudaStream_t st);
cudaError_t isa_launch_pyramid248(const float* in, size_t in_pitch, int W, int H, float* o2, size_t p2, float* o4, size_t p4, float* o8, size_t p8,
                                  cudaStream_t st);
cudaError_t isa_launch_subsample(const uint16_t* raw, size_t raw_pitch, int W, int H, unsigned cfa, float max_val, float* out,
                                 size_t out_pitch, cudaStream_t st);

// track.cu
cudaError_t isa_launch_track(const float* const* frames, size_t img_pitch, int Wl, int Hl, int T, int S, int tcx, int tcy,
                             const isa_pair_desc* pairs, int npairs, float2* grids, size_t grid_pitch, size_t grid_stride,
                             float threshold, float* scores, int* argmin, int* offsets, cudaStream_t st);
cudaError_t isa_launch_upsample(const float2* in, size_t in_pitch, size_t in_stride, float2* out, size_t out_pitch,
                                size_t out_stride, int ngrids, int oldLevel, int newLevel, int ocx, int ocy, int ncx, int ncy,
                                int oldT, int newT, cudaStream_t st);
size_t isa_solve_smem(int m, int n1);
cudaError_t isa_solve_prepare();
cudaError_t isa_launch_solve(const int* row_a, const int* row_b, const int* row_sign, const double* N0, int m, int n1,
                             float2* grids, size_t grid_pitch, size_t grid_stride, const int* row_grid, int tcx, int tcy,
                             float2* x_out, int* status, cudaStream_t st);
cudaError_t isa_launch_optimal(const float2* x, int n1, int tcx, int tcy, int ref, int trk, float2* out, size_t out_pitch,
                               cudaStream_t st);

// flow.cu
cudaError_t isa_launch_flow_from_tiles(const float2* tiles, size_t tile_pitch, int tcx, int tcy, int W, int H, float bx, float by,
                                       float rot, float2* flow, size_t flow_pitch, cudaStream_t st);
cudaError_t isa_launch_warp(const float* img, size_t img_pitch, int W, int H, const float2* flow, size_t flow_pitch, float* out,
                            size_t out_pitch, cudaStream_t st);
cudaError_t isa_launch_derivatives(const float* src, const float* tgt, size_t pitch, int W, int H, float* ix, float* iy, float* it,
                                   size_t out_pitch, cudaStream_t st);
cudaError_t isa_launch_derivatives2(const float* img, size_t pitch, int W, int H, float* ix, float* iy, size_t out_pitch,
                                    cudaStream_t st);
cudaError_t isa_launch_lk_sums(float2* flow, size_t flow_pitch, const float* ix, const float* iy, const float* it, size_t pitch, int W,
                               int H, int half, float min_det, cudaStream_t st);
cudaError_t isa_launch_lk_iteration(const float2* flow_in, float2* flow_out, size_t flow_pitch, const float* src, const float* ref,
                                    size_t img_pitch, int W, int H, int half, float min_det, cudaStream_t st, int strip_rows = 0);
// adjoint of one LK iteration (scratch: wplane one float plane, a5 and A5 five planes, gd3 three planes, all W x H floats at
// pitch W * 4) and of the tile term of the flow from tiles
cudaError_t isa_launch_lk_adjoint(const float2* f, const float2* gout, float2* gin, size_t fpitch, const float* src, const float* ref, size_t img_pitch,
                                  int W, int H, int half, float min_det, float* wplane, float* a5, float* A5, float* gd3, cudaStream_t st);
cudaError_t isa_launch_tiles_bwd(const float2* g, size_t fpitch, int W, int H, int tcx, int tcy, float2* gt, size_t tpitch, cudaStream_t st);

// robust.cu
cudaError_t isa_launch_robustness(const float* ref3, const float* mov3, size_t img_pitch, float4* mask, size_t mask_pitch, int Wh,
                                  int Hh, const float2* flow, size_t flow_pitch, int Wf, int Hf, float alpha, float beta,
                                  float thr_m, float s, float t, cudaStream_t st);
cudaError_t isa_launch_erode(const float4* in, size_t in_pitch, float4* out, size_t out_pitch, int W, int H, int size,
                             cudaStream_t st);
cudaError_t isa_launch_robustness_erode(const float* ref3, const float* mov3, size_t img_pitch, int Wh, int Hh, const float2* flow,
                                        size_t flow_pitch, int Wf, int Hf, float alpha, float beta, float thr_m, float s, float t, int size,
                                        float4* out, size_t out_pitch, cudaStream_t st);

// pipeline form of the mask: reference statistics once per burst, moved 3x3 means per frame
cudaError_t isa_launch_ref_stats(const float* ref3, size_t img_pitch, int Wh, int Hh, float4* mr, float4* sr, size_t sp, cudaStream_t st);
cudaError_t isa_launch_box3(const float* mov3, size_t img_pitch, int Wh, int Hh, float4* box, size_t sp, cudaStream_t st);
cudaError_t isa_launch_robustness_erode_tabs(const float4* mr, const float4* sr, const float4* box, size_t sp, const float* mov3, size_t img_pitch,
                                             int Wh, int Hh, const float2* flow, size_t flow_pitch, int Wf, int Hf, float alpha, float beta,
                                             float thr_m, float s, float t, int size, float4* out, size_t out_pitch, int bil, cudaStream_t st);

// prealign.cu
cudaError_t isa_launch_rotate_cubic(const float* src, size_t pitch, int W, int H, double angle_deg, float* dst, size_t dst_pitch, cudaStream_t st);
cudaError_t isa_launch_conj_mul(const float2* a, float2* b, size_t n, cudaStream_t st);
size_t isa_argmax_scratch_bytes();
cudaError_t isa_launch_argmax(const float* img, int n, void* scratch, void* out, cudaStream_t st);

// adjoint of the merge (robust.cu, merge.cu)
cudaError_t isa_launch_mask_store(const float4* mr, const float4* sr, const float4* box, size_t sp, const float* mov3, size_t img_pitch, int Wh,
                                  int Hh, const float2* flow, size_t flow_pitch, int Wf, int Hf, float alpha, float beta, float thr_m, float s,
                                  float t, float4* m_out, float4* aux_out, int bil, cudaStream_t st);
cudaError_t isa_launch_mask_flow_bwd(const float4* mr, const float4* sr, const float4* box, size_t sp, const float* mov3, size_t img_pitch, int Wh,
                                     int Hh, const float2* flow, size_t flow_pitch, int Wf, int Hf, float alpha, float beta, float t,
                                     const float4* aux, const float4* g_mask, float2* gflow, cudaStream_t st);
cudaError_t isa_launch_erode_route(const float4* m, const float4* g_eroded, size_t sp, int Wh, int Hh, int size, float4* g_mask, cudaStream_t st);
cudaError_t isa_launch_mask_param_bwd(const float4* m, const float4* aux, const float4* g_mask, size_t sp, int Wh, int Hh, float t, double* grad2,
                                      cudaStream_t st);

// merge.cu
struct isa_accum_geom {
    int W, H;          // input frame
    int Wo, Ho;        // output grid
    float s;           // merge scale
    int s_int;         // s when it is a positive integer, else 0
    int ox, oy;        // output-grid origin
    int cx0, cy0, cx1, cy1;  // inclusive source crop
    int masks_finite;  // 1: every mask value is finite (masks made by this library)
    int bilinear;      // 1: sample mode BILINEAR (the four integer shifts around s * flow, blended)
    int bx = 0, by = 0;  // thread block of the generic accumulation (0: 32 x 8)
    int yb0, yb1;      // output rows [yb0, yb1) computed by this launch (yb0 a multiple of 32)
};
struct isa_frame_in {
    const uint16_t* raw;
    const float2* flow;   // nullptr: zero flow
    const float4* mask;   // nullptr: certainty 1
};
cudaError_t isa_launch_structure_tensor(const float* img, size_t pitch, int W, int H, float* st3, size_t st_pitch, cudaStream_t st);
cudaError_t isa_launch_kernel_param(const float* st3, size_t st_pitch, int W, int H, float* out, size_t out_pitch, int out_channels,
                                    float Dth, float Dtr, float kDetail, float kDenoise, float kStretch, float kShrink,
                                    cudaStream_t st);
cudaError_t isa_launch_accumulate(const isa_accum_geom& g, unsigned cfa, const isa_frame_in* frames, int nframes,
                                  const isa_frame_in* single, size_t raw_pitch, size_t flow_pitch, size_t mask_pitch, const float* kparam, size_t kparam_pitch,
                                  int kparam_channels, const float* white, const float* black, float* acc, float* wsum,
                                  size_t out_pitch, int accumulate_into, cudaStream_t st);
bool isa_accumulate_x2_supported(unsigned cfa);
cudaError_t isa_launch_accumulate_x2(const isa_accum_geom& g, unsigned cfa, const isa_frame_in* frames, int nframes, const isa_frame_in* single,
                                     size_t raw_pitch, size_t flow_pitch, size_t mask_pitch, const float* kparam, size_t kparam_pitch,
                                     const float* white, const float* black, float* acc, float* wsum, size_t out_pitch, int accumulate_into,
                                     cudaStream_t st);
cudaError_t isa_launch_apply_weighting(float* img, size_t img_pitch, const float* acc, const float* wsum, size_t pitch, int W, int H,
                                       float thr, cudaStream_t st);

cudaError_t isa_launch_accumulate_bwd(const isa_accum_geom& g, unsigned cfa, const isa_frame_in* frames, int nframes, size_t raw_pitch,
                                      size_t flow_pitch, size_t mask_pitch, const float* kparam, size_t kparam_pitch, const float* white,
                                      const float* black, const float* out, size_t out_pitch, const float* wsum, size_t ws_pitch, const float* target,
                                      size_t tg_pitch, const float* weight, size_t wt_pitch, float* gkp, float4* gmask, size_t gmask_stride, double* loss,
                                      float2* gflow, cudaStream_t st);
cudaError_t isa_launch_kparam_bwd(const float* st3, size_t st_pitch, int W, int H, const float* gkp, float Dth, float Dtr, float kDetail,
                                  float kDenoise, float kStretch, float kShrink, double* grad6, cudaStream_t st);

// post.cu: the post-processing chain (isa_postprocess), arguments by value
struct isa_post_args {
    int crop_x, crop_y, crop_w, crop_h;
    float wb[3];
    float t1[12], t2[12];
    float amp;
    int nlut, uniform;
    float lut_x[ISA_MAX_LUT];
    float lut_c[ISA_MAX_LUT - 1][4];  // per segment k: cubic in t = v - lut_x[k], c0 + c1 t + c2 t^2 + c3 t^3
};
cudaError_t isa_launch_postprocess(const float* img, size_t pitch, const isa_post_args& a, int format, void* out, size_t out_pitch,
                                   cudaStream_t st);

// raw.cu: PEF decoding (isa_pef_decode, isa_pef_unpack)
size_t isa_pef_scratch_layout(unsigned long long nbytes, int W, int H, size_t* parts);
cudaError_t isa_launch_pef_decode(const uint8_t* data, unsigned long long nbytes, const unsigned short* table, int W, int H, void* scratch,
                                  uint16_t* out, size_t out_pitch, cudaStream_t st);
int isa_pef_max_blocks();
cudaError_t isa_launch_pef_unpack(const uint8_t* file, unsigned long long fsize, const uint32_t* offsets, const uint32_t* sizes, int nstrips,
                                  int rows_per_strip, int W, int H, int depth, uint16_t* out, size_t out_pitch, cudaStream_t st);

// api.cu: sets the calling thread's isa_last_error message and returns code
int isa_set_error(int code, const char* msg);

// raw.cu: DNG pixel data (isa_dng_decode)
size_t isa_dng_part_bytes();
void isa_dng_part_set(void* dst, int i, unsigned long long pos, unsigned long long end, int skip, const int* hdr, int out_row, int out_col,
                      const int* table, unsigned long long rowbuf);
cudaError_t isa_launch_dng(const uint8_t* file, unsigned long long fsize, int compression, const void* parts, int nparts, const uint16_t* tables,
                           uint16_t* rows, const unsigned long long* offs, const unsigned long long* cnts, int rps, int depth, const uint16_t* lin,
                           int nlin, const uint16_t* bh, const uint16_t* bv, int W, int H, int large, uint16_t* out, size_t out_pitch, int* error,
                           cudaStream_t st, int jwide_max, int ntables);
// the parallel decoder of predictor-1 parts: scratch bytes (0 = the frame does not qualify) and launch
size_t isa_dngf_scratch(const void* parts, int nparts, const uint16_t* tables, size_t ntables, int large);
size_t isa_dngf_flag_offset(const void* parts, int nparts, const uint16_t* tables, size_t ntables, int large);  // the hand-back flag in that scratch
cudaError_t isa_launch_dngf(const uint8_t* file, unsigned long long fsize, const void* parts_host, int nparts, const uint16_t* tables_host,
                            size_t ntables, const uint16_t* lin, int nlin, const uint16_t* bh, const uint16_t* bv, int W, int H, int large,
                            uint16_t* out, size_t out_pitch, int* error, void* scratch, size_t scratch_bytes, int* anomaly_host /* NULL: not read back */,
                            cudaStream_t st);
