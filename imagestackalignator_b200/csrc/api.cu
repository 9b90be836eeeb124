// C ABI (include/isa.h): argument checks, the context that owns the fused
// pipeline's buffers, and the pipeline itself, which issues the kernels in
// the order of the reference controller (ImageStackAlignatorController.cs:
// DeBayerBWGaussWB :2384-2418, TrackPatches :1601-1746, PrepareAccumulation
// :1795-1926, Accumulate :1928-1987) on the caller's stream.
#include "isa.h"
#include "isa_internal.cuh"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <limits>
#include <map>
#include <mutex>
#include <string>
#include <vector>

namespace {

thread_local std::string g_err;
thread_local int g_dng_path = -1;  // decoder of the calling thread's last isa_dng_decode: 1 parallel, 0 per part

int fail(int code, const char* fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

}  // namespace

// The calling thread's error message, for the other host files of the library.
int isa_set_error(int code, const char* msg)
{
    g_err = msg ? msg : "";
    return code;
}

namespace {

#define ISA_CK(call)                                                                         \
    do {                                                                                     \
        cudaError_t e_ = (call);                                                             \
        if (e_ != cudaSuccess) return fail(ISA_ECUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
    } while (0)
#define ISA_LAUNCH(ctx, call) \
    do {                      \
        ISA_CK(call);         \
        ++(ctx)->launches;    \
    } while (0)
#define ISA_TRY(call)            \
    do {                         \
        int s_ = (call);         \
        if (s_ != ISA_OK) return s_; \
    } while (0)

inline cudaStream_t S(void* s) { return (cudaStream_t)s; }

unsigned pack_cfa(const int cfa[4])
{
    unsigned v = 0;
    for (int i = 0; i < 4; i++) v |= (unsigned)(cfa[i] & 3) << (2 * i);
    return v;
}

bool cfa_ok(const int cfa[4])
{
    for (int i = 0; i < 4; i++)
        if (cfa[i] < 0 || cfa[i] > 2) return false;
    return true;
}

// gaussian_filter_1D (controller :2351-2382), float arithmetic as in C#.
std::vector<float> gauss_taps(float sigma)
{
    if (sigma <= 0) {
        std::vector<float> t(9, 0.f);
        t[4] = 1.f;
        return t;
    }
    int size = (int)(sigma / 0.6f - 0.4f) * 2 + 1 + 2;
    size = std::min(size, 99);
    std::vector<float> t(size);
    int c = size / 2;
    for (int i = 0; i < size; i++) {
        int x = i - c;
        t[i] = (float)std::exp((double)((float)(-(x * x)) / (2 * sigma * sigma)));
    }
    float sum = 0;
    for (int i = 0; i < size; i++) sum += t[i];
    for (int i = 0; i < size; i++) t[i] /= sum;
    return t;
}

// ---- ShiftCollection bookkeeping (ShiftCollection.cs:100-512) -------------
struct Strategy {
    int n = 0, m = 0, n1 = 0;
    std::vector<std::pair<int, int>> pairs;  // tracking order (FillShiftPairs)
    std::vector<int> idx;                    // n x n -> measurement row (FillIndexTable)
    std::vector<int> a, b, sign;             // row k of the incidence matrix = sign on [a, b)
};

int shift_count(int n, int strategy, int block)
{
    switch (strategy) {
    case ISA_TRACK_FULL: return (int)((n - 1) * ((float)n / 2.0f));
    case ISA_TRACK_ONLY_ON_REFERENCE: return n - 1;
    case ISA_TRACK_ON_REFERENCE_BLOCK: return (int)((block - 1) * ((float)block / 2.0f)) + block * (n - block);
    case ISA_TRACK_BLOCKS: return (int)(-0.5 * block * (block - 2 * n + 1));
    }
    return 0;
}

bool build_strategy(int n, int ref, int strategy, int block, Strategy& s)
{
    if (block >= n) block = n - 1;  // ShiftCollection constructor
    s = Strategy();
    s.n = n;
    s.n1 = n - 1;
    s.m = shift_count(n, strategy, block);
    s.idx.assign((size_t)n * n, -1);
    int first = 0, last = 0;
    if (strategy == ISA_TRACK_ON_REFERENCE_BLOCK) {
        if (ref < n / 2) { first = std::max(ref - block / 2, 0); last = first + block - 1; }
        else { last = std::min(ref + block / 2, n - 1); first = last - block + 1; }
    }
    auto add_row = [&](int from, int to, int a, int b, int sg) {
        s.idx[(size_t)from * n + to] = (int)s.a.size();
        s.a.push_back(a); s.b.push_back(b); s.sign.push_back(sg);
    };
    // rows in FillIndexTable order with their incidence intervals
    if (strategy == ISA_TRACK_FULL) {
        for (int d = 1; d < n; d++)
            for (int f = 0; f + d < n; f++) add_row(f, f + d, f, f + d, 1);
        for (int r = 0; r < n; r++)
            for (int t = r + 1; t < n; t++) s.pairs.push_back({r, t});
    } else if (strategy == ISA_TRACK_ONLY_ON_REFERENCE) {
        for (int t = 0; t < n; t++) {
            if (t == ref) continue;
            if (t < ref) add_row(ref, t, t, ref, -1);
            else add_row(ref, t, ref, t, 1);
            s.pairs.push_back({ref, t});
        }
    } else if (strategy == ISA_TRACK_ON_REFERENCE_BLOCK) {
        for (int sh = 0; sh < block - 1; sh++) {
            int count = block - 1 - sh;
            for (int line = 0; line < count; line++) {
                int f = line + first, t = line + first + block - count;
                add_row(f, t, f, t, 1);
                s.pairs.push_back({f, t});
            }
        }
        for (int i = 0; i < first; i++)
            for (int tb = first; tb <= last; tb++) { add_row(tb, i, i, tb, -1); s.pairs.push_back({tb, i}); }
        for (int i = last + 1; i < n; i++)
            for (int tb = first; tb <= last; tb++) { add_row(tb, i, tb, i, 1); s.pairs.push_back({tb, i}); }
    } else if (strategy == ISA_TRACK_BLOCKS) {
        for (int d = 1; d <= block; d++)
            for (int f = 0; f + d < n; f++) add_row(f, f + d, f, f + d, 1);
        for (int sh = 0; sh < block; sh++) {
            int count = (n - 1) - sh;
            for (int line = 0; line < count; line++) s.pairs.push_back({line, line + n - count});
        }
    } else {
        return false;
    }
    return (int)s.a.size() == s.m && (int)s.pairs.size() == s.m;  // "Ooups" check (ShiftCollection.cs:522-525)
}

size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

}  // namespace

int isa_static_solve_setup();

// ---------------------------------------------------------------------------
struct isa_ctx {
    int device = 0;  // current device at isa_ctx_create; the context's memory, events and streams live there
    int max_w = 0, max_h = 0, max_n = 0;
    isa_params p{};
    int max_pairs = 0, max_rows = 0, max_tiles = 0, maxcx = 0, maxcy = 0;
    int max_wo = 0, max_ho = 0;
    // device memory (one arena, carved)
    void* arena = nullptr;
    size_t arena_bytes = 0;
    uint16_t* raw_stage = nullptr;
    float *bw_track = nullptr, *bw_acc = nullptr, *tmp = nullptr;
    float* pyr[ISA_MAX_LEVELS] = {};
    float2* spec = nullptr;
    float2 *grids = nullptr, *grids_tmp = nullptr, *x = nullptr, *tiles_opt = nullptr;
    int* status = nullptr;
    int *row_a = nullptr, *row_b = nullptr, *row_sign = nullptr, *row_grid = nullptr;
    double* N0 = nullptr;
    isa_pair_desc* pair_desc = nullptr;
    const float** frame_tab = nullptr;
    float2 *flows = nullptr, *flow_tmp = nullptr;
    float *half_ref = nullptr, *half_mov = nullptr;
    float4 *ref_mr = nullptr, *ref_sr = nullptr, *mov_box = nullptr;  // robustness statistics (half resolution)
    float4* masks = nullptr;
    // adjoint sums (loss and the eight parameter gradients); the adjoint's image-sized scratch reuses buffers
    // that the forward no longer needs (see isa_merge_backward)
    double* adj_acc = nullptr;
    float *st3 = nullptr, *kparam = nullptr;
    float *acc = nullptr, *wsum = nullptr, *out_stage = nullptr;
    isa_frame_in* frame_in = nullptr;
    // full-frame transforms: plans (radices) and twiddle tables for the current frame size: rows of W / 2, the
    // unpacking factors e^{-2 pi i k / W} (k <= W / 2), columns of H
    isa_fft_plan fft_rows{}, fft_cols{};
    float2 *tw_rows = nullptr, *tw_unpack = nullptr, *tw_cols = nullptr;
    int fft_w = 0, fft_h = 0;
    cudaEvent_t ev[8] = {};
    // host entry point: frames copied in and the image copied out on a second stream, overlapped with the work
    static constexpr int kBands = 8;
    cudaStream_t copy_stream = nullptr;
    std::vector<cudaEvent_t> ev_frame;         // frame i resident
    cudaEvent_t ev_band[kBands] = {};          // output rows of band b final
    cudaEvent_t ev_free = nullptr, ev_copied = nullptr;
    int ev_count = 0;
    long launches = 0;  // kernels of this library launched by the last merge
    // caller-owned record of every level's tile search (isa_debug_track_record), or null
    int* track_rec = nullptr;
    size_t track_rec_bytes = 0;
    // caller-owned per-frame tile flows that replace the solved ones (isa_set_tile_flow), or null
    const float2* tile_override = nullptr;
    // sample mode BILINEAR only: scratch of the flow adjoint (isa_merge_backward_tiles), 25 floats per frame pixel
    float* adj_flow = nullptr;
    // launch shapes per frame size (isa_ctx_set_tuning)
    std::vector<isa_tuning> tuning;
    // set while isa_batch_graph_create captures a batch: no stage-time events, transform twiddles uploaded per burst
    bool capturing = false;
    // last call
    int last_w = 0, last_h = 0, last_n = 0, last_tcx0 = 0, last_tcy0 = 0, last_n1 = 0, last_ref = 0;
};

namespace {

size_t bw_pitch(int W) { return (size_t)W * sizeof(float); }

// floats per frame pixel of the flow adjoint's scratch: the recomputed flows of the LK iterations before the last (3 x 2), the
// warped source (1), the window-sum gradients and their box sums (5 + 5), the derivative gradients (3), the flow gradient
// ping-pong (2 x 2) and the half-res mask gradient (4 per half-res pixel = 1 per frame pixel)
constexpr size_t kAdjFlowFloats = 25;

// Host-to-device copies of the merge's small tables (pair and frame tables, solver rows, transform twiddles). Outside a
// graph capture they copy from the caller's host vectors; while isa_batch_graph_create captures a batch, they go
// through the graph's pinned arena, so that the captured copy nodes read memory that stays valid and unchanged for
// every replay.
struct HostStage {
    char* base = nullptr;
    size_t cap = 0, used = 0;
};
thread_local HostStage* g_stage = nullptr;

cudaError_t h2d(void* dst, const void* src, size_t bytes, cudaStream_t st)
{
    if (bytes == 0) return cudaSuccess;
    if (!g_stage) return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st);
    const size_t at = (g_stage->used + 15) / 16 * 16;
    if (at + bytes > g_stage->cap) return cudaErrorMemoryAllocation;
    memcpy(g_stage->base + at, src, bytes);
    g_stage->used = at + bytes;
    return cudaMemcpyAsync(dst, g_stage->base + at, bytes, cudaMemcpyHostToDevice, st);
}

int level_tiles(const isa_level& l, int W, int H, int* tcx, int* tcy)
{
    int Wl = W / l.resize_level, Hl = H / l.resize_level;
    *tcx = (Wl - 2 * l.max_shift) / l.tile_size;
    *tcy = (Hl - 2 * l.max_shift) / l.tile_size;
    return (*tcx > 0 && *tcy > 0) ? ISA_OK : ISA_EINVAL;
}

int check_params(const isa_params* p)
{
    if (!p) return fail(ISA_EINVAL, "params is NULL");
    if (p->level_count < 1 || p->level_count > ISA_MAX_LEVELS) return fail(ISA_EINVAL, "level_count %d out of range", p->level_count);
    for (int i = 0; i < p->level_count; i++) {
        const isa_level& l = p->levels[i];
        if (l.resize_level < 1 || l.tile_size < 2 || (l.tile_size & 1) || l.max_shift < 1)
            return fail(ISA_EINVAL, "level %d: resize %d tile %d shift %d invalid", i, l.resize_level, l.tile_size, l.max_shift);
    }
    if (p->levels[0].resize_level != 1) return fail(ISA_EINVAL, "the finest level must have resize_level 1");
    if (p->window_size_lk < 1 || p->window_size_lk / 2 > 15) return fail(ISA_EINVAL, "window_size_lk %d out of range", p->window_size_lk);
    if (p->erode_size < 1 || p->erode_size / 2 > 4) return fail(ISA_EINVAL, "erode_size %d out of range", p->erode_size);
    if (p->iterations_lk < 0) return fail(ISA_EINVAL, "iterations_lk < 0");
    if (p->tracking_strategy < 0 || p->tracking_strategy > 3) return fail(ISA_EINVAL, "tracking_strategy %d", p->tracking_strategy);
    if (p->merge_scale < 0 || p->merge_scale > 8) return fail(ISA_EINVAL, "merge_scale %g out of range", p->merge_scale);
    if (p->sample_mode != ISA_SAMPLE_ROUND && p->sample_mode != ISA_SAMPLE_BILINEAR) return fail(ISA_EINVAL, "sample_mode %d", p->sample_mode);
    return ISA_OK;
}

// Geometry of the accumulation for a W x H frame (see merge.cu).
void accum_geom(const isa_params* p, int W, int H, isa_accum_geom& g, float& thr)
{
    g.W = W; g.H = H;
    g.masks_finite = 0;
    g.bilinear = p->sample_mode == ISA_SAMPLE_BILINEAR;
    if (p->merge_scale > 0) {
        g.s = p->merge_scale;
        g.Wo = (int)std::lround(W * (double)p->merge_scale);
        g.Ho = (int)std::lround(H * (double)p->merge_scale);
        g.ox = g.oy = 0;
        g.cx0 = 0; g.cy0 = 0; g.cx1 = W - 1; g.cy1 = H - 1;
        thr = 0.f;
    } else if (p->super_resolution) {
        g.s = 2.f; g.Wo = W; g.Ho = H; g.ox = W / 2; g.oy = H / 2;
        g.cx0 = W / 4; g.cy0 = H / 4; g.cx1 = W / 2 - 1 + W / 4; g.cy1 = H / 2 - 1 + H / 4;
        thr = 0.f;
    } else {
        g.s = 1.f; g.Wo = W; g.Ho = H; g.ox = g.oy = 0;
        g.cx0 = 0; g.cy0 = 0; g.cx1 = W - 1; g.cy1 = H - 1;
        thr = 1.f;
    }
    float r = std::round(g.s);
    g.s_int = (r == g.s && r >= 1.f) ? (int)r : 0;
    g.yb0 = 0;
    g.yb1 = g.Ho;
}

// Plans and twiddle tables of the W x H transforms (the tables are copied on
// the caller's stream, ordered with the work that reads them).
int ensure_fft(isa_ctx* c, int W, int H, cudaStream_t st)
{
    if (c->fft_w == W && c->fft_h == H) return ISA_OK;
    if ((W & 1) || W > c->max_w || H > c->max_h) return fail(ISA_EINVAL, "transform size %dx%d", W, H);
    isa_fft_plan pr, pc;
    if (!isa_fft_plan_make(W / 2, pr) || !isa_fft_plan_make(H, pc)) return fail(ISA_EINVAL, "no FFT plan for %dx%d", W, H);
    std::vector<float2> tr(W / 2), tu(W), tc(H);
    isa_fft_twiddles(W / 2, tr.data());
    isa_fft_twiddles(W, tu.data());
    isa_fft_twiddles(H, tc.data());
    ISA_CK(h2d(c->tw_rows, tr.data(), tr.size() * sizeof(float2), st));
    ISA_CK(h2d(c->tw_unpack, tu.data(), (W / 2 + 1) * sizeof(float2), st));
    ISA_CK(h2d(c->tw_cols, tc.data(), tc.size() * sizeof(float2), st));
    // pageable sources: the copies above are staged before returning
    c->fft_rows = pr;
    c->fft_cols = pc;
    c->fft_w = W;
    c->fft_h = H;
    return ISA_OK;
}

// The forward half spectrum of a W x H real image into `spec` (pitch (W/2 + 1) * 8).
int fft_forward(isa_ctx* c, const float* img, size_t pitch, float2* spec, int W, int H, cudaStream_t st)
{
    ISA_TRY(ensure_fft(c, W, H, st));
    const size_t sp = (size_t)(W / 2 + 1) * sizeof(float2);
    ISA_LAUNCH(c, isa_launch_fft_rows_r2c(img, pitch, spec, sp, W, H, c->fft_rows, c->tw_rows, c->tw_unpack, st));
    isa_fft_filter none{};
    ISA_LAUNCH(c, isa_launch_fft_cols(spec, sp, W, H, W / 2 + 1, c->fft_cols, c->tw_cols, ISA_FFT_COLS_FWD, none, nullptr, 0, st));
    return ISA_OK;
}

void color_consts(const isa_raw_info* info, float black[3], float white[3], float scale[3], float divisor[3])
{
    for (int c = 0; c < 3; c++) {
        black[c] = info->black[c];
        white[c] = info->white[c];
        float cw = info->camera_white[c] != 0.f ? info->camera_white[c] : 1.f;
        scale[c] = 1.0f / cw;
        divisor[c] = info->white[c] / cw;
    }
}

// DeBayerBWGaussWB (controller :2384-2418) for one frame into `out`;
// `gray_out`, when given, also receives the Gaussian of the un-filtered
// gray image (the accumulation variant, skipFourierFilter = true).
inline size_t fsz_of(int W, int H) { return (size_t)W * H; }

int bw_frame(isa_ctx* c, const uint16_t* raw, size_t raw_pitch, int W, int H, const isa_raw_info* info, bool high_pass, float* out,
             const std::vector<float>& taps_hp, float* acc_out, const std::vector<float>& taps_acc, cudaStream_t st)
{
    float black[3], white[3], scale[3], divisor[3];
    color_consts(info, black, white, scale, divisor);
    const float gw_rgb[3] = {0.2989f, 0.5870f, 0.1141f}, gw_g[3] = {0.f, 1.f, 0.f};
    const float* gw = c->p.green_channel_only ? gw_g : gw_rgb;
    size_t pitch = bw_pitch(W);
    ISA_LAUNCH(c, isa_launch_demosaic_gray(raw, raw_pitch, W, H, pack_cfa(info->cfa), black, scale, divisor, gw, 1, out, pitch, nullptr, 0, st));
    if (acc_out)
        ISA_LAUNCH(c, isa_launch_gauss(out, pitch, acc_out, pitch, c->tmp, pitch, W, H, 1, taps_acc.data(), (int)taps_acc.size(), 0, st));
    if (high_pass) {
        // PreAlignment.FourierFilter: R2C rows, then per column the forward transform, fourierFilter (with the
        // 1 / (W * H) of the inverse) and the inverse transform, then C2R rows
        ISA_TRY(ensure_fft(c, W, H, st));
        const size_t sp = (size_t)(W / 2 + 1) * sizeof(float2);
        ISA_LAUNCH(c, isa_launch_fft_rows_r2c(out, pitch, c->spec, sp, W, H, c->fft_rows, c->tw_rows, c->tw_unpack, st));
        const isa_fft_filter f{1.0f, c->p.high_pass, 1.0f, c->p.high_pass_sigma, c->p.clear_axis, 1.0f / ((float)W * (float)H)};
        // columns from kf on have the coefficient 1 at every row: their forward and inverse transforms cancel (a
        // factor H), so they skip the column pass and take post_scale * H in the inverse row pass
        const int kf = isa_fft_filter_columns(W, f);
        const float kscale = f.post_scale * (float)H;
        ISA_LAUNCH(c, isa_launch_fft_cols(c->spec, sp, W, H, kf, c->fft_cols, c->tw_cols, ISA_FFT_COLS_FILTER, f, nullptr, 0, st));
        if (taps_hp.empty()) {
            ISA_LAUNCH(c, isa_launch_fft_rows_c2r(c->spec, sp, out, pitch, W, H, c->fft_rows, c->tw_rows, c->tw_unpack, 1, kf, kscale, st));
        } else {
            // inverse rows into scratch, then clamp + Gauss back into `out` in one pass
            ISA_LAUNCH(c, isa_launch_fft_rows_c2r(c->spec, sp, c->tmp, pitch, W, H, c->fft_rows, c->tw_rows, c->tw_unpack, 0, kf, kscale, st));
            ISA_LAUNCH(c, isa_launch_gauss(c->tmp, pitch, out, pitch, c->tmp + fsz_of(W, H), pitch, W, H, 1, taps_hp.data(), (int)taps_hp.size(), 1,
                                           st));
        }
        return ISA_OK;
    }
    if (!taps_hp.empty())
        ISA_LAUNCH(c, isa_launch_gauss(out, pitch, out, pitch, c->tmp, pitch, W, H, 1, taps_hp.data(), (int)taps_hp.size(), 0, st));
    return ISA_OK;
}

int check_info(const isa_raw_info* info)
{
    if (!info) return fail(ISA_EINVAL, "raw info is NULL");
    if (info->width < 16 || info->height < 16 || (info->width & 1) || (info->height & 1))
        return fail(ISA_EINVAL, "frame %dx%d: need even sizes of at least 16", info->width, info->height);
    if (!cfa_ok(info->cfa)) return fail(ISA_EINVAL, "CFA codes must be 0 (R), 1 (G) or 2 (B)");
    for (int c = 0; c < 3; c++)
        if (!(info->white[c] > 0)) return fail(ISA_EINVAL, "white level must be positive");
    return ISA_OK;
}

float prealign_rot(const isa_prealign* pre, int from, int to)
{
    if (!pre || !pre->rotations_deg) return 0.f;
    float a = pre->rotations_deg[to] - pre->rotations_deg[from];
    return a / 180.0f * (float)M_PI;
}

void prealign_shift(const isa_prealign* pre, int from, int to, float out[2])
{
    out[0] = out[1] = 0.f;
    if (!pre || !pre->shifts) return;
    out[0] = pre->shifts[2 * to] - pre->shifts[2 * from];
    out[1] = pre->shifts[2 * to + 1] - pre->shifts[2 * from + 1];
}

// Copies the solver's row tables (interval, sign, grid of each measurement
// row) and N0 = A^T A into device memory at the given addresses.
int upload_rows(int* d_a, int* d_b, int* d_sign, int* d_grid, double* d_N0, const Strategy& s, cudaStream_t st)
{
    std::vector<double> N0((size_t)s.n1 * s.n1, 0.0);
    for (int k = 0; k < s.m; k++)
        for (int i = s.a[k]; i < s.b[k]; i++)
            for (int j = s.a[k]; j < s.b[k]; j++) N0[(size_t)i * s.n1 + j] += 1.0;
    std::vector<int> rg(s.m);
    for (int k = 0; k < s.m; k++) rg[k] = k;  // grid k holds measurement row k
    ISA_CK(h2d(d_a, s.a.data(), s.m * sizeof(int), st));
    ISA_CK(h2d(d_b, s.b.data(), s.m * sizeof(int), st));
    ISA_CK(h2d(d_sign, s.sign.data(), s.m * sizeof(int), st));
    ISA_CK(h2d(d_grid, rg.data(), s.m * sizeof(int), st));
    ISA_CK(h2d(d_N0, N0.data(), N0.size() * sizeof(double), st));
    // pageable sources: the copies above complete before returning
    return ISA_OK;
}

int upload_strategy(isa_ctx* c, const Strategy& s, cudaStream_t st)
{
    return upload_rows(c->row_a, c->row_b, c->row_sign, c->row_grid, c->N0, s, st);
}

// Host buffers of isa_merge_burst_host: frames arrive on the copy stream
// (event per frame) and the image leaves on it band by band.
struct HostIo {
    bool frames_async;  // wait for ev_frame[i] before the first use of frame i
    float* host_out;    // when set: the output is copied out band by band (rows of 12 * Wo bytes)
};

// The tuning entry for W x H frames: its own, else the 0 x 0 entry, else none.
const isa_tuning* tuning_for(const isa_ctx* c, int W, int H)
{
    const isa_tuning* any = nullptr;
    for (const isa_tuning& t : c->tuning) {
        if (t.width == W && t.height == H) return &t;
        if (t.width == 0 && t.height == 0) any = &t;
    }
    return any;
}

int run_merge(isa_ctx* c, const uint16_t* raw, size_t raw_pitch, size_t frame_stride, int n, const isa_raw_info* info,
              const isa_prealign* pre, float* out, size_t out_pitch, cudaStream_t st, const HostIo* hio = nullptr)
{
    const isa_params* p = &c->p;
    ISA_TRY(check_info(info));
    const int W = info->width, H = info->height;
    if (W > c->max_w || H > c->max_h) return fail(ISA_EINVAL, "frame %dx%d exceeds the context's %dx%d", W, H, c->max_w, c->max_h);
    if (n < 2 || n > c->max_n) return fail(ISA_EINVAL, "frame count %d outside [2, %d]", n, c->max_n);
    if (!raw || !out) return fail(ISA_EINVAL, "NULL frame or output pointer");
    const int ref = pre ? pre->reference : 0;
    if (ref < 0 || ref >= n) return fail(ISA_EINVAL, "reference index %d outside [0, %d)", ref, n);
    if (raw_pitch < (size_t)W * 2 || frame_stride < raw_pitch * H) return fail(ISA_EINVAL, "raw pitch/stride too small");
    isa_accum_geom g;
    float thr;
    accum_geom(p, W, H, g, thr);
    const isa_tuning* tune = tuning_for(c, W, H);
    const int lk_rows = tune ? tune->lk_strip_rows : 0;
    if (tune) { g.bx = tune->acc_block_x; g.by = tune->acc_block_y; }
    if (out_pitch < (size_t)g.Wo * 12) return fail(ISA_EINVAL, "output pitch %zu < %d", out_pitch, g.Wo * 12);
    if (g.Wo > c->max_wo || g.Ho > c->max_ho) return fail(ISA_EINVAL, "output exceeds the context");
    Strategy strat;
    if (!build_strategy(n, ref, p->tracking_strategy, p->tracking_block_size, strat))
        return fail(ISA_EINVAL, "tracking strategy %d with block %d and %d frames is inconsistent", p->tracking_strategy,
                    p->tracking_block_size, n);
    if (strat.m > c->max_rows || strat.n1 > 64) return fail(ISA_EINVAL, "too many frame pairs for the context");
    const auto frame = [&](int i) { return (const uint16_t*)((const char*)raw + (size_t)i * frame_stride); };
    const size_t pitch = bw_pitch(W);
    const size_t fsz = (size_t)W * H;
    const unsigned cfa = pack_cfa(info->cfa);
    float black[3], white[3], scale[3], divisor[3];
    color_consts(info, black, white, scale, divisor);
    c->ev_count = 0;
    c->launches = 0;
    auto mark = [&]() -> int {
        if (c->capturing) return ISA_OK;
        ISA_CK(cudaEventRecord(c->ev[c->ev_count++], st));
        return ISA_OK;
    };
    if (c->capturing) c->fft_w = c->fft_h = 0;
    ISA_TRY(mark());
    // 1. tracking (high-pass) and accumulation images of every frame
    const std::vector<float> taps_trk = gauss_taps(p->sigma_debayer_tracking), taps_acc = gauss_taps(p->sigma_debayer_accumulation);
    for (int i = 0; i < n; i++) {
        if (hio && hio->frames_async) ISA_CK(cudaStreamWaitEvent(st, c->ev_frame[i], 0));
        ISA_TRY(bw_frame(c, frame(i), raw_pitch, W, H, info, true, c->bw_track + i * fsz, taps_trk, c->bw_acc + i * fsz, taps_acc, st));
    }
    ISA_TRY(mark());
    // 2. pyramid tile alignment, coarsest level first (TrackPatches :1640-1712)
    ISA_TRY(upload_strategy(c, strat, st));
    const int L = p->level_count;
    const size_t gpitch = (size_t)c->maxcx * sizeof(float2), gstride = gpitch * c->maxcy;
    int otcx = 0, otcy = 0, olevel = 0, oT = 0;
    float2* grids = c->grids;
    float2* grids_tmp = c->grids_tmp;
    ISA_CK(cudaMemsetAsync(grids, 0, gstride * strat.m, st));
    int tcx0 = 0, tcy0 = 0;
    // record of the tile search per level (argmin, then block offsets), finest level first
    std::vector<size_t> rec_off(L + 1, 0);
    for (int li = 0; li < L; li++) {
        int tx, ty;
        if (level_tiles(p->levels[li], W, H, &tx, &ty) != ISA_OK) return fail(ISA_EINVAL, "level %d has no tiles for %dx%d", li, W, H);
        rec_off[li + 1] = rec_off[li] + (size_t)3 * strat.m * tx * ty;
    }
    if (c->track_rec && c->track_rec_bytes < rec_off[L] * sizeof(int))
        return fail(ISA_EINVAL, "tile-search record of %zu bytes < %zu needed", c->track_rec_bytes, rec_off[L] * sizeof(int));
    // levels with resize 2, 4 and 8 (the default pyramid) from one read of each tracking image
    int lv_of[9] = {-1, -1, -1, -1, -1, -1, -1, -1, -1};
    for (int li = 0; li < L; li++)
        if (p->levels[li].resize_level >= 1 && p->levels[li].resize_level <= 8) lv_of[p->levels[li].resize_level] = li;
    const bool fused_pyramid = lv_of[2] >= 0 && lv_of[4] >= 0 && lv_of[8] >= 0;
    if (fused_pyramid)
        for (int i = 0; i < n; i++)
            ISA_LAUNCH(c, isa_launch_pyramid248(c->bw_track + i * fsz, pitch, W, H, c->pyr[lv_of[2]] + (size_t)i * (W / 2) * (H / 2), bw_pitch(W / 2),
                                                c->pyr[lv_of[4]] + (size_t)i * (W / 4) * (H / 4), bw_pitch(W / 4),
                                                c->pyr[lv_of[8]] + (size_t)i * (W / 8) * (H / 8), bw_pitch(W / 8), st));
    for (int li = L - 1; li >= 0; li--) {
        const isa_level& lv = p->levels[li];
        const int Wl = W / lv.resize_level, Hl = H / lv.resize_level;
        int tcx, tcy;
        if (level_tiles(lv, W, H, &tcx, &tcy) != ISA_OK) return fail(ISA_EINVAL, "level %d has no tiles for %dx%d", li, W, H);
        if (li == 0) { tcx0 = tcx; tcy0 = tcy; }
        if (li != L - 1) {
            ISA_LAUNCH(c, isa_launch_upsample(grids, gpitch, gstride, grids_tmp, gpitch, gstride, strat.m, olevel, lv.resize_level, otcx, otcy, tcx,
                                       tcy, oT, lv.tile_size, st));
            std::swap(grids, grids_tmp);
        }
        std::vector<const float*> fptr(n);
        size_t lpitch = bw_pitch(Wl);
        if (lv.resize_level > 1) {
            float* base = c->pyr[li];
            const bool done = fused_pyramid && (lv.resize_level == 2 || lv.resize_level == 4 || lv.resize_level == 8) && lv_of[lv.resize_level] == li;
            for (int i = 0; i < n; i++) {
                float* dst = base + (size_t)i * Wl * Hl;
                if (!done) ISA_LAUNCH(c, isa_launch_resize_box(c->bw_track + i * fsz, pitch, W, H, lv.resize_level, dst, lpitch, st));
                fptr[i] = dst;
            }
        } else {
            for (int i = 0; i < n; i++) fptr[i] = c->bw_track + i * fsz;
        }
        std::vector<isa_pair_desc> pd(strat.m);
        for (size_t k = 0; k < strat.pairs.size(); k++) {
            int r = strat.pairs[k].first, t = strat.pairs[k].second;
            float br[2], bt[2];
            prealign_shift(pre, ref, r, br);
            prealign_shift(pre, ref, t, bt);
            isa_pair_desc& d = pd[k];
            d.ref = r; d.trk = t; d.grid = strat.idx[(size_t)r * n + t];
            d.base_ref_x = br[0] / lv.resize_level; d.base_ref_y = br[1] / lv.resize_level; d.rot_ref = prealign_rot(pre, ref, r);
            d.base_trk_x = bt[0] / lv.resize_level; d.base_trk_y = bt[1] / lv.resize_level; d.rot_trk = prealign_rot(pre, ref, t);
        }
        ISA_CK(h2d(c->pair_desc + (size_t)li * c->max_pairs, pd.data(), pd.size() * sizeof(isa_pair_desc), st));
        ISA_CK(h2d(c->frame_tab + (size_t)li * c->max_n, fptr.data(), n * sizeof(float*), st));
        ISA_LAUNCH(c, isa_launch_track(c->frame_tab + (size_t)li * c->max_n, lpitch, Wl, Hl, lv.tile_size, lv.max_shift, tcx, tcy,
                                c->pair_desc + (size_t)li * c->max_pairs, strat.m, grids, gpitch, gstride, p->matching_threshold, nullptr,
                                c->track_rec ? c->track_rec + rec_off[li] : nullptr,
                                c->track_rec ? c->track_rec + rec_off[li] + (size_t)strat.m * tcx * tcy : nullptr, st));
        ISA_LAUNCH(c, isa_launch_solve(c->row_a, c->row_b, c->row_sign, c->N0, strat.m, strat.n1, grids, gpitch, gstride, c->row_grid, tcx, tcy,
                                c->x, c->status, st));
        otcx = tcx; otcy = tcy; olevel = lv.resize_level; oT = lv.tile_size;
    }
    ISA_TRY(mark());
    // 3. kernel parameters from the reference frame (PrepareAccumulation :1851-1858)
    const std::vector<float> taps_st = gauss_taps(p->sigma_structure_tensor);
    const size_t p3 = (size_t)W * 12, p4 = (size_t)W * 16;
    ISA_LAUNCH(c, isa_launch_structure_tensor(c->bw_acc + ref * fsz, pitch, W, H, c->st3, p3, st));
    ISA_LAUNCH(c, isa_launch_gauss(c->st3, p3, c->st3, p3, c->tmp, p3, W, H, 3, taps_st.data(), (int)taps_st.size(), 0, st));
    ISA_LAUNCH(c, isa_launch_kernel_param(c->st3, p3, W, H, c->kparam, p4, 4, p->dth, p->dtr, p->k_detail, p->k_denoise, p->k_stretch, p->k_shrink,
                                   st));
    ISA_TRY(mark());
    // 4. per frame: LK refinement and robustness mask (Accumulate :1961-1977)
    const int Wh = W / 2, Hh = H / 2;
    const size_t hp3 = (size_t)Wh * 12, hp4 = (size_t)Wh * 16, fp = (size_t)W * sizeof(float2);
    float maxv = 0.f;
    for (int ch = 0; ch < 3; ch++) maxv = std::max(maxv, white[ch] + black[ch]);
    ISA_LAUNCH(c, isa_launch_subsample(frame(ref), raw_pitch, W, H, cfa, maxv, c->half_ref, hp3, st));
    ISA_LAUNCH(c, isa_launch_ref_stats(c->half_ref, hp3, Wh, Hh, c->ref_mr, c->ref_sr, hp4, st));
    const int half = p->window_size_lk / 2;
    std::vector<isa_frame_in> fin;
    fin.push_back({frame(ref), nullptr, nullptr});
    for (int i = 0; i < n; i++) {
        if (i == ref) continue;
        float2* flow = c->flows + (size_t)i * fsz;
        ISA_LAUNCH(c, isa_launch_subsample(frame(i), raw_pitch, W, H, cfa, maxv, c->half_mov, hp3, st));
        const float2* tiles = c->tiles_opt;
        if (c->tile_override)
            tiles = c->tile_override + (size_t)i * tcx0 * tcy0;
        else
            ISA_LAUNCH(c, isa_launch_optimal(c->x, strat.n1, tcx0, tcy0, ref, i, c->tiles_opt, (size_t)tcx0 * sizeof(float2), st));
        float bs[2];
        prealign_shift(pre, ref, i, bs);
        // ping-pong so that the last iteration lands in `flow`
        float2* a = (p->iterations_lk & 1) ? c->flow_tmp : flow;
        float2* b = (p->iterations_lk & 1) ? flow : c->flow_tmp;
        ISA_LAUNCH(c, isa_launch_flow_from_tiles(tiles, (size_t)tcx0 * sizeof(float2), tcx0, tcy0, W, H, bs[0], bs[1], prealign_rot(pre, ref, i),
                                          a, fp, st));
        for (int it = 0; it < p->iterations_lk; it++) {
            ISA_LAUNCH(c, isa_launch_lk_iteration(a, b, fp, c->bw_acc + i * fsz, c->bw_acc + ref * fsz, pitch, W, H, half, p->min_det_lk, st,
                                                  lk_rows));
            std::swap(a, b);
        }
        float4* mask = c->masks + (size_t)i * Wh * Hh;
        ISA_LAUNCH(c, isa_launch_box3(c->half_mov, hp3, Wh, Hh, c->mov_box, hp4, st));
        ISA_LAUNCH(c, isa_launch_robustness_erode_tabs(c->ref_mr, c->ref_sr, c->mov_box, hp4, c->half_mov, hp3, Wh, Hh, flow, fp, W, H,
                                                       info->noise_alpha, info->noise_beta, p->threshold_m, p->robust_s, p->robust_t,
                                                       p->erode_size, mask, hp4, p->sample_mode == ISA_SAMPLE_BILINEAR, st));
        fin.push_back({frame(i), flow, mask});
    }
    ISA_TRY(mark());
    // 5. accumulation: reference frame first (PrepareAccumulation :1894-1902), then the others in order
    const size_t op = (size_t)g.Wo * 12;
    g.masks_finite = 1;  // the masks come from isa_launch_robustness_erode_tabs, whose values are clamped to [0, 1]
    ISA_CK(h2d(c->frame_in, fin.data(), fin.size() * sizeof(isa_frame_in), st));
    if (hio && hio->host_out) {
        // bands of output rows: accumulate, normalise, then copy out on the copy stream while the next band runs
        if (thr > 0)
            ISA_LAUNCH(c, isa_launch_demosaic_gray(frame(ref), raw_pitch, W, H, cfa, black, scale, divisor, nullptr, 0, nullptr, 0, out, out_pitch, st));
        const int rows = std::max(32, (g.Ho / isa_ctx::kBands + 31) / 32 * 32);
        int b = 0;
        for (int y0 = 0; y0 < g.Ho; y0 += rows, b++) {
            isa_accum_geom gb = g;
            gb.yb0 = y0;
            gb.yb1 = std::min(g.Ho, y0 + rows);
            const int nr = gb.yb1 - gb.yb0;
            if (p->fused_accumulate) {
                ISA_LAUNCH(c, isa_launch_accumulate(gb, cfa, c->frame_in, (int)fin.size(), nullptr, raw_pitch, fp, hp4, c->kparam, p4, 4, white, black,
                                                    c->acc, c->wsum, op, 0, st));
            } else {
                ISA_CK(cudaMemsetAsync((char*)c->acc + (size_t)y0 * op, 0, op * nr, st));
                ISA_CK(cudaMemsetAsync((char*)c->wsum + (size_t)y0 * op, 0, op * nr, st));
                for (size_t f = 0; f < fin.size(); f++)
                    ISA_LAUNCH(c, isa_launch_accumulate(gb, cfa, nullptr, 1, &fin[f], raw_pitch, fp, hp4, c->kparam, p4, 4, white, black, c->acc,
                                                        c->wsum, op, 1, st));
            }
            float* ob = (float*)((char*)out + (size_t)y0 * out_pitch);
            ISA_LAUNCH(c, isa_launch_apply_weighting(ob, out_pitch, (const float*)((const char*)c->acc + (size_t)y0 * op),
                                                     (const float*)((const char*)c->wsum + (size_t)y0 * op), op, g.Wo, nr, thr, st));
            ISA_CK(cudaEventRecord(c->ev_band[b % isa_ctx::kBands], st));
            ISA_CK(cudaStreamWaitEvent(c->copy_stream, c->ev_band[b % isa_ctx::kBands], 0));
            ISA_CK(cudaMemcpy2DAsync((char*)hio->host_out + (size_t)y0 * g.Wo * 12, (size_t)g.Wo * 12, ob, out_pitch, (size_t)g.Wo * 12, nr,
                                     cudaMemcpyDeviceToHost, c->copy_stream));
        }
        ISA_TRY(mark());
        ISA_TRY(mark());
        // the caller's stream completes only when the image has left the device
        ISA_CK(cudaEventRecord(c->ev_copied, c->copy_stream));
        ISA_CK(cudaStreamWaitEvent(st, c->ev_copied, 0));
        c->last_w = W; c->last_h = H; c->last_n = n; c->last_tcx0 = tcx0; c->last_tcy0 = tcy0; c->last_n1 = strat.n1; c->last_ref = ref;
        return ISA_OK;
    }
    if (p->fused_accumulate) {
        ISA_LAUNCH(c, isa_launch_accumulate(g, cfa, c->frame_in, (int)fin.size(), nullptr, raw_pitch, fp, hp4, c->kparam, p4, 4, white, black, c->acc, c->wsum,
                                     op, 0, st));
    } else {
        ISA_CK(cudaMemsetAsync(c->acc, 0, op * g.Ho, st));
        ISA_CK(cudaMemsetAsync(c->wsum, 0, op * g.Ho, st));
        for (size_t f = 0; f < fin.size(); f++)
            ISA_LAUNCH(c, isa_launch_accumulate(g, cfa, nullptr, 1, &fin[f], raw_pitch, fp, hp4, c->kparam, p4, 4, white, black, c->acc, c->wsum, op, 1,
                                         st));
    }
    ISA_TRY(mark());
    // 6. ApplyWeighting (:1908-1917, :1994-2002)
    if (thr > 0)
        ISA_LAUNCH(c, isa_launch_demosaic_gray(frame(ref), raw_pitch, W, H, cfa, black, scale, divisor, nullptr, 0, nullptr, 0, out, out_pitch, st));
    ISA_LAUNCH(c, isa_launch_apply_weighting(out, out_pitch, c->acc, c->wsum, op, g.Wo, g.Ho, thr, st));
    ISA_TRY(mark());
    c->last_w = W; c->last_h = H; c->last_n = n; c->last_tcx0 = tcx0; c->last_tcy0 = tcy0; c->last_n1 = strat.n1; c->last_ref = ref;
    return ISA_OK;
}

// ---- global pre-alignment ---------------------------------------------------
struct ScanResult { double x, y, ang, val; };
struct ArgMax { float v; int i; };

// PreAlignment.ScanAngles (PreAlignment.cs:176-261) of tracking image `img`
// against the reference spectrum in c->spec. Scratch in c->tmp: the rotated
// image (and its inverse transform), its spectrum, the arg-max partials and
// one (value, index) per angle.
int scan_angles(isa_ctx* c, const float* img, int W, int H, double incr, double range, double zero, cudaStream_t st, ScanResult& out)
{
    const size_t fsz = (size_t)W * H, hw = (size_t)(W / 2 + 1);
    float* rot = c->tmp;
    float2* spec = (float2*)(c->tmp + fsz);
    char* scratch = (char*)(c->tmp + fsz + (W + 2) * (size_t)H);
    scratch = (char*)(((uintptr_t)scratch + 255) & ~(uintptr_t)255);
    ArgMax* res = (ArgMax*)(scratch + isa_argmax_scratch_bytes());
    constexpr int kMaxAngles = 256;
    const float N = (float)W * (float)H;
    double maxVal = -DBL_MAX, maxAng = 0, maxX = 0, maxY = 0;
    ISA_TRY(ensure_fft(c, W, H, st));
    const size_t sp = hw * sizeof(float2);
    const isa_fft_filter none{};
    for (int phase = 0; phase < 2; phase++) {
        // the reference's loops, in the same double arithmetic
        std::vector<double> angles;
        const double step = phase == 0 ? 5 * incr : incr;
        for (double ang = zero - range; ang <= zero + range; ang += step) {
            angles.push_back(ang);
            if ((int)angles.size() > kMaxAngles) return fail(ISA_EINVAL, "more than %d rotation angles per scan", kMaxAngles);
        }
        for (size_t k = 0; k < angles.size(); k++) {
            ISA_LAUNCH(c, isa_launch_rotate_cubic(img, (size_t)W * 4, W, H, angles[k], rot, (size_t)W * 4, st));
            // R2C, conjugateComplexMulKernel against the reference spectrum, C2R (one column pass does the middle three)
            ISA_LAUNCH(c, isa_launch_fft_rows_r2c(rot, (size_t)W * 4, spec, sp, W, H, c->fft_rows, c->tw_rows, c->tw_unpack, st));
            ISA_LAUNCH(c, isa_launch_fft_cols(spec, sp, W, H, (int)hw, c->fft_cols, c->tw_cols, ISA_FFT_COLS_XCORR, none, c->spec, sp, st));
            ISA_LAUNCH(c, isa_launch_fft_rows_c2r(spec, sp, rot, (size_t)W * 4, W, H, c->fft_rows, c->tw_rows, c->tw_unpack, 0, W, 1.0f, st));
            ISA_LAUNCH(c, isa_launch_argmax(rot, (int)fsz, scratch, res + k, st));
        }
        std::vector<ArgMax> h(angles.size());
        ISA_CK(cudaMemcpyAsync(h.data(), res, h.size() * sizeof(ArgMax), cudaMemcpyDeviceToHost, st));
        ISA_CK(cudaStreamSynchronize(st));
        for (size_t k = 0; k < angles.size(); k++) {
            const float v = h[k].v / N;  // the reference divides the correlation by W * H before MaxIndex
            if (v > maxVal) {
                maxVal = v;
                maxAng = angles[k];
                maxX = h[k].i % W;
                maxY = h[k].i / W;
            }
        }
        zero = maxAng;
        range = 10 * incr;
    }
    if (maxX > W / 2) maxX -= W;
    if (maxY > H / 2) maxY -= H;
    out = ScanResult{-maxX, -maxY, maxAng, maxVal};
    return ISA_OK;
}

// PreAlignmentStore (PreAlignmentStore.cs:36-110): consecutive differences of
// the per-frame results, the reference index that minimises the remaining
// total shift, and every frame's shift and rotation relative to it.
int prealign_store(const std::vector<ScanResult>& init, float* shifts, float* rots, int* reference)
{
    const int n = (int)init.size();
    std::vector<ScanResult> basic(n, ScanResult{0, 0, 0, 0});
    for (int i = 1; i < n; i++)
        basic[i - 1] = ScanResult{init[i].x - init[i - 1].x, init[i].y - init[i - 1].y, init[i].ang - init[i - 1].ang, 0};
    int minIndex = -1;
    double minShift = DBL_MAX;
    for (int i = 0; i < n - 1; i++) {
        double ax = 0, ay = 0, bx = 0, by = 0;
        for (int j = 0; j < i; j++) { ax -= basic[j].x; ay -= basic[j].y; }
        for (int j = i; j < n - 1; j++) { bx += basic[j].x; by += basic[j].y; }
        const double sx = ax + bx, sy = ay + by;
        const double d = std::sqrt(sx * sx + sy * sy);
        if (d < minShift) { minShift = d; minIndex = i; }
    }
    for (int i = 0; i < n; i++) {
        double ax = 0, ay = 0, az = 0;
        for (int j = i; j < minIndex; j++) { ax -= basic[j].x; ay -= basic[j].y; az -= basic[j].ang; }
        for (int j = minIndex; j < i; j++) { ax += basic[j].x; ay += basic[j].y; az += basic[j].ang; }
        shifts[2 * i] = (float)ax;
        shifts[2 * i + 1] = (float)ay;
        rots[i] = (float)az;
    }
    *reference = minIndex;
    return ISA_OK;
}

}  // namespace

// ===========================================================================
extern "C" {

const char* isa_last_error(void) { return g_err.c_str(); }
const char* isa_version(void) { return "isa-b200 0.1 (sm_100a)"; }

void isa_params_default(isa_params* p)
{
    if (!p) return;
    std::memset(p, 0, sizeof *p);
    p->sigma_debayer_tracking = 0.5f;
    p->sigma_debayer_accumulation = 0.5f;
    p->high_pass = 0.01f;
    p->high_pass_sigma = 0.0025f;
    p->clear_axis = 0;
    p->matching_threshold = 1.0f;
    p->sigma_structure_tensor = 1.0f;
    p->dth = 0.001f;
    p->dtr = 0.006f;
    p->k_detail = 0.25f;
    p->k_denoise = 3.0f;
    p->k_stretch = 4.0f;
    p->k_shrink = 2.0f;
    p->iterations_lk = 3;
    p->window_size_lk = 11;
    p->erode_size = 5;
    p->min_det_lk = 0.01f;
    p->threshold_m = 100000.0f;
    p->tracking_strategy = ISA_TRACK_FULL;
    p->tracking_block_size = 5;
    p->green_channel_only = 0;
    p->level_count = 4;
    p->levels[0] = {1, 32, 2};
    for (int i = 1; i < 4; i++) p->levels[i] = {p->levels[i - 1].resize_level * 2, 32, 4};
    p->super_resolution = 0;
    p->merge_scale = 0.f;
    p->robust_s = 1.5f;
    p->robust_t = 0.12f;
    p->fused_accumulate = 1;
    p->sample_mode = ISA_SAMPLE_ROUND;
}

int isa_output_size(const isa_params* p, int width, int height, int* ow, int* oh)
{
    if (!p || !ow || !oh) return fail(ISA_EINVAL, "NULL argument");
    isa_accum_geom g;
    float thr;
    accum_geom(p, width, height, g, thr);
    *ow = g.Wo;
    *oh = g.Ho;
    return ISA_OK;
}

int isa_ctx_create(isa_ctx** out, int max_w, int max_h, int max_n, const isa_params* p)
{
    if (!out) return fail(ISA_EINVAL, "ctx out pointer is NULL");
    *out = nullptr;
    ISA_TRY(check_params(p));
    if (max_w < 16 || max_h < 16 || (max_w & 1) || (max_h & 1) || max_n < 2 || max_n > 65)
        return fail(ISA_EINVAL, "context size %dx%d x %d frames invalid", max_w, max_h, max_n);
    // the full-frame transforms hold a row (W complex values) and at least one column (2 H) in shared memory
    if ((size_t)max_w * 8 > 227 * 1024 || isa_fft_cols_per_cta(max_h) < 1)
        return fail(ISA_EINVAL, "context size %dx%d exceeds the full-frame transform's limit (W <= 29056, H <= 12800)", max_w, max_h);
    isa_ctx* c = new isa_ctx();
    if (cudaGetDevice(&c->device) != cudaSuccess) { cudaGetLastError(); delete c; return fail(ISA_ECUDA, "cudaGetDevice failed"); }
    c->max_w = max_w; c->max_h = max_h; c->max_n = max_n; c->p = *p;
    // worst case pairs over strategies for max_n frames
    c->max_rows = 0;
    for (int n = 2; n <= max_n; n++) {
        int bn = p->tracking_block_size >= n ? n - 1 : p->tracking_block_size;
        c->max_rows = std::max(c->max_rows, shift_count(n, p->tracking_strategy, bn));
    }
    c->max_pairs = c->max_rows;
    for (int i = 0; i < p->level_count; i++) {
        int tcx, tcy;
        if (level_tiles(p->levels[i], max_w, max_h, &tcx, &tcy) != ISA_OK) { delete c; return fail(ISA_EINVAL, "level %d has no tiles", i); }
        c->maxcx = std::max(c->maxcx, tcx);
        c->maxcy = std::max(c->maxcy, tcy);
    }
    c->max_tiles = c->maxcx * c->maxcy;
    isa_accum_geom g;
    float thr;
    accum_geom(p, max_w, max_h, g, thr);
    c->max_wo = g.Wo; c->max_ho = g.Ho;
    // carve one arena
    const size_t A = 256, fsz = (size_t)max_w * max_h;
    std::vector<std::pair<void**, size_t>> plan;
    auto add = [&](void** ptr, size_t bytes) { plan.push_back({ptr, align_up(std::max<size_t>(bytes, 1), A)}); };
    add((void**)&c->raw_stage, fsz * max_n * 2);
    add((void**)&c->bw_track, fsz * max_n * 4);
    add((void**)&c->bw_acc, fsz * max_n * 4);
    add((void**)&c->tmp, fsz * 3 * 4);
    for (int i = 0; i < p->level_count; i++) {
        int L = p->levels[i].resize_level;
        if (L > 1) add((void**)&c->pyr[i], (size_t)(max_w / L) * (max_h / L) * max_n * 4);
    }
    add((void**)&c->spec, (size_t)(max_w / 2 + 1) * max_h * 8);
    size_t gbytes = (size_t)c->maxcx * c->maxcy * sizeof(float2) * c->max_rows;
    add((void**)&c->grids, gbytes);
    add((void**)&c->grids_tmp, gbytes);
    add((void**)&c->x, (size_t)c->max_tiles * (max_n - 1) * sizeof(float2));
    add((void**)&c->tiles_opt, (size_t)c->max_tiles * sizeof(float2));
    add((void**)&c->status, (size_t)c->max_tiles * sizeof(int));
    add((void**)&c->row_a, c->max_rows * sizeof(int));
    add((void**)&c->row_b, c->max_rows * sizeof(int));
    add((void**)&c->row_sign, c->max_rows * sizeof(int));
    add((void**)&c->row_grid, c->max_rows * sizeof(int));
    add((void**)&c->N0, (size_t)(max_n - 1) * (max_n - 1) * sizeof(double));
    add((void**)&c->pair_desc, (size_t)c->max_pairs * ISA_MAX_LEVELS * sizeof(isa_pair_desc));
    add((void**)&c->frame_tab, (size_t)max_n * ISA_MAX_LEVELS * sizeof(float*));
    add((void**)&c->flows, fsz * max_n * sizeof(float2));
    add((void**)&c->flow_tmp, fsz * sizeof(float2));
    add((void**)&c->half_ref, fsz / 4 * 12);
    add((void**)&c->half_mov, fsz / 4 * 12);
    add((void**)&c->ref_mr, fsz / 4 * 16);
    add((void**)&c->ref_sr, fsz / 4 * 16);
    add((void**)&c->mov_box, fsz / 4 * 16);
    add((void**)&c->masks, fsz / 4 * 16 * max_n);
    add((void**)&c->st3, fsz * 12);
    add((void**)&c->kparam, fsz * 16);
    add((void**)&c->acc, (size_t)c->max_wo * c->max_ho * 12);
    add((void**)&c->wsum, (size_t)c->max_wo * c->max_ho * 12);
    add((void**)&c->out_stage, (size_t)c->max_wo * c->max_ho * 12);
    add((void**)&c->frame_in, (size_t)max_n * sizeof(isa_frame_in));
    add((void**)&c->adj_acc, 16 * sizeof(double));
    add((void**)&c->tw_rows, (size_t)(max_w / 2) * sizeof(float2));
    add((void**)&c->tw_unpack, (size_t)(max_w / 2 + 1) * sizeof(float2));
    add((void**)&c->tw_cols, (size_t)max_h * sizeof(float2));
    if (p->sample_mode == ISA_SAMPLE_BILINEAR) add((void**)&c->adj_flow, fsz * kAdjFlowFloats * sizeof(float));
    size_t total = 0;
    for (auto& e : plan) total += e.second;
    if (cudaMalloc(&c->arena, total) != cudaSuccess) {
        cudaGetLastError();
        delete c;
        return fail(ISA_ENOMEM, "device arena of %.2f GB", total / 1e9);
    }
    c->arena_bytes = total;
    size_t off = 0;
    for (auto& e : plan) { *e.first = (char*)c->arena + off; off += e.second; }
    for (int i = 0; i < 8; i++)
        if (cudaEventCreate(&c->ev[i]) != cudaSuccess) { isa_ctx_destroy(c); return fail(ISA_ECUDA, "cudaEventCreate failed"); }
    bool ok = cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking) == cudaSuccess;
    c->ev_frame.assign(max_n, nullptr);
    for (int i = 0; i < max_n && ok; i++) ok = cudaEventCreateWithFlags(&c->ev_frame[i], cudaEventDisableTiming) == cudaSuccess;
    for (int i = 0; i < isa_ctx::kBands && ok; i++) ok = cudaEventCreateWithFlags(&c->ev_band[i], cudaEventDisableTiming) == cudaSuccess;
    ok = ok && cudaEventCreateWithFlags(&c->ev_free, cudaEventDisableTiming) == cudaSuccess;
    ok = ok && cudaEventCreateWithFlags(&c->ev_copied, cudaEventDisableTiming) == cudaSuccess;
    if (!ok) { isa_ctx_destroy(c); return fail(ISA_ECUDA, "stream/event creation failed"); }
    int r = ISA_OK;
    // the static solve's set-up on this device (loads the solver's device code), so that it allocates nothing later
    r = isa_static_solve_setup();
    if (r != ISA_OK) { isa_ctx_destroy(c); return r; }
    *out = c;
    return ISA_OK;
}

int isa_ctx_destroy(isa_ctx* c)
{
    if (!c) return ISA_OK;
    for (int i = 0; i < 8; i++)
        if (c->ev[i]) cudaEventDestroy(c->ev[i]);
    for (cudaEvent_t e : c->ev_frame)
        if (e) cudaEventDestroy(e);
    for (int i = 0; i < isa_ctx::kBands; i++)
        if (c->ev_band[i]) cudaEventDestroy(c->ev_band[i]);
    if (c->ev_free) cudaEventDestroy(c->ev_free);
    if (c->ev_copied) cudaEventDestroy(c->ev_copied);
    if (c->copy_stream) cudaStreamDestroy(c->copy_stream);
    if (c->arena) cudaFree(c->arena);
    delete c;
    return ISA_OK;
}

int isa_stage_times(isa_ctx* c, float* ms, int max_count)
{
    if (!c || !ms) return fail(ISA_EINVAL, "NULL argument");
    if (c->ev_count < 2) return 0;
    ISA_CK(cudaEventSynchronize(c->ev[c->ev_count - 1]));
    int k = 0;
    for (int i = 1; i < c->ev_count && k < max_count; i++, k++) ISA_CK(cudaEventElapsedTime(&ms[k], c->ev[i - 1], c->ev[i]));
    return k;
}

long isa_launch_count(isa_ctx* c) { return c ? c->launches : -1; }

int isa_merge_burst(isa_ctx* c, const uint16_t* raw, size_t raw_pitch, size_t frame_stride, int n, const isa_raw_info* info,
                    const isa_prealign* pre, float* out, size_t out_pitch, void* stream)
{
    if (!c) return fail(ISA_EINVAL, "ctx is NULL");
    return run_merge(c, raw, raw_pitch, frame_stride, n, info, pre, out, out_pitch, S(stream));
}

namespace {

// Forward merge, then the adjoint of the weighted L2 loss: the eight parameter gradients, and with tile_grad (sample
// mode BILINEAR) the gradient of every frame's tile flow.
int merge_backward(isa_ctx* c, const uint16_t* raw, size_t raw_pitch, size_t frame_stride, int n, const isa_raw_info* info,
                   const isa_prealign* pre, const float* target, size_t target_pitch, const float* weight, size_t weight_pitch, float* out,
                   size_t out_pitch, double* loss, double* grad, float* tile_grad, cudaStream_t st)
{
    if (!c || !raw || !target || !out || !loss || !grad) return fail(ISA_EINVAL, "NULL argument");
    ISA_TRY(check_info(info));
    const isa_params* p = &c->p;
    const int W = info->width, H = info->height;
    isa_accum_geom g;
    float thr;
    accum_geom(p, W, H, g, thr);
    if (thr != 0.f) return fail(ISA_EINVAL, "the adjoint covers the merge_scale and super-resolution modes (normalisation threshold 0)");
    if (!p->fused_accumulate) return fail(ISA_EINVAL, "the adjoint needs fused_accumulate");
    if (target_pitch < (size_t)g.Wo * 12) return fail(ISA_EINVAL, "target pitch %zu < %d", target_pitch, g.Wo * 12);
    if (weight && weight_pitch < (size_t)g.Wo * 4) return fail(ISA_EINVAL, "weight pitch %zu < %d", weight_pitch, g.Wo * 4);
    if (tile_grad) {
        if (p->sample_mode != ISA_SAMPLE_BILINEAR || !c->adj_flow)
            return fail(ISA_EINVAL, "the tile-flow gradient needs a context created with sample_mode ISA_SAMPLE_BILINEAR");
        if (p->iterations_lk > 3) return fail(ISA_EINVAL, "the tile-flow gradient covers up to 3 LK iterations (%d)", p->iterations_lk);
        if (((uintptr_t)tile_grad & 7) != 0) return fail(ISA_EINVAL, "tile_grad must be 8-byte aligned");
    }
    // forward (keeps flows, masks, kernel parameters, structure tensor, sums and the frame table)
    ISA_TRY(run_merge(c, raw, raw_pitch, frame_stride, n, info, pre, out, out_pitch, st));
    const size_t fsz = (size_t)W * H;
    const int Wh = W / 2, Hh = H / 2;
    const size_t hsz = (size_t)Wh * Hh, hp4 = (size_t)Wh * 16, hp3 = (size_t)Wh * 12, fp = (size_t)W * sizeof(float2), p3 = (size_t)W * 12,
                 p4 = (size_t)W * 16, op = (size_t)g.Wo * 12;
    // scratch of the adjoint in buffers the forward has finished with: the FFT / Gauss scratch (fsz x 12 B) takes the
    // kernel-parameter gradients, the tracking images (n x fsz x 4 B) the mask-certainty gradients of every frame, the
    // LK ping-pong flow (fsz x 8 B) the recomputed mask and its auxiliaries, the accumulation images (or, for the
    // tile-flow gradient, whose LK recomputation reads them, the flow adjoint's scratch) the routed gradient; none of
    // them is read again before the next merge
    float* adj_gkp = c->tmp;
    float4* adj_gmask = (float4*)c->bw_track;
    float4* adj_m = (float4*)c->flow_tmp;
    float4* adj_aux = (float4*)((char*)c->flow_tmp + hsz * 16);
    // flow adjoint scratch (floats per frame pixel, kAdjFlowFloats in all)
    float* sc = c->adj_flow;
    float2* F[3] = {(float2*)sc, (float2*)(sc + 2 * fsz), (float2*)(sc + 4 * fsz)};
    float* wplane = sc + 6 * fsz;
    float* a5 = sc + 7 * fsz;
    float* A5 = sc + 12 * fsz;
    float* gd3 = sc + 17 * fsz;
    float2* gA = (float2*)(sc + 20 * fsz);
    float2* gB = (float2*)(sc + 22 * fsz);
    float4* adj_gm = tile_grad ? (float4*)(sc + 24 * fsz) : (float4*)c->bw_acc;
    ISA_CK(cudaMemsetAsync(adj_gkp, 0, fsz * 12, st));
    ISA_CK(cudaMemsetAsync(adj_gmask, 0, hsz * 16 * n, st));
    ISA_CK(cudaMemsetAsync(c->adj_acc, 0, 16 * sizeof(double), st));
    float black[3], white[3], scale[3], divisor[3];
    color_consts(info, black, white, scale, divisor);
    const unsigned cfa = pack_cfa(info->cfa);
    const int ref = pre ? pre->reference : 0;
    const int tcx0 = c->last_tcx0, tcy0 = c->last_tcy0;
    const size_t tsz = (size_t)tcx0 * tcy0;
    // output -> kernel parameters and mask certainties; with the tile-flow gradient frame by frame (below), each
    // launch adding its flow gradient to gA, the reference frame's here with the loss
    ISA_LAUNCH(c, isa_launch_accumulate_bwd(g, cfa, c->frame_in, tile_grad ? 1 : n, raw_pitch, fp, hp4, c->kparam, p4, white, black, out, out_pitch,
                                            c->wsum, op, target, target_pitch, weight, weight_pitch, adj_gkp, adj_gmask, hsz, c->adj_acc + 8, nullptr,
                                            st));
    if (tile_grad) ISA_CK(cudaMemsetAsync(tile_grad + 2 * ref * tsz, 0, tsz * sizeof(float2), st));
    // mask certainties -> erosion -> robustness s, t (per frame, recomputing the un-eroded mask); with the tile-flow
    // gradient also the flow: accumulation and mask -> final flow -> LK iterations (recomputed) -> tile flow
    float maxv = 0.f;
    for (int ch = 0; ch < 3; ch++) maxv = std::max(maxv, white[ch] + black[ch]);
    const int half = p->window_size_lk / 2;
    const int bil = p->sample_mode == ISA_SAMPLE_BILINEAR;
    int f = 1;
    for (int i = 0; i < n; i++) {
        if (i == ref) continue;
        const uint16_t* fr = (const uint16_t*)((const char*)raw + (size_t)i * frame_stride);
        const float2* flow = c->flows + (size_t)i * fsz;
        if (tile_grad) {
            ISA_CK(cudaMemsetAsync(gA, 0, fsz * sizeof(float2), st));
            ISA_LAUNCH(c, isa_launch_accumulate_bwd(g, cfa, c->frame_in + f, 1, raw_pitch, fp, hp4, c->kparam, p4, white, black, out, out_pitch, c->wsum,
                                                    op, target, target_pitch, weight, weight_pitch, adj_gkp, adj_gmask + (size_t)f * hsz, hsz, nullptr,
                                                    gA, st));
        }
        ISA_LAUNCH(c, isa_launch_subsample(fr, raw_pitch, W, H, cfa, maxv, c->half_mov, hp3, st));
        ISA_LAUNCH(c, isa_launch_box3(c->half_mov, hp3, Wh, Hh, c->mov_box, hp4, st));
        ISA_LAUNCH(c, isa_launch_mask_store(c->ref_mr, c->ref_sr, c->mov_box, hp4, c->half_mov, hp3, Wh, Hh, flow, fp, W, H, info->noise_alpha,
                                            info->noise_beta, p->threshold_m, p->robust_s, p->robust_t, adj_m, adj_aux, bil, st));
        ISA_CK(cudaMemsetAsync(adj_gm, 0, hsz * 16, st));
        ISA_LAUNCH(c, isa_launch_erode_route(adj_m, adj_gmask + (size_t)f * hsz, hp4, Wh, Hh, p->erode_size, adj_gm, st));
        ISA_LAUNCH(c, isa_launch_mask_param_bwd(adj_m, adj_aux, adj_gm, hp4, Wh, Hh, p->robust_t, c->adj_acc + 6, st));
        if (tile_grad) {
            ISA_LAUNCH(c, isa_launch_mask_flow_bwd(c->ref_mr, c->ref_sr, c->mov_box, hp4, c->half_mov, hp3, Wh, Hh, flow, fp, W, H, info->noise_alpha,
                                                   info->noise_beta, p->robust_t, adj_aux, adj_gm, gA, st));
            // the flows before each LK iteration, as the forward made them
            const float2* tiles = c->tiles_opt;
            if (c->tile_override)
                tiles = c->tile_override + (size_t)i * tsz;
            else
                ISA_LAUNCH(c, isa_launch_optimal(c->x, c->last_n1, tcx0, tcy0, ref, i, c->tiles_opt, (size_t)tcx0 * sizeof(float2), st));
            float bs[2];
            prealign_shift(pre, ref, i, bs);
            const int K = p->iterations_lk;
            if (K > 0)
                ISA_LAUNCH(c, isa_launch_flow_from_tiles(tiles, (size_t)tcx0 * sizeof(float2), tcx0, tcy0, W, H, bs[0], bs[1],
                                                         prealign_rot(pre, ref, i), F[0], fp, st));
            for (int k = 1; k < K; k++)
                ISA_LAUNCH(c, isa_launch_lk_iteration(F[k - 1], F[k], fp, c->bw_acc + i * fsz, c->bw_acc + ref * fsz, bw_pitch(W), W, H, half,
                                                      p->min_det_lk, st));
            float2* gcur = gA;
            float2* gnext = gB;
            for (int k = K - 1; k >= 0; k--) {
                ISA_LAUNCH(c, isa_launch_lk_adjoint(F[k], gcur, gnext, fp, c->bw_acc + i * fsz, c->bw_acc + ref * fsz, bw_pitch(W), W, H, half,
                                                    p->min_det_lk, wplane, a5, A5, gd3, st));
                std::swap(gcur, gnext);
            }
            ISA_LAUNCH(c, isa_launch_tiles_bwd(gcur, fp, W, H, tcx0, tcy0, (float2*)tile_grad + (size_t)i * tsz, (size_t)tcx0 * sizeof(float2), st));
        }
        f++;
    }
    // kernel parameters -> kDetail, kDenoise, Dth, Dtr, kStretch, kShrink (after every frame's accumulation adjoint)
    ISA_LAUNCH(c, isa_launch_kparam_bwd(c->st3, p3, W, H, adj_gkp, p->dth, p->dtr, p->k_detail, p->k_denoise, p->k_stretch, p->k_shrink,
                                        c->adj_acc, st));
    double h[9];
    ISA_CK(cudaMemcpyAsync(h, c->adj_acc, sizeof(h), cudaMemcpyDeviceToHost, st));
    ISA_CK(cudaStreamSynchronize(st));
    *loss = h[8];
    for (int k = 0; k < 8; k++) grad[k] = h[k];
    return ISA_OK;
}

}  // namespace

int isa_merge_backward(isa_ctx* c, const uint16_t* raw, size_t raw_pitch, size_t frame_stride, int n, const isa_raw_info* info,
                       const isa_prealign* pre, const float* target, size_t target_pitch, const float* weight, size_t weight_pitch, float* out,
                       size_t out_pitch, double* loss, double* grad, void* stream)
{
    return merge_backward(c, raw, raw_pitch, frame_stride, n, info, pre, target, target_pitch, weight, weight_pitch, out, out_pitch, loss, grad,
                          nullptr, S(stream));
}

int isa_merge_backward_tiles(isa_ctx* c, const uint16_t* raw, size_t raw_pitch, size_t frame_stride, int n, const isa_raw_info* info,
                             const isa_prealign* pre, const float* target, size_t target_pitch, const float* weight, size_t weight_pitch,
                             float* out, size_t out_pitch, double* loss, double* grad, float* tile_grad, void* stream)
{
    if (!tile_grad) return fail(ISA_EINVAL, "tile_grad is NULL");
    return merge_backward(c, raw, raw_pitch, frame_stride, n, info, pre, target, target_pitch, weight, weight_pitch, out, out_pitch, loss, grad,
                          tile_grad, S(stream));
}

int isa_batch_plan(const double* work, const int* burst_device, int nbursts, const int* ctx_device, int nctx, int* assignment)
{
    if (nbursts < 0 || nctx < 1 || !ctx_device || (nbursts > 0 && (!work || !burst_device || !assignment))) return fail(ISA_EINVAL, "bad plan arguments");
    std::vector<double> load(nctx, 0.0);
    int unassigned = 0;
    for (int b = 0; b < nbursts; b++) {
        int k = -1;
        for (int i = 0; i < nctx; i++)
            if ((burst_device[b] < 0 || ctx_device[i] == burst_device[b]) && (k < 0 || load[i] < load[k])) k = i;
        assignment[b] = k;
        if (k < 0)
            unassigned++;
        else
            load[k] += work[b] > 0 ? work[b] : 0.0;
    }
    return unassigned;
}

namespace {

// Device of a device pointer (-1: managed memory, which every device reaches); ISA_EINVAL for host memory.
int pointer_device(const void* ptr, int* dev)
{
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, ptr) != cudaSuccess) {
        cudaGetLastError();
        return fail(ISA_EINVAL, "not a CUDA pointer");
    }
    if (a.type == cudaMemoryTypeManaged) { *dev = -1; return ISA_OK; }
    if (a.type != cudaMemoryTypeDevice) return fail(ISA_EINVAL, "burst frames and outputs must be device memory");
    *dev = a.device;
    return ISA_OK;
}

}  // namespace

int isa_merge_batch(isa_ctx* const* ctxs, void* const* streams, int nctx, const isa_burst* bursts, int nbursts, int* status)
{
    if (!ctxs || nctx < 1 || (!bursts && nbursts > 0) || nbursts < 0) return fail(ISA_EINVAL, "bad batch arguments");
    for (int i = 0; i < nctx; i++)
        if (!ctxs[i]) return fail(ISA_EINVAL, "context %d is NULL", i);
    int caller_dev = 0;
    ISA_CK(cudaGetDevice(&caller_dev));
    // the plan: each burst to the least-loaded context on the device of its frames
    std::vector<double> work(nbursts, 0.0);
    std::vector<int> bdev(nbursts, -1), cdev(nctx), assign(nbursts, -1), pre_rc(nbursts, ISA_OK);
    for (int i = 0; i < nctx; i++) cdev[i] = ctxs[i]->device;
    for (int b = 0; b < nbursts; b++) {
        const isa_burst& u = bursts[b];
        if (!u.info || !u.raw || !u.out) { pre_rc[b] = fail(ISA_EINVAL, "burst %d: NULL argument", b); continue; }
        int od = -1;
        if (pointer_device(u.raw, &bdev[b]) != ISA_OK || pointer_device(u.out, &od) != ISA_OK) { pre_rc[b] = ISA_EINVAL; continue; }
        if (od >= 0 && bdev[b] >= 0 && od != bdev[b]) { pre_rc[b] = fail(ISA_EINVAL, "burst %d: frames and output on different devices", b); continue; }
        if (bdev[b] < 0) bdev[b] = od;
        work[b] = (double)u.info->width * u.info->height * u.n;
    }
    isa_batch_plan(work.data(), bdev.data(), nbursts, cdev.data(), nctx, assign.data());
    int first = ISA_OK;
    for (int b = 0; b < nbursts; b++) {
        const isa_burst& u = bursts[b];
        int rc = pre_rc[b];
        if (rc == ISA_OK && assign[b] < 0) rc = fail(ISA_EINVAL, "burst %d: no context on device %d", b, bdev[b]);
        if (rc == ISA_OK) {
            const int k = assign[b];
            isa_ctx* c = ctxs[k];
            const isa_params saved = c->p;
            if (u.params) {
                const isa_params& q = *u.params;
                rc = check_params(&q);
                bool same = rc == ISA_OK && q.level_count == saved.level_count && q.tracking_strategy == saved.tracking_strategy &&
                            q.tracking_block_size == saved.tracking_block_size;
                for (int l = 0; same && l < q.level_count; l++)
                    same = q.levels[l].resize_level == saved.levels[l].resize_level && q.levels[l].tile_size == saved.levels[l].tile_size &&
                           q.levels[l].max_shift == saved.levels[l].max_shift;
                if (rc == ISA_OK && !same) rc = fail(ISA_EINVAL, "burst %d: params change the pyramid levels or the tracking strategy", b);
                if (rc == ISA_OK) c->p = q;
            }
            if (rc == ISA_OK && cudaSetDevice(c->device) != cudaSuccess) {
                cudaGetLastError();
                rc = fail(ISA_ECUDA, "cudaSetDevice(%d) failed", c->device);
            }
            if (rc == ISA_OK) rc = run_merge(c, u.raw, u.raw_pitch, u.frame_stride, u.n, u.info, u.pre, u.out, u.out_pitch, S(streams ? streams[k] : nullptr));
            c->p = saved;
        }
        if (status) status[b] = rc;
        if (rc != ISA_OK && first == ISA_OK) first = rc;
    }
    cudaSetDevice(caller_dev);
    return first;
}

struct isa_batch_graph {
    int device = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    void* pinned = nullptr;  // the staged tables the graph's copy nodes read
    std::vector<isa_ctx*> ctxs;
};

int isa_batch_graph_destroy(isa_batch_graph* gr)
{
    if (!gr) return ISA_OK;
    if (gr->exec) cudaGraphExecDestroy(gr->exec);
    if (gr->graph) cudaGraphDestroy(gr->graph);
    if (gr->pinned) cudaFreeHost(gr->pinned);
    delete gr;
    return ISA_OK;
}

int isa_batch_graph_create(isa_ctx* const* ctxs, void* const* streams, int nctx, const isa_burst* bursts, int nbursts, void* origin,
                           isa_batch_graph** out)
{
    if (!out) return fail(ISA_EINVAL, "graph out pointer is NULL");
    *out = nullptr;
    if (!ctxs || !streams || nctx < 1 || !bursts || nbursts < 1 || !origin) return fail(ISA_EINVAL, "bad graph arguments");
    int dev = 0;
    ISA_CK(cudaGetDevice(&dev));
    for (int i = 0; i < nctx; i++) {
        if (!ctxs[i] || !streams[i]) return fail(ISA_EINVAL, "context or stream %d is NULL", i);
        if (ctxs[i]->device != dev) return fail(ISA_EINVAL, "context %d is on device %d, not the current device %d", i, ctxs[i]->device, dev);
        if (streams[i] == origin) return fail(ISA_EINVAL, "stream %d is the origin stream", i);
        for (int j = 0; j < i; j++)
            if (streams[j] == streams[i]) return fail(ISA_EINVAL, "streams %d and %d are the same", j, i);
    }
    // the pinned arena: per burst at most the tables of its context's maxima (twiddles, solver rows, N0, per level the
    // pair and frame tables, the frame table of the accumulation), with 16-byte alignment slack per copy
    size_t per = 0;
    for (int i = 0; i < nctx; i++) {
        const isa_ctx* c = ctxs[i];
        size_t b = ((size_t)c->max_w / 2 + (size_t)c->max_w / 2 + 1 + (size_t)c->max_h) * sizeof(float2);
        b += (size_t)c->max_rows * 4 * sizeof(int) + (size_t)(c->max_n - 1) * (c->max_n - 1) * sizeof(double);
        b += (size_t)ISA_MAX_LEVELS * ((size_t)c->max_pairs * sizeof(isa_pair_desc) + (size_t)c->max_n * sizeof(float*));
        b += (size_t)c->max_n * sizeof(isa_frame_in) + 32 * 16;
        per = std::max(per, b);
    }
    isa_batch_graph* gr = new isa_batch_graph();
    gr->device = dev;
    gr->ctxs.assign(ctxs, ctxs + nctx);
    HostStage stage;
    stage.cap = per * (size_t)nbursts;
    if (cudaHostAlloc(&gr->pinned, stage.cap, cudaHostAllocDefault) != cudaSuccess) {
        cudaGetLastError();
        delete gr;
        return fail(ISA_ENOMEM, "pinned staging of %zu bytes", stage.cap);
    }
    stage.base = (char*)gr->pinned;
    cudaEvent_t fork = nullptr;
    std::vector<cudaEvent_t> join(nctx, nullptr);
    bool ok = cudaEventCreateWithFlags(&fork, cudaEventDisableTiming) == cudaSuccess;
    for (int i = 0; i < nctx && ok; i++) ok = cudaEventCreateWithFlags(&join[i], cudaEventDisableTiming) == cudaSuccess;
    int rc = ok ? ISA_OK : fail(ISA_ECUDA, "event creation failed");
    cudaStream_t os = (cudaStream_t)origin;
    bool capturing = false;
    if (rc == ISA_OK) {
        if (cudaStreamBeginCapture(os, cudaStreamCaptureModeRelaxed) != cudaSuccess)
            rc = fail(ISA_ECUDA, "cudaStreamBeginCapture failed");
        else
            capturing = true;
    }
    if (rc == ISA_OK && cudaEventRecord(fork, os) != cudaSuccess) rc = fail(ISA_ECUDA, "fork record failed");
    for (int i = 0; i < nctx && rc == ISA_OK; i++)
        if (cudaStreamWaitEvent((cudaStream_t)streams[i], fork, 0) != cudaSuccess) rc = fail(ISA_ECUDA, "fork wait failed");
    std::vector<int> status(nbursts, ISA_OK);
    if (rc == ISA_OK) {
        g_stage = &stage;
        for (int i = 0; i < nctx; i++) ctxs[i]->capturing = true;
        rc = isa_merge_batch(ctxs, streams, nctx, bursts, nbursts, status.data());
        for (int i = 0; i < nctx; i++) ctxs[i]->capturing = false;
        g_stage = nullptr;
    }
    for (int i = 0; i < nctx && capturing; i++) {
        if (cudaEventRecord(join[i], (cudaStream_t)streams[i]) != cudaSuccess || cudaStreamWaitEvent(os, join[i], 0) != cudaSuccess)
            if (rc == ISA_OK) rc = fail(ISA_ECUDA, "join failed");
    }
    // the capture ran the host side of every merge but none of its copies: the contexts' transform tables are
    // whatever they were before, so the size they record is forgotten and the next merge uploads its own
    // (and the last merge the debug entry points describe did not run)
    for (int i = 0; i < nctx; i++) {
        ctxs[i]->fft_w = ctxs[i]->fft_h = 0;
        ctxs[i]->last_n = 0;
    }
    if (capturing) {
        cudaGraph_t graph = nullptr;
        const cudaError_t e = cudaStreamEndCapture(os, &graph);
        gr->graph = graph;
        if (e != cudaSuccess && rc == ISA_OK) rc = fail(ISA_ECUDA, "stream capture failed: %s", cudaGetErrorString(e));
    }
    if (rc == ISA_OK && cudaGraphInstantiate(&gr->exec, gr->graph, 0) != cudaSuccess) rc = fail(ISA_ECUDA, "cudaGraphInstantiate failed");
    if (fork) cudaEventDestroy(fork);
    for (cudaEvent_t e : join)
        if (e) cudaEventDestroy(e);
    if (rc != ISA_OK) {
        cudaGetLastError();
        isa_batch_graph_destroy(gr);
        return rc;
    }
    *out = gr;
    return ISA_OK;
}

int isa_batch_graph_launch(isa_batch_graph* gr, void* stream)
{
    if (!gr || !gr->exec) return fail(ISA_EINVAL, "graph is NULL");
    int dev = 0;
    ISA_CK(cudaGetDevice(&dev));
    if (dev != gr->device) return fail(ISA_EINVAL, "the graph belongs to device %d, the current device is %d", gr->device, dev);
    ISA_CK(cudaGraphLaunch(gr->exec, S(stream)));
    return ISA_OK;
}

int isa_merge_burst_host(isa_ctx* c, const uint16_t* host_raw, int n, const isa_raw_info* info, const isa_prealign* pre, float* host_out,
                         void* stream)
{
    if (!c || !host_raw || !host_out) return fail(ISA_EINVAL, "NULL argument");
    ISA_TRY(check_info(info));
    const int W = info->width, H = info->height;
    if (W > c->max_w || H > c->max_h || n < 2 || n > c->max_n) return fail(ISA_EINVAL, "burst exceeds the context");
    isa_accum_geom g;
    float thr;
    accum_geom(&c->p, W, H, g, thr);
    cudaStream_t st = S(stream);
    const size_t fb = (size_t)W * H * 2;
    // frames go in on the copy stream, one event each, once earlier work on `st` no longer reads the staging buffers
    ISA_CK(cudaEventRecord(c->ev_free, st));
    ISA_CK(cudaStreamWaitEvent(c->copy_stream, c->ev_free, 0));
    for (int i = 0; i < n; i++) {
        ISA_CK(cudaMemcpyAsync((char*)c->raw_stage + (size_t)i * fb, (const char*)host_raw + (size_t)i * fb, fb, cudaMemcpyHostToDevice,
                               c->copy_stream));
        ISA_CK(cudaEventRecord(c->ev_frame[i], c->copy_stream));
    }
    HostIo hio{true, host_out};
    const int rc = run_merge(c, c->raw_stage, (size_t)W * 2, fb, n, info, pre, c->out_stage, (size_t)g.Wo * 12, st, &hio);
    if (rc != ISA_OK) {
        // leave nothing of this call running on the copy stream past the caller's stream
        cudaEventRecord(c->ev_copied, c->copy_stream);
        cudaStreamWaitEvent(st, c->ev_copied, 0);
    }
    return rc;
}

int isa_debug_buffers(isa_ctx* c, int frame, const void** flow, size_t* flow_pitch, const void** mask, size_t* mask_pitch, const void** kparam,
                      size_t* kparam_pitch, const void** bw_track, const void** bw_acc, size_t* bw_pitch_out, const void** acc,
                      const void** wsum, size_t* acc_pitch)
{
    if (!c || c->last_n == 0) return fail(ISA_EINVAL, "no merge has run on this context");
    if (frame < 0 || frame >= c->last_n) return fail(ISA_EINVAL, "frame %d out of range", frame);
    const int W = c->last_w, H = c->last_h;
    const size_t fsz = (size_t)W * H;
    isa_accum_geom g;
    float thr;
    accum_geom(&c->p, W, H, g, thr);
    if (flow) *flow = c->flows + frame * fsz;
    if (flow_pitch) *flow_pitch = (size_t)W * 8;
    if (mask) *mask = c->masks + (size_t)frame * (W / 2) * (H / 2);
    if (mask_pitch) *mask_pitch = (size_t)(W / 2) * 16;
    if (kparam) *kparam = c->kparam;
    if (kparam_pitch) *kparam_pitch = (size_t)W * 16;
    if (bw_track) *bw_track = c->bw_track + frame * fsz;
    if (bw_acc) *bw_acc = c->bw_acc + frame * fsz;
    if (bw_pitch_out) *bw_pitch_out = (size_t)W * 4;
    if (acc) *acc = c->acc;
    if (wsum) *wsum = c->wsum;
    if (acc_pitch) *acc_pitch = (size_t)g.Wo * 12;
    return ISA_OK;
}

int isa_debug_track_record(isa_ctx* c, int* record, size_t bytes)
{
    if (!c) return fail(ISA_EINVAL, "NULL context");
    if (record && ((uintptr_t)record & 3)) return fail(ISA_EINVAL, "the record must be 4-byte aligned");
    c->track_rec = record;
    c->track_rec_bytes = record ? bytes : 0;
    return ISA_OK;
}

int isa_debug_shifts(isa_ctx* c, const void** one_to_one, int* tx, int* ty)
{
    if (!c || c->last_n == 0) return fail(ISA_EINVAL, "no merge has run on this context");
    if (one_to_one) *one_to_one = c->x;
    if (tx) *tx = c->last_tcx0;
    if (ty) *ty = c->last_tcy0;
    return ISA_OK;
}

int isa_ctx_set_params(isa_ctx* c, const isa_params* q)
{
    if (!c) return fail(ISA_EINVAL, "ctx is NULL");
    ISA_TRY(check_params(q));
    const isa_params& o = c->p;
    bool same = q->level_count == o.level_count && q->tracking_strategy == o.tracking_strategy && q->tracking_block_size == o.tracking_block_size;
    for (int l = 0; same && l < q->level_count; l++)
        same = q->levels[l].resize_level == o.levels[l].resize_level && q->levels[l].tile_size == o.levels[l].tile_size &&
               q->levels[l].max_shift == o.levels[l].max_shift;
    if (!same) return fail(ISA_EINVAL, "the parameters change the pyramid levels or the tracking strategy of the context");
    isa_accum_geom g;
    float thr;
    accum_geom(q, c->max_w, c->max_h, g, thr);
    if (g.Wo > c->max_wo || g.Ho > c->max_ho) return fail(ISA_EINVAL, "output %dx%d exceeds the context's %dx%d", g.Wo, g.Ho, c->max_wo, c->max_ho);
    c->p = *q;
    return ISA_OK;
}

int isa_ctx_set_tuning(isa_ctx* c, const isa_tuning* e, int count)
{
    if (!c || count < 0 || (count > 0 && !e)) return fail(ISA_EINVAL, "bad tuning arguments");
    for (int i = 0; i < count; i++) {
        const isa_tuning& t = e[i];
        if (t.lk_strip_rows < 0 || t.lk_strip_rows > 4096) return fail(ISA_EINVAL, "tuning %d: lk_strip_rows %d", i, t.lk_strip_rows);
        const bool block0 = t.acc_block_x == 0 && t.acc_block_y == 0;
        if (!block0 && (t.acc_block_x < 1 || t.acc_block_y < 1 || t.acc_block_x * t.acc_block_y > 256 || (t.acc_block_x * t.acc_block_y) % 32 != 0))
            return fail(ISA_EINVAL, "tuning %d: accumulation block %d x %d", i, t.acc_block_x, t.acc_block_y);
    }
    c->tuning.assign(e, e + count);
    return ISA_OK;
}

int isa_set_tile_flow(isa_ctx* c, const float* tiles)
{
    if (!c) return fail(ISA_EINVAL, "ctx is NULL");
    if (((uintptr_t)tiles & 7) != 0) return fail(ISA_EINVAL, "tile flows must be 8-byte aligned");
    c->tile_override = (const float2*)tiles;
    return ISA_OK;
}

int isa_tile_flow(isa_ctx* c, float* tiles, int* tcx, int* tcy, void* stream)
{
    if (!c || c->last_n == 0) return fail(ISA_EINVAL, "no merge has run on this context");
    if (tcx) *tcx = c->last_tcx0;
    if (tcy) *tcy = c->last_tcy0;
    if (!tiles) return ISA_OK;
    if (((uintptr_t)tiles & 7) != 0) return fail(ISA_EINVAL, "tile flows must be 8-byte aligned");
    cudaStream_t st = S(stream);
    const size_t tsz = (size_t)c->last_tcx0 * c->last_tcy0;
    float2* out = (float2*)tiles;
    for (int i = 0; i < c->last_n; i++) {
        if (i == c->last_ref)
            ISA_CK(cudaMemsetAsync(out + i * tsz, 0, tsz * sizeof(float2), st));
        else if (c->tile_override)
            ISA_CK(cudaMemcpyAsync(out + i * tsz, c->tile_override + i * tsz, tsz * sizeof(float2), cudaMemcpyDeviceToDevice, st));
        else
            ISA_CK(isa_launch_optimal(c->x, c->last_n1, c->last_tcx0, c->last_tcy0, c->last_ref, i, out + i * tsz,
                                      (size_t)c->last_tcx0 * sizeof(float2), st));
    }
    return ISA_OK;
}

// ---- operator API -----------------------------------------------------------
#define ISA_REQ(cond, msg)                          \
    do {                                            \
        if (!(cond)) return fail(ISA_EINVAL, "%s", msg); \
    } while (0)

int isa_tracking_pairs(int n, int ref, int strategy, int block, int* pairs, int* rows, int max_pairs)
{
    if (n < 2 || ref < 0 || ref >= n) return fail(ISA_EINVAL, "frame count or reference out of range");
    Strategy s;
    if (!build_strategy(n, ref, strategy, block, s)) return fail(ISA_EINVAL, "inconsistent tracking strategy");
    if (pairs || rows) {
        if (max_pairs < s.m) return fail(ISA_EINVAL, "%d pairs do not fit in %d", s.m, max_pairs);
        for (int k = 0; k < s.m; k++) {
            if (pairs) { pairs[2 * k] = s.pairs[k].first; pairs[2 * k + 1] = s.pairs[k].second; }
            if (rows) {
                rows[3 * k] = s.a[k]; rows[3 * k + 1] = s.b[k]; rows[3 * k + 2] = s.sign[k];
            }
        }
    }
    return s.m;
}

int isa_debayer_full(const uint16_t* raw, size_t raw_pitch, int W, int H, const int cfa[4], const float black[3], const float scale[3],
                     const float divisor[3], float* out, size_t out_pitch, void* stream)
{
    ISA_REQ(raw && out && cfa && black && scale && divisor, "NULL argument");
    ISA_REQ(W > 0 && H > 0 && raw_pitch >= (size_t)W * 2 && out_pitch >= (size_t)W * 12, "bad size or pitch");
    ISA_REQ(cfa_ok(cfa), "bad CFA code");
    ISA_CK(isa_launch_demosaic_gray(raw, raw_pitch, W, H, pack_cfa(cfa), black, scale, divisor, nullptr, 0, nullptr, 0, out, out_pitch,
                                    S(stream)));
    return ISA_OK;
}

int isa_gamma_srgb(float* img, size_t pitch, int W, int H, void* stream)
{
    ISA_REQ(img && W > 0 && H > 0 && pitch >= (size_t)W * 12, "bad argument");
    ISA_CK(isa_launch_gamma(img, pitch, W, H, S(stream)));
    return ISA_OK;
}

int isa_bw_image(isa_ctx* c, const uint16_t* raw, size_t raw_pitch, int W, int H, const isa_raw_info* info, float sigma, int high_pass,
                 float* out, size_t out_pitch, void* stream)
{
    ISA_REQ(c && raw && out && info, "NULL argument");
    ISA_TRY(check_info(info));
    ISA_REQ(info->width == W && info->height == H, "info size differs from width/height");
    ISA_REQ(W <= c->max_w && H <= c->max_h, "frame exceeds the context");
    ISA_REQ(out_pitch == (size_t)W * 4 && raw_pitch >= (size_t)W * 2, "out pitch must be width * 4");
    ISA_REQ(!high_pass || ((uintptr_t)out & 7) == 0, "out must be 8-byte aligned for the high-pass (rows are read as complex pairs)");
    std::vector<float> taps = gauss_taps(sigma), none;
    return bw_frame(c, raw, raw_pitch, W, H, info, high_pass != 0, out, taps, nullptr, none, S(stream));
}

int isa_prealign_burst(isa_ctx* c, const uint16_t* raw, size_t raw_pitch, size_t frame_stride, int n, const isa_raw_info* info, float increment_deg,
                       float range_deg, const float* roll_deg, float* shifts, float* rotations_deg, int* reference, double* scan, void* stream)
{
    ISA_REQ(c && raw && info && shifts && rotations_deg && reference, "NULL argument");
    ISA_TRY(check_info(info));
    const int W = info->width, H = info->height;
    ISA_REQ(W <= c->max_w && H <= c->max_h && n >= 2 && n <= c->max_n, "burst exceeds the context");
    ISA_REQ(raw_pitch >= (size_t)W * 2 && frame_stride >= raw_pitch * H, "bad frame layout");
    ISA_REQ(increment_deg > 0.f && range_deg >= 0.f, "increment must be positive and range non-negative");
    ISA_REQ((size_t)W * H >= 4096, "frames too small for the pre-alignment scratch");
    cudaStream_t st = S(stream);
    const size_t fsz = (size_t)W * H;
    // tracking images of every frame (DeBayerBWGaussWB with the high-pass, controller :1474-1478)
    const std::vector<float> taps = gauss_taps(c->p.sigma_debayer_tracking), none;
    for (int i = 0; i < n; i++)
        ISA_TRY(bw_frame(c, (const uint16_t*)((const char*)raw + (size_t)i * frame_stride), raw_pitch, W, H, info, true, c->bw_track + i * fsz, taps,
                         nullptr, none, st));
    // reference spectrum (SetReferenceImage, PreAlignment.cs:164-175): frame 0
    ISA_TRY(fft_forward(c, c->bw_track, (size_t)W * 4, c->spec, W, H, st));
    std::vector<ScanResult> init(n, ScanResult{0, 0, 0, 0});
    const float roll0 = roll_deg ? -roll_deg[0] : 0.f;
    for (int i = 1; i < n; i++) {
        const float rollt = roll_deg ? -roll_deg[i] : 0.f;
        ISA_TRY(scan_angles(c, c->bw_track + i * fsz, W, H, (double)increment_deg, (double)range_deg, (double)(rollt - roll0), st, init[i]));
    }
    if (scan)
        for (int i = 0; i < n; i++) {
            scan[4 * i] = init[i].x; scan[4 * i + 1] = init[i].y; scan[4 * i + 2] = init[i].ang; scan[4 * i + 3] = init[i].val;
        }
    return prealign_store(init, shifts, rotations_deg, reference);
}

int isa_fourier_filter(void* spec, size_t pitch, int W, int H, float lp, float hp, float lps, float hps, int clear_axis, float post_scale,
                       void* stream)
{
    ISA_REQ(spec && W > 1 && H > 0 && pitch >= (size_t)(W / 2 + 1) * 8, "bad argument");
    ISA_CK(isa_launch_fourier_filter((float2*)spec, pitch, W, H, 1, 0, lp, hp, lps, hps, clear_axis, post_scale, S(stream)));
    return ISA_OK;
}

int isa_gauss_filter(const float* in, size_t in_pitch, float* out, size_t out_pitch, float* tmp, size_t tmp_pitch, int W, int H, int C,
                     float sigma, void* stream)
{
    ISA_REQ(in && out && tmp && W > 0 && H > 0 && (C == 1 || C == 3), "bad argument");
    ISA_REQ(in_pitch >= (size_t)W * C * 4 && out_pitch >= (size_t)W * C * 4 && tmp_pitch >= (size_t)W * C * 4, "pitch too small");
    std::vector<float> t = gauss_taps(sigma);
    ISA_CK(isa_launch_gauss(in, in_pitch, out, out_pitch, tmp, tmp_pitch, W, H, C, t.data(), (int)t.size(), 0, S(stream)));
    return ISA_OK;
}

int isa_resize_box(const float* in, size_t in_pitch, int W, int H, int level, float* out, size_t out_pitch, void* stream)
{
    ISA_REQ(in && out && level >= 1 && W >= level && H >= level, "bad argument");
    ISA_REQ(in_pitch >= (size_t)W * 4 && out_pitch >= (size_t)(W / level) * 4, "pitch too small");
    ISA_CK(isa_launch_resize_box(in, in_pitch, W, H, level, out, out_pitch, S(stream)));
    return ISA_OK;
}

int isa_track_level(const float* const* frames, size_t frame_pitch, int W, int H, int T, int Smax, int tcx, int tcy, const isa_track_pair* pairs,
                    int npairs, void* grids, size_t grid_pitch, size_t grid_stride, float threshold, float* scores, int* argmin, void* stream)
{
    ISA_REQ(frames && pairs && grids && npairs > 0, "NULL argument");
    ISA_REQ(tcx > 0 && tcy > 0 && (W - 2 * Smax) / T >= tcx && (H - 2 * Smax) / T >= tcy, "tile counts exceed the frame");
    ISA_REQ(grid_pitch >= (size_t)tcx * 8 && grid_stride >= grid_pitch * tcy, "grid pitch/stride too small");
    static_assert(sizeof(isa_track_pair) == sizeof(isa_pair_desc), "pair layout");
    cudaError_t e = isa_launch_track(frames, frame_pitch, W, H, T, Smax, tcx, tcy, (const isa_pair_desc*)pairs, npairs, (float2*)grids, grid_pitch,
                                     grid_stride, threshold, scores, argmin, nullptr, S(stream));
    if (e == cudaErrorInvalidValue) return fail(ISA_EINVAL, "tile size %d / max shift %d not supported", T, Smax);
    ISA_CK(e);
    return ISA_OK;
}

int isa_upsample_shifts(const void* in, size_t in_pitch, size_t in_stride, void* out, size_t out_pitch, size_t out_stride, int ngrids, int oldLevel,
                        int newLevel, int ocx, int ocy, int ncx, int ncy, int oT, int nT, void* stream)
{
    ISA_REQ(in && out && in != out && ngrids > 0 && ocx > 0 && ocy > 0 && ncx > 0 && ncy > 0 && newLevel > 0 && nT > 0, "bad argument");
    ISA_CK(isa_launch_upsample((const float2*)in, in_pitch, in_stride, (float2*)out, out_pitch, out_stride, ngrids, oldLevel, newLevel, ocx, ocy, ncx,
                               ncy, oT, nT, S(stream)));
    return ISA_OK;
}

int isa_solve_shifts(isa_ctx* c, int n, int ref, int strategy, int block, void* grids, size_t grid_pitch, size_t grid_stride, int tcx, int tcy,
                     void* x, int* status, void* stream)
{
    ISA_REQ(c && grids && x && status && tcx > 0 && tcy > 0, "bad argument");
    ISA_REQ(n >= 2 && n <= c->max_n && ref >= 0 && ref < n, "frame count or reference out of range");
    Strategy s;
    ISA_REQ(build_strategy(n, ref, strategy, block, s), "inconsistent tracking strategy");
    ISA_REQ(s.m <= c->max_rows, "too many pairs for the context");
    ISA_TRY(upload_strategy(c, s, S(stream)));
    cudaError_t e = isa_launch_solve(c->row_a, c->row_b, c->row_sign, c->N0, s.m, s.n1, (float2*)grids, grid_pitch, grid_stride, c->row_grid, tcx, tcy,
                                     (float2*)x, status, S(stream));
    if (e == cudaErrorInvalidValue) return fail(ISA_EINVAL, "solver shared memory exceeds the limit (m=%d, n-1=%d)", s.m, s.n1);
    ISA_CK(e);
    return ISA_OK;
}

int isa_optimal_shifts(const void* x, int n, int tcx, int tcy, int ref, int trk, void* out, size_t out_pitch, void* stream)
{
    ISA_REQ(x && out && n >= 2 && tcx > 0 && tcy > 0 && ref >= 0 && ref < n && trk >= 0 && trk < n, "bad argument");
    ISA_CK(isa_launch_optimal((const float2*)x, n - 1, tcx, tcy, ref, trk, (float2*)out, out_pitch, S(stream)));
    return ISA_OK;
}

int isa_flow_from_tiles(const void* tiles, size_t tile_pitch, int tcx, int tcy, int W, int H, const float base[2], float rot, void* flow,
                        size_t flow_pitch, void* stream)
{
    ISA_REQ(tiles && flow && base && tcx > 0 && tcy > 0 && W > 0 && H > 0, "bad argument");
    ISA_CK(isa_launch_flow_from_tiles((const float2*)tiles, tile_pitch, tcx, tcy, W, H, base[0], base[1], rot, (float2*)flow, flow_pitch,
                                      S(stream)));
    return ISA_OK;
}

int isa_warp(const float* img, size_t img_pitch, int W, int H, const void* flow, size_t flow_pitch, float* out, size_t out_pitch, void* stream)
{
    ISA_REQ(img && flow && out && W > 0 && H > 0, "bad argument");
    ISA_CK(isa_launch_warp(img, img_pitch, W, H, (const float2*)flow, flow_pitch, out, out_pitch, S(stream)));
    return ISA_OK;
}

int isa_derivatives(const float* src, const float* tgt, size_t pitch, int W, int H, float* ix, float* iy, float* it, size_t out_pitch, void* stream)
{
    ISA_REQ(src && tgt && ix && iy && it && W > 0 && H > 0, "bad argument");
    ISA_CK(isa_launch_derivatives(src, tgt, pitch, W, H, ix, iy, it, out_pitch, S(stream)));
    return ISA_OK;
}

int isa_derivatives2(const float* img, size_t pitch, int W, int H, float* ix, float* iy, size_t out_pitch, void* stream)
{
    ISA_REQ(img && ix && iy && W > 0 && H > 0, "bad argument");
    ISA_CK(isa_launch_derivatives2(img, pitch, W, H, ix, iy, out_pitch, S(stream)));
    return ISA_OK;
}

int isa_lucas_kanade(void* flow, size_t flow_pitch, const float* ix, const float* iy, const float* it, size_t pitch, int W, int H, float min_det,
                     int window, void* stream)
{
    ISA_REQ(flow && ix && iy && it && W > 0 && H > 0 && window >= 1, "bad argument");
    ISA_CK(isa_launch_lk_sums((float2*)flow, flow_pitch, ix, iy, it, pitch, W, H, window / 2, min_det, S(stream)));
    return ISA_OK;
}

int isa_lk_iteration(const void* flow_in, void* flow_out, size_t flow_pitch, const float* src, const float* ref, size_t img_pitch, int W, int H,
                     float min_det, int window, void* stream)
{
    ISA_REQ(flow_in && flow_out && flow_in != flow_out && src && ref && W > 0 && H > 0, "bad argument");
    ISA_REQ(window >= 1 && window / 2 <= 15, "window size out of range");
    ISA_CK(isa_launch_lk_iteration((const float2*)flow_in, (float2*)flow_out, flow_pitch, src, ref, img_pitch, W, H, window / 2, min_det,
                                   S(stream)));
    return ISA_OK;
}

int isa_lk_refine(const float* src, const float* ref, size_t img_pitch, int W, int H, const void* tiles, size_t tile_pitch, int tcx, int tcy,
                  const float base[2], float rot, int iterations, float min_det, int window, void* flow, void* flow_scratch, size_t flow_pitch,
                  void* stream)
{
    ISA_REQ(src && ref && tiles && base && flow && flow_scratch && flow != flow_scratch && iterations >= 0, "bad argument");
    ISA_REQ(window >= 1 && window / 2 <= 15, "window size out of range");
    float2* a = (iterations & 1) ? (float2*)flow_scratch : (float2*)flow;
    float2* b = (iterations & 1) ? (float2*)flow : (float2*)flow_scratch;
    ISA_CK(isa_launch_flow_from_tiles((const float2*)tiles, tile_pitch, tcx, tcy, W, H, base[0], base[1], rot, a, flow_pitch, S(stream)));
    for (int i = 0; i < iterations; i++) {
        ISA_CK(isa_launch_lk_iteration(a, b, flow_pitch, src, ref, img_pitch, W, H, window / 2, min_det, S(stream)));
        std::swap(a, b);
    }
    return ISA_OK;
}

int isa_debayer_subsample(const uint16_t* raw, size_t raw_pitch, int W, int H, const int cfa[4], float max_value, float* out, size_t out_pitch,
                          void* stream)
{
    ISA_REQ(raw && out && cfa && W >= 2 && H >= 2 && cfa_ok(cfa) && max_value != 0.f, "bad argument");
    ISA_CK(isa_launch_subsample(raw, raw_pitch, W, H, pack_cfa(cfa), max_value, out, out_pitch, S(stream)));
    return ISA_OK;
}

int isa_robustness_mask(const float* ref3, const float* mov3, size_t img_pitch, void* mask, size_t mask_pitch, int Wh, int Hh, const void* flow,
                        size_t flow_pitch, int Wf, int Hf, float alpha, float beta, float thr_m, float s, float t, void* stream)
{
    ISA_REQ(ref3 && mov3 && mask && flow && Wh >= 3 && Hh >= 3 && Wf > 0 && Hf > 0, "bad argument");
    ISA_CK(isa_launch_robustness(ref3, mov3, img_pitch, (float4*)mask, mask_pitch, Wh, Hh, (const float2*)flow, flow_pitch, Wf, Hf, alpha, beta,
                                 thr_m, s, t, S(stream)));
    return ISA_OK;
}

int isa_erode(const void* in, size_t in_pitch, void* out, size_t out_pitch, int W, int H, int size, void* stream)
{
    ISA_REQ(in && out && in != out && W > 0 && H > 0 && size >= 1, "bad argument");
    ISA_CK(isa_launch_erode((const float4*)in, in_pitch, (float4*)out, out_pitch, W, H, size, S(stream)));
    return ISA_OK;
}

int isa_robustness_erode(const float* ref3, const float* mov3, size_t img_pitch, int Wh, int Hh, const void* flow, size_t flow_pitch, int Wf, int Hf,
                         float alpha, float beta, float thr_m, float s, float t, int erode_size, void* out, size_t out_pitch, void* stream)
{
    ISA_REQ(ref3 && mov3 && flow && out && Wh >= 3 && Hh >= 3 && erode_size >= 1 && erode_size / 2 <= 4, "bad argument");
    ISA_CK(isa_launch_robustness_erode(ref3, mov3, img_pitch, Wh, Hh, (const float2*)flow, flow_pitch, Wf, Hf, alpha, beta, thr_m, s, t, erode_size,
                                       (float4*)out, out_pitch, S(stream)));
    return ISA_OK;
}

int isa_structure_tensor(const float* img, size_t pitch, int W, int H, float* out, size_t out_pitch, void* stream)
{
    ISA_REQ(img && out && W > 0 && H > 0 && out_pitch >= (size_t)W * 12, "bad argument");
    ISA_CK(isa_launch_structure_tensor(img, pitch, W, H, out, out_pitch, S(stream)));
    return ISA_OK;
}

int isa_kernel_param(const float* st3, size_t st_pitch, int W, int H, float* out, size_t out_pitch, int oc, float dth, float dtr, float kd, float kn,
                     float ks, float kh, void* stream)
{
    ISA_REQ(st3 && out && W > 0 && H > 0 && (oc == 3 || oc == 4), "bad argument");
    ISA_REQ(oc == 3 || (const void*)st3 != (const void*)out, "4-channel output cannot alias the tensor");
    ISA_CK(isa_launch_kernel_param(st3, st_pitch, W, H, out, out_pitch, oc, dth, dtr, kd, kn, ks, kh, S(stream)));
    return ISA_OK;
}

int isa_accumulate(const uint16_t* raw, size_t raw_pitch, int W, int H, const int cfa[4], float* acc, float* wsum, size_t out_pitch, int Wo, int Ho,
                   const void* mask, size_t mask_pitch, const float* kparam, size_t kparam_pitch, int kc, const void* flow, size_t flow_pitch,
                   const float white[3], const float black[3], float scale, int ox, int oy, const int crop[4], void* stream)
{
    ISA_REQ(raw && acc && wsum && kparam && cfa && white && black && crop, "NULL argument");
    ISA_REQ(W >= 2 && H >= 2 && !(W & 1) && !(H & 1) && Wo > 0 && Ho > 0 && (kc == 3 || kc == 4) && scale > 0, "bad size");
    ISA_REQ(crop[0] >= 0 && crop[1] >= 0 && crop[2] < W && crop[3] < H && crop[0] <= crop[2] && crop[1] <= crop[3], "crop outside the frame");
    ISA_REQ(cfa_ok(cfa), "bad CFA code");
    isa_accum_geom g;
    g.W = W; g.H = H; g.Wo = Wo; g.Ho = Ho; g.s = scale; g.ox = ox; g.oy = oy;
    g.cx0 = crop[0]; g.cy0 = crop[1]; g.cx1 = crop[2]; g.cy1 = crop[3];
    g.masks_finite = 0;
    g.bilinear = 0;
    g.yb0 = 0;
    g.yb1 = Ho;
    float r = std::round(scale);
    g.s_int = (r == scale && r >= 1.f) ? (int)r : 0;
    isa_frame_in f{raw, (const float2*)flow, (const float4*)mask};
    ISA_CK(isa_launch_accumulate(g, pack_cfa(cfa), nullptr, 1, &f, raw_pitch, flow_pitch, mask_pitch, kparam, kparam_pitch, kc, white, black, acc,
                                 wsum, out_pitch, 1, S(stream)));
    return ISA_OK;
}

int isa_apply_weighting(float* img, const float* acc, const float* wsum, size_t pitch, int W, int H, float thr, void* stream)
{
    ISA_REQ(img && acc && wsum && W > 0 && H > 0 && pitch >= (size_t)W * 12, "bad argument");
    ISA_CK(isa_launch_apply_weighting(img, pitch, acc, wsum, pitch, W, H, thr, S(stream)));
    return ISA_OK;
}

}  // extern "C"

// ---- shift solve without a context ------------------------------------------
// isa_solve_shifts needs an isa_ctx only for its row tables, and creating a
// context allocates device memory. Some hosts cannot do that at the point
// where they align tiles: the device memory belongs to another allocator
// that has handed it all out, or the caller works under a fixed memory
// budget, or it must not enter cudaMalloc because an allocation can
// synchronise the device and stall work on other streams. For them the row
// tables live in this file-scope device array, created with the module and
// kept until the process exits on every GPU that loads the library.
namespace {

constexpr int kStaticMaxRows = 2048;  // measurement rows (frame pairs)
constexpr int kStaticMaxN1 = 64;      // one-to-one shifts (frames - 1)

struct StaticSolveTables {
    int a[kStaticMaxRows], b[kStaticMaxRows], sign[kStaticMaxRows], grid[kStaticMaxRows];
    double N0[kStaticMaxN1 * kStaticMaxN1];
};

static __device__ __align__(256) unsigned char g_solve_scratch[sizeof(StaticSolveTables)];

// Device address of g_solve_scratch. In host code the symbol is only a
// handle, so the address is asked for (with the device current) once per
// device and CUDA context, and kept with the context's unique id: after a
// cudaDeviceReset the device code is loaded again in a new context and the
// array may move, so a new id triggers a new look-up. The same set-up loads
// the solver's device code, so that a later call loads nothing.
typedef int (*CtxGetCurrentFn)(void**);                     // CUresult cuCtxGetCurrent(CUcontext*)
typedef int (*CtxGetIdFn)(void*, unsigned long long*);      // CUresult cuCtxGetId(CUcontext, unsigned long long*)

struct StaticScratchSlot {
    unsigned long long ctx_id = 0;
    StaticSolveTables* addr = nullptr;
};
std::mutex g_scratch_lock;
StaticScratchSlot g_scratch_slot[64];

// The current context's unique id (cuCtxGetId through the runtime's driver
// entry points, so the library needs no link to the driver library); 0 when
// no context is current yet.
int current_ctx_id(unsigned long long* id)
{
    static CtxGetCurrentFn get_current = nullptr;
    static CtxGetIdFn get_id = nullptr;
    if (!get_current || !get_id) {
        cudaDriverEntryPointQueryResult q1, q2;
        void *f1 = nullptr, *f2 = nullptr;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f1, 12000, cudaEnableDefault, &q1) != cudaSuccess || !f1 ||
            cudaGetDriverEntryPointByVersion("cuCtxGetId", &f2, 12000, cudaEnableDefault, &q2) != cudaSuccess || !f2)
            return fail(ISA_ECUDA, "the driver does not provide cuCtxGetCurrent / cuCtxGetId");
        get_current = (CtxGetCurrentFn)f1;
        get_id = (CtxGetIdFn)f2;
    }
    void* ctx = nullptr;
    *id = 0;
    if (get_current(&ctx) != 0) return fail(ISA_ECUDA, "cuCtxGetCurrent failed");
    if (ctx && get_id(ctx, id) != 0) return fail(ISA_ECUDA, "cuCtxGetId failed");
    return ISA_OK;
}

int static_tables(StaticSolveTables** out)
{
    int dev = 0;
    ISA_CK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return fail(ISA_EINVAL, "device ordinal %d out of range", dev);
    std::lock_guard<std::mutex> lock(g_scratch_lock);
    unsigned long long id = 0;
    ISA_TRY(current_ctx_id(&id));
    StaticScratchSlot& slot = g_scratch_slot[dev];
    if (!slot.addr || id == 0 || id != slot.ctx_id) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_solve_scratch);  // loads this file's device code on the device
        if (e != cudaSuccess) return fail(ISA_ECUDA, "cudaGetSymbolAddress(g_solve_scratch): %s", cudaGetErrorString(e));
        e = isa_solve_prepare();
        if (e != cudaSuccess) return fail(ISA_ECUDA, "loading the solver: %s", cudaGetErrorString(e));
        ISA_TRY(current_ctx_id(&id));
        slot.addr = (StaticSolveTables*)p;
        slot.ctx_id = id;
    }
    *out = slot.addr;
    return ISA_OK;
}

}  // namespace

// The static solve's set-up on the current device, also run by isa_ctx_create.
int isa_static_solve_setup()
{
    StaticSolveTables* t = nullptr;
    return static_tables(&t);
}

extern "C" int isa_solve_shifts_static(int n, int ref, int strategy, int block, void* grids, size_t grid_pitch, size_t grid_stride, int tcx,
                                       int tcy, void* x, int* status, void* stream)
{
    ISA_REQ(grids && x && status && tcx > 0 && tcy > 0, "bad argument");
    ISA_REQ(n >= 2 && ref >= 0 && ref < n, "frame count or reference out of range");
    if (n - 1 > kStaticMaxN1) return fail(ISA_EINVAL, "%d frames exceed the static limit of %d", n, kStaticMaxN1 + 1);
    Strategy s;
    ISA_REQ(build_strategy(n, ref, strategy, block, s), "inconsistent tracking strategy");
    if (s.m > kStaticMaxRows) return fail(ISA_EINVAL, "%d frame pairs exceed the static limit of %d", s.m, kStaticMaxRows);
    StaticSolveTables* t = nullptr;
    ISA_TRY(static_tables(&t));
    // every entry the kernel reads (m rows, n1 x n1 of N0) is rewritten here
    ISA_TRY(upload_rows(t->a, t->b, t->sign, t->grid, t->N0, s, S(stream)));
    cudaError_t e = isa_launch_solve(t->a, t->b, t->sign, t->N0, s.m, s.n1, (float2*)grids, grid_pitch, grid_stride, t->grid, tcx, tcy, (float2*)x,
                                     status, S(stream));
    if (e == cudaErrorInvalidValue) return fail(ISA_EINVAL, "solver shared memory exceeds the limit (m=%d, n-1=%d)", s.m, s.n1);
    ISA_CK(e);
    return ISA_OK;
}


// ---- colour and tone post-processing, TIFF output ----

namespace {

struct M3 { double a[3][3]; };

// DNGMatrix operator * (DNGMatrix.cs:232-254): sums from 0.0 in column order
M3 mat_mul(const M3& x, const M3& y)
{
    M3 r;
    for (int j = 0; j < 3; j++)
        for (int k = 0; k < 3; k++) {
            double s = 0.0;
            for (int m = 0; m < 3; m++) s += x.a[j][m] * y.a[m][k];
            r.a[j][k] = s;
        }
    return r;
}

// DNGMatrix.Invert3x3 (DNGMatrix.cs:440-486): adjugate over the determinant
bool mat_inv3(const M3& m, M3& out)
{
    const double a00 = m.a[0][0], a01 = m.a[0][1], a02 = m.a[0][2], a10 = m.a[1][0], a11 = m.a[1][1], a12 = m.a[1][2], a20 = m.a[2][0],
                 a21 = m.a[2][1], a22 = m.a[2][2];
    double t[3][3];
    t[0][0] = a11 * a22 - a21 * a12;
    t[0][1] = a21 * a02 - a01 * a22;
    t[0][2] = a01 * a12 - a11 * a02;
    t[1][0] = a20 * a12 - a10 * a22;
    t[1][1] = a00 * a22 - a20 * a02;
    t[1][2] = a10 * a02 - a00 * a12;
    t[2][0] = a10 * a21 - a20 * a11;
    t[2][1] = a20 * a01 - a00 * a21;
    t[2][2] = a00 * a11 - a10 * a01;
    const double det = a00 * t[0][0] + a01 * t[1][0] + a02 * t[2][0];
    if (!(std::fabs(det) >= 1e-10)) return false;  // NEAR_ZERO (DNGMatrix.cs:34)
    for (int j = 0; j < 3; j++)
        for (int k = 0; k < 3; k++) out.a[j][k] = t[j][k] / det;
    return true;
}

// DNGColorSpace(toPCS) (DNGColorSpace.cs:45-65): rows scaled so that RGB
// white (1, 1, 1) maps to the PCS white (D50 xy (0.3457, 0.3585) as XYZ,
// DNGxyCoord.cs:79-101, 175-181, 211-214); fromPCS is its inverse.
bool color_space(const M3& toPCS, M3& to, M3& from)
{
    const double x = 0.3457, y = 0.3585;  // inside the pinning range of XYtoXYZ, x + y < 0.999999
    const double W2[3] = {x / y, 1.0, (1.0 - x - y) / y};
    for (int j = 0; j < 3; j++) {
        double w1 = 0.0;
        for (int m = 0; m < 3; m++) w1 += toPCS.a[j][m] * 1.0;
        const double s = W2[j] / w1;
        for (int k = 0; k < 3; k++) to.a[j][k] = s * toPCS.a[j][k];
    }
    return mat_inv3(to, from);
}

void twist_of(const M3& m, float t[12])
{
    for (int i = 0; i < 3; i++) {
        for (int j = 0; j < 3; j++) t[i * 4 + j] = (float)m.a[i][j];
        t[i * 4 + 3] = 0.f;
    }
}

int check_post(const isa_post_params* pp, int width, int height)
{
    ISA_REQ(pp, "NULL post-processing parameters");
    ISA_REQ(pp->crop_x >= 0 && pp->crop_y >= 0 && pp->crop_w > 0 && pp->crop_h > 0 && pp->crop_x + pp->crop_w <= width &&
                pp->crop_y + pp->crop_h <= height,
            "crop outside the image");
    if (!(pp->lut_x && pp->lut_y && pp->nlut >= 4 && pp->nlut <= ISA_MAX_LUT)) return fail(ISA_EINVAL, "LUT needs 4 to %d levels", ISA_MAX_LUT);
    for (int i = 1; i < pp->nlut; i++)
        if (!(pp->lut_x[i] > pp->lut_x[i - 1])) return fail(ISA_EINVAL, "LUT levels must increase strictly (level %d)", i);
    for (int i = 0; i < pp->nlut; i++)
        if (!std::isfinite(pp->lut_x[i]) || !std::isfinite(pp->lut_y[i])) return fail(ISA_EINVAL, "LUT entry %d is not finite", i);
    return ISA_OK;
}

// LUTCubic as the cubic through the four nearest levels: for segment k
// (x[k] <= v < x[k + 1]) the levels i0 .. i0 + 3, i0 = clamp(k - 1, 0, n - 4),
// in FP64: Newton divided differences on the nodes z_j = x[i0 + j] - x[k],
// expanded to c0 + c1 t + c2 t^2 + c3 t^3 in t = v - x[k], then rounded to float.
void lut_coefficients(const float* x, const float* y, int n, float (*c)[4])
{
    for (int k = 0; k < n - 1; k++) {
        const int i0 = std::min(std::max(k - 1, 0), n - 4);
        double z[4], a[4];
        for (int j = 0; j < 4; j++) {
            z[j] = (double)x[i0 + j] - (double)x[k];
            a[j] = (double)y[i0 + j];
        }
        for (int o = 1; o < 4; o++)
            for (int j = 3; j >= o; j--) a[j] = (a[j] - a[j - 1]) / (z[j] - z[j - o]);
        // p(t) = a0 + (t - z0)(a1 + (t - z1)(a2 + (t - z2) a3)), expanded from the inside out
        double p[4] = {a[3], 0.0, 0.0, 0.0};  // coefficients of t^0 .. t^3 of the partial polynomial
        int deg = 0;
        for (int j = 2; j >= 0; j--) {
            // p <- p * (t - z_j) + a_j
            double q[4] = {0.0, 0.0, 0.0, 0.0};
            for (int d = 0; d <= deg; d++) {
                q[d + 1] += p[d];
                q[d] -= z[j] * p[d];
            }
            q[0] += a[j];
            deg++;
            for (int d = 0; d < 4; d++) p[d] = q[d];
        }
        for (int d = 0; d < 4; d++) c[k][d] = (float)p[d];
    }
}

void post_args(const isa_post_params* pp, isa_post_args& a)
{
    a.crop_x = pp->crop_x; a.crop_y = pp->crop_y; a.crop_w = pp->crop_w; a.crop_h = pp->crop_h;
    for (int c = 0; c < 3; c++) a.wb[c] = pp->camera_white[c];
    for (int i = 0; i < 12; i++) { a.t1[i] = pp->twist1[i]; a.t2[i] = pp->twist2[i]; }
    a.amp = (float)std::pow(2.0, (double)pp->exposure);  // (float)Math.Pow(2.0, Exposure) (:2243)
    a.nlut = pp->nlut;
    a.uniform = 1;
    lut_coefficients(pp->lut_x, pp->lut_y, pp->nlut, a.lut_c);
    for (int i = 0; i < pp->nlut; i++) {
        a.lut_x[i] = pp->lut_x[i];
        // near-uniform levels (within half a step of i / (n - 1)): the kernel's guess is off by at most one level
        if (!(std::fabs((double)pp->lut_x[i] - (double)i / (pp->nlut - 1)) <= 0.5 / (pp->nlut - 1))) a.uniform = 0;
    }
}

void put16(std::vector<unsigned char>& b, size_t at, uint16_t v) { b[at] = v & 255; b[at + 1] = v >> 8; }
void put32(std::vector<unsigned char>& b, size_t at, uint32_t v)
{
    for (int i = 0; i < 4; i++) b[at + i] = (v >> (8 * i)) & 255;
}

}  // namespace

int isa_color_twists(const double camera_to_pcs[9], float twist1[12], float twist2[12])
{
    ISA_REQ(camera_to_pcs && twist1 && twist2, "NULL argument");
    // DNGColorSpace.ProPhoto and .sRGB50 (DNGColorSpace.cs:35-42)
    const M3 prophoto{{{0.7976749, 0.1351917, 0.0313534}, {0.2880402, 0.7118741, 0.0000857}, {0.0000000, 0.0000000, 0.8252100}}};
    const M3 srgb50{{{0.4360747, 0.3850649, 0.1430804}, {0.2225045, 0.7168786, 0.0606169}, {0.0139322, 0.0971045, 0.7141733}}};
    M3 pp_to, pp_from, s_to, s_from, cam;
    ISA_REQ(color_space(prophoto, pp_to, pp_from) && color_space(srgb50, s_to, s_from), "colour space matrix is singular");
    for (int j = 0; j < 3; j++)
        for (int k = 0; k < 3; k++) cam.a[j][k] = camera_to_pcs[j * 3 + k];
    twist_of(mat_mul(pp_from, cam), twist1);      // ProPhoto.FromPCS * cameraToXYZ (:2227)
    twist_of(mat_mul(s_from, pp_to), twist2);     // sRGB50.FromPCS * ProPhoto.ToPCS (:2239)
    return ISA_OK;
}

int isa_postprocess(const float* img, size_t pitch, int width, int height, const isa_post_params* pp, int format, void* out, size_t out_pitch,
                    void* stream)
{
    ISA_REQ(img && out && width > 0 && height > 0 && pitch >= (size_t)width * 12, "bad image argument");
    if (format != ISA_POST_RGB16 && format != ISA_POST_BGRA8) return fail(ISA_EINVAL, "unknown output format %d", format);
    ISA_TRY(check_post(pp, width, height));
    ISA_REQ(out_pitch >= (size_t)pp->crop_w * (format == ISA_POST_RGB16 ? 6 : 4) && (format == ISA_POST_RGB16 || out_pitch % 4 == 0) &&
                (format == ISA_POST_RGB16 ? ((uintptr_t)out & 1) == 0 && out_pitch % 2 == 0 : ((uintptr_t)out & 3) == 0),
            "bad output pitch or alignment");
    isa_post_args a;
    post_args(pp, a);
    ISA_CK(isa_launch_postprocess(img, pitch, a, format, out, out_pitch, S(stream)));
    return ISA_OK;
}

int isa_save_tiff16(const char* path, const uint16_t* rgb, int width, int height)
{
    ISA_REQ(path && rgb && width > 0 && height > 0, "bad argument");
    const uint64_t nbytes = (uint64_t)width * height * 3 * 2;
    ISA_REQ(nbytes <= 0xffffffffull - 200, "image too large for a 32-bit TIFF");
    // header, the IFD of 13 entries in the order of ImageFileDirectory(width, height)
    // (ImageFileDirectory.cs:75-92), then the out-of-line values in the same
    // order (BitsPerSample, XResolution, YResolution, Make), then the strip
    std::vector<unsigned char> b(200, 0);
    b[0] = 0x49; b[1] = 0x49; b[2] = 0x2A; b[3] = 0; put32(b, 4, 8);
    put16(b, 8, 13);
    size_t e = 10;
    const auto entry = [&](uint16_t tag, uint16_t type, uint32_t count, uint32_t value) {
        put16(b, e, tag); put16(b, e + 2, type); put32(b, e + 4, count); put32(b, e + 8, value);
        e += 12;
    };
    const uint32_t data_at = 200;
    entry(256, 4, 1, (uint32_t)width);             // ImageWidth, LONG
    entry(257, 4, 1, (uint32_t)height);            // ImageLength, LONG
    entry(258, 3, 3, 170);                         // BitsPerSample 16, 16, 16 (out of line)
    entry(259, 3, 1, 1);                           // Compression: none
    entry(262, 3, 1, 2);                           // PhotometricInterpretation: RGB
    entry(273, 4, 1, data_at);                     // StripOffsets
    entry(277, 3, 1, 3);                           // SamplesPerPixel
    entry(278, 4, 1, (uint32_t)height);            // RowsPerStrip
    entry(279, 4, 1, (uint32_t)nbytes);            // StripByteCounts
    entry(282, 5, 1, 176);                         // XResolution 720/10
    entry(283, 5, 1, 184);                         // YResolution 720/10
    entry(296, 3, 1, 1);                           // ResolutionUnit: none
    entry(271, 2, 8, 192);                         // Make "MK TIFF\0"
    put32(b, e, 0);                                // no next IFD; e + 4 == 170
    put16(b, 170, 16); put16(b, 172, 16); put16(b, 174, 16);
    put32(b, 176, 720); put32(b, 180, 10);
    put32(b, 184, 720); put32(b, 188, 10);
    std::memcpy(&b[192], "MK TIFF", 8);
    FILE* f = std::fopen(path, "wb");
    if (!f) return fail(ISA_EINVAL, "cannot open %s for writing", path);
    bool ok = std::fwrite(b.data(), 1, b.size(), f) == b.size();
    // uint16 little-endian samples (BinaryWriter.Write(ushort))
    std::vector<unsigned char> row((size_t)width * 6);
    for (int y = 0; ok && y < height; y++) {
        const uint16_t* r = rgb + (size_t)y * width * 3;
        for (size_t i = 0; i < (size_t)width * 3; i++) { row[2 * i] = r[i] & 255; row[2 * i + 1] = r[i] >> 8; }
        ok = std::fwrite(row.data(), 1, row.size(), f) == row.size();
    }
    ok = (std::fclose(f) == 0) && ok;
    if (!ok) return fail(ISA_EINVAL, "writing %s failed", path);
    return ISA_OK;
}

int isa_save_as_16bit_tiff(const float* img, size_t pitch, int width, int height, const isa_post_params* pp, const char* path, void* stream)
{
    ISA_REQ(path, "NULL path");
    ISA_TRY(check_post(pp, width, height));
    const size_t bytes = (size_t)pp->crop_w * pp->crop_h * 6;
    void* d = nullptr;
    ISA_CK(cudaMallocAsync(&d, bytes, S(stream)));
    std::vector<uint16_t> h((size_t)pp->crop_w * pp->crop_h * 3);
    int rc = isa_postprocess(img, pitch, width, height, pp, ISA_POST_RGB16, d, (size_t)pp->crop_w * 6, stream);
    if (rc == ISA_OK) {
        cudaError_t e = cudaMemcpyAsync(h.data(), d, bytes, cudaMemcpyDeviceToHost, S(stream));
        if (e == cudaSuccess) e = cudaStreamSynchronize(S(stream));
        if (e != cudaSuccess) rc = fail(ISA_ECUDA, "copying the image to the host: %s", cudaGetErrorString(e));
    }
    cudaFreeAsync(d, S(stream));
    if (rc != ISA_OK) return rc;
    return isa_save_tiff16(path, h.data(), pp->crop_w, pp->crop_h);
}

// ---- PEF raw decoding ----

int isa_pef_huff_table(const uint8_t* mn, size_t n, int big_endian, uint16_t table[4097])
{
    ISA_REQ(mn && table, "NULL argument");
    std::memset(table, 0, 4097 * sizeof(uint16_t));
    const auto rd16 = [&](size_t i) -> unsigned {
        return big_endian ? (unsigned)(mn[i] << 8 | mn[i + 1]) : (unsigned)(mn[i + 1] << 8 | mn[i]);
    };
    ISA_REQ(n >= 2, "maker note too short");
    const int dep = (int)((rd16(0) + 12) & 15);
    if (n < (size_t)(14 + 3 * dep)) return fail(ISA_EINVAL, "maker note too short for %d codes", dep);
    for (int c = 0; c < dep; c++) {
        const unsigned code = rd16(14 + 2 * (size_t)c), len = mn[14 + 2 * (size_t)dep + c];
        // the fill loop of MNHuffmanTable: entries code + 1 .. through the 4096 >> len peeks that start with the code (mod 4096)
        for (unsigned i = code; i <= ((code + (4096u >> (len & 31)) - 1) & 4095u);) {
            ++i;
            if (i > 4096) break;
            table[i] = (uint16_t)(len << 8 | (unsigned)c);
        }
        table[0] = 12;
    }
    return dep;
}

size_t isa_pef_decode_scratch(size_t nbytes, int width, int height)
{
    if (width <= 0 || height <= 0) return 0;
    size_t parts[14];
    return isa_pef_scratch_layout(nbytes, width, height, parts);
}

int isa_pef_decode(const uint8_t* data, size_t nbytes, const uint16_t* table, int width, int height, void* scratch, size_t scratch_bytes,
                   uint16_t* out, size_t out_pitch, void* stream)
{
    ISA_REQ(data && table && scratch && out && width > 0 && height > 0 && nbytes > 0, "bad argument");
    ISA_REQ(out_pitch >= (size_t)width * 2 && out_pitch % 2 == 0, "bad output pitch");
    ISA_REQ(scratch_bytes >= isa_pef_decode_scratch(nbytes, width, height), "scratch too small (isa_pef_decode_scratch)");
    if ((nbytes * 8 / 1024 + 2 + 255) / 256 > (size_t)isa_pef_max_blocks()) return fail(ISA_EINVAL, "stream of %zu bytes too long", nbytes);
    ISA_REQ(table[0] == 12, "decode table must peek 12 bits (table[0] == 12)");
    for (int i = 1; i < 4097; i++) {
        const unsigned len = table[i] >> 8, cat = table[i] & 255;
        if (table[i] != 0 && (len < 1 || len > 12 || cat > 15)) return fail(ISA_EINVAL, "unsupported table entry %d (length %u, category %u)", i, len, cat);
    }
    ISA_CK(isa_launch_pef_decode(data, nbytes, table, width, height, scratch, out, out_pitch, S(stream)));
    return ISA_OK;
}

int isa_pef_unpack(const uint8_t* file, size_t file_size, const uint32_t* offsets, const uint32_t* sizes, int nstrips, int rows_per_strip, int width,
                   int height, int bit_depth, uint16_t* out, size_t out_pitch, void* stream)
{
    ISA_REQ(file && offsets && sizes && out && width > 0 && height > 0 && rows_per_strip > 0, "bad argument");
    ISA_REQ(nstrips >= 1 && nstrips <= 512, "1 to 512 strips");
    ISA_REQ(bit_depth >= 1 && bit_depth <= 16, "bit depth 1 to 16");
    ISA_REQ((long long)nstrips * rows_per_strip >= height, "the strips do not cover the frame");
    ISA_REQ(out_pitch >= (size_t)width * 2 && out_pitch % 2 == 0, "bad output pitch");
    ISA_CK(isa_launch_pef_unpack(file, file_size, offsets, sizes, nstrips, rows_per_strip, width, height, bit_depth, out, out_pitch, S(stream)));
    return ISA_OK;
}

int isa_pef_levels(const int cfa[4], const float* black_point, int n_black, float white_level, const float white_point[4], float scaling,
                   int bit_depth, float black[3], float white[3], float white_balance[3])
{
    ISA_REQ(cfa && white_point && black && white && white_balance, "NULL argument");
    ISA_REQ(cfa_ok(cfa), "CFA codes must be 0, 1, 2");
    ISA_REQ(n_black == 0 || (black_point && (n_black == 1 || n_black == 3 || n_black == 4)), "1, 3 or 4 black point values");
    const float white_all = white_level > 0 ? white_level : (float)std::pow(2.0, (double)bit_depth);
    float b[3] = {0.f, 0.f, 0.f};
    if (n_black == 1) {
        b[0] = b[1] = b[2] = black_point[0];
    } else if (n_black == 3) {
        b[0] = black_point[0]; b[1] = black_point[1]; b[2] = black_point[2];
    } else if (n_black == 4) {
        int ir = -1, ib = -1, ig1 = -1, ig2 = -1;
        for (int i = 0; i < 4; i++) {
            if (cfa[i] == 0 && ir < 0) ir = i;
            if (cfa[i] == 2 && ib < 0) ib = i;
            // the reference's loop: the first green, then the last green (:240-251)
            if (cfa[i] == 1 && ig1 < 0) ig1 = i;
            if (cfa[i] == 1 && ig1 >= 0) ig2 = i;
        }
        ISA_REQ(ir >= 0 && ib >= 0 && ig1 >= 0, "CFA without red, green and blue");
        b[0] = black_point[ir];
        b[2] = black_point[ib];
        b[1] = std::max(black_point[ig1], black_point[ig2]);
    }
    for (int c = 0; c < 3; c++) {
        black[c] = b[c];
        white[c] = white_all - b[c];
    }
    white_balance[0] = white_point[0] / scaling;
    white_balance[1] = white_point[1] / scaling;
    white_balance[2] = white_point[3] / scaling;
    return ISA_OK;
}

// ---- DNG colour specification (CameraToPCS and CameraWhite) ----
// Restates DNGColorSpec (PefFile/DNGColorSpec.cs:31-647), DNGTemperature
// (PefFile/DNGTemperature.cs, xy -> temperature) and DNGxyCoord
// (PefFile/DNGxyCoord.cs), all in FP64 with the reference's operation order.

namespace {

// Robertson's isotemperature lines (Robertson 1968, as tabulated in
// Wyszecki & Stiles): reciprocal megakelvin, u, v, slope.
const double kRobertson[31][4] = {
    {0, 0.18006, 0.26352, -0.24341},   {10, 0.18066, 0.26589, -0.25479},  {20, 0.18133, 0.26846, -0.26876},  {30, 0.18208, 0.27119, -0.28539},
    {40, 0.18293, 0.27407, -0.30470},  {50, 0.18388, 0.27709, -0.32675},  {60, 0.18494, 0.28021, -0.35156},  {70, 0.18611, 0.28342, -0.37915},
    {80, 0.18740, 0.28668, -0.40955},  {90, 0.18880, 0.28997, -0.44278},  {100, 0.19032, 0.29326, -0.47888}, {125, 0.19462, 0.30141, -0.58204},
    {150, 0.19962, 0.30921, -0.70471}, {175, 0.20525, 0.31647, -0.84901}, {200, 0.21142, 0.32312, -1.0182},  {225, 0.21807, 0.32909, -1.2168},
    {250, 0.22511, 0.33439, -1.4512},  {275, 0.23247, 0.33904, -1.7298},  {300, 0.24010, 0.34308, -2.0637},  {325, 0.24702, 0.34655, -2.4681},
    {350, 0.25591, 0.34951, -2.9641},  {375, 0.26400, 0.35200, -3.5814},  {400, 0.27218, 0.35407, -4.3633},  {425, 0.28039, 0.35577, -5.3762},
    {450, 0.28863, 0.35714, -6.7262},  {475, 0.29685, 0.35823, -8.5955},  {500, 0.30505, 0.35907, -11.324},  {525, 0.31320, 0.35968, -15.628},
    {550, 0.32129, 0.36011, -23.325},  {575, 0.32931, 0.36038, -40.770},  {600, 0.33724, 0.36051, -116.45}};

struct XY { double x, y; };
const XY kD50{0.3457, 0.3585};

struct V3 { double v[3]; };

V3 xy_to_xyz(XY c)
{
    double x = std::max(0.000001, std::min(c.x, 0.999999)), y = std::max(0.000001, std::min(c.y, 0.999999));
    if (x + y > 0.999999) {
        const double s = 0.999999 / (x + y);
        x *= s;
        y *= s;
    }
    return V3{{x / y, 1.0, (1.0 - x - y) / y}};
}

XY xyz_to_xy(const V3& c)
{
    const double total = c.v[0] + c.v[1] + c.v[2];
    if (total > 0.0) return XY{c.v[0] / total, c.v[1] / total};
    return kD50;
}

V3 mat_vec(const M3& m, const V3& a)
{
    V3 r;
    for (int j = 0; j < 3; j++) {
        double s = 0.0;
        for (int k = 0; k < 3; k++) s += m.a[j][k] * a.v[k];
        r.v[j] = s;
    }
    return r;
}

double max3(const V3& a) { return std::max(a.v[0], std::max(a.v[1], a.v[2])); }

M3 diag(const V3& a)
{
    M3 m{};
    for (int j = 0; j < 3; j++) m.a[j][j] = a.v[j];
    return m;
}

M3 ident3() { return diag(V3{{1.0, 1.0, 1.0}}); }

M3 scaled(double s, const M3& m)
{
    M3 r = m;
    for (int j = 0; j < 3; j++)
        for (int k = 0; k < 3; k++) r.a[j][k] *= s;
    return r;
}

M3 mat_add(const M3& a, const M3& b)
{
    M3 r = a;
    for (int j = 0; j < 3; j++)
        for (int k = 0; k < 3; k++) r.a[j][k] += b.a[j][k];
    return r;
}

M3 inv_or_throw(const M3& m, bool& ok)
{
    M3 r{};
    if (!mat_inv3(m, r)) ok = false;
    return r;
}

// DNGTemperature.xyCoord setter (DNGTemperature.cs:181-258): the temperature only.
double temperature_of(XY c)
{
    const double u = 2.0 * c.x / (1.5 - c.x + 6.0 * c.y);
    const double v = 3.0 * c.y / (1.5 - c.x + 6.0 * c.y);
    double last_dt = 0.0;
    for (int index = 1; index <= 30; index++) {
        double du = 1.0, dv = kRobertson[index][3];
        const double len = std::sqrt(1.0 + dv * dv);
        du /= len;
        dv /= len;
        const double uu = u - kRobertson[index][1], vv = v - kRobertson[index][2];
        double dt = -uu * dv + vv * du;
        if (dt <= 0.0 || index == 30) {
            if (dt > 0.0) dt = 0.0;
            dt = -dt;
            const double f = index == 1 ? 0.0 : dt / (last_dt + dt);
            return 1.0E6 / (kRobertson[index - 1][0] * f + kRobertson[index][0] * (1.0 - f));
        }
        last_dt = dt;
    }
    return 0.0;
}

// ConvertIlluminantToTemperature (DNGColorSpec.cs:122-172), EXIF LightSource codes.
double illuminant_temperature(int code)
{
    switch (code) {
    case 1: return 5500.0;                        // daylight
    case 2: return (3800.0 + 4500.0) * 0.5;       // fluorescent
    case 3: return 2850.0;                        // tungsten
    case 4: return 5500.0;                        // flash
    case 9: return 5500.0;                        // fine weather
    case 10: return 6500.0;                       // cloudy
    case 11: return 7500.0;                       // shade
    case 12: return (5700.0 + 7100.0) * 0.5;      // daylight fluorescent
    case 13: return (4600.0 + 5500.0) * 0.5;      // day white fluorescent
    case 14: return (3800.0 + 4500.0) * 0.5;      // cool white fluorescent
    case 15: return (3250.0 + 3800.0) * 0.5;      // white fluorescent
    case 16: return (2600.0 + 3250.0) * 0.5;      // warm white fluorescent
    case 17: return 2850.0;                       // standard light A
    case 18: return 5500.0;                       // B
    case 19: return 6500.0;                       // C
    case 20: return 5500.0;                       // D55
    case 21: return 6500.0;                       // D65
    case 22: return 7500.0;                       // D75
    case 23: return 5000.0;                       // D50
    case 24: return 3200.0;                       // ISO studio tungsten
    default: return 0.0;                          // unknown, other
    }
}

// MapWhiteMatrix (DNGColorSpec.cs:38-65): linearised Bradford adaptation white1 -> white2.
M3 map_white(XY w1, XY w2, bool& ok)
{
    const M3 Mb{{{0.8951, 0.2664, -0.1614}, {-0.7502, 1.7135, 0.0367}, {0.0389, -0.0685, 1.0296}}};
    V3 a = mat_vec(Mb, xy_to_xyz(w1)), b = mat_vec(Mb, xy_to_xyz(w2));
    for (int j = 0; j < 3; j++) {
        a.v[j] = std::max(a.v[j], 0.0);
        b.v[j] = std::max(b.v[j], 0.0);
    }
    M3 A{};
    for (int j = 0; j < 3; j++) A.a[j][j] = std::max(0.1, std::min(a.v[j] > 0.0 ? b.v[j] / a.v[j] : 10.0, 10.0));
    return mat_mul(mat_mul(inv_or_throw(Mb, ok), A), Mb);
}

struct ColorSpec {
    double t1, t2;
    M3 cm1, cm2, fm1, fm2, cc1, cc2, ab;
    bool cm2_set, fm1_set, fm2_set;
};

// NormalizeForwardMatrix (DNGColorSpec.cs:105-120)
M3 normalize_forward(const M3& m, bool& ok)
{
    const V3 xyz = mat_vec(m, V3{{1.0, 1.0, 1.0}});
    return mat_mul(mat_mul(diag(xy_to_xyz(kD50)), inv_or_throw(diag(xyz), ok)), m);
}

// FindXYZtoCamera (DNGColorSpec.cs:531-645); forward / calibration optional outputs.
M3 find_xyz_to_camera(const ColorSpec& s, XY white, M3* fm, bool* fm_set, M3* cc)
{
    const double T = temperature_of(white);
    double g;
    if (T <= s.t1) g = 1.0;
    else if (T >= s.t2) g = 0.0;
    else {
        const double invT = 1.0 / T;
        g = (invT - (1.0 / s.t2)) / ((1.0 / s.t1) - (1.0 / s.t2));
    }
    const auto mix = [&](const M3& a, const M3& b) { return g >= 1.0 ? a : (g <= 0.0 ? b : mat_add(scaled(g, a), scaled(1.0 - g, b))); };
    if (fm) {
        if (s.fm1_set && s.fm2_set) { *fm = mix(s.fm1, s.fm2); *fm_set = true; }
        else if (s.fm1_set) { *fm = s.fm1; *fm_set = true; }
        else if (s.fm2_set) { *fm = s.fm2; *fm_set = true; }
        else *fm_set = false;
    }
    if (cc) *cc = mix(s.cc1, s.cc2);
    return mix(s.cm1, s.cm2);
}

// NeutralToXY (DNGColorSpec.cs:490-529)
XY neutral_to_xy(const ColorSpec& s, const V3& neutral, bool& ok)
{
    XY last = kD50;
    for (int pass = 0; pass < 30; pass++) {
        const M3 xyz_to_cam = find_xyz_to_camera(s, last, nullptr, nullptr, nullptr);
        XY next = xyz_to_xy(mat_vec(inv_or_throw(xyz_to_cam, ok), neutral));
        if (std::fabs(next.x - last.x) + std::fabs(next.y - last.y) < 0.0000001) return next;
        if (pass == 29) {
            next.x = (last.x + next.x) * 0.5;
            next.y = (last.y + next.y) * 0.5;
        }
        last = next;
    }
    return last;
}

// The WhiteXY setter (DNGColorSpec.cs:404-466) for three channels.
void set_white(const ColorSpec& s, XY white, M3& camera_to_pcs, V3& camera_white, bool& ok)
{
    M3 fm{}, cc{};
    bool fm_set = false;
    const M3 cm = find_xyz_to_camera(s, white, &fm, &fm_set, &cc);
    camera_white = mat_vec(cm, xy_to_xyz(white));
    const double ws = 1.0 / max3(camera_white);
    for (int j = 0; j < 3; j++) camera_white.v[j] = std::max(0.001, std::min(ws * camera_white.v[j], 1.0));
    M3 pcs_to_camera = mat_mul(cm, map_white(kD50, white, ok));
    const double scale = max3(mat_vec(pcs_to_camera, xy_to_xyz(kD50)));
    pcs_to_camera = scaled(1.0 / scale, pcs_to_camera);
    if (fm_set) {
        const M3 ind_to_ref = inv_or_throw(mat_mul(s.ab, cc), ok);
        const V3 ref_white = mat_vec(ind_to_ref, camera_white);
        camera_to_pcs = mat_mul(mat_mul(fm, inv_or_throw(diag(ref_white), ok)), ind_to_ref);
    } else {
        camera_to_pcs = inv_or_throw(pcs_to_camera, ok);
    }
}

M3 m3_of(const double* p)
{
    M3 m;
    for (int j = 0; j < 3; j++)
        for (int k = 0; k < 3; k++) m.a[j][k] = p[j * 3 + k];
    return m;
}

int color_spec_out(const ColorSpec& s, XY white, double camera_to_pcs[9], double camera_white[3], double white_xy[2])
{
    bool ok = true;
    M3 c2p{};
    V3 cw{};
    set_white(s, white, c2p, cw, ok);
    if (!ok) return fail(ISA_ESINGULAR, "a colour matrix is singular");
    for (int j = 0; j < 3; j++)
        for (int k = 0; k < 3; k++) camera_to_pcs[j * 3 + k] = c2p.a[j][k];
    for (int j = 0; j < 3; j++) camera_white[j] = cw.v[j];
    if (white_xy) { white_xy[0] = white.x; white_xy[1] = white.y; }
    return ISA_OK;
}

}  // namespace

int isa_dng_color_spec(const isa_dng_color_tags* t, double camera_to_pcs[9], double camera_white[3], double white_xy[2])
{
    ISA_REQ(t && camera_to_pcs && camera_white, "NULL argument");
    ISA_REQ(t->as_shot_white_xy || t->as_shot_neutral, "one of AsShotWhiteXY and AsShotNeutral is needed (DNG specification)");
    bool ok = true;
    ColorSpec s;
    s.t1 = illuminant_temperature(t->illuminant1);
    s.t2 = illuminant_temperature(t->illuminant2);
    s.cm1 = t->color_matrix1 ? m3_of(t->color_matrix1) : ident3();
    s.cm2_set = t->color_matrix2 != nullptr;
    s.cm2 = s.cm2_set ? m3_of(t->color_matrix2) : M3{};
    s.fm1_set = t->forward_matrix1 != nullptr;
    s.fm2_set = t->forward_matrix2 != nullptr;
    s.fm1 = s.fm1_set ? m3_of(t->forward_matrix1) : M3{};
    s.fm2 = s.fm2_set ? m3_of(t->forward_matrix2) : M3{};
    s.cc1 = t->camera_calibration1 ? m3_of(t->camera_calibration1) : ident3();
    s.cc2 = t->camera_calibration2 ? m3_of(t->camera_calibration2) : ident3();
    s.ab = t->analog_balance ? diag(V3{{t->analog_balance[0], t->analog_balance[1], t->analog_balance[2]}}) : ident3();
    if (s.fm1_set) s.fm1 = normalize_forward(s.fm1, ok);
    s.cm1 = mat_mul(mat_mul(s.ab, s.cc1), s.cm1);
    if (!s.cm2_set || s.t1 <= 0.0 || s.t2 <= 0.0 || s.t1 == s.t2) {
        s.t1 = s.t2 = 5000.0;
        s.cm2 = s.cm1;
        s.fm2 = s.fm1;
        s.fm2_set = s.fm1_set;
        s.cc2 = s.cc1;
    } else {
        if (s.fm2_set) s.fm2 = normalize_forward(s.fm2, ok);
        s.cm2 = mat_mul(mat_mul(s.ab, s.cc2), s.cm2);
        if (s.t1 > s.t2) {
            std::swap(s.t1, s.t2);
            std::swap(s.cm1, s.cm2);
            std::swap(s.fm1, s.fm2);
            std::swap(s.fm1_set, s.fm2_set);
            std::swap(s.cc1, s.cc2);
        }
    }
    XY white;
    if (t->as_shot_white_xy) {
        white = XY{t->as_shot_white_xy[0], t->as_shot_white_xy[1]};
    } else {
        V3 vec{{t->as_shot_neutral[0], t->as_shot_neutral[1], t->as_shot_neutral[2]}};
        const double unify = 1.0 / max3(vec);
        for (int j = 0; j < 3; j++) vec.v[j] = unify * vec.v[j];
        white = neutral_to_xy(s, vec, ok);
    }
    if (!ok) return fail(ISA_ESINGULAR, "a colour matrix is singular");
    return color_spec_out(s, white, camera_to_pcs, camera_white, white_xy);
}

int isa_pef_color_spec(const float white_balance[3], double camera_to_pcs[9], double camera_white[3], double white_xy[2])
{
    ISA_REQ(white_balance && camera_to_pcs && camera_white, "NULL argument");
    for (int c = 0; c < 3; c++)
        if (!(white_balance[c] > 0.f) || !std::isfinite(white_balance[c])) return fail(ISA_EINVAL, "white balance must be positive");
    // PEFFile.SetMembers (PEFFile.cs:310-312): identity colour matrices under D50 for both illuminants
    bool ok = true;
    ColorSpec s;
    s.t1 = s.t2 = 5000.0;
    s.cm1 = s.cm2 = ident3();
    s.cm2_set = true;
    s.fm1_set = s.fm2_set = false;
    s.fm1 = s.fm2 = M3{};
    s.cc1 = s.cc2 = ident3();
    s.ab = ident3();
    // DNGColorSpec(..., float[] whiteBalance) (DNGColorSpec.cs:248-266): neutral = 1 / wb in float, scaled by 1 / max
    V3 vec;
    for (int c = 0; c < 3; c++) vec.v[c] = (double)(1.0f / white_balance[c]);
    const double unify = 1.0 / max3(vec);
    for (int c = 0; c < 3; c++) vec.v[c] = unify * vec.v[c];
    const XY white = neutral_to_xy(s, vec, ok);
    if (!ok) return fail(ISA_ESINGULAR, "a colour matrix is singular");
    return color_spec_out(s, white, camera_to_pcs, camera_white, white_xy);
}

int isa_profile_color_spec(const double* color_matrix1, const double* color_matrix2, int illuminant1, int illuminant2,
                           const float white_balance[3], double camera_to_pcs[9], double camera_white[3], double white_xy[2])
{
    ISA_REQ(white_balance && camera_to_pcs && camera_white, "NULL argument");
    for (int c = 0; c < 3; c++)
        if (!(white_balance[c] > 0.f) || !std::isfinite(white_balance[c])) return fail(ISA_EINVAL, "white balance must be positive");
    // DNGColorSpec.cs:175-266 is the tag constructor without forward matrices,
    // calibration and analog balance, its neutral being 1 / wb in float
    double neutral[3];
    for (int c = 0; c < 3; c++) neutral[c] = (double)(1.0f / white_balance[c]);
    isa_dng_color_tags t{};
    t.color_matrix1 = color_matrix1;
    t.color_matrix2 = color_matrix2;
    t.illuminant1 = illuminant1;
    t.illuminant2 = illuminant2;
    t.as_shot_neutral = neutral;
    return isa_dng_color_spec(&t, camera_to_pcs, camera_white, white_xy);
}

// ---- Raw-file metadata ----

int isa_noise_model(int iso, const int* isos, const double* alpha, const double* beta, int n, double ab[2])
{
    ISA_REQ(ab && n >= 0 && (n == 0 || (isos && alpha && beta)), "NULL argument or negative count");
    if (n == 0) {
        ab[0] = ab[1] = 0.0;
        return ISA_OK;
    }
    int index = -1;  // the last ISO not above the asked one (ExtraCameraProfiles.cs:171-179)
    for (int i = n - 1; i >= 0; i--)
        if (isos[i] <= iso) {
            index = i;
            break;
        }
    if (index == n - 1) {
        ab[0] = alpha[n - 1];
        ab[1] = beta[n - 1];
    } else if (index < 0) {
        ab[0] = alpha[0];
        ab[1] = beta[0];
    } else {
        const double w = ((double)iso - (double)isos[index + 1]) / ((double)isos[index] - (double)isos[index + 1]);
        ab[0] = w * alpha[index] + (1.0 - w) * alpha[index + 1];
        ab[1] = w * beta[index] + (1.0 - w) * beta[index + 1];
    }
    return ISA_OK;
}

int isa_crop_window(int left, int top, int cropped_width, int cropped_height, int width, int height, int crop[4])
{
    ISA_REQ(crop, "NULL argument");
    crop[0] = std::max(2, left);
    crop[1] = std::max(2, top);
    crop[2] = cropped_width - std::max(0, (left + cropped_width) - (width - 2));
    crop[3] = cropped_height - std::max(0, (top + cropped_height) - (height - 2));
    return ISA_OK;
}

namespace {

// C#'s Math.Max(float, float): NaN when either is NaN.
float cs_maxf(float a, float b)
{
    if (a != a || b != b) return std::numeric_limits<float>::quiet_NaN();
    return a > b ? a : b;
}

// (int) of a tag's rational, truncated toward zero; false when it does not fit.
bool to_int(double v, int& out)
{
    if (!(v > -2147483649.0 && v < 2147483648.0)) return false;
    out = (int)v;
    return true;
}

}  // namespace

int isa_dng_levels(const isa_dng_level_tags* t, isa_raw_levels* out, uint16_t* black_h, uint16_t* black_v)
{
    ISA_REQ(t && out && t->cfa_pattern && t->camera_white, "NULL argument");
    ISA_REQ(t->width > 0 && t->height > 0, "bad size");
    ISA_REQ(t->cfa_repeat_w == 2 && t->cfa_repeat_h == 2, "the CFA repeat pattern must be 2 x 2 (DNGFile.cs:706-712)");
    const int W = t->width, H = t->height;
    int cfa[4];
    for (int i = 0; i < 4; i++) cfa[i] = t->cfa_pattern[i];
    ISA_REQ(cfa_ok(cfa), "CFA codes must be 0, 1, 2");
    // CFAPlaneColor: plane order and the reordering twist (:719-746)
    int plane[3] = {0, 1, 2};
    float twist[12] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0};
    int identity = 1;
    if (t->plane_color) {
        ISA_REQ(t->n_plane_color == 3, "CFAPlaneColor must hold three planes");
        for (int k = 0; k < 12; k++) twist[k] = 0.f;
        for (int i = 0; i < 3; i++) {
            const int color = t->plane_color[i];
            ISA_REQ(color >= 0 && color <= 2, "CFAPlaneColor names a colour other than red, green, blue");
            plane[i] = color;
            twist[color * 4 + i] = 1.f;
            if (color != i) identity = 0;
        }
    }
    // BlackLevel (:757-824), on the CFA as stored (before the active-area shift)
    float black[3] = {0.f, 0.f, 0.f};
    if (t->black_level) {
        const double* bl = t->black_level;
        if (t->n_black == 1) {
            black[0] = black[1] = black[2] = (float)bl[0];
        } else if (t->n_black == 3) {
            for (int i = 0; i < 3; i++) black[plane[i]] = (float)bl[i];
        } else if (t->n_black == 4) {
            int ir = -1, ib = -1, ig1 = -1, ig2 = -1;
            for (int i = 0; i < 4; i++)
                if (cfa[i] == 0) { ir = i; break; }
            for (int i = 0; i < 4; i++)
                if (cfa[i] == 2) { ib = i; break; }
            for (int i = 0; i < 4; i++) {  // the first green, then the last (:809-818)
                if (cfa[i] == 1 && ig1 == -1) ig1 = i;
                if (cfa[i] == 1 && ig1 != -1) ig2 = i;
            }
            ISA_REQ(ir >= 0 && ib >= 0 && ig1 >= 0, "a CFA without red, green and blue has no per-position black levels");
            black[0] = (float)bl[ir];
            black[2] = (float)bl[ib];
            black[1] = cs_maxf((float)bl[ig1], (float)bl[ig2]);
        }
    }
    const float white_all = (float)t->white_level;
    float white[3];
    for (int c = 0; c < 3; c++) white[c] = white_all - black[c];
    float wb[3];
    for (int i = 0; i < 3; i++) wb[plane[i]] = 1.0f / (float)t->camera_white[i];
    // ActiveArea and DefaultCrop (:861-948)
    int crop_left = 0, crop_top = 0, crop_w = W, crop_h = H;
    const int* aa = t->active_area;
    if (aa) {
        const int top = aa[0], left = aa[1], bottom = aa[2], right = aa[3];
        crop_left += left;
        crop_top += top;
        crop_w = right - left;
        crop_h = bottom - top;
        if (top % 2 != 0) {
            const int c0 = cfa[0], c1 = cfa[1];
            cfa[0] = cfa[2];
            cfa[1] = cfa[3];
            cfa[2] = c0;
            cfa[3] = c1;
        }
        if (left % 2 != 0) {
            const int c0 = cfa[0], c2 = cfa[2];
            cfa[0] = cfa[1];
            cfa[2] = cfa[3];
            cfa[1] = c0;
            cfa[3] = c2;
        }
    }
    if (t->default_crop_origin && t->default_crop_size) {
        int left, top, w, h;  // entry 0 of each tag for both coordinates, as the reference reads them (:910-915)
        ISA_REQ(to_int(t->default_crop_origin[0], left) && to_int(t->default_crop_size[0], w), "crop out of range");
        top = left;
        h = w;
        crop_left += left;
        crop_top += top;
        crop_w = w;
        crop_h = h;
    }
    int crop[4];
    isa_crop_window(crop_left, crop_top, crop_w, crop_h, W, H, crop);
    // NoiseProfile (:950-967), then an ExtraCameraProfiles noise model with alpha != 0 (:296-320)
    float alpha = 0.f, beta = 0.f;
    if (t->noise_profile) {
        ISA_REQ(t->n_noise >= 2, "NoiseProfile needs two values");
        if (t->n_noise > 2) {
            ISA_REQ(plane[1] * 2 + 1 < t->n_noise, "NoiseProfile too short for the green plane");
            alpha = (float)t->noise_profile[plane[1] * 2];
            beta = (float)t->noise_profile[plane[1] * 2 + 1];
        } else {
            alpha = (float)t->noise_profile[0];
            beta = (float)t->noise_profile[1];
        }
    }
    if (t->n_profile > 0) {
        double ab[2];
        if (isa_noise_model(t->iso, t->profile_iso, t->profile_alpha, t->profile_beta, t->n_profile, ab) != ISA_OK) return ISA_EINVAL;
        if (ab[0] != 0.0) {
            alpha = (float)ab[0];
            beta = (float)ab[1];
        }
    }
    // BlackLevelDeltaV / H placed in the active area (:324-372); the white
    // level loses the largest black of a decoded pixel (:607-609), which for
    // non-negative deltas over a fully decoded frame is max(V) + max(H)
    const int off_v = aa ? aa[0] : 0, off_h = aa ? aa[1] : 0;
    const int border_bottom = aa ? H - aa[2] : 0, border_right = aa ? W - aa[3] : 0;
    int max_v = 0, max_h = 0;
    if (black_v) std::memset(black_v, 0, sizeof(uint16_t) * (size_t)H);
    if (black_h) std::memset(black_h, 0, sizeof(uint16_t) * (size_t)W);
    if (t->black_delta_v) {
        ISA_REQ(t->n_delta_v + off_v + border_bottom == H && off_v >= 0 && t->n_delta_v >= 0, "BlackLevelDeltaV does not fit the image height");
        for (int i = 0; i < t->n_delta_v; i++) {
            const double v = t->black_delta_v[i];
            ISA_REQ(v > -1.0 && v < 65536.0, "BlackLevelDeltaV value outside 0..65535");
            const int u = (uint16_t)(int)v;
            max_v = std::max(max_v, u);
            if (black_v) black_v[off_v + i] = (uint16_t)u;
        }
    }
    if (t->black_delta_h) {
        ISA_REQ(t->n_delta_h + off_h + border_right == W && off_h >= 0 && t->n_delta_h >= 0, "BlackLevelDeltaH does not fit the image width");
        for (int i = 0; i < t->n_delta_h; i++) {
            const double v = t->black_delta_h[i];
            ISA_REQ(v > -1.0 && v < 65536.0, "BlackLevelDeltaH value outside 0..65535");
            const int u = (uint16_t)(int)v;
            max_h = std::max(max_h, u);
            if (black_h) black_h[off_h + i] = (uint16_t)u;
        }
    }
    const int max_black = max_v + max_h;
    isa_raw_levels r{};
    r.info.width = W;
    r.info.height = H;
    for (int i = 0; i < 4; i++) r.info.cfa[i] = cfa[i];
    for (int c = 0; c < 3; c++) {
        r.info.black[c] = black[c];
        r.info.white[c] = white[c] - (float)max_black;
        r.info.camera_white[c] = (float)t->camera_white[c];
        r.white_balance[c] = wb[c];
    }
    r.info.noise_alpha = alpha;
    r.info.noise_beta = beta;
    for (int k = 0; k < 12; k++) r.color_twist[k] = twist[k];
    r.color_twist_identity = identity;
    for (int k = 0; k < 4; k++) r.crop[k] = crop[k];
    *out = r;
    return ISA_OK;
}

// ---- DNG pixel data ----

namespace {

// ljpeg_start (DNGFile.cs:94-170) on the host: the frame header, the
// Huffman tables (make_decoder_ref, :73-92) and the entropy data's offset.
struct Lj92Header {
    int algo = 0, bits = 0, high = 0, wide = 0, clrs = 0, sraw = 0, psv = 0, restart = 0x7fffffff;
    std::string huff[20];   // per table: the 16 code-length counts and the values make_decoder_ref reads
    int huff_of[20];
    size_t data = 0;
};

// make_decoder_ref's table (1 + 2^max entries, entry 0 = max) from a table's counts and values.
std::vector<uint16_t> lj92_table(const std::string& spec)
{
    const uint8_t* cnt = (const uint8_t*)spec.data();
    int max;
    for (max = 16; max > 0 && cnt[max - 1] == 0; max--) ;
    std::vector<uint16_t> t((size_t)1 + ((size_t)1 << max), 0);
    t[0] = (uint16_t)max;
    size_t dp = 16;
    int hh = 1;
    for (int ln = 1; ln <= max; ln++)
        for (int i = 0; i < cnt[ln - 1]; i++, ++dp)
            for (int j = 0; j < 1 << (max - ln); j++)
                if (hh <= 1 << max) t[hh++] = (uint16_t)(ln << 8 | (uint8_t)spec[dp]);
    return t;
}

// The reader's segment buffer: zero at every call's start, as the reference
// allocates a fresh one (DNGFile.cs:98); the bytes a call wrote are cleared
// when it returns.
struct SegmentBuffer {
    std::vector<uint8_t>& data;
    size_t used = 0;
    explicit SegmentBuffer(std::vector<uint8_t>& d) : data(d) {}
    ~SegmentBuffer() { std::memset(data.data(), 0, std::min(used, data.size())); }
};

bool lj92_start(const uint8_t* d, size_t n, Lj92Header& h)
{
    size_t pos = 0;
    const auto rd = [&]() -> int { return pos < n ? d[pos++] : (pos++, -1); };
    for (int c = 0; c < 20; c++) h.huff_of[c] = -1;
    rd();
    if (rd() != 0xd8) return false;
    static thread_local std::vector<uint8_t> buffer(0x10000);
    SegmentBuffer seg(buffer);
    std::vector<uint8_t>& data = buffer;
    int tag;
    do {
        seg.used = std::max<size_t>(seg.used, 4);
        for (int k = 0; k < 4; k++) {
            const int b = rd();
            if (b < 0) return false;
            data[k] = (uint8_t)b;
        }
        tag = data[0] << 8 | data[1];
        const int len = (data[2] << 8 | data[3]) - 2;
        if (tag <= 0xff00) return false;
        seg.used = std::max<size_t>(seg.used, (size_t)std::max(len, 0));
        for (int got = 0; got < len; got++) {
            const int b = rd();
            if (b < 0) { pos--; break; }
            data[got] = (uint8_t)b;
        }
        switch (tag) {
        case 0xffc3:
            h.sraw = ((data[7] >> 4) * (data[7] & 15) - 1) & 3;
            h.algo = tag & 0xff;
            h.bits = data[0];
            h.high = data[1] << 8 | data[2];
            h.wide = data[3] << 8 | data[4];
            h.clrs = data[5] + h.sraw;
            break;
        case 0xffc1:
        case 0xffc0:
            h.algo = tag & 0xff;
            h.bits = data[0];
            h.high = data[1] << 8 | data[2];
            h.wide = data[3] << 8 | data[4];
            h.clrs = data[5] + h.sraw;
            break;
        case 0xffc4: {
            size_t dp = 0;
            int c;
            while (dp < (size_t)std::max(len, 0) && ((c = data[dp++]) & -20) == 0) {
                // make_decoder_ref: counts of lengths 1..16, then the values (expanded by lj92_table)
                const size_t cnt0 = dp;
                dp += 16;
                int max;
                for (max = 16; max > 0 && data[cnt0 + max - 1] == 0; max--) ;
                std::string spec((const char*)&data[cnt0], 16);
                for (int ln = 1; ln <= max; ln++)
                    for (int i = 0; i < data[cnt0 + ln - 1]; i++, ++dp) spec.push_back((char)(dp < data.size() ? data[dp] : 0));
                h.huff[c] = spec;
                h.huff_of[c] = c;
            }
            break;
        }
        case 0xffda:
            h.psv = data[1 + data[0] * 2];
            h.bits -= data[3 + data[0] * 2] & 15;
            break;
        case 0xffdd:
            h.restart = data[0] << 8 | data[1];
            break;
        }
    } while (tag != 0xffda);
    for (int c = 0; c < 19; c++)
        if (h.huff_of[c + 1] < 0) h.huff_of[c + 1] = h.huff_of[c];
    h.data = pos;
    return true;
}

struct DngPlan {
    std::vector<unsigned char> parts;       // Lj92Part records
    std::vector<uint16_t> tables;           // distinct tables, concatenated
    size_t row_samples = 0;                 // two-row buffers of all parts, in uint16
    int nparts = 0;
    int jwide_max = 1;                      // the widest row of samples
};

int dng_plan(const uint8_t* file, size_t fsize, const isa_dng_layout* L, int W, int H, DngPlan& plan)
{
    plan.nparts = L->n;
    plan.parts.assign((size_t)L->n * isa_dng_part_bytes(), 0);
    std::map<std::string, int> seen;
    int row = 0, col = 0;
    for (int t = 0; t < L->n; t++) {
        const size_t o = L->offsets[t];
        const size_t end = std::min<size_t>(fsize, o + (size_t)L->byte_counts[t]);
        Lj92Header h;
        const bool ok = o < fsize && lj92_start(file + o, end - o, h) && h.algo == 0xc3;
        int hdr[7] = {h.bits, h.high, h.wide, h.clrs, h.sraw, h.psv, h.restart};
        int tab[6] = {0, 0, 0, 0, 0, 0};
        bool skip = !ok;
        if (ok) {
            if (h.clrs < 1 || h.clrs > 6 || h.wide < 1 || h.high < 0 || h.bits < 1 || h.bits > 16 || h.restart <= 0)
                return fail(ISA_EINVAL, "part %d: unsupported lossless-JPEG header (%d components, %d bits)", t, h.clrs, h.bits);
            for (int c = 0; c < h.clrs; c++) {
                const int k = h.huff_of[c];
                if (k < 0) return fail(ISA_EINVAL, "part %d: no Huffman table for component %d", t, c);
                auto it = seen.find(h.huff[k]);
                if (it == seen.end()) {
                    it = seen.emplace(h.huff[k], (int)plan.tables.size()).first;
                    const std::vector<uint16_t> t = lj92_table(h.huff[k]);
                    plan.tables.insert(plan.tables.end(), t.begin(), t.end());
                }
                tab[c] = it->second;
            }
        }
        const int orow = L->tiled ? row : t * L->rows_per_strip, ocol = L->tiled ? col : 0;
        const unsigned long long rb = plan.row_samples;
        if (ok) {
            plan.row_samples += (size_t)2 * h.wide * h.clrs + 8;
            plan.jwide_max = std::max(plan.jwide_max, h.wide * h.clrs);
        }
        isa_dng_part_set(plan.parts.data(), t, (unsigned long long)(o + h.data), (unsigned long long)end, skip ? 1 : 0, hdr, orow, ocol, tab, rb);
        if (L->tiled) {
            col += L->tile_width;
            if (col >= W) { col = 0; row += L->tile_height; }
        }
    }
    (void)H;
    return ISA_OK;
}

size_t align256(size_t v) { return (v + 255) / 256 * 256; }

}  // namespace

int isa_dng_check(const isa_dng_layout* L, int width, int height)
{
    ISA_REQ(L && width > 0 && height > 0 && L->n >= 1 && L->offsets && L->byte_counts, "bad DNG layout");
    ISA_REQ(L->compression == 7 || (L->compression == 1 && !L->tiled), "lossless JPEG tiles/strips or uncompressed strips only");
    ISA_REQ(!L->tiled || (L->tile_width > 0 && L->tile_height > 0), "tile size");
    ISA_REQ(L->tiled || L->rows_per_strip > 0, "rows per strip");
    ISA_REQ(L->compression != 1 || (L->bit_depth >= 1 && L->bit_depth <= 16), "bit depth 1 to 16");
    ISA_REQ(!L->linearization || L->nlin > 0, "empty linearisation table");
    return ISA_OK;
}

namespace {

// Scratch of isa_dng_decode for a checked layout and, for lossless JPEG, its plan.
size_t dng_scratch_bytes(const isa_dng_layout* L, int width, int height, const DngPlan& plan)
{
    size_t s = align256((size_t)L->n * 16) + align256((size_t)L->n * 8) + align256((size_t)L->n * 8) + align256(64);
    s += align256((size_t)width * 2) + align256((size_t)height * 2) + align256((size_t)std::max(L->nlin, 1) * 2);
    if (L->compression == 7) {
        s += align256(plan.parts.size()) + align256(plan.tables.size() * 2 + 2) + align256(plan.row_samples * 2 + 16);
        s += align256(isa_dngf_scratch(plan.parts.data(), plan.nparts, plan.tables.data(), plan.tables.size(), L->dng_version_large));
    }
    return s;
}

}  // namespace

size_t isa_dng_decode_scratch(const uint8_t* file_host, size_t file_size, const isa_dng_layout* L, int width, int height)
{
    if (!file_host || isa_dng_check(L, width, height) != ISA_OK) return 0;
    DngPlan plan;
    if (L->compression == 7 && dng_plan(file_host, file_size, L, width, height, plan) != ISA_OK) return 0;
    return dng_scratch_bytes(L, width, height, plan);
}

int isa_dng_decode_path(void) { return g_dng_path; }

namespace {

constexpr int kDngErr0 = 0x7fffffff;  // no part failed

// The device buffers of one isa_dng_decode call inside its scratch (the order of dng_scratch_bytes).
struct DngBuffers {
    unsigned long long* offs;
    unsigned long long* cnts;
    int* err;
    uint16_t *bh, *bv, *lin;
    void* parts = nullptr;
    uint16_t* tables = nullptr;
    uint16_t* rows = nullptr;
    char* fast = nullptr;
    size_t fast_bytes = 0;
};

DngBuffers dng_buffers(char* base, const isa_dng_layout* L, int width, int height, const DngPlan& plan)
{
    DngBuffers b;
    size_t o = 0;
    const auto take = [&](size_t bytes) { char* p = base + o; o += align256(bytes); return p; };
    take((size_t)L->n * 16);
    b.offs = (unsigned long long*)take((size_t)L->n * 8);
    b.cnts = (unsigned long long*)take((size_t)L->n * 8);
    b.err = (int*)take(64);
    b.bh = (uint16_t*)take((size_t)width * 2);
    b.bv = (uint16_t*)take((size_t)height * 2);
    b.lin = (uint16_t*)take((size_t)std::max(L->nlin, 1) * 2);
    if (L->compression == 7) {
        b.parts = take(plan.parts.size());
        b.tables = (uint16_t*)take(plan.tables.size() * 2 + 2);
        b.rows = (uint16_t*)take(plan.row_samples * 2 + 16);
        b.fast_bytes = isa_dngf_scratch(plan.parts.data(), plan.nparts, plan.tables.data(), plan.tables.size(), L->dng_version_large);
        if (b.fast_bytes > 0) b.fast = take(b.fast_bytes);
    }
    return b;
}

// Checks, plan and the uploads every decode starts with; the output is cleared.
int dng_prologue(const uint8_t* file_host, const uint8_t* file_dev, size_t file_size, const isa_dng_layout* L, int width, int height,
                 void* scratch, size_t scratch_bytes, uint16_t* out, size_t out_pitch, cudaStream_t st, DngPlan& plan, DngBuffers& b)
{
    ISA_REQ(file_host && file_dev && scratch && out, "NULL argument");
    ISA_TRY(isa_dng_check(L, width, height));
    ISA_REQ(out_pitch >= (size_t)width * 2 && out_pitch % 2 == 0, "bad output pitch");
    if (L->compression == 7) ISA_TRY(dng_plan(file_host, file_size, L, width, height, plan));
    ISA_REQ(scratch_bytes >= dng_scratch_bytes(L, width, height, plan), "scratch too small (isa_dng_decode_scratch)");
    if (L->compression == 7 && (size_t)4 * (4096 + 4 * (size_t)plan.jwide_max + 64) > 227 * 1024)
        return fail(ISA_EINVAL, "rows of %d samples exceed the decoder's shared-memory row buffers", plan.jwide_max);
    b = dng_buffers((char*)scratch, L, width, height, plan);
    std::vector<unsigned long long> offs(L->n), cnts(L->n);
    for (int i = 0; i < L->n; i++) { offs[i] = L->offsets[i]; cnts[i] = L->byte_counts[i]; }
    ISA_CK(cudaMemcpyAsync(b.offs, offs.data(), offs.size() * 8, cudaMemcpyHostToDevice, st));
    ISA_CK(cudaMemcpyAsync(b.cnts, cnts.data(), cnts.size() * 8, cudaMemcpyHostToDevice, st));
    ISA_CK(cudaMemcpyAsync(b.err, &kDngErr0, sizeof(int), cudaMemcpyHostToDevice, st));
    if (L->black_h) ISA_CK(cudaMemcpyAsync(b.bh, L->black_h, (size_t)width * 2, cudaMemcpyHostToDevice, st));
    if (L->black_v) ISA_CK(cudaMemcpyAsync(b.bv, L->black_v, (size_t)height * 2, cudaMemcpyHostToDevice, st));
    if (L->linearization) ISA_CK(cudaMemcpyAsync(b.lin, L->linearization, (size_t)L->nlin * 2, cudaMemcpyHostToDevice, st));
    ISA_CK(cudaMemset2DAsync(out, out_pitch, 0, (size_t)width * 2, height, st));
    if (L->compression == 7) {
        ISA_CK(cudaMemcpyAsync(b.parts, plan.parts.data(), plan.parts.size(), cudaMemcpyHostToDevice, st));
        if (!plan.tables.empty()) ISA_CK(cudaMemcpyAsync(b.tables, plan.tables.data(), plan.tables.size() * 2, cudaMemcpyHostToDevice, st));
    }
    return ISA_OK;
}

int dng_launch_fast(const uint8_t* file_dev, size_t file_size, const isa_dng_layout* L, int width, int height, uint16_t* out, size_t out_pitch,
                    const DngPlan& plan, const DngBuffers& b, int* anomaly_host, cudaStream_t st)
{
    ISA_CK(isa_launch_dngf(file_dev, file_size, plan.parts.data(), plan.nparts, plan.tables.data(), plan.tables.size(),
                           L->linearization ? b.lin : nullptr, L->nlin, L->black_h ? b.bh : nullptr, L->black_v ? b.bv : nullptr, width, height,
                           L->dng_version_large, out, out_pitch, b.err, b.fast, b.fast_bytes, anomaly_host, st));
    return ISA_OK;
}

int dng_error(int err)
{
    if (err != kDngErr0) return fail(ISA_EINVAL, "part %d: a decoded sample exceeds the frame's bit depth (the reference stops there)", err);
    return ISA_OK;
}

// The per-part reader (every layout; the frames the parallel decoder hands back), synchronised.
int dng_sequential(const uint8_t* file_dev, size_t file_size, const isa_dng_layout* L, int width, int height, uint16_t* out, size_t out_pitch,
                   const DngPlan& plan, const DngBuffers& b, bool clear, cudaStream_t st)
{
    if (clear) {
        ISA_CK(cudaMemcpyAsync(b.err, &kDngErr0, sizeof(int), cudaMemcpyHostToDevice, st));
        ISA_CK(cudaMemset2DAsync(out, out_pitch, 0, (size_t)width * 2, height, st));
    }
    g_dng_path = L->compression == 7 ? 0 : -1;
    ISA_CK(isa_launch_dng(file_dev, file_size, L->compression, b.parts, L->n, b.tables, b.rows, b.offs, b.cnts, L->rows_per_strip, L->bit_depth,
                          L->linearization ? b.lin : nullptr, L->nlin, L->black_h ? b.bh : nullptr, L->black_v ? b.bv : nullptr, width, height,
                          L->dng_version_large, out, out_pitch, b.err, st, plan.jwide_max, (int)plan.tables.size()));
    int err = kDngErr0;
    ISA_CK(cudaMemcpyAsync(&err, b.err, sizeof(int), cudaMemcpyDeviceToHost, st));
    ISA_CK(cudaStreamSynchronize(st));
    return dng_error(err);
}

// After the parallel decoder: its flags, and the per-part reader when it handed the frame back.
int dng_settle(const uint8_t* file_dev, size_t file_size, const isa_dng_layout* L, int width, int height, uint16_t* out, size_t out_pitch,
               const DngPlan& plan, const DngBuffers& b, cudaStream_t st)
{
    const size_t flag = isa_dngf_flag_offset(plan.parts.data(), plan.nparts, plan.tables.data(), plan.tables.size(), L->dng_version_large);
    int anomaly = 1, err = kDngErr0;
    ISA_CK(cudaStreamSynchronize(st));
    ISA_CK(cudaMemcpy(&anomaly, b.fast + flag, sizeof(int), cudaMemcpyDeviceToHost));
    ISA_CK(cudaMemcpy(&err, b.err, sizeof(int), cudaMemcpyDeviceToHost));
    if (anomaly == 0) {
        g_dng_path = 1;
        return dng_error(err);
    }
    return dng_sequential(file_dev, file_size, L, width, height, out, out_pitch, plan, b, true, st);
}

}  // namespace

int isa_dng_decode(const uint8_t* file_host, const uint8_t* file_dev, size_t file_size, const isa_dng_layout* L, int width, int height,
                   void* scratch, size_t scratch_bytes, uint16_t* out, size_t out_pitch, void* stream)
{
    g_dng_path = -1;
    cudaStream_t st = S(stream);
    DngPlan plan;
    DngBuffers b;
    ISA_TRY(dng_prologue(file_host, file_dev, file_size, L, width, height, scratch, scratch_bytes, out, out_pitch, st, plan, b));
    if (b.fast) {
        ISA_TRY(dng_launch_fast(file_dev, file_size, L, width, height, out, out_pitch, plan, b, nullptr, st));
        return dng_settle(file_dev, file_size, L, width, height, out, out_pitch, plan, b, st);
    }
    return dng_sequential(file_dev, file_size, L, width, height, out, out_pitch, plan, b, false, st);
}

int isa_dng_decode_begin(const uint8_t* file_host, const uint8_t* file_dev, size_t file_size, const isa_dng_layout* L, int width, int height,
                         void* scratch, size_t scratch_bytes, uint16_t* out, size_t out_pitch, void* stream)
{
    g_dng_path = -1;
    cudaStream_t st = S(stream);
    DngPlan plan;
    DngBuffers b;
    ISA_TRY(dng_prologue(file_host, file_dev, file_size, L, width, height, scratch, scratch_bytes, out, out_pitch, st, plan, b));
    if (b.fast) return dng_launch_fast(file_dev, file_size, L, width, height, out, out_pitch, plan, b, nullptr, st);
    return dng_sequential(file_dev, file_size, L, width, height, out, out_pitch, plan, b, false, st);
}

int isa_dng_decode_finish(const uint8_t* file_host, const uint8_t* file_dev, size_t file_size, const isa_dng_layout* L, int width, int height,
                          void* scratch, size_t scratch_bytes, uint16_t* out, size_t out_pitch, void* stream)
{
    g_dng_path = -1;
    ISA_REQ(file_host && file_dev && scratch && out, "NULL argument");
    ISA_TRY(isa_dng_check(L, width, height));
    ISA_REQ(out_pitch >= (size_t)width * 2 && out_pitch % 2 == 0, "bad output pitch");
    cudaStream_t st = S(stream);
    DngPlan plan;
    if (L->compression == 7) ISA_TRY(dng_plan(file_host, file_size, L, width, height, plan));
    ISA_REQ(scratch_bytes >= dng_scratch_bytes(L, width, height, plan), "scratch too small (isa_dng_decode_scratch)");
    const DngBuffers b = dng_buffers((char*)scratch, L, width, height, plan);
    if (!b.fast) {  // isa_dng_decode_begin already decoded it with the per-part reader and waited
        g_dng_path = L->compression == 7 ? 0 : -1;
        return ISA_OK;
    }
    return dng_settle(file_dev, file_size, L, width, height, out, out_pitch, plan, b, st);
}
