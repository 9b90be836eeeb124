/*
 * isa.h -- C ABI of the B200 burst-merge library (libisa.so).
 *
 * Drop-in for the GPU hot path of ImageStackAlignator (PEFStudioDX): the
 * per-kernel operator wrappers (PEFStudioDX/*Kernels.cs, one CudaKernel
 * subclass per __global__) and the controller steps that chain them
 * (ImageStackAlignatorController.cs TrackPatches :1601, PrepareAccumulation
 * :1795, Accumulate :1928). Every declaration names the reference interface
 * it replaces.
 *
 * Conventions
 *  - Images are device pointers with a row pitch in bytes, channels
 *    interleaved, as the reference's NPPImage_* buffers: float (32fC1),
 *    float2 flow (32fC2), float3 RGB (32fC3), float4 masks / kernels (32fC4),
 *    uint16 Bayer frames (16uC1).
 *  - CFA: int cfa[4] = colour codes at (row 0, col 0), (0, 1), (1, 0), (1, 1);
 *    R = 0, G = 1, B = 2 (RawFile.BayerColor, PefFile/RawFile.cs:30-39,
 *    set through c_cfaPattern in DeBayerKernels.cs:53-63).
 *  - Every call returns an int status (ISA_OK or a negative ISA_E* code) and
 *    never throws; isa_last_error() gives the message of the calling
 *    thread's last failure. Work is ordered on the caller's stream (a
 *    cudaStream_t passed as void*, NULL = legacy default stream). Per-op
 *    entry points allocate nothing; isa_ctx owns all scratch of the fused
 *    pipeline and is created once (isa_ctx_create) per maximum size.
 *  - An isa_ctx must not be used by two host threads at once.
 */
#ifndef ISA_H
#define ISA_H

#include <stddef.h>
#include <stdint.h>

#if defined(_WIN32)
#define ISA_API __declspec(dllexport)
#elif defined(__GNUC__)
#define ISA_API __attribute__((visibility("default")))
#else
#define ISA_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define ISA_OK 0
#define ISA_EINVAL (-1)      /* bad size, pointer or parameter */
#define ISA_ECUDA (-2)       /* a CUDA runtime call or kernel launch failed */
#define ISA_ESINGULAR (-3)   /* reported per tile in the solver status array, never returned */
#define ISA_ETIMEDOUT (-4)   /* reserved for bounded waits */
#define ISA_ENOMEM (-5)      /* device allocation failed (isa_ctx_create only) */

#define ISA_MAX_LEVELS 8

/* Tracking strategies of ShiftCollection.TrackingStrategy (ShiftCollection.cs:36-47). */
#define ISA_TRACK_FULL 0
#define ISA_TRACK_ONLY_ON_REFERENCE 1
#define ISA_TRACK_ON_REFERENCE_BLOCK 2
#define ISA_TRACK_BLOCKS 3

/* How the accumulation and the robustness mask read a frame at the flow.
 * ROUND: at the integer shift round(s * flow) and round(flow / 2), as the
 * reference does (DeBayerKernels.cu:310-311, 403-404; RobustnessModell.cu:
 * 401-402); the merge is piecewise constant in the flow. BILINEAR: the
 * contributions at the four integer shifts around the flow, blended with
 * the bilinear weights of its fractional part (equal to ROUND at integer
 * flow); the merge is continuous in the flow and isa_merge_backward_tiles
 * returns its gradient with respect to the tile flow. No counterpart in the
 * reference. */
#define ISA_SAMPLE_ROUND 0
#define ISA_SAMPLE_BILINEAR 1

/* PatchTrackingLevel (PatchTrackingLevel.cs:27-63). */
typedef struct isa_level {
    int resize_level;
    int tile_size;
    int max_shift;
} isa_level;

/* Controller parameters with the reference names and defaults
 * (ImageStackAlignatorController.cs:443-675), plus extensions that default
 * to the reference behaviour. */
typedef struct isa_params {
    float sigma_debayer_tracking;     /* 0.5    :450 */
    float sigma_debayer_accumulation; /* 0.5    :459 */
    float high_pass;                  /* 0.01   :468 */
    float high_pass_sigma;            /* 0.0025 :477 */
    int clear_axis;                   /* 0      :486 */
    float matching_threshold;         /* 1.0    :495 */
    float sigma_structure_tensor;     /* 1.0    :522 */
    float dth;                        /* 0.001  :531 */
    float dtr;                        /* 0.006  :540 */
    float k_detail;                   /* 0.25   :549 */
    float k_denoise;                  /* 3.0    :558 */
    float k_stretch;                  /* 4.0    :567 */
    float k_shrink;                   /* 2.0    :576 */
    int iterations_lk;                /* 3      :585 */
    int window_size_lk;               /* 11     :594 */
    int erode_size;                   /* 5      :603 */
    float min_det_lk;                 /* 0.01   :612 */
    float threshold_m;                /* 1e5    :621 */
    int tracking_strategy;            /* FULL   :657 */
    int tracking_block_size;          /* 5      :666 */
    int green_channel_only;           /* 0      :675 */
    int level_count;                  /* 4: (1,32,2) then (2*prev,32,4) (:1572-1586) */
    isa_level levels[ISA_MAX_LEVELS];
    /* extensions */
    int super_resolution;             /* SuperResolution (:648): 2x over the central crop */
    float merge_scale;                /* 0 = reference modes; > 0: the whole frame at this scale */
    float robust_s;                   /* 1.5, literal at RobustnessModell.cu:472 */
    float robust_t;                   /* 0.12, literal at RobustnessModell.cu:476 */
    int fused_accumulate;             /* 1: all frames in one accumulation pass (same sums, same order) */
    int sample_mode;                  /* ISA_SAMPLE_ROUND (reference) or ISA_SAMPLE_BILINEAR (differentiable in the flow) */
} isa_params;

/* RawFile metadata the merge uses (PefFile/RawFile.cs:94-119). white excludes black. */
typedef struct isa_raw_info {
    int width, height;
    int cfa[4];
    float black[3];
    float white[3];
    float camera_white[3];            /* AsShot white balance (DNGColorSpec CameraWhite), 1 = none */
    float noise_alpha, noise_beta;    /* NoiseModelA / NoiseModelB */
} isa_raw_info;

/* PreAlignmentStore state (PreAlignmentStore.cs:27-150); NULL arrays = all zero. */
typedef struct isa_prealign {
    const float* shifts;              /* n x 2, host memory */
    const float* rotations_deg;       /* n, host memory */
    int reference;                    /* ReferenceIndex */
} isa_prealign;

typedef struct isa_ctx isa_ctx;

/* One burst of a batch (isa_merge_batch). */
typedef struct isa_burst {
    const uint16_t* raw;         /* device, n frames; frame i at raw + i * frame_stride bytes, rows at raw_pitch */
    size_t raw_pitch, frame_stride;
    int n;
    const isa_raw_info* info;
    const isa_prealign* pre;     /* NULL: no pre-alignment */
    const struct isa_params* params;  /* NULL: the context's parameters */
    float* out;                  /* device float3 image of isa_output_size(), rows at out_pitch */
    size_t out_pitch;
} isa_burst;

/* ---- context, parameters, errors --------------------------------------- */
ISA_API void isa_params_default(isa_params* p);
ISA_API const char* isa_last_error(void);
ISA_API const char* isa_version(void);
/* Allocates every buffer of the fused pipeline for frames up to
 * max_width x max_height and max_frames (replaces the allocations of
 * PatchTracker.AllocateDeviceMemory PatchTracker.cs:96-117, OpticalFlow
 * OpticalFlow.cs:115-138, ShiftCollection ShiftCollection.cs:490-560 and
 * the controller buffers :1832-1849). */
ISA_API int isa_ctx_create(isa_ctx** ctx, int max_width, int max_height, int max_frames, const isa_params* p);
ISA_API int isa_ctx_destroy(isa_ctx* ctx);
/* Replaces the context's parameters between calls (a parameter fit, for
 * instance). The pyramid levels, the tracking strategy and block size must
 * stay those of isa_ctx_create, and the output of a max_width x max_height
 * frame must still fit the context; else ISA_EINVAL and the parameters are
 * unchanged. Allocates nothing. No counterpart in the reference, whose
 * controller reads its properties at each run. */
ISA_API int isa_ctx_set_params(isa_ctx* ctx, const isa_params* p);
/* Launch shapes chosen by a tuner for frames of width x height (0 x 0: any
 * size without an entry of its own); 0 in a field keeps the library's
 * choice. lk_strip_rows: rows per CTA strip of the LK iteration (else the
 * wave-filling choice); acc_block_x, acc_block_y: thread block of the
 * accumulation at scales other than 2 and in sample mode BILINEAR (else
 * 32 x 8; x y <= 256). */
typedef struct isa_tuning {
    int width, height;
    int lk_strip_rows;
    int acc_block_x, acc_block_y;
} isa_tuning;
/* Sets the context's tuning table (copied; count 0 clears it). Each merge
 * uses the entry of its frame size, else the 0 x 0 entry, else the
 * library's choices. The shapes change the order of no sum: results do not
 * depend on them. ISA_EINVAL for a shape out of range. No counterpart in the
 * reference. */
ISA_API int isa_ctx_set_tuning(isa_ctx* ctx, const isa_tuning* entries, int count);
/* Output size of the merge for a frame size under p. */
ISA_API int isa_output_size(const isa_params* p, int width, int height, int* out_width, int* out_height);
/* Stage times (ms) of the last isa_merge_burst call, in order: tracking
 * images, tile alignment, kernel parameters, LK + robustness, accumulation,
 * finalize. Synchronises the context's events. Returns the count written. */
ISA_API int isa_stage_times(isa_ctx* ctx, float* ms, int max_count);
/* Number of this library's kernels the last isa_merge_burst launched
 * (every kernel of the merge, the full-frame FFTs included). */
ISA_API long isa_launch_count(isa_ctx* ctx);

/* ---- fused pipeline ------------------------------------------------------ */
/* Whole forward merge of one burst (TrackPatches :1601 + PrepareAccumulation
 * :1795 + Accumulate :1928 + ApplyWeighting :1994-2002). raw: n frames of
 * width x height uint16, frame i at raw + i * frame_stride bytes, rows at
 * raw_pitch. out: float3 image of isa_output_size() with out_pitch. */
ISA_API int isa_merge_burst(isa_ctx* ctx, const uint16_t* raw, size_t raw_pitch, size_t frame_stride, int n, const isa_raw_info* info,
                    const isa_prealign* pre, float* out, size_t out_pitch, void* stream);
/* Forward merge plus the adjoint of the weighted L2 loss
 *   L = sum over output pixels p and channels c of weight_p (out - target)^2
 * with respect to the merge parameters, in this order: k_detail, k_denoise,
 * dth, dtr, k_stretch, k_shrink (through the kernel shape,
 * kernel.cu:628-700, and the kernel weights of the accumulation,
 * DeBayerKernels.cu:290-468) and robust_s, robust_t (through the robustness
 * mask, RobustnessModell.cu:29-157, and its erosion). No counterpart in the
 * reference, which has no gradients. Runs isa_merge_burst into `out`
 * (output size, out_pitch), then the adjoint with tile-level recomputation
 * of the masks instead of stored per-frame weights; writes *loss and
 * grad[8] (host) and synchronises `stream`. target: float3 image of the
 * output size; weight: one float per output pixel (NULL = all 1).
 * The loss is piecewise smooth: an output channel whose certainty-weighted
 * weight sum reaches exactly zero is set to 0 (ApplyWeighting), a jump, and
 * the mask clamps and the erosion's minimum have kinks; the gradient is
 * that of the smooth piece at the parameters (a zero weight excludes pixels
 * near such jumps). No flow gradient is returned here: in sample mode
 * ROUND it is zero almost everywhere (the accumulation and the mask read
 * the frames at round(s * flow) and round(flow / 2), and the mask's flow
 * term M only switches the gain at a threshold); in sample mode BILINEAR
 * isa_merge_backward_tiles returns it. Covers the
 * merge_scale and super-resolution modes (normalisation threshold 0) with
 * fused_accumulate. Allocates nothing: the adjoint's scratch is context
 * memory the forward has finished with, so afterwards the tracking and
 * accumulation images of isa_debug_buffers hold adjoint scratch, not the
 * forward's images. */
ISA_API int isa_merge_backward(isa_ctx* ctx, const uint16_t* raw, size_t raw_pitch, size_t frame_stride, int n, const isa_raw_info* info,
                               const isa_prealign* pre, const float* target, size_t target_pitch, const float* weight, size_t weight_pitch,
                               float* out, size_t out_pitch, double* loss, double* grad, void* stream);
/* isa_merge_backward plus the gradient of the loss with respect to every
 * frame's tile flow (the per-tile shifts of the finest level that
 * CreateFlowFieldFromTiles, opticalFlow.cu:48-95, spreads over the frame):
 * tile_grad (device, 8-byte aligned) receives n x tiles_y x tiles_x float2,
 * frame i at tile_grad + 2 i tiles_x tiles_y, zero for the reference frame
 * (isa_tile_flow gives tiles_x, tiles_y). The chain is the adjoint of the
 * accumulation (DeBayerKernels.cu:290-468) and of the robustness mask
 * (RobustnessModell.cu:29-157) with respect to the final flow, of each LK
 * iteration (warp, derivatives, window sums and 2x2 solve,
 * opticalFlow.cu:28-325; the flows before each iteration are recomputed
 * from the tile flow) and of the flow from tiles. Needs a context created
 * with sample_mode ISA_SAMPLE_BILINEAR (the merge is then continuous in the
 * flow; its scratch, 100 B per frame pixel, is allocated with the context)
 * and at most 3 LK iterations. The mask's flow term M only switches its gain
 * at a threshold and the LK solve leaves a pixel unchanged below minDet:
 * the gradient is that of the smooth piece. No counterpart in the reference. */
ISA_API int isa_merge_backward_tiles(isa_ctx* ctx, const uint16_t* raw, size_t raw_pitch, size_t frame_stride, int n, const isa_raw_info* info,
                                     const isa_prealign* pre, const float* target, size_t target_pitch, const float* weight, size_t weight_pitch,
                                     float* out, size_t out_pitch, double* loss, double* grad, float* tile_grad, void* stream);
/* Tile flows in place of the solved ones: while `tiles` (device, caller-owned,
 * 8-byte aligned; n x tiles_y x tiles_x float2, frame i at tiles + 2 i
 * tiles_x tiles_y, the reference frame's entry unused) is set, each merge
 * spreads these over the frame instead of the tile alignment's
 * (isa_optimal_shifts) result; the tile alignment still runs. NULL returns
 * to the solved flows. Used to evaluate the merge at chosen tile flows
 * (finite differences, fits). No counterpart in the reference. */
ISA_API int isa_set_tile_flow(isa_ctx* ctx, const float* tiles);
/* The tile flows of the last merge (the solved ones, or those set with
 * isa_set_tile_flow), in isa_set_tile_flow's layout, into `tiles` (device,
 * 8-byte aligned; NULL: only the grid size) on `stream`; tiles_x, tiles_y:
 * the finest level's tile counts. */
ISA_API int isa_tile_flow(isa_ctx* ctx, float* tiles, int* tiles_x, int* tiles_y, void* stream);
/* Many bursts of different sizes, frame counts, CFA layouts, bit depths and
 * merge scales (no counterpart in the reference, whose controller merges one
 * burst). The contexts may live on different devices (each on the device
 * that was current at its isa_ctx_create; streams[i], or the legacy default
 * stream when streams is NULL, must belong to ctxs[i]'s device). Each burst
 * goes to the context with the least work queued so far (W * H * n, in burst
 * order, deterministic; isa_batch_plan) among those on the device that holds
 * its frames, and is merged on that context's stream with that device
 * current; contexts run concurrently, so small bursts that cannot fill a GPU
 * alone overlap, and several GPUs share one batch. Returns after enqueuing
 * all bursts, with the caller's current device restored; the caller
 * synchronises the streams. A burst's params may differ from its context's
 * in the merge mode and scale and in the scalar parameters, but must keep
 * the context's pyramid levels and tracking strategy, and its frames and
 * output (on the same device) must fit the context. status[b] (optional,
 * host) receives each burst's result; the return value is the first
 * failure, or ISA_OK. */
ISA_API int isa_merge_batch(isa_ctx* const* ctxs, void* const* streams, int nctx, const isa_burst* bursts, int nbursts, int* status);
/* The assignment isa_merge_batch makes, on the host alone: burst b (work
 * work[b] > 0, data on device burst_device[b], or -1 for memory every
 * device reaches) goes to the context k with the least work assigned so far
 * among those with ctx_device[k] == burst_device[b] (any context for -1);
 * ties go to the lowest index. assignment[b] receives k, or -1 when no
 * context is on the burst's device. Returns the number of unassigned
 * bursts, or ISA_EINVAL for bad arguments. */
ISA_API int isa_batch_plan(const double* work, const int* burst_device, int nbursts, const int* ctx_device, int nctx, int* assignment);
/* A batch captured once as a CUDA graph and replayed (no counterpart in the
 * reference). isa_batch_graph_create captures what isa_merge_batch would
 * enqueue for `bursts` on ctxs / streams (all on the current device; the
 * streams distinct, not the legacy default stream, and not `origin`),
 * forked from and joined back to the `origin` stream, into a graph whose
 * host-to-device table copies read a pinned arena the graph owns; it runs
 * nothing. isa_batch_graph_launch replays the whole batch on `stream`: the
 * same frames and outputs (the bursts' device buffers must stay allocated;
 * their contents may change between replays), with one launch on the host.
 * While a graph runs, its contexts must not be used by other calls; merging
 * other bursts on them between replays is fine (every table the graph reads
 * is copied in by the graph itself). Stage times (isa_stage_times) are not
 * recorded by replays, and after isa_batch_graph_create the debug entry
 * points (isa_debug_buffers, isa_debug_shifts, isa_tile_flow) report no
 * merge until the next direct merge. */
typedef struct isa_batch_graph isa_batch_graph;
ISA_API int isa_batch_graph_create(isa_ctx* const* ctxs, void* const* streams, int nctx, const isa_burst* bursts, int nbursts, void* origin,
                                   isa_batch_graph** graph);
ISA_API int isa_batch_graph_launch(isa_batch_graph* graph, void* stream);
ISA_API int isa_batch_graph_destroy(isa_batch_graph* graph);
/* The same with host buffers: frames are copied in and the image copied out
 * on `stream` (pinned host memory gives full PCIe speed). */
ISA_API int isa_merge_burst_host(isa_ctx* ctx, const uint16_t* host_raw, int n, const isa_raw_info* info, const isa_prealign* pre,
                         float* host_out, void* stream);
/* Intermediates of the last isa_merge_burst (device pointers owned by ctx,
 * valid until the next call): per-frame dense flow (float2, W x H), eroded
 * robustness mask (float4, W/2 x H/2), kernel parameters (float4, W x H),
 * tracking images (float), accumulation sums (float3, output size). */
ISA_API int isa_debug_buffers(isa_ctx* ctx, int frame, const void** flow, size_t* flow_pitch, const void** mask, size_t* mask_pitch,
                      const void** kparam, size_t* kparam_pitch, const void** bw_track, const void** bw_acc, size_t* bw_pitch,
                      const void** acc, const void** wsum, size_t* acc_pitch);
/* Tile-alignment intermediates of the last isa_merge_burst: one-to-one shifts
 * of the finest level (tiles x (n-1) float2, device) and its tile counts. */
ISA_API int isa_debug_shifts(isa_ctx* ctx, const void** one_to_one, int* tiles_x, int* tiles_y);
/* Records every level's tile search of the following isa_merge_burst calls
 * into `record` (device, caller-owned, 4-byte aligned; NULL stops recording):
 * per level, finest first, m x tiles int32 first-minimum indices of the L2
 * maps (findMinimum, kernel.cu:422-546; -1 when no minimum), then m x tiles
 * int32 pairs (x, y) of the search block's integer offset (the rounded
 * pre-shift, PatchTracker.cs:225-253); m = the strategy's pair count in
 * isa_tracking_pairs order, tiles = tiles_x * tiles_y of the level. A merge
 * whose record needs more than `bytes` fails with ISA_EINVAL. No counterpart
 * in the reference: it exposes the integer tile shifts for parity checks. */
ISA_API int isa_debug_track_record(isa_ctx* ctx, int* record, size_t bytes);

/* ShiftCollection pair bookkeeping (ShiftCollection.cs:100-512), host only:
 * returns the pair count m; pairs (m x 2, optional) = (reference, toTrack)
 * in tracking order (FillShiftPairs / GetShiftPairs); rows (m x 3, optional)
 * = incidence interval [a, b) and sign of measurement row k (FillIndexTable
 * order, CreateShiftMatrix). */
ISA_API int isa_tracking_pairs(int n, int reference, int strategy, int block_size, int* pairs, int* rows, int max_pairs);

/* ---- operator API: one entry point per reference kernel wrapper ----------- */
/* DeBayerFullRes (controller :1268-1311): NPP Convert + Set(0) +
 * deBayerGreenKernel (DeBayerKernels.cs:36-44) + deBayerRedBlueKernel
 * (DeBayerKernels.cs:72-80) + NPP Div by divisor. out: float3. */
ISA_API int isa_debayer_full(const uint16_t* raw, size_t raw_pitch, int width, int height, const int cfa[4], const float black[3],
                     const float scale[3], const float divisor[3], float* out, size_t out_pitch, void* stream);
/* GammasRGBKernel (BasicKernels.cs:243-257), in place on float3. */
ISA_API int isa_gamma_srgb(float* img, size_t pitch, int width, int height, void* stream);
/* DeBayerBWGaussWB (controller :2384-2418) for one frame: demosaic, gamma,
 * gray, optional Fourier high-pass + clamp (PreAlignment.FourierFilter
 * PreAlignment.cs:268-281), Gaussian. Needs ctx for the FFT tables and
 * spectrum; with high_pass, out must be 8-byte aligned. */
ISA_API int isa_bw_image(isa_ctx* ctx, const uint16_t* raw, size_t raw_pitch, int width, int height, const isa_raw_info* info,
                 float sigma, int high_pass, float* out, size_t out_pitch, void* stream);
/* Global pre-alignment of a burst (ComputePreAlignment, controller
 * :1451-1528): the tracking image of every frame, then for every frame
 * i >= 1 PreAlignment.ScanAngles (PreAlignment.cs:176-261) against frame 0
 * -- a coarse scan of rotation angles over [zero - range, zero + range] in
 * steps of 5 * increment and a fine scan of +-10 increments around the coarse
 * best, each angle a cubic rotation about the frame centre, a full-frame FFT
 * cross-correlation and the position of its maximum -- with
 * zero = roll[0] - roll[i] (camera roll angles in degrees; NULL = 0). The
 * results go through PreAlignmentStore (PreAlignmentStore.cs:36-110):
 * shifts (n x 2), rotations_deg (n) and the reference index that minimises
 * the total shift, the inputs of isa_prealign. scan (optional, n x 4): the
 * raw ScanAngles results (x, y, angle, correlation) of each frame against
 * frame 0. Host outputs; synchronises `stream`. Frames need at least 4096
 * pixels. Reference controller defaults: increment 0.1, range 1.0. */
ISA_API int isa_prealign_burst(isa_ctx* ctx, const uint16_t* raw, size_t raw_pitch, size_t frame_stride, int n, const isa_raw_info* info,
                               float increment_deg, float range_deg, const float* roll_deg, float* shifts, float* rotations_deg, int* reference,
                               double* scan, void* stream);
/* fourierFilterKernel (BasicKernels.cs:81-100) on a (width/2+1) x height
 * half spectrum (float2), times post_scale. */
ISA_API int isa_fourier_filter(void* spectrum, size_t pitch, int width, int height, float lp, float hp, float lps, float hps, int clear_axis,
                       float post_scale, void* stream);
/* NPP FilterGaussBorder with gaussian_filter_1D(sigma) taps (controller
 * :2351-2382) and replicate border; channels 1 or 3; tmp: same size as in. */
ISA_API int isa_gauss_filter(const float* in, size_t in_pitch, float* out, size_t out_pitch, float* tmp, size_t tmp_pitch, int width, int height,
                     int channels, float sigma, void* stream);
/* NPP ResizeSqrPixel SuperSampling by 1/level (controller :1688-1703). */
ISA_API int isa_resize_box(const float* in, size_t in_pitch, int width, int height, int level, float* out, size_t out_pitch, void* stream);
/* PatchTracker.Track (PatchTracker.cs:317-360) for a batch of pairs at one
 * level: frames = device array of level-image pointers; pairs = device
 * array of isa_track_pair; grids = per-pair preShift grids (float2), grid k
 * at grids + k * grid_stride bytes, rows at grid_pitch; updated in place
 * (preShift += found shift). scores / argmin (optional, device): per pair
 * and tile the (2S+1)^2 L2 map and the index of its first minimum. */
typedef struct isa_track_pair {
    int reference, to_track, grid;
    float base_shift_ref[2], rotation_ref;   /* PreAlignmentStore GetShift/level, GetRotation (radians) */
    float base_shift_trk[2], rotation_trk;
} isa_track_pair;
ISA_API int isa_track_level(const float* const* frames, size_t frame_pitch, int width, int height, int tile_size, int max_shift, int tiles_x,
                    int tiles_y, const isa_track_pair* pairs, int npairs, void* grids, size_t grid_pitch, size_t grid_stride,
                    float threshold, float* scores, int* argmin, void* stream);
/* upsampleShiftsKernel (BasicKernels.cs:219-233) over ngrids grids. */
ISA_API int isa_upsample_shifts(const void* in, size_t in_pitch, size_t in_stride, void* out, size_t out_pitch, size_t out_stride, int ngrids,
                        int old_level, int new_level, int old_count_x, int old_count_y, int new_count_x, int new_count_y,
                        int old_tile_size, int new_tile_size, void* stream);
/* ShiftCollection.MinimizeCUBLAS (ShiftCollection.cs:738-822) for one level:
 * strategy/reference/n define the incidence matrix; grids as in
 * isa_track_level, grid k holding measurement row k (FillIndexTable order);
 * rewritten with the consistent pair shifts. one_to_one (device, tiles x
 * (n-1) float2) and status (device, tiles: -1 converged, -3 singular,
 * >= 0 row removed in the tenth round) are outputs. Needs ctx scratch. */
ISA_API int isa_solve_shifts(isa_ctx* ctx, int n, int reference, int strategy, int block_size, void* grids, size_t grid_pitch,
                     size_t grid_stride, int tiles_x, int tiles_y, void* one_to_one, int* status, void* stream);
/* The same solve for callers that cannot allocate device memory where they
 * align tiles (their device memory is owned by another allocator, they run
 * under a fixed budget, or they must not risk the device-wide synchronisation
 * an allocation can cause). No counterpart in the reference: it replaces
 * isa_solve_shifts' context scratch by a library-owned static device array
 * that every GPU loading the library keeps until exit. Limits: at most 2048
 * frame pairs and 65 frames (ISA_EINVAL beyond). Allocates nothing once set
 * up on a device. The set-up happens in the first call on each device (and
 * CUDA context), or in isa_ctx_create on that device: it loads the library's
 * device code there -- CUDA loads it lazily, and loading allocates the
 * code's globals, this array among them, and can synchronise the device --
 * and looks up the array's address. So make one call per device at
 * initialisation, before any stream capture. All calls share the array:
 * calls that overlap on the GPU (different streams, or several host
 * threads) race and must be serialised by the caller. Inputs and outputs as
 * isa_solve_shifts. */
ISA_API int isa_solve_shifts_static(int n, int reference, int strategy, int block_size, void* grids, size_t grid_pitch, size_t grid_stride,
                                    int tiles_x, int tiles_y, void* one_to_one, int* status, void* stream);
/* getOptimalShiftsKernel (ShiftMinimizerKernels.cs): shift of frame
 * to_track relative to reference from the one-to-one shifts. */
ISA_API int isa_optimal_shifts(const void* one_to_one, int n, int tiles_x, int tiles_y, int reference, int to_track, void* out,
                       size_t out_pitch, void* stream);
/* CreateFlowFieldFromTiles (OpticalFlowKernels.cs:59-83). base_shift: 2 floats (host). */
ISA_API int isa_flow_from_tiles(const void* tiles, size_t tile_pitch, int tiles_x, int tiles_y, int width, int height, const float base_shift[2],
                        float base_rotation, void* flow, size_t flow_pitch, void* stream);
/* WarpingKernel (OpticalFlowKernels.cs:31-56). */
ISA_API int isa_warp(const float* img, size_t img_pitch, int width, int height, const void* flow, size_t flow_pitch, float* out, size_t out_pitch,
             void* stream);
/* ComputeDerivativesKernel (OpticalFlowKernels.cs:86-114). */
ISA_API int isa_derivatives(const float* src, const float* tgt, size_t pitch, int width, int height, float* ix, float* iy, float* it,
                    size_t out_pitch, void* stream);
/* ComputeDerivatives2Kernel (OpticalFlowKernels.cs:117-140). */
ISA_API int isa_derivatives2(const float* img, size_t pitch, int width, int height, float* ix, float* iy, size_t out_pitch, void* stream);
/* LukasKanadeKernel (OpticalFlowKernels.cs:143-173) on derivative images. */
ISA_API int isa_lucas_kanade(void* flow, size_t flow_pitch, const float* ix, const float* iy, const float* it, size_t pitch, int width, int height,
                     float min_det, int window_size, void* stream);
/* One fused LK iteration: warp + derivatives + LK (OpticalFlow.cs:151-158);
 * flow_in and flow_out must differ. */
ISA_API int isa_lk_iteration(const void* flow_in, void* flow_out, size_t flow_pitch, const float* src, const float* ref, size_t img_pitch, int width,
                     int height, float min_det, int window_size, void* stream);
/* OpticalFlow.LucasKanade (OpticalFlow.cs:147-164): flow from tiles then
 * `iterations` fused iterations; scratch: a second flow buffer. */
ISA_API int isa_lk_refine(const float* src, const float* ref, size_t img_pitch, int width, int height, const void* tiles, size_t tile_pitch,
                  int tiles_x, int tiles_y, const float base_shift[2], float base_rotation, int iterations, float min_det,
                  int window_size, void* flow, void* flow_scratch, size_t flow_pitch, void* stream);
/* DeBayersSubSampleKernel (DeBayerKernels.cs:84-118): 2x2 quad -> float3. */
ISA_API int isa_debayer_subsample(const uint16_t* raw, size_t raw_pitch, int width, int height, const int cfa[4], float max_value, float* out,
                          size_t out_pitch, void* stream);
/* RobustnessModellKernel (RobustnessModellKernel.cs:30-66); s and t are the
 * reference literals 1.5 / 0.12 unless changed. mask border untouched. */
ISA_API int isa_robustness_mask(const float* ref3, const float* moved3, size_t img_pitch, void* mask, size_t mask_pitch, int half_width,
                        int half_height, const void* flow, size_t flow_pitch, int flow_width, int flow_height, float alpha, float beta,
                        float threshold_m, float s, float t, void* stream);
/* NPP ErodeBorder (controller :1976) on float4, square all-ones mask. */
ISA_API int isa_erode(const void* in, size_t in_pitch, void* out, size_t out_pitch, int width, int height, int size, void* stream);
/* Mask + erosion fused (border pixels 1, as after controller :1891). */
ISA_API int isa_robustness_erode(const float* ref3, const float* moved3, size_t img_pitch, int half_width, int half_height, const void* flow,
                         size_t flow_pitch, int flow_width, int flow_height, float alpha, float beta, float threshold_m, float s, float t,
                         int erode_size, void* out, size_t out_pitch, void* stream);
/* computeStructureTensorKernel + ComputeDerivatives2Kernel (BasicKernels.cs:285-301). out: float3. */
ISA_API int isa_structure_tensor(const float* img, size_t pitch, int width, int height, float* out, size_t out_pitch, void* stream);
/* computeKernelParamKernel (BasicKernels.cs:303-318): float3 tensor ->
 * out (3 or 4 channels; may alias st when channels == 3). */
ISA_API int isa_kernel_param(const float* st, size_t st_pitch, int width, int height, float* out, size_t out_pitch, int out_channels, float dth,
                     float dtr, float k_detail, float k_denoise, float k_stretch, float k_shrink, void* stream);
/* AccumulateImagesKernel / AccumulateImagesSuperResKernel
 * (DeBayerKernels.cs:121-211), generalised: output out_width x out_height at
 * scale s with output-grid origin (ox, oy) and inclusive source crop
 * crop[4] = x0, y0, x1, y1. Reference plain: s = 1, origin 0, crop = frame;
 * super-resolution: s = 2, origin (W/2, H/2), crop = central W/2 x H/2.
 * acc / wsum: float3 read-modify-write. flow NULL = zero, mask NULL = 1. */
ISA_API int isa_accumulate(const uint16_t* raw, size_t raw_pitch, int width, int height, const int cfa[4], float* acc, float* wsum,
                   size_t out_pitch, int out_width, int out_height, const void* mask, size_t mask_pitch, const float* kparam,
                   size_t kparam_pitch, int kparam_channels, const void* flow, size_t flow_pitch, const float white[3],
                   const float black[3], float scale, int ox, int oy, const int crop[4], void* stream);
/* ApplyWeightingKernel (BasicKernels.cs:259-284): img (fallback in, result out). */
ISA_API int isa_apply_weighting(float* img, const float* acc, const float* wsum, size_t pitch, int width, int height, float threshold,
                        void* stream);

/* ---- Colour and tone post-processing and 16-bit TIFF output ----
 * The controller's SaveAs16BitTiff (ImageStackAlignatorController.cs:2197-2260)
 * and ProcessColorsAndShow (:2262-2320) after ApplyWeighting: NPP
 * ThresholdLTGT to [0, CameraWhite], ColorTwist camera -> ProPhoto,
 * ThresholdLTGT to [0, 1], LUTCubic (tone curve), ColorTwist ProPhoto ->
 * sRGB (D50), Mul 2^Exposure, GammasRGB (kernel.cu:290-332), Mul 65535 (or
 * 255), ROI = the raw file's crop, Convert with NppRoundMode.Near. */
#define ISA_MAX_LUT 512
typedef struct isa_post_params {
    int crop_x, crop_y, crop_w, crop_h;   /* RawFile CropLeft, CropTop, CroppedWidth, CroppedHeight */
    float camera_white[3];                /* DNGColorSpec.CameraWhite: per-channel upper clamp */
    float twist1[12];                     /* camera -> ProPhoto, 3 x 4 row-major (isa_color_twists) */
    float twist2[12];                     /* ProPhoto -> sRGB (D50), 3 x 4 row-major */
    const float* lut_x;                   /* host: LUT levels, strictly increasing (the controller's LUTx, 256 entries i/255) */
    const float* lut_y;                   /* host: LUT values at the levels (defaultLUT) */
    int nlut;                             /* 4 .. ISA_MAX_LUT */
    float exposure;                       /* Exposure (:793, default 0): the image is scaled by 2^exposure before the gamma */
} isa_post_params;

enum { ISA_POST_RGB16 = 0,  /* SaveAs16BitTiff: uint16 R, G, B per pixel */
       ISA_POST_BGRA8 = 1   /* ProcessColorsAndShow: uint8 B, G, R, 255 per pixel (the WPF Bgra32 bitmap) */ };

/* The two 3 x 4 colour twists of SaveAs16BitTiff (:2226-2240) from the
 * colour spec's CameraToPCS (row-major 3 x 3, camera -> XYZ D50), in FP64 as
 * DNGColorSpace (DNGColorSpace.cs:36-65: ProPhoto and sRGB50 matrices scaled
 * so that RGB white maps to the D50 PCS white, inverted with
 * DNGMatrix.Invert3x3, DNGMatrix.cs:440-486), then cast to float with a zero
 * offset column (DNGMatrix.GetAs3x4Array, DNGMatrix.cs:181-193). Host only. */
ISA_API int isa_color_twists(const double camera_to_pcs[9], float twist1[12], float twist2[12]);
/* The post-processing chain on a float3 image (device, width x height,
 * pitch bytes) into `out` (device, crop_w x crop_h, format ISA_POST_*,
 * out_pitch bytes). One fused pass; the LUT is interpolated with the cubic
 * through the four nearest levels (NPP's LUTCubic does not publish its
 * polynomial), as per-segment coefficients computed on the host in FP64 and
 * evaluated in FP32 by Horner's rule. */
ISA_API int isa_postprocess(const float* img, size_t pitch, int width, int height, const isa_post_params* pp, int format, void* out,
                            size_t out_pitch, void* stream);
/* ImageFileDirectory(width, height).SaveAsTiff (PefFile/ImageFileDirectory.cs:75-123):
 * little-endian baseline TIFF, 13 tags, one strip of uint16 RGB (host,
 * width x height x 3, row-major). Host only. */
ISA_API int isa_save_tiff16(const char* path, const uint16_t* rgb, int width, int height);
/* SaveAs16BitTiff from a device float3 image: isa_postprocess (ISA_POST_RGB16)
 * on `stream`, copy to the host, isa_save_tiff16. Synchronises `stream`. */
ISA_API int isa_save_as_16bit_tiff(const float* img, size_t pitch, int width, int height, const isa_post_params* pp, const char* path,
                                   void* stream);

/* ---- Raw decoding of Pentax PEF frames ----
 * The pixel data of PEFFile (PefFile/PEFFile.cs:81-156) and the levels of
 * PEFFile.SetMembers (:176-280). The TIFF/Exif/maker-note container is
 * parsed by the host; these entry points take the parsed values. */
/* MNHuffmanTable (PefFile/PentaxMakerNotesEntry.cs:4555-4613): the decode
 * table (4097 entries, table[0] = 12) from the HuffmanTable maker-note
 * bytes, in the file's byte order. Returns the number of codes (>= 0) or
 * ISA_EINVAL. Host only. */
ISA_API int isa_pef_huff_table(const uint8_t* maker_note, size_t n, int big_endian, uint16_t table[4097]);
/* Device scratch isa_pef_decode needs for `nbytes` of stream and a width x height frame. */
ISA_API size_t isa_pef_decode_scratch(size_t nbytes, int width, int height);
/* The compressed strip (PEFFile.cs:81-111) of one frame: `data` (device,
 * nbytes) is the strip, `table` (host) from isa_pef_huff_table (code
 * lengths 1..12, categories 0..15), `out` uint16 width x height (device).
 * Decodes in parallel without host round trips: 1024-bit chunks decoded
 * from each of their 27 candidate starts, the start maps chained, a scan of
 * the symbol counts, the differences, then prefix sums that undo the
 * prediction. Reads past the data see zeros. Streams up to about 1.9 Gbit. */
ISA_API int isa_pef_decode(const uint8_t* data, size_t nbytes, const uint16_t* table, int width, int height, void* scratch, size_t scratch_bytes,
                           uint16_t* out, size_t out_pitch, void* stream);
/* The uncompressed branch (PEFFile.cs:116-156): `file` (device, file_size
 * bytes) holds nstrips strips at offsets[s], sizes[s] (host arrays, at most
 * 512 strips) of rows_per_strip rows of `bit_depth`-bit values (1..16), MSB
 * first; the reader's left-over bits carry from one strip to the next. */
ISA_API int isa_pef_unpack(const uint8_t* file, size_t file_size, const uint32_t* offsets, const uint32_t* sizes, int nstrips, int rows_per_strip,
                           int width, int height, int bit_depth, uint16_t* out, size_t out_pitch, void* stream);
/* PEFFile.SetMembers levels (PEFFile.cs:199-260): black per R, G, B from
 * one, three or four (per CFA position; green = max of the two greens)
 * BlackPoint values, white = WhiteLevel (or 2^bit_depth when white_level
 * <= 0) minus black, white balance = WhitePoint[0, 1, 3] / DataScaling.
 * cfa as isa_raw_info. Host only. */
ISA_API int isa_pef_levels(const int cfa[4], const float* black_point, int n_black, float white_level, const float white_point[4], float scaling,
                           int bit_depth, float black[3], float white[3], float white_balance[3]);

/* ---- DNG colour specification ----
 * DNGColorSpec (PefFile/DNGColorSpec.cs:31-647) with DNGTemperature and
 * DNGxyCoord, in FP64: the colour matrix (and forward matrix, camera
 * calibration) interpolated by the white point's temperature between the
 * two calibration illuminants, the white point from AsShotWhiteXY or found
 * from AsShotNeutral, then CameraWhite and CameraToPCS (camera -> XYZ D50),
 * the inputs of isa_color_twists and isa_post_params. Host only. */
typedef struct isa_dng_color_tags {
    const double* color_matrix1;        /* 9, row-major (ColorMatrix1); NULL = identity */
    const double* color_matrix2;        /* 9 or NULL */
    int illuminant1, illuminant2;       /* CalibrationIlluminant1/2, EXIF LightSource codes; 0 = absent/unknown */
    const double* forward_matrix1;      /* 9 or NULL */
    const double* forward_matrix2;      /* 9 or NULL */
    const double* camera_calibration1;  /* 9 or NULL = identity (the reference reads CameraCalibration1 for both) */
    const double* camera_calibration2;  /* 9 or NULL = identity */
    const double* analog_balance;       /* 3 or NULL = 1 */
    const double* as_shot_neutral;      /* 3 or NULL */
    const double* as_shot_white_xy;     /* 2 or NULL; used when given */
} isa_dng_color_tags;
ISA_API int isa_dng_color_spec(const isa_dng_color_tags* tags, double camera_to_pcs[9], double camera_white[3], double white_xy[2]);
/* The colour spec PEFFile.SetMembers builds (PEFFile.cs:310-312): identity
 * colour matrices under D50 and the white point of the neutral 1 / white
 * balance (isa_pef_levels' white_balance). */
ISA_API int isa_pef_color_spec(const float white_balance[3], double camera_to_pcs[9], double camera_white[3], double white_xy[2]);

/* ---- Raw decoding of DNG frames ----
 * The pixel data of DNGFile (PefFile/DNGFile.cs:372-600): lossless-JPEG
 * (compression 7) tiles or strips, decoded with the reference's dcraw
 * reader (predictors 1..7, restart markers, 0xFF byte skipping), or
 * uncompressed strips (compression 1: 16-bit little-endian samples, or
 * packed MSB-first samples of bit_depth bits); then the linearisation
 * table and the black-level deltas: out = max(0, lin[min(v, nlin - 1)] -
 * black_h[col] - black_v[row]). Lossless-JPEG headers are parsed from
 * `file_host`; the data is read from `file_dev` (the same bytes on the
 * device), by the parallel decoder for predictor-1 parts without restarts
 * inside a part and one Huffman table, else by one warp per part
 * (isa_dng_decode_path). */
typedef struct isa_dng_layout {
    int tiled;                       /* 1: TileWidth/TileLength/TileOffsets/TileByteCounts; 0: strips */
    int tile_width, tile_height;     /* tiles */
    int rows_per_strip;              /* strips */
    int n;                           /* tiles or strips */
    const uint32_t* offsets;         /* host: n byte offsets in the file */
    const uint32_t* byte_counts;     /* host: n byte counts */
    int compression;                 /* 7 = lossless JPEG, 1 = none (strips only) */
    int bit_depth;                   /* BitsPerSample of uncompressed strips */
    int dng_version_large;           /* DNGVersion absent or its second byte > 1 (a category-16 code means -32768) */
    const uint16_t* linearization;   /* host LinearizationTable or NULL */
    int nlin;
    const uint16_t* black_h;         /* host, width entries: BlackLevelDeltaH placed in the active area, or NULL */
    const uint16_t* black_v;         /* host, height entries: BlackLevelDeltaV, or NULL */
} isa_dng_layout;
ISA_API size_t isa_dng_decode_scratch(const uint8_t* file_host, size_t file_size, const isa_dng_layout* layout, int width, int height);
/* Decodes into `out` (device, uint16 width x height; pixels no part covers
 * are 0) and synchronises `stream`; ISA_EINVAL where the reference would
 * stop (a sample above the frame's bit depth). */
ISA_API int isa_dng_decode(const uint8_t* file_host, const uint8_t* file_dev, size_t file_size, const isa_dng_layout* layout, int width, int height,
                           void* scratch, size_t scratch_bytes, uint16_t* out, size_t out_pitch, void* stream);
/* isa_dng_decode in two halves, so that a host decodes many frames with one
 * wait: begin does the checks, the uploads and, when the frame qualifies for
 * the parallel decoder, enqueues it on `stream` and returns at once (other
 * frames decode with the per-part reader inside begin, synchronised);
 * finish, with the same arguments and the scratch untouched in between,
 * waits for `stream`, reads the decoder's flags and decodes a handed-back
 * frame with the per-part reader. The output is complete after finish. */
ISA_API int isa_dng_decode_begin(const uint8_t* file_host, const uint8_t* file_dev, size_t file_size, const isa_dng_layout* layout, int width,
                                 int height, void* scratch, size_t scratch_bytes, uint16_t* out, size_t out_pitch, void* stream);
ISA_API int isa_dng_decode_finish(const uint8_t* file_host, const uint8_t* file_dev, size_t file_size, const isa_dng_layout* layout, int width,
                                  int height, void* scratch, size_t scratch_bytes, uint16_t* out, size_t out_pitch, void* stream);
/* Which decoder the calling thread's last isa_dng_decode used: 1 = the
 * parallel one (lossless-JPEG parts with predictor 1, no restart inside a
 * part, one Huffman table: chunks decoded from every candidate start, as
 * isa_pef_decode), 0 = one warp per part with the reference's sequential
 * reader (every other layout, and frames the parallel decoder hands back),
 * -1 = none (an argument error or uncompressed strips). */
ISA_API int isa_dng_decode_path(void);

/* ---- Raw-file metadata: DNG levels, camera profiles ----
 * DNGFile.SetMembers (PefFile/DNGFile.cs:714-951) and the DNGFile
 * constructor (:288-372, :607-609): CFA layout, black and white per colour,
 * white balance, plane reordering, crop window and noise model, from the
 * parsed tag values. Host only. */
typedef struct isa_dng_level_tags {
    int width, height;                /* ImageWidth, ImageLength of the raw IFD */
    const uint8_t* cfa_pattern;       /* CFAPattern, 4 codes (0 red, 1 green, 2 blue) */
    int cfa_repeat_w, cfa_repeat_h;   /* CFARepeatPatternDim; anything but 2 x 2 is rejected (:706-712) */
    const int* plane_color;           /* CFAPlaneColor or NULL (= 0, 1, 2) */
    int n_plane_color;                /* must be 3 when given (:727-730) */
    const double* black_level;        /* BlackLevel values or NULL; 1, 3 (per plane) or 4 (per CFA position) are used */
    int n_black;
    double white_level;               /* WhiteLevel[0] */
    const double* camera_white;       /* 3: CameraWhite of the colour spec (isa_dng_color_spec) */
    const int* active_area;           /* ActiveArea top, left, bottom, right, or NULL */
    const double* default_crop_origin;/* DefaultCropOrigin or NULL (the reference reads entry 0 for left and top) */
    const double* default_crop_size;  /* DefaultCropSize or NULL (entry 0 for width and height) */
    const double* noise_profile;      /* NoiseProfile of the raw IFD, else of IFD 0, or NULL */
    int n_noise;                      /* >= 2 */
    const double* black_delta_h;      /* BlackLevelDeltaH values or NULL (truncated to uint16) */
    int n_delta_h;                    /* must equal the active area's width (:358-365) */
    const double* black_delta_v;      /* BlackLevelDeltaV values or NULL */
    int n_delta_v;                    /* must equal the active area's height (:341-350) */
    /* ExtraCameraProfiles noise model for this camera (:296-320): used when it gives alpha != 0 */
    int iso;                          /* ISOSpeedRatings */
    const int* profile_iso;           /* NoiseModel.Iso ascending, or NULL */
    const double* profile_alpha;
    const double* profile_beta;
    int n_profile;
} isa_dng_level_tags;

typedef struct isa_raw_levels {
    isa_raw_info info;                /* width, height, cfa (shifted for an odd active-area origin), black,
                                         white (WhiteLevel - black - the largest black delta), camera_white, noise */
    float white_balance[3];           /* 1 / CameraWhite, per plane (:836-841) */
    float color_twist[12];            /* 3 x 4 plane reordering of CFAPlaneColor (identity when absent) */
    int color_twist_identity;
    int crop[4];                      /* CropLeft, CropTop, CroppedWidth, CroppedHeight (at least 2 pixels off each edge) */
} isa_raw_levels;

/* Fills `out` and, when not NULL, black_h (width entries) and black_v
 * (height entries) with the black-level deltas placed in the active area,
 * as isa_dng_layout takes them. ISA_EINVAL where the reference throws. */
ISA_API int isa_dng_levels(const isa_dng_level_tags* tags, isa_raw_levels* out, uint16_t* black_h, uint16_t* black_v);

/* NoiseModel.GetValue (PefFile/ExtraCameraProfiles.cs:164-199): alpha and
 * beta at `iso` from a profile's ascending ISO list, linear between the two
 * neighbours, clamped to the ends; (0, 0) for an empty list. */
ISA_API int isa_noise_model(int iso, const int* isos, const double* alpha, const double* beta, int n, double ab[2]);

/* The crop rule of DNGFile.SetMembers (:944-948) and
 * RawFile.LoadExtraCameraProfile (PefFile/RawFile.cs:246-261): at least two
 * pixels off the left and top, the size shortened to end two pixels before
 * the right and bottom edges. crop = left, top, width, height. */
ISA_API int isa_crop_window(int left, int top, int cropped_width, int cropped_height, int width, int height, int crop[4]);

/* DNGColorSpec(colorMatrix1, colorMatrix2, illuminant1, illuminant2,
 * whiteBalance) (PefFile/DNGColorSpec.cs:175-266), the colour spec of an
 * ExtraCameraProfiles entry (RawFile.cs:264-268): color_matrix2 may be NULL,
 * illuminants are EXIF LightSource codes, the white point is that of the
 * neutral 1 / white_balance. isa_pef_color_spec is the identity / D50 case. */
ISA_API int isa_profile_color_spec(const double* color_matrix1, const double* color_matrix2, int illuminant1, int illuminant2,
                                   const float white_balance[3], double camera_to_pcs[9], double camera_white[3], double white_xy[2]);

/* ---- DNG container ----
 * The TIFF structure RawFile reads (PefFile/RawFile.cs:56-90: byte order,
 * magic 42, the IFD chain), SubIFDs, and the tags DNGFile and DNGColorSpec
 * read: the raw IFD is the first IFD of the chain whose
 * PhotometricInterpretation is CFA, else the first CFA SubIFD of the last
 * IFD of the chain that has one (DNGFile.cs:621-660); colour tags come from
 * IFD 0, else the raw IFD (DNGColorSpec.cs:94-103), CameraCalibration1
 * serving both illuminants as the reference reads it; the ISO from the Exif
 * IFD, else the raw IFD, else IFD 0. Host only; ISA_EINVAL where the
 * reference cannot read the file. */
typedef struct isa_dng_file isa_dng_file;
ISA_API int isa_dng_open(const uint8_t* file, size_t size, isa_dng_file** out);
ISA_API int isa_dng_close(isa_dng_file* f);
/* Views into the parsed file, valid until isa_dng_close (any output may be
 * NULL): the pixel layout for isa_dng_decode (black deltas left NULL: place
 * them with isa_dng_levels), the level tags for isa_dng_levels (camera_white
 * left NULL: take it from isa_dng_color_spec) and the colour tags. */
ISA_API int isa_dng_file_info(const isa_dng_file* f, isa_dng_layout* layout, isa_dng_level_tags* levels, isa_dng_color_tags* color, int* width,
                              int* height);
/* The camera roll angle (degrees) of a Pentax maker note carried in IFD 0's
 * DNGPrivateData (DNGFile.cs:676-685, MNLevelInfo): 1 and the angle when
 * present, 0 and 0.0 when not. Per frame, the roll angles are the `roll`
 * input of isa_prealign_burst, as ComputePreAlignment uses them. */
ISA_API int isa_dng_roll_angle(const isa_dng_file* f, float* roll_deg);

/* ---- PEF container ----
 * PEFFile.SetMembers (PefFile/PEFFile.cs:176-312): the raw image of IFD 0,
 * the Exif IFD's ISO and CFA pattern (ExifCFAPattern,
 * PefFile/ExifEntry.cs:2529-2542) and the Pentax maker note
 * (PentaxMakerNotes, PefFile/PentaxMakerNotes.cs:26-198: "AOC\0" or
 * "PENTAX \0" header, its own byte order) with HuffmanTable, BlackPoint,
 * WhitePoint, WhiteLevel and DataScaling. The fields feed
 * isa_pef_huff_table, isa_pef_levels and isa_pef_decode / isa_pef_unpack.
 * Host only; ISA_EINVAL where the reference cannot read the file. */
typedef struct isa_pef_file isa_pef_file;
typedef struct isa_pef_info {
    int width, height, bit_depth;
    int cfa[4];
    int nstrips, rows_per_strip;
    const uint32_t* strip_offsets;    /* nstrips byte offsets in the file */
    const uint32_t* strip_sizes;
    int compressed;                   /* a HuffmanTable and a single strip: the Huffman branch (PEFFile.cs:87) */
    const uint8_t* huffman_table;     /* the HuffmanTable entry's bytes (isa_pef_huff_table), or NULL */
    size_t huffman_bytes;
    int huffman_big_endian;           /* the maker note's byte order */
    const float* black_point;         /* BlackPoint values or NULL */
    int n_black;
    float white_level;                /* WhiteLevel, or -1 when absent (2^bit_depth then) */
    float white_point[4];             /* WhitePoint */
    float scaling;                    /* DataScaling */
    int iso;                          /* ISOSpeedRatings (0 when absent) */
    float roll_angle;                 /* LevelInfo roll angle in degrees (PEFFile.cs:278-282), 0 when absent */
    int roll_angle_present;
} isa_pef_info;
ISA_API int isa_pef_open(const uint8_t* file, size_t size, isa_pef_file** out);
ISA_API int isa_pef_close(isa_pef_file* f);
/* The parsed values, valid until isa_pef_close. */
ISA_API int isa_pef_file_info(const isa_pef_file* f, isa_pef_info* info);

#ifdef __cplusplus
}
#endif
#endif
