/*
 * isa_oracle.c -- CPU restatement (FP64 by default) of the ImageStackAlignator
 * burst-merge hot path.
 *
 * TEST INFRASTRUCTURE ONLY. This file is the checker that the CUDA path is
 * compared against; nothing in the shipped library links, loads or calls it.
 * Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg use it.
 *
 * Every function restates one reference kernel or one library step and cites
 * the reference file:line it follows (paths relative to the reference
 * project). Library steps with no source in the reference (NPP, cuFFT,
 * cuBLAS) are restated from their documented mathematical definition.
 * The frequency-domain part of the high-pass (the FFT itself) is done by
 * numpy in oracle/pipeline.py; this file provides the filter mask.
 *
 * Layout conventions (chosen for numpy callers): every image is a contiguous
 * row-major array without pitch; multi-channel images interleave channels
 * (H x W x C). CFA codes follow the reference enum (DeBayerKernels.cu:28-37):
 * R=0, G=1, B=2; cfa[(y & 1) * 2 + (x & 1)] is the colour at (x, y).
 *
 * Build: REAL defaults to double; -DISA_ORACLE_REAL=float gives an FP32 copy
 * of the library steps for the host baseline.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <float.h>

#ifndef ISA_ORACLE_REAL
#define ISA_ORACLE_REAL double
#endif
typedef ISA_ORACLE_REAL real;

#define EXPORT __attribute__((visibility("default")))

static inline int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

/* Reflect a texel index with the edge texel repeated (period 2n): the
 * documented mirror addressing of a CUDA texture (CUDA C Programming Guide,
 * "Texture Fetching"). Used where the reference samples through a mirror
 * texture (opticalFlow.cu:28-45, 97-148, 151-185; RobustnessModell.cu:47-61). */
static inline int mirror_index(int i, int n) {
    int p = 2 * n;
    int j = i % p;
    if (j < 0) j += p;
    return j >= n ? p - 1 - j : j;
}

/* Exact bilinear sample of channel c of a (h x w x ch) image at texel-space
 * position (xb, yb) = (u*w - 0.5, v*h - 0.5); mode 0 clamps, 1 mirrors.
 * (The hardware keeps 8 fractional bits of the weights; exact weights here.) */
static real bilinear(const real* img, int w, int h, int ch, int c, real xb, real yb, int mirror) {
    real fx = floor(xb), fy = floor(yb);
    int i = (int)fx, j = (int)fy;
    real a = xb - fx, b = yb - fy;
    int i0, i1, j0, j1;
    if (mirror) { i0 = mirror_index(i, w); i1 = mirror_index(i + 1, w); j0 = mirror_index(j, h); j1 = mirror_index(j + 1, h); }
    else { i0 = clampi(i, 0, w - 1); i1 = clampi(i + 1, 0, w - 1); j0 = clampi(j, 0, h - 1); j1 = clampi(j + 1, 0, h - 1); }
    /* texels with zero weight are not read, so a non-finite neighbour only
     * affects samples that actually weight it */
    real v = 0;
    if (a != 1 && b != 1) v += (1 - a) * (1 - b) * img[((size_t)j0 * w + i0) * ch + c];
    if (a != 0 && b != 1) v += a * (1 - b) * img[((size_t)j0 * w + i1) * ch + c];
    if (a != 1 && b != 0) v += (1 - a) * b * img[((size_t)j1 * w + i0) * ch + c];
    if (a != 0 && b != 0) v += a * b * img[((size_t)j1 * w + i1) * ch + c];
    return v;
}

/* ------------------------------------------------------------------------ */
/* A1: full-resolution demosaic.                                             */
/* ImageStackAlignatorController.cs:1268-1311 (DeBayerFullRes): u16 -> float, */
/* decoded image cleared to 0, green by DeBayerKernels.cu:55-150, red/blue by */
/* DeBayerKernels.cu:153-231, then per-channel division (NPP Div, :1304-1306). */
/* ------------------------------------------------------------------------ */
EXPORT void orc_debayer_full(const uint16_t* raw, int W, int H, const int* cfa,
                             const real* black, const real* scale, const real* divisor, real* rgb)
{
    size_t n = (size_t)W * H;
    real* g = (real*)calloc(n, sizeof(real));
    memset(rgb, 0, n * 3 * sizeof(real));
#define LIN(xx, yy, c) (((real)raw[(size_t)(yy) * W + (xx)] - black[c]) * scale[c])
    /* green plane (DeBayerKernels.cu:55-150); 2-px border stays 0 */
    for (int y = 2; y < H - 2; y++)
        for (int x = 2; x < W - 2; x++) {
            int col = cfa[(y & 1) * 2 + (x & 1)];
            real v = 0;
            if (col == 1) {
                v = LIN(x, y, 1);
            } else if (col == 0 || col == 2) {
                real p = LIN(x, y, col);
                real hm2 = LIN(x - 2, y, col), hp2 = LIN(x + 2, y, col);
                real hm1 = LIN(x - 1, y, 1), hp1 = LIN(x + 1, y, 1);
                real vm2 = LIN(x, y - 2, col), vp2 = LIN(x, y + 2, col);
                real vm1 = LIN(x, y - 1, 1), vp1 = LIN(x, y + 1, 1);
                real gradH = 0.5 * fabs(hp1 - hm1), gradV = 0.5 * fabs(vp1 - vm1);
                real lapH = 0.25 * fabs(2 * p - hm2 - hp2), lapV = 0.25 * fabs(2 * p - vm2 - vp2);
                real estH = 0.125 * (-hm2 + 4 * hm1 + 2 * p + 4 * hp1 - hp2);
                real estV = 0.125 * (-vm2 + 4 * vm1 + 2 * p + 4 * vp1 - vp2);
                real wH = (gradV + lapV) / (gradH + gradV + lapH + lapV + 0.000000001);
                v = wH * estH + (1 - wH) * estV;
            }
            g[(size_t)y * W + x] = v;
        }
    /* red / blue by colour differences to green (DeBayerKernels.cu:153-231) */
#define GP(xx, yy) g[(size_t)(yy) * W + (xx)]
    for (int y = 2; y < H - 2; y++)
        for (int x = 2; x < W - 2; x++) {
            int col = cfa[(y & 1) * 2 + (x & 1)];
            int rowNext = cfa[(y & 1) * 2 + ((x + 1) & 1)];
            real gc = GP(x, y), r = 0, b = 0;
            if (col == 1) {
                /* horizontal neighbours carry the colour of this row */
                int hc = rowNext == 0 ? 0 : 2, vc = rowNext == 0 ? 2 : 0;
                real h = gc + 0.5 * ((LIN(x - 1, y, hc) - GP(x - 1, y)) + (LIN(x + 1, y, hc) - GP(x + 1, y)));
                real v = gc + 0.5 * ((LIN(x, y - 1, vc) - GP(x, y - 1)) + (LIN(x, y + 1, vc) - GP(x, y + 1)));
                if (hc == 0) { r = h; b = v; } else { b = h; r = v; }
            } else if (col == 0 || col == 2) {
                int oc = col == 0 ? 2 : 0;
                real own = LIN(x, y, col);
                real other = gc + 0.25 * ((LIN(x - 1, y - 1, oc) - GP(x - 1, y - 1)) + (LIN(x + 1, y - 1, oc) - GP(x + 1, y - 1)) +
                                          (LIN(x + 1, y + 1, oc) - GP(x + 1, y + 1)) + (LIN(x - 1, y + 1, oc) - GP(x - 1, y + 1)));
                if (col == 0) { r = own; b = other; } else { b = own; r = other; }
            }
            real* o = rgb + ((size_t)y * W + x) * 3;
            o[0] = r; o[1] = gc; o[2] = b;
        }
#undef GP
#undef LIN
    for (size_t i = 0; i < n; i++)
        for (int c = 0; c < 3; c++) rgb[i * 3 + c] /= divisor[c];
    free(g);
}

/* A2: sRGB gamma with NaN -> 0 and clamp to [0,1] (kernel.cu:290-332). The
 * constants are the reference's float literals (e.g. 1.0f / 2.4f is a float
 * quotient), carried into double exactly. */
EXPORT void orc_gamma_srgb(real* rgb, int W, int H)
{
    const real knee = (real)0.0031308f, slope = (real)12.92f, gain = (real)(1.0f + 0.055f);
    const real expo = (real)(1.0f / 2.4f), off = (real)0.055f;
    size_t n = (size_t)W * H * 3;
    for (size_t i = 0; i < n; i++) {
        real v = rgb[i];
        if (isnan(v)) v = 0;
        v = v < 0 ? 0 : (v > 1 ? 1 : v);
        rgb[i] = v <= knee ? slope * v : gain * pow(v, expo) - off;
    }
}

/* GammasRGB (kernel.cu:290-332) in float exactly as the reference's float
 * code: float literals, powf, each operation rounded on its own (no
 * contraction on this target). Used by the FP32 post-processing restatement
 * (oracle/post.py). n values in place. */
EXPORT void orc_gamma_srgb_f32(float* v, size_t n)
{
    for (size_t i = 0; i < n; i++) {
        float x = v[i];
        if (isnan(x)) x = 0.0f;
        x = fmaxf(fminf(x, 1.0f), 0.0f);
        if (x <= 0.0031308f) {
            x = 12.92f * x;
        } else {
            const float p = powf(x, 1.0f / 2.4f);
            const float g = (1.0f + 0.055f) * p;
            x = g - 0.055f;
        }
        v[i] = x;
    }
}

/* A2: NPP ColorToGray (controller :2404-2408): gray = sum_c w_c * rgb_c. */
EXPORT void orc_color_to_gray(const real* rgb, int W, int H, const real* w, real* gray)
{
    size_t n = (size_t)W * H;
    for (size_t i = 0; i < n; i++) gray[i] = w[0] * rgb[i * 3] + w[1] * rgb[i * 3 + 1] + w[2] * rgb[i * 3 + 2];
}

/* A2: frequency-domain filter coefficient of kernel.cu:704-779 for the
 * (W/2+1) x H half spectrum, including the clearAxis rule; the caller
 * multiplies both parts of each complex bin by it. */
EXPORT void orc_fourier_filter_mask(int W, int H, real lp, real hp, real lps, real hps, int clearAxis, real* mask)
{
    int Wc = W / 2 + 1;
    lp = lp - lps;
    hp = hp + hps;
    for (int y = 0; y < H; y++)
        for (int x = 0; x < Wc; x++) {
            real mx = x, my = y;
            if (my > H * 0.5) my = -(H - my);
            mx /= W; my /= H;
            real d = sqrt(mx * mx + my * my);
            real f = 0;
            if (lp > 0) { if (d <= lp) f = 1; }
            else { if (d <= 1.0) f = 1; }
            if (lps > 0) {
                real f2 = (1.0 - f) * exp(-((d - lp) * (d - lp) / (2 * lps * lps)));
                if (f2 > 0.001) f = f2;
            }
            if (lps > 0 && lp == 0 && hp == 0 && hps == 0) f = exp(-((d - lp) * (d - lp) / (2 * lps * lps)));
            if (hp > 0) {
                real f2 = d >= hp ? 1 : 0;
                f *= f2;
                if (hps > 0) {
                    real f3 = (1.0 - f2) * exp(-((d - hp) * (d - hp) / (2 * hps * hps)));
                    if (f3 > 0.001) f = f3;
                }
            }
            if (x < clearAxis || fabs(my) * H < clearAxis) f = 0;
            mask[(size_t)y * Wc + x] = f;
        }
}

/* A2: NPP ThresholdLTGT(0, 0, 1, 1) (PreAlignment.cs:280): clamp to [0,1]. */
EXPORT void orc_clamp01(real* img, size_t n)
{
    for (size_t i = 0; i < n; i++) img[i] = img[i] < 0 ? 0 : (img[i] > 1 ? 1 : img[i]);
}

/* Gaussian taps of gaussian_filter_1D (controller :2351-2382); returns the
 * tap count (at most 99). sigma <= 0 gives the 9-tap identity. */
EXPORT int orc_gauss_taps(real sigma, real* taps)
{
    if (sigma <= 0) {
        for (int i = 0; i < 9; i++) taps[i] = i == 4 ? 1 : 0;
        return 9;
    }
    int size = (int)(sigma / 0.6 - 0.4) * 2 + 1 + 2;
    if (size > 99) size = 99;
    int c = size / 2;
    real sum = 0;
    for (int i = 0; i < size; i++) {
        int x = i - c;
        taps[i] = exp(-(x * x) / (2 * sigma * sigma));
        sum += taps[i];
    }
    for (int i = 0; i < size; i++) taps[i] /= sum;
    return size;
}

/* NPP FilterGaussBorder with user taps and replicate border (controller
 * :2414, :1855): the separable filter applied along x then y to each of the
 * C interleaved channels. */
EXPORT void orc_gauss_filter(const real* in, int W, int H, int C, const real* taps, int n, real* out)
{
    int c0 = n / 2;
    real* tmp = (real*)malloc((size_t)W * H * C * sizeof(real));
    for (int y = 0; y < H; y++)
        for (int x = 0; x < W; x++)
            for (int c = 0; c < C; c++) {
                real s = 0;
                for (int k = 0; k < n; k++) s += taps[k] * in[((size_t)y * W + clampi(x + k - c0, 0, W - 1)) * C + c];
                tmp[((size_t)y * W + x) * C + c] = s;
            }
    for (int y = 0; y < H; y++)
        for (int x = 0; x < W; x++)
            for (int c = 0; c < C; c++) {
                real s = 0;
                for (int k = 0; k < n; k++) s += taps[k] * tmp[((size_t)clampi(y + k - c0, 0, H - 1) * W + x) * C + c];
                out[((size_t)y * W + x) * C + c] = s;
            }
    free(tmp);
}

/* NPP ResizeSqrPixel super-sampling by 1/L (controller :1696-1697): each
 * output pixel is the mean of its L x L source block; output is (W/L) x (H/L). */
EXPORT void orc_resize_box(const real* in, int W, int H, int L, real* out)
{
    int Wo = W / L, Ho = H / L;
    for (int y = 0; y < Ho; y++)
        for (int x = 0; x < Wo; x++) {
            real s = 0;
            for (int j = 0; j < L; j++)
                for (int i = 0; i < L; i++) s += in[(size_t)(y * L + j) * W + x * L + i];
            out[(size_t)y * Wo + x] = s / (L * L);
        }
}

/* ------------------------------------------------------------------------ */
/* A3: PatchTracker.Track for one frame pair at one level                    */
/* (PatchTracker.cs:317-360). Template tiles: kernel.cu:175-228; search      */
/* tiles: kernel.cu:234-288; L2 map = squaredSum + box filter - 2 CC         */
/* (kernel.cu:29-171, cuFFT CC with fft-shift indexing), which for |s| <= S  */
/* equals the direct sum of squared differences computed here; minimum and   */
/* sub-pixel fit: kernel.cu:413-546; preShift += result (:355-358).          */
/* ------------------------------------------------------------------------ */
static const real FIT_A11[9] = {0.25, -0.5, 0.25, 0.5, -1.0, 0.5, 0.25, -0.5, 0.25};
static const real FIT_A22[9] = {0.25, 0.5, 0.25, -0.5, -1.0, -0.5, 0.25, 0.5, 0.25};
static const real FIT_A12[9] = {0.25, 0, -0.25, 0, 0, 0, -0.25, 0, 0.25};
static const real FIT_B1[9] = {-0.125, 0, 0.125, -0.25, 0, 0.25, -0.125, 0, 0.125};
static const real FIT_B2[9] = {-0.125, -0.25, -0.125, 0, 0, 0, 0.125, 0.25, 0.125};

/* The integer pixel offset of a tile: rotation about the image centre plus
 * the negated base shift, rounded (kernel.cu:203-221, 262-281). */
static void tile_offset(int tx, int ty, int T, int Wl, int Hl, const real* base, real rot, real addx, real addy, int* ox, int* oy,
                        real* unrounded)
{
    real sf = sin(rot), cf = cos(rot);
    real sx = addx + cf * -base[0] - sf * -base[1];
    real sy = addy + sf * -base[0] + cf * -base[1];
    real pcx = tx * T + T / 2 - Wl / 2, pcy = ty * T + T / 2 - Hl / 2;
    sx += cf * pcx - sf * pcy - pcx;
    sy += sf * pcx + cf * pcy - pcy;
    *ox = (int)round(sx);
    *oy = (int)round(sy);
    if (unrounded) { unrounded[0] = sx; unrounded[1] = sy; }
}

/* scores (optional): tiles x (2S+1)^2 L2 maps; argmin (optional): index of
 * the first strict minimum per tile; offsets (optional): tiles x 2, the
 * search block's offset before rounding (PatchTracker.cs:225-253).
 * preShift: tcy x tcx float pairs. */
EXPORT void orc_track_pair(const real* imgTrack, const real* imgRef, int Wl, int Hl, int T, int S, int tcx, int tcy,
                           real* preShift, const real* baseRef, real rotRef, const real* baseTrk, real rotTrk,
                           real threshold, real* scores, int* argmin, real* offsets)
{
    int B = T + 2 * S, D = 2 * S + 1;
    real* tpl = (real*)malloc((size_t)T * T * sizeof(real));
    real* blk = (real*)malloc((size_t)B * B * sizeof(real));
    real* map = (real*)malloc((size_t)D * D * sizeof(real));
    for (int ty = 0; ty < tcy; ty++)
        for (int tx = 0; tx < tcx; tx++) {
            int t = ty * tcx + tx;
            int ox, oy;
            tile_offset(tx, ty, T, Wl, Hl, baseRef, rotRef, 0, 0, &ox, &oy, NULL);
            for (int y = 0; y < T; y++)
                for (int x = 0; x < T; x++) {
                    int ix = clampi(tx * T + S + x + ox, 0, Wl - 1), iy = clampi(ty * T + S + y + oy, 0, Hl - 1);
                    tpl[y * T + x] = imgRef[(size_t)iy * Wl + ix];
                }
            real* ps = preShift + (size_t)t * 2;
            tile_offset(tx, ty, T, Wl, Hl, baseTrk, rotTrk, ps[0], ps[1], &ox, &oy, offsets ? offsets + (size_t)t * 2 : NULL);
            for (int y = 0; y < B; y++)
                for (int x = 0; x < B; x++) {
                    int ix = clampi(tx * T + x + ox, 0, Wl - 1), iy = clampi(ty * T + y + oy, 0, Hl - 1);
                    blk[y * B + x] = imgTrack[(size_t)iy * Wl + ix];
                }
            for (int sy = 0; sy < D; sy++)
                for (int sx = 0; sx < D; sx++) {
                    real s = 0;
                    for (int y = 0; y < T; y++)
                        for (int x = 0; x < T; x++) {
                            real d = tpl[y * T + x] - blk[(y + sy) * B + x + sx];
                            s += d * d;
                        }
                    map[sy * D + sx] = s;
                }
            if (scores) memcpy(scores + (size_t)t * D * D, map, (size_t)D * D * sizeof(real));
            real mn = DBL_MAX, mx = -DBL_MAX;
            int mi = -1;
            for (int i = 0; i < D * D; i++) {
                if (map[i] > mx) mx = map[i];
                if (map[i] < mn) { mn = map[i]; mi = i; }
            }
            if (argmin) argmin[t] = mi;
            int cy = mi / D, cx = mi - cy * D;
            real rx, ry;
            if (cx < 1 || cy < 1 || cx >= 2 * S || cy >= 2 * S) {
                rx = 0; ry = 0;
            } else {
                real a11 = 0, a22 = 0, a12 = 0, b1 = 0, b2 = 0;
                for (int k = 0; k < 9; k++) {
                    real v = map[(cy + k / 3 - 1) * D + cx + k % 3 - 1];
                    a11 += FIT_A11[k] * v; a22 += FIT_A22[k] * v; a12 += FIT_A12[k] * v;
                    b1 += FIT_B1[k] * v; b2 += FIT_B2[k] * v;
                }
                if (a11 < 0) a11 = 0;
                if (a22 < 0) a22 = 0;
                real det = a11 * a22 - a12 * a12;
                if (det < 0) { a12 = 0; det = a11 * a22; }
                rx = cx; ry = cy;
                if (det != 0) {
                    real mux = (a22 * b1 - a12 * b2) / det, muy = (a11 * b2 - a12 * b1) / det;
                    if (fabs(mux) > 1) mux = 0;
                    if (fabs(muy) > 1) muy = 0;
                    rx -= mux; ry -= muy;
                }
                rx -= S; ry -= S;
            }
            if (threshold + mn > mx) { rx = 0; ry = 0; }
            ps[0] += rx;
            ps[1] += ry;
        }
    free(tpl); free(blk); free(map);
}

/* A4: UpSampleShifts (kernel.cu:552-598). in: ocy x ocx pairs, out: ncy x ncx. */
EXPORT void orc_upsample_shifts(const real* in, real* out, int oldLevel, int newLevel, int ocx, int ocy, int ncx, int ncy, int oldT, int newT)
{
    real f = (real)oldLevel * oldT / (real)(newLevel * newT);
    for (int ny = 0; ny < ncy; ny++)
        for (int nx = 0; nx < ncx; nx++) {
            real ox = nx / f, oy = ny / f;
            int x0 = (int)floor(ox), x1 = (int)ceil(ox), y0 = (int)floor(oy), y1 = (int)ceil(oy);
            x0 = x0 < ocx - 1 ? x0 : ocx - 1; x1 = x1 < ocx - 1 ? x1 : ocx - 1;
            y0 = y0 < ocy - 1 ? y0 : ocy - 1; y1 = y1 < ocy - 1 ? y1 : ocy - 1;
            real wx = 1.0 - (x1 - ox), wy = 1.0 - (y1 - oy);
            for (int c = 0; c < 2; c++) {
                real v00 = in[((size_t)y0 * ocx + x0) * 2 + c], v10 = in[((size_t)y0 * ocx + x1) * 2 + c];
                real v01 = in[((size_t)y1 * ocx + x0) * 2 + c], v11 = in[((size_t)y1 * ocx + x1) * 2 + c];
                real t0 = v00 + (v10 - v00) * wx, t1 = v01 + (v11 - v01) * wx;
                out[((size_t)ny * ncx + nx) * 2 + c] = (t0 + (t1 - t0) * wy) * (oldLevel / (real)newLevel);
            }
        }
}

/* ------------------------------------------------------------------------ */
/* A5: ShiftCollection.MinimizeCUBLAS (ShiftCollection.cs:738-822) with the */
/* kernels of ShiftMinimizerKernels.cu:81-140 (outlier rule) and :143-176.  */
/* Per tile: up to 10 rounds of x = (A^T A)^-1 A^T b; after each solve the  */
/* pair with the largest squared residual above 1 is removed (its row of A  */
/* and its measurement zeroed). The final pair shifts are A_orig x.         */
/* A is m x n1 row-major (row = pair, column = one-to-one shift).           */
/* meas: tiles x m x 2 (in: measured, out: re-synthesised); x: tiles x n1 x 2;*/
/* status: -1 converged, -3 singular (previous solve kept), >=0 the pair    */
/* removed in the tenth round.                                              */
/* ------------------------------------------------------------------------ */
static int invert_spd(double* a, double* inv, int n)
{
    /* Gauss-Jordan with partial pivoting; singular if a pivot is below a
     * relative bound. a is destroyed. */
    double scale = 0;
    for (int i = 0; i < n; i++) scale = fmax(scale, fabs(a[i * n + i]));
    for (int i = 0; i < n * n; i++) inv[i] = 0;
    for (int i = 0; i < n; i++) inv[i * n + i] = 1;
    for (int c = 0; c < n; c++) {
        int p = c;
        for (int r = c + 1; r < n; r++) if (fabs(a[r * n + c]) > fabs(a[p * n + c])) p = r;
        if (!(fabs(a[p * n + c]) > 1e-12 * (scale > 0 ? scale : 1))) return 1;
        if (p != c)
            for (int k = 0; k < n; k++) {
                double t = a[c * n + k]; a[c * n + k] = a[p * n + k]; a[p * n + k] = t;
                t = inv[c * n + k]; inv[c * n + k] = inv[p * n + k]; inv[p * n + k] = t;
            }
        double d = a[c * n + c];
        for (int k = 0; k < n; k++) { a[c * n + k] /= d; inv[c * n + k] /= d; }
        for (int r = 0; r < n; r++) {
            if (r == c) continue;
            double f = a[r * n + c];
            if (f == 0) continue;
            for (int k = 0; k < n; k++) { a[r * n + k] -= f * a[c * n + k]; inv[r * n + k] -= f * inv[c * n + k]; }
        }
    }
    return 0;
}

EXPORT void orc_solve_shifts(const real* Aorig, int m, int n1, int tiles, real* meas, real* x, int* status)
{
    double* A = (double*)malloc((size_t)m * n1 * sizeof(double));
    double* b = (double*)malloc((size_t)m * 2 * sizeof(double));
    double* N = (double*)malloc((size_t)n1 * n1 * sizeof(double));
    double* Ni = (double*)malloc((size_t)n1 * n1 * sizeof(double));
    double* sol = (double*)malloc((size_t)n1 * 2 * sizeof(double));
    double* rhs = (double*)malloc((size_t)n1 * 2 * sizeof(double));
    for (int t = 0; t < tiles; t++) {
        for (int i = 0; i < m * n1; i++) A[i] = Aorig[i];
        for (int i = 0; i < m * 2; i++) b[i] = meas[(size_t)t * m * 2 + i];
        for (int i = 0; i < n1 * 2; i++) sol[i] = 0;
        int st = -1;
        for (int round_ = 0; round_ < 10; round_++) {
            for (int i = 0; i < n1; i++)
                for (int j = 0; j < n1; j++) {
                    double s = 0;
                    for (int k = 0; k < m; k++) s += A[k * n1 + i] * A[k * n1 + j];
                    N[i * n1 + j] = s;
                }
            if (invert_spd(N, Ni, n1)) { st = -3; break; }
            for (int i = 0; i < n1; i++)
                for (int c = 0; c < 2; c++) {
                    double s = 0;
                    for (int k = 0; k < m; k++) s += A[k * n1 + i] * b[k * 2 + c];
                    rhs[i * 2 + c] = s;
                }
            for (int i = 0; i < n1; i++)
                for (int c = 0; c < 2; c++) {
                    double s = 0;
                    for (int j = 0; j < n1; j++) s += Ni[i * n1 + j] * rhs[j * 2 + c];
                    sol[i * 2 + c] = s;
                }
            /* largest squared residual above 1 (checkForOutliers,
             * ShiftMinimizerKernels.cu:104-117); residuals within a relative
             * 1e-9 of the largest count as ties and the lowest row wins, so the
             * choice does not depend on rounding when two rows are equal in
             * exact arithmetic */
            double worst = 1;
            int wi = -1;
            for (int pass = 0; pass < 2; pass++) {
                double thr = worst * (1 - 1e-9);
                for (int k = 0; k < m; k++) {
                    double px = 0, py = 0;
                    for (int j = 0; j < n1; j++) { px += A[k * n1 + j] * sol[j * 2]; py += A[k * n1 + j] * sol[j * 2 + 1]; }
                    double dx = b[k * 2] - px, dy = b[k * 2 + 1] - py;
                    double d = dx * dx + dy * dy;
                    if (pass == 0) { if (d > worst) { worst = d; wi = k; } }
                    else if (wi >= 0 && d >= thr && d > 1) { wi = k; break; }
                }
                if (wi < 0) break;
            }
            st = wi;
            if (wi < 0) break;
            b[wi * 2] = 0; b[wi * 2 + 1] = 0;
            for (int j = 0; j < n1; j++) A[wi * n1 + j] = 0;
        }
        status[t] = st;
        for (int i = 0; i < n1 * 2; i++) x[(size_t)t * n1 * 2 + i] = sol[i];
        for (int k = 0; k < m; k++) {
            double px = 0, py = 0;
            for (int j = 0; j < n1; j++) { px += Aorig[k * n1 + j] * sol[j * 2]; py += Aorig[k * n1 + j] * sol[j * 2 + 1]; }
            meas[((size_t)t * m + k) * 2] = px;
            meas[((size_t)t * m + k) * 2 + 1] = py;
        }
    }
    free(A); free(b); free(N); free(Ni); free(sol); free(rhs);
}

/* A5 end: getOptimalShifts (ShiftMinimizerKernels.cu:179-218): the shift of
 * frame `trk` relative to `ref` as a signed sum of one-to-one shifts.
 * x: tiles x n1 x 2; out: tiles x 2. */
EXPORT void orc_optimal_shifts(const real* x, int n1, int tiles, int ref, int trk, real* out)
{
    for (int t = 0; t < tiles; t++) {
        const real* r = x + (size_t)t * n1 * 2;
        real sx = 0, sy = 0;
        if (ref < trk) for (int i = ref; i < trk; i++) { sx += r[i * 2]; sy += r[i * 2 + 1]; }
        else if (trk < ref) for (int i = trk; i < ref; i++) { sx -= r[i * 2]; sy -= r[i * 2 + 1]; }
        out[t * 2] = sx; out[t * 2 + 1] = sy;
    }
}

/* ------------------------------------------------------------------------ */
/* A6: Lucas-Kanade refinement (OpticalFlow.cs:147-164).                     */
/* ------------------------------------------------------------------------ */
/* CreateFlowFieldFromTiles (opticalFlow.cu:48-94): rotation/base term plus
 * the tile grid sampled bilinearly (clamp) over the whole frame. */
EXPORT void orc_flow_from_tiles(const real* tiles, int tcx, int tcy, int W, int H, const real* base, real rot, real* flow)
{
    real c = cos(rot), s = sin(rot);
    for (int y = 0; y < H; y++)
        for (int x = 0; x < W; x++) {
            real fx = c * -base[0] - s * -base[1];
            real fy = s * -base[0] + c * -base[1];
            real pcx = x - W / 2, pcy = y - H / 2;
            fx += c * pcx - s * pcy - pcx;
            fy += s * pcx + c * pcy - pcy;
            real xb = (x + 0.5) / W * tcx - 0.5, yb = (y + 0.5) / H * tcy - 0.5;
            fx += bilinear(tiles, tcx, tcy, 2, 0, xb, yb, 0);
            fy += bilinear(tiles, tcx, tcy, 2, 1, xb, yb, 0);
            flow[((size_t)y * W + x) * 2] = fx;
            flow[((size_t)y * W + x) * 2 + 1] = fy;
        }
}

/* WarpingKernel (opticalFlow.cu:28-45): out(x) = img sampled bilinearly with
 * mirror addressing at x + flow(x). */
EXPORT void orc_warp(const real* img, int W, int H, const real* flow, real* out)
{
    for (int y = 0; y < H; y++)
        for (int x = 0; x < W; x++) {
            const real* f = flow + ((size_t)y * W + x) * 2;
            out[(size_t)y * W + x] = bilinear(img, W, H, 1, 0, x + f[0], y + f[1], 1);
        }
}

static inline real at_m(const real* img, int W, int H, int x, int y) {
    return img[(size_t)mirror_index(y, H) * W + mirror_index(x, W)];
}
/* five-tap difference of the reference: (f(+2) - 8 f(+1) + 8 f(-1) - f(-2)) / 12 */
static inline real d5x(const real* f, int W, int H, int x, int y) {
    return (at_m(f, W, H, x + 2, y) - 8 * at_m(f, W, H, x + 1, y) + 8 * at_m(f, W, H, x - 1, y) - at_m(f, W, H, x - 2, y)) / 12;
}
static inline real d5y(const real* f, int W, int H, int x, int y) {
    return (at_m(f, W, H, x, y + 2) - 8 * at_m(f, W, H, x, y + 1) + 8 * at_m(f, W, H, x, y - 1) - at_m(f, W, H, x, y - 2)) / 12;
}

/* ComputeDerivativesKernel (opticalFlow.cu:97-148). */
EXPORT void orc_derivatives(const real* src, const real* tgt, int W, int H, real* Ix, real* Iy, real* It)
{
    for (int y = 0; y < H; y++)
        for (int x = 0; x < W; x++) {
            size_t i = (size_t)y * W + x;
            Ix[i] = (d5x(src, W, H, x, y) + d5x(tgt, W, H, x, y)) * 0.5;
            It[i] = src[i] - tgt[i];
            Iy[i] = (d5y(src, W, H, x, y) + d5y(tgt, W, H, x, y)) * 0.5;
        }
}

/* ComputeDerivatives2Kernel (opticalFlow.cu:151-185). */
EXPORT void orc_derivatives2(const real* img, int W, int H, real* Ix, real* Iy)
{
    for (int y = 0; y < H; y++)
        for (int x = 0; x < W; x++) {
            Ix[(size_t)y * W + x] = d5x(img, W, H, x, y);
            Iy[(size_t)y * W + x] = d5y(img, W, H, x, y);
        }
}

/* 2x2 pseudo-inverse of the windowed normal matrix exactly as
 * opticalFlow.cu:229-290 forms it (angles from atan2, singular values from
 * the sums of squares, the `min(sigma1, sigma1)` test against minDet kept).
 * Returns 0 when the reference leaves the pixel untouched. */
static int lk_pinv(real a, real b, real c, real d, real minDet, real* M)
{
    real th = 0.5 * atan2(2 * a * c + 2 * b * d, a * a + b * b - c * c - d * d);
    real ct = cos(th), st = sin(th);
    real S1 = a * a + b * b + c * c + d * d;
    real S2 = sqrt((a * a + b * b - c * c - d * d) * (a * a + b * b - c * c - d * d) + 4 * (a * c + b * d) * (a * c + b * d));
    real s1 = sqrt((S1 + S2) / 2), s2 = sqrt((S1 - S2) / 2);
    if (s1 < minDet) return 0; /* the reference tests min(sigma1, sigma1) */
    s1 = s1 != 0 ? 1 / s1 : 0;
    s2 = s2 != 0 ? 1 / s2 : 0;
    real ep = 0.5 * atan2(2 * a * b + 2 * c * d, a * a - b * b + c * c - d * d);
    real ce = cos(ep), se = sin(ep);
    real q11 = (a * ct + c * st) * ce + (b * ct + d * st) * se;
    real q22 = (a * st - c * ct) * se + (-b * st + d * ct) * ce;
    q11 = q11 > 0 ? 1 : (q11 < 0 ? -1 : 0);
    q22 = q22 > 0 ? 1 : (q22 < 0 ? -1 : 0);
    real V0 = q11 * ce, V1 = -q22 * se, V2 = q11 * se, V3 = q22 * ce;
    /* S * U^T with U^T = [ct st; -st ct] */
    real m0 = s1 * ct, m1 = s1 * st, m2 = s2 * -st, m3 = s2 * ct;
    M[0] = V0 * m0 + V1 * m2;
    M[1] = V0 * m1 + V1 * m3;
    M[2] = V2 * m0 + V3 * m2;
    M[3] = V2 * m1 + V3 * m3;
    return 1;
}

/* lucasKanadeOptim (opticalFlow.cu:190-325): flow += pinv(sum grad grad^T)
 * * sum grad * It over a (2h+1)^2 window, for pixels at least h from the
 * border; NaN updates become 0. */
EXPORT void orc_lucas_kanade(real* flow, const real* Ix, const real* Iy, const real* It, int W, int H, int h, real minDet)
{
    for (int y = h; y < H - h; y++)
        for (int x = h; x < W - h; x++) {
            real sxx = 0, sxy = 0, syy = 0, sxt = 0, syt = 0;
            for (int j = -h; j <= h; j++)
                for (int i = -h; i <= h; i++) {
                    size_t k = (size_t)(y + j) * W + x + i;
                    sxx += Ix[k] * Ix[k]; sxy += Ix[k] * Iy[k]; syy += Iy[k] * Iy[k];
                    sxt += Ix[k] * It[k]; syt += Iy[k] * It[k];
                }
            real M[4];
            if (!lk_pinv(sxx, sxy, sxy, syy, minDet, M)) continue;
            real u = M[0] * sxt + M[1] * syt, v = M[2] * sxt + M[3] * syt;
            if (isnan(u)) u = 0;
            if (isnan(v)) v = 0;
            flow[((size_t)y * W + x) * 2] += u;
            flow[((size_t)y * W + x) * 2 + 1] += v;
        }
}

/* ------------------------------------------------------------------------ */
/* A7: robustness mask.                                                      */
/* ------------------------------------------------------------------------ */
/* deBayersSubSample3 (DeBayerKernels.cu:244-283): each 2x2 CFA quad to one
 * RGB pixel, greens averaged, all divided by maxVal (black not removed).
 * raw: H x W; out: (H/2) x (W/2) x 3. */
EXPORT void orc_debayer_subsample(const uint16_t* raw, int W, int H, const int* cfa, real maxVal, real* out)
{
    int Wh = W / 2, Hh = H / 2;
    real f = 1.0 / maxVal;
    for (int y = 0; y < Hh; y++)
        for (int x = 0; x < Wh; x++) {
            real p[3] = {0, 0, 0};
            for (int ix = 0; ix < 2; ix++)
                for (int iy = 0; iy < 2; iy++) {
                    int col = cfa[iy * 2 + ix];
                    real v = raw[(size_t)(2 * y + iy) * W + 2 * x + ix];
                    if (col == 1) p[1] += v * f * 0.5;
                    else if (col == 0) p[0] = v * f;
                    else if (col == 2) p[2] = v * f;
                }
            real* o = out + ((size_t)y * Wh + x) * 3;
            o[0] = p[0]; o[1] = p[1]; o[2] = p[2];
        }
}

/* ComputeRobustnessMask (RobustnessModell.cu:29-157). ref/moved: Hh x Wh x 3;
 * flow: full-resolution (2Hh x 2Wh x 2 in the reference, any Wf x Hf here)
 * sampled bilinearly with mirror addressing at the half-res pixel's
 * normalized position; mask: Hh x Wh x 4, border pixels left untouched.
 * The running max/min of the reference compares each tap with the centre
 * only, so M depends on the last tap; kept as is. s and t are the literals
 * 1.5 and 0.12 of the reference. */
/* bil = 0: the moved 3x3 mean at round(flow / 2) (RobustnessModell.cu:401-402);
 * bil = 1 (sample mode BILINEAR, no counterpart in the reference): the
 * moved means at the four integer offsets around flow / 2, blended with the
 * bilinear weights of its fractional part, so that the mask is continuous in
 * the flow. */
static void robustness_mask_mode(const real* ref, const real* mov, int Wh, int Hh, const real* flow, int Wf, int Hf,
                                 real alpha, real beta, real thresholdM, real s_lit, real t_lit, real* mask, int bil)
{
    for (int y = 1; y < Hh - 1; y++)
        for (int x = 1; x < Wh - 1; x++) {
            real cxb = (x + 0.5) / Wh * Wf - 0.5, cyb = (y + 0.5) / Hh * Hf - 0.5;
            real fx = bilinear(flow, Wf, Hf, 2, 0, cxb, cyb, 1), fy = bilinear(flow, Wf, Hf, 2, 1, cxb, cyb, 1);
            real mxx = fx, mxy = fy, mnx = fx, mny = fy;
            for (int j = -2; j <= 2; j++)
                for (int i = -2; i <= 2; i++) {
                    real xb = (x + i + 0.5) / Wh * Wf - 0.5, yb = (y + j + 0.5) / Hh * Hf - 0.5;
                    real sx = bilinear(flow, Wf, Hf, 2, 0, xb, yb, 1), sy = bilinear(flow, Wf, Hf, 2, 1, xb, yb, 1);
                    mxx = fmax(sx, fx); mxy = fmax(sy, fy);
                    mnx = fmin(sx, fx); mny = fmin(sy, fy);
                }
            real mr[3] = {0, 0, 0}, mm[3] = {0, 0, 0}, sd[3] = {0, 0, 0};
            for (int j = -1; j <= 1; j++)
                for (int i = -1; i <= 1; i++) {
                    const real* p = ref + ((size_t)(y + j) * Wh + x + i) * 3;
                    for (int c = 0; c < 3; c++) mr[c] += p[c];
                }
            int shx, shy, nc;
            real bx = 0, by = 0;
            if (bil) {
                real hx = fx * 0.5, hy = fy * 0.5;
                shx = (int)floor(hx); shy = (int)floor(hy);
                bx = hx - shx; by = hy - shy;
                nc = 4;
            } else {
                shx = (int)round(fx * 0.5); shy = (int)round(fy * 0.5);
                nc = 1;
            }
            for (int k = 0; k < nc; k++) {
                int dx = k & 1, dy = k >> 1;
                real wk = bil ? (dx ? bx : 1 - bx) * (dy ? by : 1 - by) : 1;
                real box[3] = {0, 0, 0};
                for (int j = -1; j <= 1; j++)
                    for (int i = -1; i <= 1; i++) {
                        int qy = clampi(y + shy + dy + j, 0, Hh - 1), qx = clampi(x + shx + dx + i, 0, Wh - 1);
                        const real* q = mov + ((size_t)qy * Wh + qx) * 3;
                        for (int c = 0; c < 3; c++) box[c] += q[c];
                    }
                for (int c = 0; c < 3; c++) mm[c] += wk * (box[c] / 9);
            }
            for (int c = 0; c < 3; c++) mr[c] /= 9;
            real md = (fabs(mr[0] - mm[0]) + fabs(mr[1] - mm[1]) + fabs(mr[2] - mm[2])) / 3;
            mxx *= 0.5 * md; mxy *= 0.5 * md; mnx *= 0.5 * md; mny *= 0.5 * md;
            real M = sqrt((mxx - mnx) * (mxx - mnx) + (mxy - mny) * (mxy - mny));
            for (int j = -1; j <= 1; j++)
                for (int i = -1; i <= 1; i++) {
                    const real* p = ref + ((size_t)(y + j) * Wh + x + i) * 3;
                    for (int c = 0; c < 3; c++) sd[c] += (p[c] - mr[c]) * (p[c] - mr[c]);
                }
            real* o = mask + ((size_t)y * Wh + x) * 4;
            real sgain = M > thresholdM ? 0 : s_lit;
            for (int c = 0; c < 3; c++) {
                real sr = sqrt(sd[c] / 9);
                real smd = sqrt(alpha * mr[c] + beta);
                if (c == 1) smd /= (real)sqrtf(2.0f); /* the float constant of the reference */
                real dist = fabs(mr[c] - mm[c]) * (sr * sr / (sr * sr + smd * smd));
                real sig = fmax(smd, sr);
                real v = sgain * exp(-dist * dist / (sig * sig)) - t_lit;
                o[c] = fmax(fmin(v, 1.0), 0.0);
            }
            o[3] = M;
        }
}

EXPORT void orc_robustness_mask(const real* ref, const real* mov, int Wh, int Hh, const real* flow, int Wf, int Hf,
                                real alpha, real beta, real thresholdM, real s_lit, real t_lit, real* mask)
{
    robustness_mask_mode(ref, mov, Wh, Hh, flow, Wf, Hf, alpha, beta, thresholdM, s_lit, t_lit, mask, 0);
}

EXPORT void orc_robustness_mask_bil(const real* ref, const real* mov, int Wh, int Hh, const real* flow, int Wf, int Hf,
                                    real alpha, real beta, real thresholdM, real s_lit, real t_lit, real* mask)
{
    robustness_mask_mode(ref, mov, Wh, Hh, flow, Wf, Hf, alpha, beta, thresholdM, s_lit, t_lit, mask, 1);
}

/* NPP ErodeBorder with an all-ones size x size mask, anchor size/2 and
 * replicate border (controller :1976): per-channel minimum. */
EXPORT void orc_erode(const real* in, int W, int H, int C, int size, real* out)
{
    int a = size / 2;
    for (int y = 0; y < H; y++)
        for (int x = 0; x < W; x++)
            for (int c = 0; c < C; c++) {
                real m = DBL_MAX;
                for (int j = 0; j < size; j++)
                    for (int i = 0; i < size; i++) {
                        real v = in[((size_t)clampi(y + j - a, 0, H - 1) * W + clampi(x + i - a, 0, W - 1)) * C + c];
                        if (v < m) m = v;
                    }
                out[((size_t)y * W + x) * C + c] = m;
            }
}

/* ------------------------------------------------------------------------ */
/* A8: structure tensor and kernel parameters.                               */
/* ------------------------------------------------------------------------ */
/* ComputeStructureTensor (kernel.cu:601-625): (dx^2, dy^2, dx dy). */
EXPORT void orc_structure_tensor(const real* dx, const real* dy, int W, int H, real* out)
{
    size_t n = (size_t)W * H;
    for (size_t i = 0; i < n; i++) { out[i * 3] = dx[i] * dx[i]; out[i * 3 + 1] = dy[i] * dy[i]; out[i * 3 + 2] = dx[i] * dy[i]; }
}

/* ComputeKernelParam (kernel.cu:628-700): in place, (a11,a22,a12) -> the
 * inverse kernel covariance (b22/det, b11/det, -b12/det). */
EXPORT void orc_kernel_param(real* st, int W, int H, real Dth, real Dtr, real kDetail, real kDenoise, real kStretch, real kShrink)
{
    size_t n = (size_t)W * H;
    for (size_t i = 0; i < n; i++) {
        real a11 = st[i * 3], a22 = st[i * 3 + 1], a12 = st[i * 3 + 2];
        real hlp = sqrt((a22 - a11) * (a22 - a11) + 4 * a12 * a12);
        real c = 2 * a12, s = a22 - a11 + hlp;
        real nrm = sqrt(c * c + s * s);
        if (nrm > 0) { c /= nrm; s /= nrm; } else { c = 1; s = 0; }
        real l1 = (a11 + a22 + hlp) / 2, l2 = (a11 + a22 - hlp) / 2;
        real A = 1 + sqrt((l1 - l2) * (l1 - l2) / ((l1 + l2) * (l1 + l2)));
        real D = 1 - sqrt(l1) / Dtr + Dth;
        D = fmax(fmin(1.0, D), 0.0); /* fmin/fmax return the non-NaN operand, like fminf/fmaxf */
        real k1 = (1 - D) * (kDetail * kStretch * A) + D * kDetail * kDenoise;
        real k2 = (1 - D) * (kDetail / kShrink * A) + D * kDetail * kDenoise;
        k1 *= k1; k2 *= k2;
        real x2 = c, y2 = s, x1 = s, y1 = -c;
        real b11 = k1 * x1 * x1 + x2 * x2 * k2;
        real b12 = k1 * x1 * y1 + x2 * y2 * k2;
        real b22 = k1 * y1 * y1 + y2 * y2 * k2;
        real det = b11 * b22 - b12 * b12 + 0.0000000001;
        st[i * 3] = b22 / det; st[i * 3 + 1] = b11 / det; st[i * 3 + 2] = -b12 / det;
    }
}

/* ------------------------------------------------------------------------ */
/* A9: kernel-weighted Bayer accumulation, generalised to merge scale s.     */
/* accumulateImages (DeBayerKernels.cu:290-376) is s = 1, origin 0, crop =   */
/* the whole frame; accumulateImagesSuperRes (DeBayerKernels.cu:379-468) is  */
/* s = 2, origin (W/2, H/2), crop = the central W/2 x H/2 of the frame.      */
/* Output pixel (x,y) samples kernel parameters (clamp) and flow (mirror)    */
/* bilinearly at input position ((x+0.5+ox)/s, (y+0.5+oy)/s); the shift is  */
/* round(s*flow); each of the 25 taps reads the raw sample at                */
/* floor((x+px+sx+ox)/s) clamped to the crop, the certainty of the unshifted */
/* tap's half-resolution pixel, and adds to the channel of the CFA colour.   */
/* raw: H x W; acc, wsum: Ho x Wo x 3; mask: (H/2) x (W/2) x 4;              */
/* kparam: H x W x kc (kc = 3 or 4); flow: H x W x 2.                        */
/* crop: x0, y0, x1, y1 inclusive.                                           */
/* ------------------------------------------------------------------------ */
/* bil = 0: the frame is read at the integer shift round(s * flow)
 * (DeBayerKernels.cu:310-311, 403-404); bil = 1 (sample mode BILINEAR, no
 * counterpart in the reference): the contributions at the four integer
 * shifts around s * flow, blended with the bilinear weights of its
 * fractional part, so that the merge is continuous in the flow. */
static void accumulate_mode(const uint16_t* raw, int W, int H, const int* cfa, real* acc, real* wsum, int Wo, int Ho,
                            const real* mask, const real* kparam, int kc, const real* flow,
                            const real* white, const real* black, real s, int ox, int oy, const int* crop, int bil)
{
    int Wm = W / 2;
    for (int y = 1; y < Ho - 1; y++)
        for (int x = 1; x < Wo - 1; x++) {
            real xb = (x + 0.5 + ox) / s - 0.5, yb = (y + 0.5 + oy) / s - 0.5;
            real k0 = bilinear(kparam, W, H, kc, 0, xb, yb, 0);
            real k1 = bilinear(kparam, W, H, kc, 1, xb, yb, 0);
            real k2 = bilinear(kparam, W, H, kc, 2, xb, yb, 0);
            real fx = bilinear(flow, W, H, 2, 0, xb, yb, 1), fy = bilinear(flow, W, H, 2, 1, xb, yb, 1);
            int sx0, sy0, nc;
            real bx = 0, by = 0;
            if (bil) {
                real hx = fx * s, hy = fy * s;
                sx0 = (int)floor(hx); sy0 = (int)floor(hy);
                bx = hx - sx0; by = hy - sy0;
                nc = 4;
            } else {
                sx0 = (int)round(fx * s); sy0 = (int)round(fy * s);
                nc = 1;
            }
            real* a = acc + ((size_t)y * Wo + x) * 3;
            real* w = wsum + ((size_t)y * Wo + x) * 3;
            real wts[25];
            for (int py = -2; py <= 2; py++)
                for (int px = -2; px <= 2; px++) {
                    real q = px * px * k0 + 2 * px * py * k2 + py * py * k1;
                    real wt = exp(-0.5 * q);
                    if (!isfinite(wt)) wt = px * py == 0 ? 1 : 0;
                    wts[(py + 2) * 5 + px + 2] = wt;
                }
            for (int k = 0; k < nc; k++) {
                int sx = sx0 + (k & 1), sy = sy0 + (k >> 1);
                real wk = bil ? ((k & 1) ? bx : 1 - bx) * ((k >> 1) ? by : 1 - by) : 1;
                if (wk == 0) continue;
                for (int py = -2; py <= 2; py++)
                    for (int px = -2; px <= 2; px++) {
                        int qx = clampi((int)floor((x + px + sx + ox) / s), crop[0], crop[2]);
                        int qy = clampi((int)floor((y + py + sy + oy) / s), crop[1], crop[3]);
                        int ux = clampi((int)floor((x + px + ox) / s), crop[0], crop[2]);
                        int uy = clampi((int)floor((y + py + oy) / s), crop[1], crop[3]);
                        int col = cfa[(qy & 1) * 2 + (qx & 1)];
                        real wt = wts[(py + 2) * 5 + px + 2];
                        if (col < 0 || col > 2) continue;
                        real v = ((real)raw[(size_t)qy * W + qx] - black[col]) / white[col];
                        real cert = mask[((size_t)(uy / 2) * Wm + ux / 2) * 4 + col];
                        if (!isfinite(cert)) cert = 0;
                        if (bil) cert *= wk;
                        a[col] += v * wt * cert;
                        w[col] += wt * cert;
                    }
            }
        }
}

EXPORT void orc_accumulate(const uint16_t* raw, int W, int H, const int* cfa, real* acc, real* wsum, int Wo, int Ho,
                           const real* mask, const real* kparam, int kc, const real* flow,
                           const real* white, const real* black, real s, int ox, int oy, const int* crop)
{
    accumulate_mode(raw, W, H, cfa, acc, wsum, Wo, Ho, mask, kparam, kc, flow, white, black, s, ox, oy, crop, 0);
}

EXPORT void orc_accumulate_bil(const uint16_t* raw, int W, int H, const int* cfa, real* acc, real* wsum, int Wo, int Ho,
                               const real* mask, const real* kparam, int kc, const real* flow,
                               const real* white, const real* black, real s, int ox, int oy, const int* crop)
{
    accumulate_mode(raw, W, H, cfa, acc, wsum, Wo, Ho, mask, kparam, kc, flow, white, black, s, ox, oy, crop, 1);
}

/* A10: ApplyWeighting (kernel.cu:336-391): per channel, where w < thr the
 * fallback `img` value and one unit of weight are added; out = num / den or
 * 0. img is read as the fallback and overwritten with the result. */
EXPORT void orc_apply_weighting(real* img, const real* acc, const real* wsum, int W, int H, real thr)
{
    size_t n = (size_t)W * H * 3;
    for (size_t i = 0; i < n; i++) {
        real v = acc[i], w = wsum[i];
        if (w < thr) { v += img[i]; w += 1; }
        img[i] = w != 0 ? v / w : 0;
    }
}

/* ---- Raw decoding (PEF) ----
 * MNHuffmanTable (PefFile/PentaxMakerNotesEntry.cs:4555-4613): the maker
 * note's bytes hold a u16 (dep - 12), 12 bytes not used, dep u16 code words
 * left-aligned in 12 bits and dep u8 code lengths (all u16 in the file's
 * byte order). The decode table has table[0] = 12 and, for each code c,
 * table[1 + i] = len << 8 | c over the 4096 >> len peeks i that start with
 * the code. */
EXPORT int orc_pef_huff_table(const uint8_t* mn, int n, int big_endian, uint16_t* table)
{
    uint16_t code[16], len[16];
    memset(table, 0, 4097 * sizeof(uint16_t));
    if (n < 2) return -1;
#define RD16(p) (big_endian ? (uint16_t)((p)[0] << 8 | (p)[1]) : (uint16_t)((p)[1] << 8 | (p)[0]))
    const int dep = (RD16(mn) + 12) & 15;
    if (n < 14 + 3 * dep) return -1;
    for (int c = 0; c < dep; c++) code[c] = RD16(mn + 14 + 2 * c);
    for (int c = 0; c < dep; c++) len[c] = mn[14 + 2 * dep + c];
#undef RD16
    for (int c = 0; c < dep; c++) {
        for (int i = code[c]; i <= ((code[c] + (4096 >> len[c]) - 1) & 4095);) table[++i] = (uint16_t)(len[c] << 8 | c);
        table[0] = 12;
    }
    return dep;
}

/* The bit reader of PEFFile (getbithuff, PEFFile.cs:35-69): bytes are
 * appended to a 32-bit buffer while fewer than nbits are valid; reads past
 * the end of the data give zero bytes. */
typedef struct { const uint8_t* d; size_t n, pos; uint32_t buf; int vbits; } orc_bits;

static uint32_t orc_getbithuff(orc_bits* b, int nbits, const uint16_t* huff)
{
    if (nbits > 25) return 0;
    if (nbits == 0 || b->vbits < 0) return 0;
    while (b->vbits < nbits) {
        uint32_t c = b->pos < b->n ? b->d[b->pos] : 0;
        b->pos++;
        b->buf = (b->buf << 8) + (uint8_t)c;
        b->vbits += 8;
    }
    uint32_t c = b->buf << (32 - b->vbits) >> (32 - nbits);
    if (huff) {
        b->vbits -= huff[c] >> 8;
        c = (uint8_t)huff[c];
    } else {
        b->vbits -= nbits;
    }
    return c;
}

/* PEFFile(aFileName) compressed branch (PEFFile.cs:81-111): one strip,
 * ljpeg_diff per pixel in raster order, the first two columns predicted
 * from the pixel two rows up (vpred), the others from the pixel two
 * columns left (hpred), stored as (ushort). The shift by len - 1 uses the
 * 5-bit shift count of C# (len = 0 gives diff = 0). */
EXPORT void orc_pef_decode(const uint8_t* data, size_t n, const uint16_t* huff, int W, int H, uint16_t* out)
{
    orc_bits b = {data, n, 0, 0, 0};
    int vpred[2][2] = {{0, 0}, {0, 0}}, hpred[2] = {0, 0};
    for (int row = 0; row < H; row++)
        for (int col = 0; col < W; col++) {
            const int len = (int)orc_getbithuff(&b, huff[0], huff + 1);
            int diff = (int)orc_getbithuff(&b, len, NULL);
            if ((diff & (int)(1u << ((len - 1) & 31))) == 0) diff -= (int)((1u << (len & 31)) - 1);
            if (col < 2) hpred[col] = vpred[row & 1][col] += diff;
            else hpred[col & 1] += diff;
            out[(size_t)row * W + col] = (uint16_t)hpred[col & 1];
        }
}

/* PEFFile(aFileName) uncompressed branch (PEFFile.cs:116-156): per strip,
 * rows_per_strip rows of W values of `depth` bits, MSB first; the bit
 * buffer and its count carry over from one strip to the next. Rows past H
 * are not written (the reference would throw there). */
EXPORT void orc_pef_unpack(const uint8_t* file, size_t file_size, const uint32_t* offsets, const uint32_t* sizes, int nstrips, int rows_per_strip,
                           int W, int H, int depth, uint16_t* out)
{
    uint32_t bitbuf = 0;
    int bitoff = 0;
    for (int s = 0; s < nstrips; s++) {
        const uint8_t* d = file + offsets[s];
        const size_t nd = offsets[s] < file_size ? (size_t)sizes[s] : 0;
        size_t pos = 0;
        for (int line = 0; line < rows_per_strip; line++)
            for (int px = 0; px < W; px++) {
                const int row = s * rows_per_strip + line;
                while (bitoff < depth) {
                    uint32_t v = pos < nd ? d[pos] : 0;
                    bitbuf = (bitbuf << 8) + v;
                    bitoff += 8;
                    pos++;
                }
                uint32_t v = bitbuf << (32 - bitoff) >> (32 - depth);
                bitoff -= depth;
                if (row < H) out[(size_t)row * W + px] = (uint16_t)v;
            }
    }
}

/* Test-stream synthesis (not part of the reference, which only decodes):
 * the inverse of orc_pef_decode for a code book (code[c] left-aligned in 12
 * bits, len[c]) covering categories 0 .. ncodes-1. Returns the bytes
 * written, or -1 if `cap` is too small or a difference needs a category
 * the book lacks. The last byte is zero-padded. */
EXPORT long orc_pef_encode(const uint16_t* img, int W, int H, const uint16_t* code, const uint8_t* len, int ncodes, uint8_t* out, size_t cap)
{
    uint64_t acc = 0;
    int nacc = 0;
    size_t w = 0;
    int vpred[2][2] = {{0, 0}, {0, 0}}, hpred[2] = {0, 0};
#define PUT(v, nb)                                                   \
    do {                                                             \
        acc = (acc << (nb)) | ((uint64_t)(v) & ((1ull << (nb)) - 1)); \
        nacc += (nb);                                                \
        while (nacc >= 8) {                                          \
            if (w >= cap) return -1;                                 \
            out[w++] = (uint8_t)(acc >> (nacc - 8));                 \
            nacc -= 8;                                               \
        }                                                            \
    } while (0)
    for (int row = 0; row < H; row++)
        for (int col = 0; col < W; col++) {
            const int v = img[(size_t)row * W + col];
            const int pred = col < 2 ? vpred[row & 1][col] : hpred[col & 1];
            const int diff = v - pred;
            int ssss = 0;
            while ((abs(diff) >> ssss) != 0) ssss++;
            if (ssss >= ncodes || len[ssss] == 0) return -1;
            PUT(code[ssss] >> (12 - len[ssss]), len[ssss]);
            if (ssss > 0) PUT(diff >= 0 ? diff : diff - 1, ssss);
            if (col < 2) hpred[col] = vpred[row & 1][col] = v;
            else hpred[col & 1] = v;
        }
    if (nacc > 0) {
        if (w >= cap) return -1;
        out[w++] = (uint8_t)(acc << (8 - nacc));
    }
#undef PUT
    return (long)w;
}

/* ---- Raw decoding (DNG) ----
 * The lossless-JPEG reader of DNGFile (PefFile/DNGFile.cs:40-285, dcraw's
 * ljpeg_start / ljpeg_row / getbithuff / ljpeg_diff) and the tile / strip
 * assembly with black-level deltas and linearisation (:323-600). A stream
 * is a byte range; ReadByte past its end gives -1. */
typedef struct {
    const uint8_t* d;
    long n, pos;
    uint32_t bitbuf;
    int vbits;
} orc_mstream;

static int ms_byte(orc_mstream* s) { return s->pos >= 0 && s->pos < s->n ? s->d[s->pos++] : (s->pos++, -1); }

typedef struct {
    int algo, bits, high, wide, clrs, sraw, psv, restart;
    int vpred[6];
    uint16_t* huff[20];
    uint16_t* own[20];
} orc_jhead;

/* make_decoder_ref (DNGFile.cs:73-92): the 1 + 2^max lookup table. */
static uint16_t* orc_make_decoder(const uint8_t** source, const uint8_t* end)
{
    const uint8_t* count = (*source += 16) - 17;
    int max;
    for (max = 16; max > 0 && count[max] == 0; max--) ;
    uint16_t* huff = (uint16_t*)calloc((size_t)1 + ((size_t)1 << max), sizeof(uint16_t));
    huff[0] = (uint16_t)max;
    int h = 1;
    for (int len = 1; len <= max; len++)
        for (int i = 0; i < count[len]; i++, ++*source)
            for (int j = 0; j < 1 << (max - len); j++)
                if (h <= 1 << max) huff[h++] = (uint16_t)(len << 8 | (*source < end ? **source : 0));
    return huff;
}

static void orc_jhead_free(orc_jhead* jh)
{
    for (int c = 0; c < 20; c++) free(jh->own[c]);
}

/* ljpeg_start (DNGFile.cs:94-170). Returns 1 and leaves s at the entropy data, or 0. */
static int orc_ljpeg_start(orc_jhead* jh, orc_mstream* s)
{
    static uint8_t data[0x10000];
    memset(jh, 0, sizeof(*jh));
    jh->restart = 0x7fffffff;
    ms_byte(s);
    if (ms_byte(s) != 0xd8) return 0;
    int tag;
    do {
        for (int k = 0; k < 4; k++) {
            const int b = ms_byte(s);
            if (b < 0) return 0;
            data[k] = (uint8_t)b;
        }
        tag = data[0] << 8 | data[1];
        const int len = (data[2] << 8 | data[3]) - 2;
        if (tag <= 0xff00) return 0;
        int got = 0;
        for (; got < len; got++) {
            const int b = ms_byte(s);
            if (b < 0) { s->pos--; break; }
            data[got] = (uint8_t)b;
        }
        switch (tag) {
        case 0xffc3:
            jh->sraw = ((data[7] >> 4) * (data[7] & 15) - 1) & 3;
            jh->algo = tag & 0xff;
            jh->bits = data[0];
            jh->high = data[1] << 8 | data[2];
            jh->wide = data[3] << 8 | data[4];
            jh->clrs = data[5] + jh->sraw;
            break;
        case 0xffc1:
        case 0xffc0:
            jh->algo = tag & 0xff;
            jh->bits = data[0];
            jh->high = data[1] << 8 | data[2];
            jh->wide = data[3] << 8 | data[4];
            jh->clrs = data[5] + jh->sraw;
            break;
        case 0xffc4: {
            const uint8_t* dp = data;
            int c;
            while (dp < data + len && ((c = *dp++) & -20) == 0) {
                free(jh->own[c]);
                jh->own[c] = jh->huff[c] = orc_make_decoder(&dp, data + len);
            }
            break;
        }
        case 0xffda:
            jh->psv = data[1 + data[0] * 2];
            jh->bits -= data[3 + data[0] * 2] & 15;
            break;
        case 0xffdd:
            jh->restart = data[0] << 8 | data[1];
            break;
        }
    } while (tag != 0xffda);
    for (int c = 0; c < 19; c++)
        if (!jh->huff[c + 1]) jh->huff[c + 1] = jh->huff[c];
    return 1;
}

/* getbithuff of DNGFile (:234-268): the byte after a 0xFF is skipped; past the end 0xFF bytes. */
static uint32_t orc_dng_bits(orc_mstream* s, int nbits, const uint16_t* huff)
{
    if (nbits > 25) return 0;
    if (nbits < 0) { s->vbits = 0; s->bitbuf = 0; return 0; }
    if (nbits == 0 || s->vbits < 0) return 0;
    while (s->vbits < nbits) {
        const int c = ms_byte(s);
        if (c == 255) ms_byte(s);
        s->bitbuf = (s->bitbuf << 8) + (uint8_t)c;
        s->vbits += 8;
    }
    uint32_t c = s->bitbuf << (32 - s->vbits) >> (32 - nbits);
    if (huff) {
        s->vbits -= huff[c] >> 8;
        c = (uint8_t)huff[c];
    } else {
        s->vbits -= nbits;
    }
    return c;
}

static int orc_ljpeg_diff(orc_mstream* s, const uint16_t* huff, int large)
{
    const int len = (int)orc_dng_bits(s, huff[0], huff + 1);
    if (len == 16 && large) return -32768;
    int diff = (int)orc_dng_bits(s, len, NULL);
    if ((diff & (int)(1u << ((len - 1) & 31))) == 0) diff -= (int)((1u << (len & 31)) - 1);
    return diff;
}

/* ljpeg_row (DNGFile.cs:173-228) into rowbuf (2 rows of wide * clrs). Returns the row or NULL. */
static uint16_t* orc_ljpeg_row(orc_jhead* jh, orc_mstream* s, int jrow, uint16_t* rowbuf, int large)
{
    if ((long)jrow * jh->wide % jh->restart == 0) {
        for (int c = 0; c < 6; c++) jh->vpred[c] = 1 << (jh->bits - 1);
        if (jrow > 0) {
            s->pos -= 2;
            uint16_t mark = 0;
            int c;
            do mark = (uint16_t)((mark << 8) + (c = ms_byte(s)));
            while (s->pos < s->n - 1 && mark >> 4 != 0xffd);
        }
        orc_dng_bits(s, -1, NULL);
    }
    uint16_t* row[3];
    for (int c = 0; c < 3; c++) row[c] = rowbuf + (size_t)jh->wide * jh->clrs * ((jrow + c) & 1);
    int spred = 0;
    for (int col = 0; col < jh->wide; col++)
        for (int c = 0; c < jh->clrs; c++) {
            const int diff = orc_ljpeg_diff(s, jh->huff[c], large);
            int pred;
            if (jh->sraw > 0 && c <= jh->sraw && (col | c) > 0) pred = spred;
            else if (col > 0) pred = row[0][-jh->clrs];
            else pred = (jh->vpred[c] += diff) - diff;
            if (jrow > 0 && col > 0) switch (jh->psv) {
                case 1: break;
                case 2: pred = row[1][0]; break;
                case 3: pred = row[1][-jh->clrs]; break;
                case 4: pred = pred + row[1][0] - row[1][-jh->clrs]; break;
                case 5: pred = pred + ((row[1][0] - row[1][-jh->clrs]) >> 1); break;
                case 6: pred = row[1][0] + ((pred - row[1][-jh->clrs]) >> 1); break;
                case 7: pred = (pred + row[1][0]) >> 1; break;
                default: pred = 0; break;
                }
            if ((*row[0] = (uint16_t)(pred + diff)) >> jh->bits) return NULL;
            if (c <= jh->sraw) spred = *row[0];
            row[0]++; row[1]++;
        }
    return row[2];
}

static inline uint16_t orc_dng_value(unsigned v, int row, int col, const uint16_t* lin, int nlin, const uint16_t* bh, const uint16_t* bv)
{
    const int black = (bh ? bh[col] : 0) + (bv ? bv[row] : 0);
    const int x = lin ? (int)lin[v < (unsigned)nlin ? v : (unsigned)(nlin - 1)] : (int)v;
    return (uint16_t)(x - black > 0 ? x - black : 0);
}

/* DNGFile pixel data (:372-600). compression 7 = lossless JPEG, 1 = none.
 * tiled: tiles of tw x th in row-major tile order; else strips of rps rows.
 * Returns 0, or -1 where the reference would stop with an exception. */
EXPORT int orc_dng_decode(const uint8_t* file, size_t file_size, int tiled, int tw, int th, int rps, int nparts, const uint32_t* offsets,
                          const uint32_t* counts, int compression, int bit_depth, int large, const uint16_t* lin, int nlin,
                          const uint16_t* bh, const uint16_t* bv, int W, int H, uint16_t* out)
{
    memset(out, 0, (size_t)W * H * 2);
    int row = 0, col = 0;
    for (int t = 0; t < nparts; t++) {
        const long o = offsets[t];
        const long n = (o + (long)counts[t] <= (long)file_size) ? (long)counts[t] : (o < (long)file_size ? (long)file_size - o : 0);
        if (compression == 7) {
            orc_mstream s = {file + o, n, 0, 0, 0};
            orc_jhead jh;
            int ret = orc_ljpeg_start(&jh, &s);
            if (ret > 0 && jh.algo == 0xc3) {
                const int jwide = jh.wide * jh.clrs;
                uint16_t* rowbuf = (uint16_t*)calloc((size_t)jh.wide * jh.clrs * 2 + 8, sizeof(uint16_t));
                for (int jrow = 0; jrow < jh.high; jrow++) {
                    const uint16_t* rp = orc_ljpeg_row(&jh, &s, jrow, rowbuf + 4, large);
                    if (!rp) { free(rowbuf); orc_jhead_free(&jh); return -1; }
                    for (int jcol = 0; jcol < jwide; jcol++) {
                        const int r = tiled ? row + jrow : t * rps + jrow, c = tiled ? col + jcol : jcol;
                        if (c < W && r < H) out[(size_t)r * W + c] = orc_dng_value(rp[jcol], r, c, lin, nlin, bh, bv);
                    }
                }
                free(rowbuf);
            }
            orc_jhead_free(&jh);
            if (tiled) {
                col += tw;
                if (col >= W) { col = 0; row += th; }
            }
        } else if (compression == 1 && !tiled) {
            const uint8_t* d = file + o;
            if (bit_depth == 16) {
                for (long p = 0; p < n / 2; p++) {
                    const int r = t * rps + (int)(p / W), c = (int)(p % W);
                    if (r >= H) return -1;
                    out[(size_t)r * W + c] = orc_dng_value((unsigned)(d[2 * p] | d[2 * p + 1] << 8), r, c, lin, nlin, bh, bv);
                }
            } else if (bit_depth < 16) {
                uint32_t bitbuf = 0;
                int offset = 0;
                long pos = 0;
                for (int line = 0; line < rps; line++)
                    for (int px = 0; px < W; px++) {
                        const int r = t * rps + line;
                        while (offset < bit_depth) {
                            const uint32_t v = pos < n ? d[pos] : 0;
                            bitbuf = (bitbuf << 8) + v;
                            offset += 8;
                            pos++;
                        }
                        const uint32_t v = bitbuf << (32 - offset) >> (32 - bit_depth);
                        offset -= bit_depth;
                        if (r >= H) continue;
                        out[(size_t)r * W + px] = orc_dng_value(v, r, px, lin, nlin, bh, bv);
                    }
            }
        } else {
            return -1;
        }
    }
    return 0;
}

/* Test-tile synthesis (the reference only decodes): one lossless-JPEG tile
 * of `wide` x `high` samples with `clrs` components (interleaved), one DC
 * table of the given code lengths per category for all components,
 * predictor psv, optional restart interval (in MCUs, a multiple of wide),
 * with byte stuffing and RSTn markers. Returns bytes written or -1. */
EXPORT long orc_lj92_encode(const uint16_t* img, int wide, int high, int clrs, int bits, int psv, int restart, const uint8_t* lens, int ncat,
                            uint8_t* out, size_t cap)
{
    size_t w = 0;
#define OUTB(b) do { if (w >= cap) return -1; out[w++] = (uint8_t)(b); } while (0)
    /* canonical codes from the lengths */
    uint16_t code[17];
    {
        int c = 0;
        for (int len = 1; len <= 16; len++) {
            for (int k = 0; k < ncat; k++)
                if (lens[k] == len) code[k] = (uint16_t)c++;
            c <<= 1;
        }
    }
    OUTB(0xFF); OUTB(0xD8);
    /* SOF3 */
    OUTB(0xFF); OUTB(0xC3);
    const int lsof = 8 + 3 * clrs;
    OUTB(lsof >> 8); OUTB(lsof & 255); OUTB(bits); OUTB(high >> 8); OUTB(high & 255); OUTB(wide >> 8); OUTB(wide & 255); OUTB(clrs);
    for (int c = 0; c < clrs; c++) { OUTB(c + 1); OUTB(0x11); OUTB(0); }
    /* DHT: table 0 */
    int nv = 0;
    for (int k = 0; k < ncat; k++) nv += lens[k] > 0;
    OUTB(0xFF); OUTB(0xC4);
    const int ldht = 2 + 1 + 16 + nv;
    OUTB(ldht >> 8); OUTB(ldht & 255); OUTB(0x00);
    for (int len = 1; len <= 16; len++) {
        int cnt = 0;
        for (int k = 0; k < ncat; k++) cnt += lens[k] == len;
        OUTB(cnt);
    }
    for (int len = 1; len <= 16; len++)
        for (int k = 0; k < ncat; k++)
            if (lens[k] == len) OUTB(k);
    if (restart > 0) { OUTB(0xFF); OUTB(0xDD); OUTB(0); OUTB(4); OUTB(restart >> 8); OUTB(restart & 255); }
    /* SOS */
    OUTB(0xFF); OUTB(0xDA);
    const int lsos = 6 + 2 * clrs;
    OUTB(lsos >> 8); OUTB(lsos & 255); OUTB(clrs);
    for (int c = 0; c < clrs; c++) { OUTB(c + 1); OUTB(0x00); }
    OUTB(psv); OUTB(0); OUTB(0);
    uint64_t acc = 0;
    int nacc = 0, rst = 0;
#define PUTBITS(v, nb) do { acc = (acc << (nb)) | ((uint64_t)(v) & ((1ull << (nb)) - 1)); nacc += (nb); \
        while (nacc >= 8) { const uint8_t b_ = (uint8_t)(acc >> (nacc - 8)); nacc -= 8; OUTB(b_); if (b_ == 0xFF) OUTB(0x00); } } while (0)
#define FLUSH() do { if (nacc > 0) { const int pad_ = 8 - nacc; PUTBITS((1u << pad_) - 1, pad_); } } while (0)
    const int W = wide * clrs;
    for (int r = 0; r < high; r++) {
        if (restart > 0 && r > 0 && ((long)r * wide) % restart == 0) {
            FLUSH();
            OUTB(0xFF); OUTB(0xD0 + (rst & 7));
            rst++;
        }
        const int fresh = restart > 0 ? ((long)r * wide) % restart == 0 : r == 0;
        for (int col = 0; col < wide; col++)
            for (int c = 0; c < clrs; c++) {
                const int x = img[(size_t)r * W + col * clrs + c];
                int pred;
                const int left = col > 0 ? img[(size_t)r * W + (col - 1) * clrs + c] : 0;
                const int up = r > 0 ? img[(size_t)(r - 1) * W + col * clrs + c] : 0;
                const int ul = (r > 0 && col > 0) ? img[(size_t)(r - 1) * W + (col - 1) * clrs + c] : 0;
                if (col == 0) pred = fresh ? 1 << (bits - 1) : up;   /* vpred: reset at restarts */
                else pred = left;
                if (r > 0 && col > 0) switch (psv) {                     /* the previous row survives restarts */
                    case 1: break;
                    case 2: pred = up; break;
                    case 3: pred = ul; break;
                    case 4: pred = left + up - ul; break;
                    case 5: pred = left + ((up - ul) >> 1); break;
                    case 6: pred = up + ((left - ul) >> 1); break;
                    case 7: pred = (left + up) >> 1; break;
                    default: pred = 0; break;
                    }
                int diff = (x - pred) & 0xFFFF;
                if (diff >= 32768) diff -= 65536;
                int ssss = 0;
                while ((abs(diff) >> ssss) != 0) ssss++;
                if (ssss >= ncat || lens[ssss] == 0) return -1;
                PUTBITS(code[ssss], lens[ssss]);
                if (ssss > 0) PUTBITS(diff >= 0 ? diff : diff - 1, ssss);
            }
    }
    FLUSH();
    OUTB(0xFF); OUTB(0xD9);
#undef PUTBITS
#undef FLUSH
#undef OUTB
    return (long)w;
}
