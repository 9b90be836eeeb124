// Full-frame FFTs of the path, hand-written: the frequency-domain high-pass
// of the tracking images (PreAlignment.FourierFilter, PreAlignment.cs:268-281:
// R2C, fourierFilter kernel.cu:704-779, C2R, / (W * H)) and the
// cross-correlation of the pre-alignment's angle scan (PreAlignment.cs:
// 176-261: R2C, conjugateComplexMulKernel kernel.cu:395-411, C2R).
//
// A W x H real frame (W even) is transformed as the reference's cuFFT plans
// do, unnormalised, into the (W/2 + 1) x H half spectrum:
//   rows:    each row is read as N = W/2 complex values z[n] = x[2n] + i x[2n+1],
//            transformed, and unpacked to X[k] = E[k] + e^{-2 pi i k / W} O[k],
//            E = (Z[k] + conj Z[N-k]) / 2, O = (Z[k] - conj Z[N-k]) / 2i;
//   columns: each column of bins is transformed forward, multiplied (by the
//            filter coefficient, or by the conjugate of a reference
//            spectrum), and transformed back, in one kernel;
//   rows:    Z'[k] = (X[k] + conj X[N-k]) + i e^{2 pi i k / W} (X[k] - conj X[N-k])
//            is transformed back and re-interleaved (x[2n], x[2n+1]) = z'[n].
// One transform lives in shared memory; the stages are Stockham (natural
// order, ping-pong buffers) of radix 8, 4, 2, 5 and 3, and any other prime
// factor p is one stage that pairs outputs r and p - r (sums and differences
// of inputs a and p - a, then cosine and sine sums). Twiddles come from a
// table of e^{-2 pi i k / n} computed in double precision on the host; the
// inverse transform is the forward one between two conjugations.
#include "isa_internal.cuh"

#include <algorithm>
#include <cmath>
#include <vector>

namespace {

__device__ __forceinline__ float2 cmul(float2 a, float2 b) { return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmuli(float2 a) { return make_float2(-a.y, a.x); }    // i * a
__device__ __forceinline__ float2 cmulmi(float2 a) { return make_float2(a.y, -a.x); }  // -i * a
__device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
__device__ __forceinline__ float2 conjf2(float2 a) { return make_float2(a.x, -a.y); }

// Shared-memory index of element i of a transform buffer: one pad slot per 16
// elements, so the strided writes of the early Stockham stages (stride R)
// fall on different banks.
__device__ __forceinline__ int pad(int i) { return i + (i >> 4); }
__host__ __device__ constexpr int padded(int n) { return n + (n >> 4) + 1; }

// q = n / d by multiply-high with m = 2^32 / d + 1 (exact for n, d < 2^15; d = 1 handled by the caller's m = 0).
__device__ __forceinline__ int qdiv(int n, unsigned m) { return m ? (int)__umulhi((unsigned)n, m) : n; }

// Asynchronous 8-byte global -> shared copies (many in flight per thread), then a wait for all of them.
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem)
{
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory"); }

// Forward DFTs of size 2, 3, 4, 5, 8 in place (X[r] = sum_a v[a] e^{-2 pi i a r / R}).
__device__ __forceinline__ void dft(float2 (&v)[2])
{
    const float2 a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
}

__device__ __forceinline__ void dft(float2 (&v)[4])
{
    const float2 a0 = cadd(v[0], v[2]), a1 = csub(v[0], v[2]), a2 = cadd(v[1], v[3]), a3 = cmulmi(csub(v[1], v[3]));
    v[0] = cadd(a0, a2);
    v[2] = csub(a0, a2);
    v[1] = cadd(a1, a3);
    v[3] = csub(a1, a3);
}

__device__ __forceinline__ void dft(float2 (&v)[8])
{
    constexpr float h = 0.70710678118654752f;
    float2 u0[4], u1[4];
#pragma unroll
    for (int a = 0; a < 4; a++) {
        u0[a] = cadd(v[a], v[a + 4]);
        u1[a] = csub(v[a], v[a + 4]);
    }
    // u1[a] *= e^{-2 pi i a / 8}
    u1[1] = make_float2(h * (u1[1].x + u1[1].y), h * (u1[1].y - u1[1].x));
    u1[2] = cmulmi(u1[2]);
    u1[3] = make_float2(h * (u1[3].y - u1[3].x), -h * (u1[3].x + u1[3].y));
    dft(u0);
    dft(u1);
#pragma unroll
    for (int r = 0; r < 4; r++) {
        v[2 * r] = u0[r];
        v[2 * r + 1] = u1[r];
    }
}

__device__ __forceinline__ void dft(float2 (&v)[3])
{
    constexpr float s = 0.86602540378443865f;  // sin(2 pi / 3)
    const float2 t = cadd(v[1], v[2]), d = csub(v[1], v[2]);
    const float2 m = make_float2(v[0].x - 0.5f * t.x, v[0].y - 0.5f * t.y);
    const float2 q = cscale(cmulmi(d), s);
    v[0] = cadd(v[0], t);
    v[1] = cadd(m, q);
    v[2] = csub(m, q);
}

__device__ __forceinline__ void dft(float2 (&v)[5])
{
    constexpr float c1 = 0.30901699437494742f, c2 = -0.80901699437494742f;  // cos(2 pi / 5), cos(4 pi / 5)
    constexpr float s1 = 0.95105651629515357f, s2 = 0.58778525229247313f;   // sin(2 pi / 5), sin(4 pi / 5)
    const float2 A = cadd(v[1], v[4]), B = cadd(v[2], v[3]), Da = csub(v[1], v[4]), Db = csub(v[2], v[3]);
    const float2 m1 = make_float2(v[0].x + c1 * A.x + c2 * B.x, v[0].y + c1 * A.y + c2 * B.y);
    const float2 m2 = make_float2(v[0].x + c2 * A.x + c1 * B.x, v[0].y + c2 * A.y + c1 * B.y);
    const float2 q1 = cmulmi(make_float2(s1 * Da.x + s2 * Db.x, s1 * Da.y + s2 * Db.y));
    const float2 q2 = cmulmi(make_float2(s2 * Da.x - s1 * Db.x, s2 * Da.y - s1 * Db.y));
    v[0] = cadd(v[0], cadd(A, B));
    v[1] = cadd(m1, q1);
    v[4] = csub(m1, q1);
    v[2] = cadd(m2, q2);
    v[3] = csub(m2, q2);
}

// One Stockham stage of radix R over T transforms of length L (transform t at
// offset t * L): butterfly j reads in[j + a L / R], multiplies by
// e^{-2 pi i a (j mod Ns) / (Ns R)} and writes the R outputs to
// out[(j / Ns) Ns R + j mod Ns + r Ns].
template <int R>
__device__ __forceinline__ void stage_small(const float2* __restrict__ in, float2* __restrict__ out, int L, int LP, int T, int Ns, unsigned mns,
                                            const float2* __restrict__ tw)
{
    const int nb = L / R, unit = L / (Ns * R);
    for (int t = 0; t < T; t++) {
        const float2* src = in + (size_t)t * LP;
        float2* dst = out + (size_t)t * LP;
        for (int j = threadIdx.x; j < nb; j += blockDim.x) {
            const int jq = qdiv(j, mns), jj = j - jq * Ns;
            float2 v[R];
#pragma unroll
            for (int a = 0; a < R; a++) {
                const float2 x = src[pad(j + a * nb)];
                v[a] = (a > 0 && jj > 0) ? cmul(x, __ldg(tw + a * jj * unit)) : x;
            }
            dft(v);
            const int d0 = jq * Ns * R + jj;
#pragma unroll
            for (int r = 0; r < R; r++) dst[pad(d0 + r * Ns)] = v[r];
        }
    }
}

// A stage of odd prime radix p (any size). First the twiddled inputs of each
// butterfly are folded into v0, S_a = v_a + v_{p-a} and D_a = v_a - v_{p-a}
// (a = 1 .. (p-1)/2), stored in `out` at the butterfly's output places; then
// X_0 = v0 + sum S_a and, per r = 1 .. (p-1)/2, with theta = 2 pi a r / p,
// P = sum S_a cos(theta), Q = sum D_a sin(theta): X_r = v0 + P - iQ,
// X_{p-r} = v0 + P + iQ, written to `in` (the stage's result stays there).
// Each work item of the second part makes four pairs r from one pass over
// S and D; roots (p of them, e^{-2 pi i k / p}) come from `roots`.
__device__ void stage_prime(float2* __restrict__ in, float2* __restrict__ out, int L, int LP, int T, int Ns, unsigned mns, int p,
                            const float2* __restrict__ tw, const float2* __restrict__ roots)
{
    const int nb = L / p, unit = L / (Ns * p), h = (p - 1) / 2;
    // (butterfly, a) items: a = 0 copies v0, a >= 1 makes S_a and D_a
    for (int idx = threadIdx.x; idx < nb * T * (h + 1); idx += blockDim.x) {
        const int t = idx / (nb * (h + 1)), rem = idx - t * nb * (h + 1);
        const int j = rem / (h + 1), a = rem - j * (h + 1);
        const float2* src = in + (size_t)t * LP;
        float2* dst = out + (size_t)t * LP;
        const int jq = qdiv(j, mns), jj = j - jq * Ns;
        const int d0 = jq * Ns * p + jj;
        if (a == 0) {
            dst[pad(d0)] = src[pad(j)];
        } else {
            float2 xa = src[pad(j + a * nb)], xb = src[pad(j + (p - a) * nb)];
            if (jj > 0) {
                xa = cmul(xa, __ldg(tw + a * jj * unit));
                xb = cmul(xb, __ldg(tw + (p - a) * jj * unit));
            }
            dst[pad(d0 + a * Ns)] = cadd(xa, xb);        // S_a
            dst[pad(d0 + (p - a) * Ns)] = csub(xa, xb);  // D_a
        }
    }
    __syncthreads();
    const int ng = (h + 4) / 4;  // groups: g = 0 also makes X_0
    for (int idx = threadIdx.x; idx < nb * T * ng; idx += blockDim.x) {
        const int t = idx / (nb * ng), rem = idx - t * nb * ng;
        const int j = rem / ng, g = rem - j * ng;
        const float2* sd = out + (size_t)t * LP;
        float2* res = in + (size_t)t * LP;
        const int jq = qdiv(j, mns), jj = j - jq * Ns;
        const int d0 = jq * Ns * p + jj;
        const float2 v0 = sd[pad(d0)];
        const int r0 = 1 + 4 * g;
        float2 P[4], Q[4];
        int k[4];
#pragma unroll
        for (int u = 0; u < 4; u++) { P[u] = make_float2(0.f, 0.f); Q[u] = make_float2(0.f, 0.f); k[u] = 0; }
        float2 s0 = v0;
        for (int a = 1; a <= h; a++) {
            const float2 S = sd[pad(d0 + a * Ns)], D = sd[pad(d0 + (p - a) * Ns)];
            if (g == 0) s0 = cadd(s0, S);
#pragma unroll
            for (int u = 0; u < 4; u++) {
                k[u] += r0 + u;
                if (k[u] >= p) k[u] -= p;
                const float2 w = roots[k[u]];  // (cos theta, -sin theta)
                P[u].x = fmaf(S.x, w.x, P[u].x);
                P[u].y = fmaf(S.y, w.x, P[u].y);
                Q[u].x = fmaf(D.x, -w.y, Q[u].x);
                Q[u].y = fmaf(D.y, -w.y, Q[u].y);
            }
        }
        if (g == 0) res[pad(d0)] = s0;
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const int r = r0 + u;
            if (r <= h) {
                const float2 m = cadd(v0, P[u]), q = cmulmi(Q[u]);
                res[pad(d0 + r * Ns)] = cadd(m, q);
                res[pad(d0 + (p - r) * Ns)] = csub(m, q);
            }
        }
    }
}

// T forward transforms of length L in b0 (b1: scratch of the same size;
// roots: room for the largest prime radix's roots); returns the buffer
// holding the result.
__device__ float2* fft_smem(float2* b0, float2* b1, int L, int T, const isa_fft_plan& pl, const float2* __restrict__ tw, float2* roots)
{
    const int LP = padded(L);  // transform t at b + t * LP, element i at pad(i)
    int Ns = 1;
    for (int s = 0; s < pl.nst; s++) {
        const int R = pl.radix[s];
        const unsigned m = pl.mns[s];
        switch (R) {
        case 8: stage_small<8>(b0, b1, L, LP, T, Ns, m, tw); break;
        case 4: stage_small<4>(b0, b1, L, LP, T, Ns, m, tw); break;
        case 2: stage_small<2>(b0, b1, L, LP, T, Ns, m, tw); break;
        case 5: stage_small<5>(b0, b1, L, LP, T, Ns, m, tw); break;
        case 3: stage_small<3>(b0, b1, L, LP, T, Ns, m, tw); break;
        default:
            for (int k = threadIdx.x; k < R; k += blockDim.x) roots[k] = __ldg(tw + k * (L / R));
            __syncthreads();
            stage_prime(b0, b1, L, LP, T, Ns, m, R, tw, roots);
            break;
        }
        __syncthreads();
        if (R == 8 || R == 4 || R == 2 || R == 5 || R == 3) {
            float2* x = b0;
            b0 = b1;
            b1 = x;
        }
        Ns *= R;
    }
    return b0;
}

constexpr int kRowThreads = 256, kColThreads = 512;
#ifndef ISA_FFT_COL_SMEM_KB
#define ISA_FFT_COL_SMEM_KB 200  // shared memory of a column CTA (three 4000-row columns): wide rows of bins beat occupancy
#endif
constexpr size_t kColSmem = (size_t)ISA_FFT_COL_SMEM_KB * 1024;

// Roots needed by the plan's stages of prime radix above 5 (0 if none).
int max_prime(const isa_fft_plan& pl)
{
    int m = 0;
    for (int s = 0; s < pl.nst; s++) {
        const int r = pl.radix[s];
        if (r != 2 && r != 3 && r != 4 && r != 5 && r != 8 && r > m) m = r;
    }
    return m;
}

// Rows, real to half spectrum (one row per CTA).
__global__ void __launch_bounds__(kRowThreads) k_fft_rows_r2c(const float* __restrict__ in, size_t in_pitch, float2* __restrict__ spec, size_t spec_pitch,
                                                             int W, isa_fft_plan pl, const float2* __restrict__ tw_n, const float2* __restrict__ tw_w)
{
    extern __shared__ __align__(16) float2 fsm[];
    const int N = W / 2, y = blockIdx.x, NP = padded(N);
    float2* b0 = fsm;
    float2* b1 = fsm + NP;
    const float2* row = (const float2*)isa::row_ptr(in, in_pitch, y);
    for (int n = threadIdx.x; n < N; n += blockDim.x) cp_async8(b0 + pad(n), row + n);
    cp_async_wait_all();
    __syncthreads();
    const float2* Z = fft_smem(b0, b1, N, 1, pl, tw_n, fsm + 2 * NP);
    float2* out = isa::row_ptr(spec, spec_pitch, y);
    for (int k = threadIdx.x; k <= N; k += blockDim.x) {
        const float2 zk = Z[pad(k == N ? 0 : k)], zn = conjf2(Z[pad(k == 0 ? 0 : N - k)]);
        const float2 E = cscale(cadd(zk, zn), 0.5f);
        const float2 O = cscale(cmulmi(csub(zk, zn)), 0.5f);  // (zk - zn) / 2i
        out[k] = cadd(E, cmul(__ldg(tw_w + k), O));
    }
}

// Rows, half spectrum to real (one row per CTA); optionally clamped to [0, 1];
// bins k >= kfrom are first multiplied by kscale.
__global__ void __launch_bounds__(kRowThreads) k_fft_rows_c2r(const float2* __restrict__ spec, size_t spec_pitch, float* __restrict__ out, size_t out_pitch,
                                                             int W, isa_fft_plan pl, const float2* __restrict__ tw_n, const float2* __restrict__ tw_w,
                                                             int clamp01, int kfrom, float kscale)
{
    extern __shared__ __align__(16) float2 fsm[];
    const int N = W / 2, y = blockIdx.x, NP = padded(N);
    float2* X = fsm;           // N + 1 bins (unpadded), then the scratch buffer once X is consumed
    float2* b0 = fsm + NP;     // conj Z'
    float2* b1 = fsm;
    const float2* srow = isa::row_ptr(spec, spec_pitch, y);
    for (int k = threadIdx.x; k <= N; k += blockDim.x) cp_async8(X + k, srow + k);
    cp_async_wait_all();
    __syncthreads();
    // bins whose column transform was skipped (the column's filter is 1 throughout) take its factor here
    if (kfrom <= N) {
        for (int k = kfrom + threadIdx.x; k <= N; k += blockDim.x) X[k] = cscale(X[k], kscale);
        __syncthreads();
    }
    for (int k = threadIdx.x; k < N; k += blockDim.x) {
        const float2 xk = X[k], xn = conjf2(X[N - k]);
        const float2 w = conjf2(__ldg(tw_w + k));  // e^{+2 pi i k / W}
        const float2 zp = cadd(cadd(xk, xn), cmuli(cmul(w, csub(xk, xn))));
        b0[pad(k)] = conjf2(zp);
    }
    __syncthreads();
    const float2* z = fft_smem(b0, b1, N, 1, pl, tw_n, fsm + 2 * NP);
    float2* orow = (float2*)isa::row_ptr(out, out_pitch, y);
    for (int n = threadIdx.x; n < N; n += blockDim.x) {
        float2 v = conjf2(z[pad(n)]);
        if (clamp01) {
            v.x = fminf(fmaxf(v.x, 0.f), 1.f);
            v.y = fminf(fmaxf(v.y, 0.f), 1.f);
        }
        orow[n] = v;
    }
}

// Columns of the half spectrum, C per CTA: forward transform, then (mode
// FILTER) the fourierFilter coefficient times post_scale or (mode XCORR) the
// conjugate of ref, then the inverse transform; mode FWD stores the forward
// transform.
__global__ void __launch_bounds__(kColThreads) k_fft_cols(float2* __restrict__ spec, size_t spec_pitch, int W, int H, int ncols, int C, isa_fft_plan pl,
                                                         const float2* __restrict__ tw_h, int mode, isa_fft_filter f, const float2* __restrict__ ref,
                                                         size_t ref_pitch)
{
    extern __shared__ __align__(16) float2 fsm[];
    const int x0 = blockIdx.x * C;
    const int nc = min(C, ncols - x0);
    const int HP = padded(H);
    float2* b0 = fsm;
    float2* b1 = fsm + (size_t)C * HP;
    // column c at b0 + c * HP (padded); a row's nc bins are contiguous in memory
    for (int i = threadIdx.x; i < nc * H; i += blockDim.x) {
        const int y = i / nc, c = i - y * nc;
        cp_async8(b0 + (size_t)c * HP + pad(y), isa::row_ptr(spec, spec_pitch, y) + x0 + c);
    }
    cp_async_wait_all();
    __syncthreads();
    float2* roots = fsm + (size_t)2 * C * HP;
    float2* F = fft_smem(b0, b1, H, nc, pl, tw_h, roots);
    float2* G = F == b0 ? b1 : b0;
    if (mode != ISA_FFT_COLS_FWD) {
        for (int i = threadIdx.x; i < nc * H; i += blockDim.x) {
            const int c = i / H, y = i - c * H;
            float2& e = F[(size_t)c * HP + pad(y)];
            float2 v = e;
            if (mode == ISA_FFT_COLS_FILTER) {
                v = cscale(v, isa::fourier_mask(x0 + c, y, W, H, f.lp, f.hp, f.lps, f.hps, f.clear_axis) * f.post_scale);
            } else {
                v = cmul(conjf2(__ldg(isa::row_ptr(ref, ref_pitch, y) + x0 + c)), v);
            }
            e = conjf2(v);
        }
        __syncthreads();
        F = fft_smem(F, G, H, nc, pl, tw_h, roots);
        for (int i = threadIdx.x; i < nc * H; i += blockDim.x) {
            const int c = i / H, y = i - c * H;
            float2& e = F[(size_t)c * HP + pad(y)];
            e = conjf2(e);
        }
        __syncthreads();
    }
    for (int i = threadIdx.x; i < nc * H; i += blockDim.x) {
        const int y = i / nc, c = i - y * nc;
        isa::row_ptr(spec, spec_pitch, y)[x0 + c] = F[(size_t)c * HP + pad(y)];
    }
}

}  // namespace

int isa_fft_filter_columns(int W, const isa_fft_filter& f)
{
    const int Wc = W / 2 + 1;
    // fourierFilter with lp - lps <= 0 and no axis clearing is 1 wherever dist >= hp + hps (the low-pass part is 1 for
    // every dist <= 1, and dist <= sqrt(1/2)); dist >= mx = x / W, evaluated in float as the device does
    const float lp = f.lp - f.lps, hp = f.hp + f.hps;
    if (f.clear_axis > 0 || lp > 0.f) return Wc;
    if (f.lps > 0 && lp == 0 && hp == 0 && f.hps == 0) return Wc;
    if (!(hp > 0.f)) return 0;
    for (int x = 0; x < Wc; x++) {
        float mx = (float)x;
        mx /= W;
        if (mx >= hp) return x;
    }
    return Wc;
}

bool isa_fft_plan_make(int n, isa_fft_plan& p)
{
    p.n = n;
    p.nst = 0;
    if (n < 1) return false;
    int m = n;
    auto push = [&](int r) {
        if (p.nst >= ISA_FFT_MAX_STAGES) return false;
        p.radix[p.nst++] = r;
        m /= r;
        return true;
    };
    while (m % 8 == 0) if (!push(8)) return false;
    while (m % 4 == 0) if (!push(4)) return false;
    while (m % 2 == 0) if (!push(2)) return false;
    while (m % 5 == 0) if (!push(5)) return false;
    while (m % 3 == 0) if (!push(3)) return false;
    for (int q = 7; m > 1 && (long long)q * q <= m; q += 2)
        while (m % q == 0) if (!push(q)) return false;
    if (m > 1 && !push(m)) return false;
    int ns = 1;
    for (int st = 0; st < p.nst; st++) {
        p.ns[st] = ns;
        p.mns[st] = ns == 1 ? 0u : (unsigned)(0x100000000ull / (unsigned long long)ns + 1);
        ns *= p.radix[st];
    }
    return true;
}

void isa_fft_twiddles(int n, float2* out)
{
    const double a = -2.0 * M_PI / n;
    for (int k = 0; k < n; k++) out[k] = make_float2((float)std::cos(a * k), (float)std::sin(a * k));
}

int isa_fft_cols_per_cta(int H)
{
    // the roots of a prime factor of H take at most H / 7 entries
    const size_t roots = (size_t)(H / 7 + 1) * sizeof(float2);
    const size_t col = (size_t)2 * padded(H) * sizeof(float2);
    const size_t budget = std::max(kColSmem, col + roots);  // at least one column
    if (budget > 227 * 1024) return 0;
    const int c = (int)((budget - roots) / col);
    return c < 1 ? 0 : (c > 16 ? 16 : c);
}

cudaError_t isa_launch_fft_rows_r2c(const float* in, size_t in_pitch, float2* spec, size_t spec_pitch, int W, int H, const isa_fft_plan& pn,
                                    const float2* tw_n, const float2* tw_w, cudaStream_t st)
{
    const size_t smem = (size_t)(2 * padded(W / 2) + max_prime(pn)) * sizeof(float2);  // two padded buffers of W / 2, prime roots
    if (smem > 227 * 1024 || (W & 1) || pn.n != W / 2 || ((uintptr_t)in & 7) || (in_pitch & 7) || ((uintptr_t)spec & 7) || (spec_pitch & 7))
        return cudaErrorInvalidValue;
    cudaError_t e = cudaFuncSetAttribute(k_fft_rows_r2c, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    k_fft_rows_r2c<<<H, kRowThreads, smem, st>>>(in, in_pitch, spec, spec_pitch, W, pn, tw_n, tw_w);
    return cudaGetLastError();
}

cudaError_t isa_launch_fft_rows_c2r(const float2* spec, size_t spec_pitch, float* out, size_t out_pitch, int W, int H, const isa_fft_plan& pn,
                                    const float2* tw_n, const float2* tw_w, int clamp01, int kfrom, float kscale, cudaStream_t st)
{
    const size_t smem = (size_t)(2 * padded(W / 2) + max_prime(pn)) * sizeof(float2);  // N + 1 bins / scratch, conj Z', prime roots
    if (smem > 227 * 1024 || (W & 1) || pn.n != W / 2 || ((uintptr_t)out & 7) || (out_pitch & 7) || ((uintptr_t)spec & 7) || (spec_pitch & 7))
        return cudaErrorInvalidValue;
    cudaError_t e = cudaFuncSetAttribute(k_fft_rows_c2r, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    k_fft_rows_c2r<<<H, kRowThreads, smem, st>>>(spec, spec_pitch, out, out_pitch, W, pn, tw_n, tw_w, clamp01, kfrom, kscale);
    return cudaGetLastError();
}

cudaError_t isa_launch_fft_cols(float2* spec, size_t spec_pitch, int W, int H, int ncols, const isa_fft_plan& ph, const float2* tw_h, int mode,
                                const isa_fft_filter& f, const float2* ref, size_t ref_pitch, cudaStream_t st)
{
    const int C = isa_fft_cols_per_cta(H);
    if (C < 1 || ph.n != H || ((uintptr_t)spec & 7) || (spec_pitch & 7) || (mode == ISA_FFT_COLS_XCORR && (!ref || ((uintptr_t)ref & 7) || (ref_pitch & 7))))
        return cudaErrorInvalidValue;
    const size_t smem = ((size_t)2 * C * padded(H) + max_prime(ph)) * sizeof(float2);
    cudaError_t e = cudaFuncSetAttribute(k_fft_cols, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    if (ncols < 0 || ncols > W / 2 + 1) return cudaErrorInvalidValue;
    if (ncols == 0) return cudaSuccess;
    k_fft_cols<<<(ncols + C - 1) / C, kColThreads, smem, st>>>(spec, spec_pitch, W, H, ncols, C, ph, tw_h, mode, f, ref, ref_pitch);
    return cudaGetLastError();
}
