// Raw decoding of Pentax PEF frames on the GPU (PEFFile, PefFile/PEFFile.cs:81-156).
//
// Compressed frames are one bitstream of lossless-JPEG style symbols (a
// Huffman-coded difference category, then that many difference bits) in
// raster order, each difference relative to the pixel two columns left, or
// for the first two columns two rows up. The reference decodes it with one
// sequential bit reader. Here the stream is first copied into zero-padded
// big-endian 32-bit words (every symbol is then read with two aligned loads
// and a funnel shift), and cut into chunks of PEF_CHUNK bits. The first
// symbol boundary at or past a chunk's start lies within PEF_K bits of it
// (a symbol is at most 12 + 15 bits), so:
//   1. every chunk is decoded from each of its PEF_K candidate starts (a
//      warp per chunk, a lane per candidate, positions only) to the first
//      boundary at or past its end: per candidate the next chunk's
//      candidate and the symbol count, or "stopped" at an empty table
//      entry -- a map over PEF_K states. This stream format barely
//      resynchronises (most of each symbol is raw difference bits), so the
//      candidates are decoded, not guessed;
//   2. the maps are chained from chunk 0's state 0 in three levels (32
//      chunks per warp, 32 warps per block, blocks in order), then walked
//      back down: every chunk's true start, count and local offset;
//   3. a scan of the block totals gives each chunk's first pixel, and every
//      chunk decodes again from its true start, writing its differences;
//   4. column prefix sums (first two columns, per row parity) and row prefix
//      sums (per column parity) undo the prediction, in 32-bit wrap-around
//      arithmetic, stored as the low 16 bits.
// Reads past the end of the data see zero bytes, as the reference's bit
// reader does at the end of its file region; an empty table entry consumes
// nothing, after which every remaining pixel repeats the last value (the
// reference's reader then returns zero differences).
//
// Uncompressed frames (`isa_pef_unpack`): W values of `depth` bits per row,
// MSB first, strips of rows_per_strip rows whose bit buffer carries over from
// one strip to the next; one thread per value.
#include "isa_internal.cuh"

#include <algorithm>
#include <vector>

namespace {

constexpr int PEF_NT = 256;
constexpr unsigned long long PEF_CHUNK = 1024;  // bits per chunk
constexpr int PEF_MAX_STRIPS = 512;
constexpr int PEF_K = 27;          // candidate starts per chunk: a symbol is at most 12 + 15 bits
constexpr int PEF_CB = 1024;       // chunks per block of the map composition (32 warps x 32 chunks)
constexpr unsigned PEF_STOP = 255; // state after an empty table entry

struct PefTable {
    unsigned short t[4097];
};

// Zero-padded big-endian words of the stream: word i = bytes 4i .. 4i + 3.
__global__ void k_pef_words(const uint8_t* __restrict__ data, unsigned long long nbytes, unsigned long long nwords, unsigned* __restrict__ words)
{
    for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < nwords; i += (unsigned long long)gridDim.x * blockDim.x) {
        unsigned w = 0;
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const unsigned long long b = 4 * i + k;
            w = (w << 8) | (b < nbytes ? (unsigned)__ldg(data + b) : 0u);
        }
        words[i] = w;
    }
}

// The 32 bits starting at bit p, MSB first (zero past the padded copy).
__device__ __forceinline__ unsigned bits32(const unsigned* __restrict__ words, unsigned long long nwords, unsigned long long p)
{
    const unsigned long long w = p >> 5;
    const unsigned hi = w < nwords ? __ldg(words + w) : 0u, lo = w + 1 < nwords ? __ldg(words + w + 1) : 0u;
    return __funnelshift_l(lo, hi, (unsigned)(p & 31));
}

// One symbol at bit p: the table entry's code length and category (0 length: empty entry).
__device__ __forceinline__ int pef_decode_at(unsigned x, const unsigned short* tab, int& adv)
{
    const unsigned t = tab[1 + (x >> 20)];
    const int clen = (int)(t >> 8), ssss = (int)(t & 255);
    adv = clen == 0 ? 0 : clen + ssss;
    if (ssss == 0) return 0;
    int v = (int)((x << clen) >> (32 - ssss));
    if ((v & (1 << (ssss - 1))) == 0) v -= (1 << ssss) - 1;
    return v;
}

// The decode table and the advance table (code length + category, 0 for an
// empty entry) into device memory once, so that every CTA copies them from
// global memory (coalesced) rather than from kernel parameters read with a
// different address per thread.
__global__ void k_pef_tables(const __grid_constant__ PefTable T, unsigned short* __restrict__ tab, uint8_t* __restrict__ adv)
{
    for (int i = threadIdx.x; i < 4097; i += blockDim.x) {
        const unsigned t = T.t[i];
        tab[i] = (unsigned short)t;
        if (i > 0) adv[i - 1] = (t >> 8) == 0 ? 0 : (uint8_t)((t >> 8) + (t & 255));
    }
}

__device__ __forceinline__ void load_table(unsigned short* s, const unsigned short* __restrict__ g)
{
    for (int i = threadIdx.x; i < 4097; i += blockDim.x) s[i] = g[i];
    __syncthreads();
}

// Step 1: a warp per chunk (grid-stride): the chunk's 33 words staged in
// shared memory, lane k < PEF_K follows candidate start k (advance table only).
constexpr int PEF_CW = 34;  // words a chunk's decode reads: 32, the next one, and one spare

__global__ void __launch_bounds__(PEF_NT) k_pef_map(const unsigned* __restrict__ words, const uint8_t* __restrict__ gadv, int nchunks,
                                                    uint8_t* __restrict__ nextk, uint16_t* __restrict__ cntk)
{
    __shared__ __align__(16) uint8_t adv[4096];
    __shared__ unsigned cw[PEF_NT / 32][PEF_CW];
    for (int i = threadIdx.x; i < 1024; i += blockDim.x) ((unsigned*)adv)[i] = ((const unsigned*)gadv)[i];
    __syncthreads();
    const int warp = threadIdx.x >> 5, k = threadIdx.x & 31;
    for (int i = blockIdx.x * (PEF_NT / 32) + warp; i < nchunks; i += gridDim.x * (PEF_NT / 32)) {
        for (int t = k; t < PEF_CW; t += 32) cw[warp][t] = __ldg(words + (size_t)i * 32 + t);
        __syncwarp();
        if (k < PEF_K) {
            unsigned p = (unsigned)k, c = 0;
            bool stop = false;
            // two symbols per step while both must start inside the chunk (a symbol is at most 27 bits)
            while (p < PEF_CHUNK - 64) {
                const unsigned w1 = p >> 5;
                const unsigned a1 = adv[__funnelshift_l(cw[warp][w1 + 1], cw[warp][w1], p & 31) >> 20];
                if (a1 == 0) { stop = true; break; }
                p += a1;
                const unsigned w2 = p >> 5;
                const unsigned a2 = adv[__funnelshift_l(cw[warp][w2 + 1], cw[warp][w2], p & 31) >> 20];
                if (a2 == 0) { c += 1; stop = true; break; }
                p += a2;
                c += 2;
            }
            while (!stop && p < PEF_CHUNK) {
                const unsigned w = p >> 5;
                const unsigned a = adv[__funnelshift_l(cw[warp][w + 1], cw[warp][w], p & 31) >> 20];
                if (a == 0) { stop = true; break; }
                p += a;
                c++;
            }
            nextk[(size_t)i * 32 + k] = stop ? PEF_STOP : (uint8_t)(p - PEF_CHUNK);
            cntk[(size_t)i * 32 + k] = (uint16_t)c;
        }
        __syncwarp();
    }
}

// Step 2a: per block of PEF_CB = 32 x 32 chunks, the 32-chunk map of each
// warp (lane j follows state j) and the block's map.
__global__ void __launch_bounds__(1024) k_pef_compose(const uint8_t* __restrict__ nextk, int nchunks, uint8_t* __restrict__ sub_map,
                                                      uint8_t* __restrict__ block_map)
{
    __shared__ uint8_t m[PEF_CB][32];
    __shared__ uint8_t sm[32][32];
    const int c0 = blockIdx.x * PEF_CB, n = min(PEF_CB, nchunks - c0);
    for (int t = threadIdx.x; t < n * 32; t += blockDim.x) m[t >> 5][t & 31] = nextk[(size_t)c0 * 32 + t];
    __syncthreads();
    const int warp = threadIdx.x >> 5, j = threadIdx.x & 31;
    unsigned s = j < PEF_K ? (unsigned)j : PEF_STOP;
    for (int q = warp * 32; q < min(n, warp * 32 + 32) && s != PEF_STOP; q++) s = m[q][s];
    sm[warp][j] = (uint8_t)s;
    sub_map[((size_t)blockIdx.x * 32 + warp) * 32 + j] = (uint8_t)s;
    __syncthreads();
    if (warp == 0) {
        unsigned b = j < PEF_K ? (unsigned)j : PEF_STOP;
        for (int w = 0; w < 32 && b != PEF_STOP; w++) b = sm[w][b];
        block_map[(size_t)blockIdx.x * 32 + j] = (uint8_t)b;
    }
}

// Step 2b: one thread walks the block maps from state 0: every block's entry state and the state after the last chunk.
__global__ void k_pef_chain(const uint8_t* __restrict__ block_map, int nblocks, uint8_t* __restrict__ block_in, unsigned* __restrict__ final_state)
{
    extern __shared__ uint8_t bm[];
    for (int t = threadIdx.x; t < nblocks * 32; t += blockDim.x) bm[t] = block_map[t];
    __syncthreads();
    if (threadIdx.x != 0) return;
    unsigned s = 0;
    for (int b = 0; b < nblocks; b++) {
        block_in[b] = (uint8_t)s;
        if (s != PEF_STOP) s = bm[b * 32 + s];
    }
    *final_state = s;
}

// Step 2c: down the levels. Warp entry states from the block's entry state,
// then lane 0 of each warp walks its 32 chunks (true start, count); the
// counts are scanned within the block (local offsets and the block total).
// After a stop every later chunk has count 0, so totals need no stop flag.
__global__ void __launch_bounds__(1024) k_pef_walk(const uint8_t* __restrict__ nextk, const uint16_t* __restrict__ cntk, const uint8_t* __restrict__ sub_map,
                                                   const uint8_t* __restrict__ block_in, int nchunks, unsigned long long* __restrict__ start,
                                                   unsigned* __restrict__ loc, unsigned* __restrict__ block_total)
{
    __shared__ uint8_t wentry[32];
    __shared__ unsigned wtot[32];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int c0 = blockIdx.x * PEF_CB, n = min(PEF_CB, nchunks - c0);
    if (threadIdx.x == 0) {
        unsigned s = block_in[blockIdx.x];
        for (int w = 0; w < 32; w++) {
            wentry[w] = (uint8_t)s;
            if (s != PEF_STOP) s = sub_map[((size_t)blockIdx.x * 32 + w) * 32 + s];
        }
    }
    __syncthreads();
    if (lane == 0) {
        unsigned s = wentry[warp];
        for (int q = 0; q < 32; q++) {
            const int ci = warp * 32 + q;
            if (ci >= n) break;
            const int i = c0 + ci;
            if (s == PEF_STOP) {
                start[i] = (unsigned long long)i * PEF_CHUNK;
                loc[i] = 0;
                continue;
            }
            start[i] = (unsigned long long)i * PEF_CHUNK + s;
            loc[i] = cntk[(size_t)i * 32 + s];
            s = nextk[(size_t)i * 32 + s];
        }
    }
    __syncwarp();
    const int ci = warp * 32 + lane;
    const unsigned my = ci < n ? loc[c0 + ci] : 0u;
    unsigned x = my;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) wtot[warp] = x;
    __syncthreads();
    unsigned wpre = 0;
    for (int w = 0; w < warp; w++) wpre += wtot[w];
    if (ci < n) loc[c0 + ci] = wpre + x - my;
    if (threadIdx.x == 0) {
        unsigned tot = 0;
        for (int w = 0; w < 32; w++) tot += wtot[w];
        block_total[blockIdx.x] = tot;
    }
}

// Step 3a: exclusive scan of the block totals (one CTA); boff[nblocks] = all symbols.
__global__ void __launch_bounds__(1024) k_pef_scan(const unsigned* __restrict__ block_total, int nblocks, unsigned long long* __restrict__ boff)
{
    __shared__ unsigned long long wsum[32];
    __shared__ unsigned long long carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int base = 0; base < nblocks; base += 1024) {
        const int i = base + threadIdx.x;
        const unsigned long long v = i < nblocks ? block_total[i] : 0ull;
        unsigned long long x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned long long y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) wsum[warp] = x;
        __syncthreads();
        if (warp == 0) {
            unsigned long long w = wsum[lane];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const unsigned long long y = __shfl_up_sync(0xffffffffu, w, o);
                if (lane >= o) w += y;
            }
            wsum[lane] = w;
        }
        __syncthreads();
        if (i < nblocks) boff[i] = carry + (warp ? wsum[warp - 1] : 0ull) + x - v;
        __syncthreads();
        if (threadIdx.x == 0) carry += wsum[31];
        __syncthreads();
    }
    if (threadIdx.x == 0) boff[nblocks] = carry;
}

// Step 3b: the differences of every chunk at its pixel offset (one thread
// per chunk; the CTA's 256 consecutive chunks staged in shared memory with
// one skew word per 32, so that the lanes' chunks fall in different banks).
__global__ void __launch_bounds__(PEF_NT) k_pef_emit(const unsigned* __restrict__ words, unsigned long long nwords, const unsigned short* __restrict__ gtab,
                                                     int nchunks, int nblocks, const unsigned long long* __restrict__ start,
                                                     const unsigned* __restrict__ loc, const unsigned long long* __restrict__ boff,
                                                     unsigned long long npix, int16_t* __restrict__ diff)
{
    __shared__ unsigned short tab[4097];
    __shared__ unsigned cw[PEF_NT * 33 + 2];
    const int c0 = blockIdx.x * PEF_NT;
    for (int j = threadIdx.x; j < PEF_NT * 32 + 2; j += PEF_NT) {
        const unsigned long long g = (unsigned long long)c0 * 32 + j;
        cw[j + (j >> 5)] = g < nwords ? __ldg(words + g) : 0u;
    }
    load_table(tab, gtab);
    const int t = threadIdx.x, i = c0 + t;
    if (i >= nchunks) return;
    const unsigned long long total = boff[nblocks], limit = total < npix ? total : npix;
    unsigned long long o = boff[i / PEF_CB] + loc[i];
    if (o >= limit) return;
    unsigned p = (unsigned)(start[i] - (unsigned long long)i * PEF_CHUNK);
    const unsigned* cb = cw + 33 * t;
    while (p < PEF_CHUNK && o < limit) {
        const unsigned w = p >> 5;
        const unsigned x = __funnelshift_l(cb[w + 1 + ((w + 1) >> 5)], cb[w], p & 31);
        int a;
        const int d = pef_decode_at(x, tab, a);
        if (a == 0) break;
        p += a;
        diff[o++] = (int16_t)d;
    }
}

// After the last chunk: pixels the chunks did not reach (a stream that ends
// early reads zero bytes; after a stop the differences are zero). One thread.
__global__ void k_pef_tail(const unsigned* __restrict__ words, unsigned long long nwords, const unsigned short* __restrict__ gtab, int nchunks, int nblocks,
                           const unsigned* __restrict__ final_state, const unsigned long long* __restrict__ boff, unsigned long long npix,
                           int16_t* __restrict__ diff)
{
    unsigned long long o = boff[nblocks];
    if (o >= npix) return;
    const unsigned s = *final_state;
    if (s != PEF_STOP) {
        unsigned long long p = (unsigned long long)nchunks * PEF_CHUNK + s;
        while (o < npix) {
            int a;
            const int d = pef_decode_at(bits32(words, nwords, p), gtab, a);
            if (a == 0) break;
            p += a;
            diff[o++] = (int16_t)d;
        }
    }
    for (; o < npix; o++) diff[o] = 0;
}

// Prediction of the first two columns: running sums down the rows of one
// parity (vpred[row & 1][col]), one warp per (row parity, column).
__global__ void k_pef_cols(const int16_t* __restrict__ diff, int W, int H, int* __restrict__ colsum)
{
    const int lane = threadIdx.x & 31, seq = threadIdx.x >> 5;  // 4 warps: (parity, column)
    const int par = seq >> 1, col = seq & 1;
    if (col >= W) return;
    unsigned carry = 0;
    for (int base = par; base < H; base += 64) {
        const int row = base + 2 * lane;
        unsigned x = row < H ? (unsigned)diff[(size_t)row * W + col] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (row < H) colsum[(size_t)row * 2 + col] = (int)(carry + x);
        carry += __shfl_sync(0xffffffffu, x, 31);
    }
}

// Row prediction: value(row, col) = colsum(row, col & 1) + sum of the row's
// differences at columns 2 .. col of the same parity. One CTA per row.
__global__ void __launch_bounds__(PEF_NT) k_pef_rows(const int16_t* __restrict__ diff, const int* __restrict__ colsum, int W, int H,
                                                     uint16_t* __restrict__ out, size_t out_pitch)
{
    __shared__ unsigned ws[2][PEF_NT / 32];
    __shared__ unsigned carry[2];
    const int row = blockIdx.x;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int16_t* drow = diff + (size_t)row * W;
    uint16_t* orow = isa::row_ptr(out, out_pitch, row);
    if (threadIdx.x < 2) carry[threadIdx.x] = threadIdx.x < W ? (unsigned)colsum[(size_t)row * 2 + threadIdx.x] : 0u;
    __syncthreads();
    // columns in pairs: thread t of a pass owns columns 2 (base + t) and 2 (base + t) + 1
    for (int base = 1; 2 * base < W; base += PEF_NT) {
        const int c0 = 2 * (base + threadIdx.x);
        unsigned e = c0 < W ? (unsigned)drow[c0] : 0u, od = c0 + 1 < W ? (unsigned)drow[c0 + 1] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned ye = __shfl_up_sync(0xffffffffu, e, o), yo = __shfl_up_sync(0xffffffffu, od, o);
            if (lane >= o) { e += ye; od += yo; }
        }
        if (lane == 31) { ws[0][warp] = e; ws[1][warp] = od; }
        __syncthreads();
        unsigned pe = carry[0], po = carry[1];
        for (int w = 0; w < warp; w++) { pe += ws[0][w]; po += ws[1][w]; }
        if (c0 < W) orow[c0] = (uint16_t)(pe + e);
        if (c0 + 1 < W) orow[c0 + 1] = (uint16_t)(po + od);
        __syncthreads();
        if (threadIdx.x == 0) {
            unsigned te = 0, to = 0;
            for (int w = 0; w < PEF_NT / 32; w++) { te += ws[0][w]; to += ws[1][w]; }
            carry[0] += te;
            carry[1] += to;
        }
        __syncthreads();
    }
    if (threadIdx.x < 2 && threadIdx.x < W) orow[threadIdx.x] = (uint16_t)colsum[(size_t)row * 2 + threadIdx.x];
}

// Uncompressed strips: value v of strip s (v = line * W + px) is bits
// [v * depth, + depth) of the strip's virtual stream: the carry_bits bits
// the previous strip left in the reader's buffer, then the strip's bytes.
struct UnpackStrip {
    unsigned long long off, size;   // the strip's bytes in the file
    unsigned long long carry_src;   // file byte whose low carry_bits bits precede the strip's bytes (~0: zero bits)
    unsigned carry_bits;
};

struct UnpackArgs {
    int nstrips;
    UnpackStrip s[PEF_MAX_STRIPS];
};

__device__ __forceinline__ unsigned file_byte(const uint8_t* __restrict__ file, unsigned long long fsize, unsigned long long i)
{
    return i < fsize ? (unsigned)__ldg(file + i) : 0u;
}

__device__ __forceinline__ unsigned strip_bits(const uint8_t* __restrict__ file, unsigned long long fsize, const UnpackStrip& s,
                                               unsigned long long b, int depth)
{
    unsigned long long v = 0;
    int got = 0;
    while (got < depth) {
        const unsigned long long p = b + got;
        if (p < s.carry_bits) {
            const unsigned cv = s.carry_src == ~0ull ? 0u : file_byte(file, fsize, s.carry_src);
            const int take = (int)min((unsigned long long)(depth - got), s.carry_bits - p);
            const int lo = (int)(s.carry_bits - p) - take;  // bit index (from 0 = LSB) of the last bit taken
            v = (v << take) | ((cv >> lo) & ((1u << take) - 1));
            got += take;
            continue;
        }
        const unsigned long long q = p - s.carry_bits, byte = q >> 3;
        const int sh = (int)(q & 7), take = min(8 - sh, depth - got);
        const unsigned x = byte < s.size ? file_byte(file, fsize, s.off + byte) : 0u;
        v = (v << take) | ((x >> (8 - sh - take)) & ((1u << take) - 1));
        got += take;
    }
    return (unsigned)v;
}

__global__ void k_pef_unpack(const uint8_t* __restrict__ file, unsigned long long fsize, const __grid_constant__ UnpackArgs A, int rows_per_strip,
                             int W, int H, int depth, uint16_t* __restrict__ out, size_t out_pitch)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= W || y >= H) return;
    const int s = y / rows_per_strip, line = y - s * rows_per_strip;
    const unsigned long long b = ((unsigned long long)line * W + x) * depth;
    isa::row_ptr(out, out_pitch, y)[x] = (uint16_t)strip_bits(file, fsize, A.s[s], b, depth);
}

}  // namespace

size_t isa_pef_scratch_layout(unsigned long long nbytes, int W, int H, size_t* parts)
{
    const unsigned long long nchunks = (nbytes * 8 + PEF_CHUNK - 1) / PEF_CHUNK + 1;
    const unsigned long long nblocks = (nchunks + PEF_CB - 1) / PEF_CB;
    const unsigned long long nwords = nchunks * 32 + 64;  // every chunk's staged words lie inside
    size_t o = 0;
    const auto take = [&](int k, size_t bytes) { parts[k] = o; o += (bytes + 255) / 256 * 256; };
    take(0, nwords * 4);           // big-endian words of the stream
    take(1, nchunks * 8);          // true start of each chunk
    take(2, nchunks * 32);         // next state per (chunk, candidate)
    take(3, nchunks * 64);         // count per (chunk, candidate)
    take(4, nchunks * 4);          // local offsets
    take(5, nblocks * 32 * 32);    // warp (32-chunk) maps
    take(6, nblocks * 32);         // block maps
    take(7, nblocks + 32);         // block entry states, then the final state at the next 16-byte boundary
    take(8, nblocks * 4);          // block totals
    take(9, (nblocks + 1) * 8);    // block offsets, total
    take(10, (size_t)W * H * 2);   // differences (|d| < 2^15)
    take(11, (size_t)H * 2 * 4);   // column sums
    take(12, 4097 * 2);            // decode table
    take(13, 4096);                // advance table
    return o;
}

int isa_pef_max_blocks() { return (227 * 1024) / 32; }

cudaError_t isa_launch_pef_decode(const uint8_t* data, unsigned long long nbytes, const unsigned short* table, int W, int H, void* scratch,
                                  uint16_t* out, size_t out_pitch, cudaStream_t st)
{
    size_t part[14];
    isa_pef_scratch_layout(nbytes, W, H, part);
    char* base = (char*)scratch;
    const int nchunks = (int)((nbytes * 8 + PEF_CHUNK - 1) / PEF_CHUNK) + 1;  // one spare chunk past the data
    const int nblocks = (nchunks + PEF_CB - 1) / PEF_CB;
    const unsigned long long nwords = (unsigned long long)nchunks * 32 + 64;
    if (nblocks > isa_pef_max_blocks()) return cudaErrorInvalidValue;
    unsigned* words = (unsigned*)(base + part[0]);
    unsigned long long* start = (unsigned long long*)(base + part[1]);
    uint8_t* nextk = (uint8_t*)(base + part[2]);
    uint16_t* cntk = (uint16_t*)(base + part[3]);
    unsigned* loc = (unsigned*)(base + part[4]);
    uint8_t* sub_map = (uint8_t*)(base + part[5]);
    uint8_t* block_map = (uint8_t*)(base + part[6]);
    uint8_t* block_in = (uint8_t*)(base + part[7]);
    unsigned* final_state = (unsigned*)(base + part[7] + (nblocks + 15) / 16 * 16);
    unsigned* block_total = (unsigned*)(base + part[8]);
    unsigned long long* boff = (unsigned long long*)(base + part[9]);
    int16_t* diff = (int16_t*)(base + part[10]);
    int* colsum = (int*)(base + part[11]);
    unsigned short* gtab = (unsigned short*)(base + part[12]);
    uint8_t* gadv = (uint8_t*)(base + part[13]);
    PefTable T;
    for (int i = 0; i < 4097; i++) T.t[i] = table[i];
    k_pef_tables<<<1, 1024, 0, st>>>(T, gtab, gadv);
    k_pef_words<<<(unsigned)std::min<unsigned long long>((nwords + 255) / 256, 148 * 16), 256, 0, st>>>(data, nbytes, nwords, words);
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const unsigned mapg = (unsigned)std::min<long long>((nchunks + PEF_NT / 32 - 1) / (PEF_NT / 32), (long long)sms * 8);
    k_pef_map<<<mapg, PEF_NT, 0, st>>>(words, gadv, nchunks, nextk, cntk);
    k_pef_compose<<<nblocks, 1024, 0, st>>>(nextk, nchunks, sub_map, block_map);
    const size_t chain_smem = (size_t)nblocks * 32;
    cudaError_t e = cudaFuncSetAttribute(k_pef_chain, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)std::max<size_t>(chain_smem, 1));
    if (e != cudaSuccess) return e;
    k_pef_chain<<<1, 256, chain_smem, st>>>(block_map, nblocks, block_in, final_state);
    k_pef_walk<<<nblocks, 1024, 0, st>>>(nextk, cntk, sub_map, block_in, nchunks, start, loc, block_total);
    k_pef_scan<<<1, 1024, 0, st>>>(block_total, nblocks, boff);
    const unsigned long long npix = (unsigned long long)W * H;
    k_pef_emit<<<(unsigned)((nchunks + PEF_NT - 1) / PEF_NT), PEF_NT, 0, st>>>(words, nwords, gtab, nchunks, nblocks, start, loc, boff, npix, diff);
    k_pef_tail<<<1, 1, 0, st>>>(words, nwords, gtab, nchunks, nblocks, final_state, boff, npix, diff);
    k_pef_cols<<<1, 128, 0, st>>>(diff, W, H, colsum);
    k_pef_rows<<<H, PEF_NT, 0, st>>>(diff, colsum, W, H, out, out_pitch);
    return cudaGetLastError();
}

// Strip descriptors from the file layout: strip s starts at offsets[s] with
// the bits the previous strips left in the reader's buffer (PEFFile.cs:124-155).
cudaError_t isa_launch_pef_unpack(const uint8_t* file, unsigned long long fsize, const uint32_t* offsets, const uint32_t* sizes, int nstrips,
                                  int rows_per_strip, int W, int H, int depth, uint16_t* out, size_t out_pitch, cudaStream_t st)
{
    if (nstrips < 1 || nstrips > PEF_MAX_STRIPS) return cudaErrorInvalidValue;
    UnpackArgs A;
    A.nstrips = nstrips;
    unsigned long long carry_src = ~0ull;
    unsigned carry_bits = 0;
    const unsigned long long need = (unsigned long long)rows_per_strip * W * depth;
    for (int s = 0; s < nstrips; s++) {
        A.s[s] = UnpackStrip{offsets[s], sizes[s], carry_src, carry_bits};
        // bytes this strip consumes; the bits left over are the low bits of the last one
        const unsigned long long bytes = need > carry_bits ? (need - carry_bits + 7) / 8 : 0;
        const unsigned long long left = carry_bits + bytes * 8 - need;
        if (bytes > 0) carry_src = bytes <= sizes[s] ? (unsigned long long)offsets[s] + bytes - 1 : ~0ull;
        carry_bits = (unsigned)left;
    }
    dim3 b(256), g((W + 255) / 256, H);
    k_pef_unpack<<<g, b, 0, st>>>(file, fsize, A, rows_per_strip, W, H, depth, out, out_pitch);
    return cudaGetLastError();
}

// ---- DNG pixel data (DNGFile, PefFile/DNGFile.cs:372-600) ----
//
// Lossless-JPEG tiles or strips: one thread per tile / strip decodes its
// stream sequentially with the reference's reader (dcraw's ljpeg_row,
// getbithuff and ljpeg_diff: the byte after a 0xFF is skipped, restart
// markers are searched from two bytes back, predictors 1..7, the first
// column from vpred), headers parsed and Huffman tables built on the host.
// Values then pass the linearisation table and the black-level deltas:
// out = max(0, lin[min(v, n - 1)] - black_h[col] - black_v[row]).
// Uncompressed strips: one thread per value.

namespace {

struct Lj92Part {
    unsigned long long pos, end;   // entropy data start and end of the part's bytes in the file
    int skip;                      // ljpeg_start failed or not a lossless frame: nothing written
    int bits, high, wide, clrs, sraw, psv, restart;
    int out_row, out_col;          // where the part's first sample goes
    int table[6];                  // table offsets (in uint16) per component
    unsigned long long rowbuf;     // offset (in uint16) of the part's two-row buffer
};

struct DngArgs {
    const uint8_t* file;
    unsigned long long fsize;
    const Lj92Part* parts;
    int nparts;
    const uint16_t* tables;
    uint16_t* rows;
    const uint16_t* lin;
    int nlin;
    const uint16_t* bh;
    const uint16_t* bv;
    int W, H, large;
    uint16_t* out;
    size_t out_pitch;
    int* error;
};

__device__ __forceinline__ uint16_t dng_value(const DngArgs& A, unsigned v, int row, int col)
{
    const int black = (A.bh ? (int)A.bh[col] : 0) + (A.bv ? (int)A.bv[row] : 0);
    const int x = A.lin ? (int)A.lin[v < (unsigned)A.nlin ? v : (unsigned)(A.nlin - 1)] : (int)v;
    return (uint16_t)(x - black > 0 ? x - black : 0);
}

// The reader of one tile, run by lane 0 of the tile's warp. The warp keeps
// a DNG_WIN-byte window of the tile's bytes in shared memory (loaded with
// coalesced reads by all lanes) and slides it whenever fewer than
// DNG_MARGIN bytes remain ahead of the reader: one column of samples reads
// at most 6 components x 2 calls x 8 bytes.
constexpr int DNG_WIN = 4096, DNG_MARGIN = 256, DNG_WARPS = 4;

struct DngReader {
    const uint8_t* win;    // shared window: bytes [base, base + DNG_WIN) of the tile
    long long base, n, pos;
    unsigned bitbuf;
    int vbits;
    __device__ __forceinline__ int byte()
    {
        long long i = pos - base;
        i = i < 0 ? 0 : (i >= DNG_WIN ? DNG_WIN - 1 : i);  // the margin keeps i in range; the clamp only guards the memory
        const int v = (pos >= 0 && pos < n) ? (int)win[i] : -1;
        pos++;
        return v;
    }
    __device__ __forceinline__ unsigned bits(int nbits, const uint16_t* huff)
    {
        if (nbits > 25) return 0;
        if (nbits == 0 || vbits < 0) return 0;
        while (vbits < nbits) {
            const int c = byte();
            if (c == 255) byte();
            bitbuf = (bitbuf << 8) + (uint8_t)c;
            vbits += 8;
        }
        unsigned c = bitbuf << (32 - vbits) >> (32 - nbits);
        if (huff) {
            vbits -= huff[c] >> 8;
            c = (uint8_t)huff[c];
        } else {
            vbits -= nbits;
        }
        return c;
    }
    __device__ __forceinline__ int diff(const uint16_t* huff, int large)
    {
        const int len = (int)bits(huff[0], huff + 1);
        if (len == 16 && large) return -32768;
        int d = (int)bits(len, nullptr);
        if ((d & (int)(1u << ((len - 1) & 31))) == 0) d -= (int)((1u << (len & 31)) - 1);
        return d;
    }
};

// Warp per tile: lane 0 decodes sample by sample (the reference's order and
// arithmetic), the warp keeps the byte window filled and converts and stores
// each finished row. Row buffers live in shared memory.
__global__ void __launch_bounds__(32 * DNG_WARPS) k_dng_lj92(const DngArgs A, int jwide_max, int ntab)
{
    extern __shared__ __align__(16) unsigned char dsm[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // all Huffman tables of the frame when they fit (ntab > 0 entries), then per warp the window and the rows
    uint16_t* stab = (uint16_t*)dsm;
    for (int i = threadIdx.x; i < ntab; i += blockDim.x) stab[i] = A.tables[i];
    __syncthreads();
    const uint16_t* tabs = ntab > 0 ? stab : A.tables;
    uint8_t* win = dsm + (size_t)(ntab * 2 + 15) / 16 * 16 + (size_t)warp * (DNG_WIN + 4 * (size_t)jwide_max + 64);
    uint16_t* rowbuf = (uint16_t*)(win + DNG_WIN);
    int* svpred = (int*)(win + DNG_WIN + 4 * (size_t)jwide_max);        // 6 predictors
    int* stable = svpred + 8;                                             // 6 table offsets
    const int t = blockIdx.x * DNG_WARPS + warp;
    if (t >= A.nparts) return;  // whole warp
    const Lj92Part* PP = A.parts + t;
    if (PP->skip) return;
    if (lane < 6) stable[lane] = PP->table[lane];
    struct {
        unsigned long long pos, end;
        int bits, high, wide, clrs, sraw, psv, restart, out_row, out_col;
    } P{PP->pos, PP->end, PP->bits, PP->high, PP->wide, PP->clrs, PP->sraw, PP->psv, PP->restart, PP->out_row, PP->out_col};
    __syncwarp();
    const uint8_t* src = A.file + P.pos;
    const long long n = (long long)(P.end - P.pos);
    long long base = 0;
    const auto load = [&](long long b) {
        __syncwarp();
        base = b;
        for (int i = lane; i < DNG_WIN; i += 32) {
            const long long q = b + i;
            win[i] = (q >= 0 && q < n) ? __ldg(src + q) : (uint8_t)0;
        }
        __syncwarp();
    };
    load(0);
    DngReader r{win, 0, n, 0, 0u, 0};
    const int jwide = P.wide * P.clrs;
    bool failed = false;
    for (int jrow = 0; jrow < P.high; jrow++) {
        const bool restart = (long long)jrow * P.wide % P.restart == 0;
        if (restart && jrow > 0) {
            // seek back 2 bytes, then read until a 0xFFDx marker (or the last byte)
            long long p = __shfl_sync(0xffffffffu, r.pos, 0) - 2;
            if (p < base || p + DNG_MARGIN > base + DNG_WIN) load(p - 8);
            if (lane == 0) { r.base = base; r.pos = p; }
            unsigned short mark = 0;
            while (true) {
                bool done = false;
                if (lane == 0) {
                    while (r.pos < base + DNG_WIN - 8) {
                        const int c = r.byte();
                        mark = (unsigned short)((mark << 8) + c);
                        if (!(r.pos < r.n - 1 && mark >> 4 != 0xffd)) { done = true; break; }
                    }
                }
                if (__shfl_sync(0xffffffffu, done, 0)) break;
                load(__shfl_sync(0xffffffffu, r.pos, 0) - 8);
                if (lane == 0) r.base = base;
            }
        }
        if (lane == 0 && restart) {
            for (int c = 0; c < 6; c++) svpred[c] = 1 << (P.bits - 1);
            r.bitbuf = 0;
            r.vbits = 0;
        }
        uint16_t* row0 = rowbuf + (size_t)jwide * (jrow & 1);
        const uint16_t* row1 = rowbuf + (size_t)jwide * ((jrow + 1) & 1);
        int spred = 0;
        for (int col = 0; col < P.wide; col++) {
            const long long p = __shfl_sync(0xffffffffu, r.pos, 0);
            if (p + DNG_MARGIN > base + DNG_WIN) {
                load(p - 8);
                if (lane == 0) r.base = base;
            }
            if (lane == 0) {
                for (int c = 0; c < P.clrs; c++) {
                    const int d = r.diff(tabs + stable[c], A.large);
                    int pred;
                    if (P.sraw > 0 && c <= P.sraw && (col | c) > 0) pred = spred;
                    else if (col > 0) pred = row0[col * P.clrs + c - P.clrs];
                    else pred = (svpred[c] += d) - d;
                    if (jrow > 0 && col > 0) {
                        const int up = row1[col * P.clrs + c], ul = row1[col * P.clrs + c - P.clrs];
                        switch (P.psv) {
                        case 1: break;
                        case 2: pred = up; break;
                        case 3: pred = ul; break;
                        case 4: pred = pred + up - ul; break;
                        case 5: pred = pred + ((up - ul) >> 1); break;
                        case 6: pred = up + ((pred - ul) >> 1); break;
                        case 7: pred = (pred + up) >> 1; break;
                        default: pred = 0; break;
                        }
                    }
                    const uint16_t v = (uint16_t)(pred + d);
                    row0[col * P.clrs + c] = v;
                    if (v >> P.bits) { failed = true; break; }
                    if (c <= P.sraw) spred = v;
                }
            }
            if (__shfl_sync(0xffffffffu, failed, 0)) break;
        }
        failed = __shfl_sync(0xffffffffu, failed, 0);
        if (failed) break;
        __syncwarp();
        // the finished row, converted and stored by the whole warp
        const int orow = P.out_row + jrow;
        if (orow < A.H) {
            uint16_t* o = isa::row_ptr(A.out, A.out_pitch, orow);
            for (int jcol = lane; jcol < jwide; jcol += 32) {
                const int ocol = P.out_col + jcol;
                if (ocol < A.W) o[ocol] = dng_value(A, row0[jcol], orow, ocol);
            }
        }
        __syncwarp();
    }
    if (failed && lane == 0) atomicMin(A.error, t);
}

// Uncompressed strips: 16-bit little-endian samples filling rows strip by
// strip, or MSB-first samples of `depth` bits with the bit count reset at
// each strip.
__global__ void k_dng_plain(const DngArgs A, const unsigned long long* __restrict__ offs, const unsigned long long* __restrict__ cnts, int rps,
                            int depth)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= A.W || y >= A.H) return;
    const int s = y / rps, line = y - s * rps;
    if (s >= A.nparts) return;
    const unsigned long long v = (unsigned long long)line * A.W + x;
    unsigned val;
    if (depth == 16) {
        if (2 * v + 1 >= cnts[s]) return;  // the strip holds data.Length / 2 samples
        const unsigned long long b = offs[s] + 2 * v;
        const unsigned lo = b < A.fsize ? __ldg(A.file + b) : 0u, hi = b + 1 < A.fsize ? __ldg(A.file + b + 1) : 0u;
        val = lo | hi << 8;
    } else {
        const unsigned long long bit = v * depth;
        unsigned long long acc = 0;
        for (unsigned long long q = bit >> 3; q <= (bit + depth - 1) >> 3; q++) {
            const unsigned long long b = offs[s] + q;
            acc = (acc << 8) | ((q < cnts[s] && b < A.fsize) ? __ldg(A.file + b) : 0u);
        }
        const unsigned long long nb = (((bit + depth - 1) >> 3) - (bit >> 3) + 1) * 8;
        val = (unsigned)((acc >> (nb - (bit & 7) - depth)) & ((1ull << depth) - 1));
    }
    isa::row_ptr(A.out, A.out_pitch, y)[x] = dng_value(A, val, y, x);
}

}  // namespace

size_t isa_dng_part_bytes() { return sizeof(Lj92Part); }

void isa_dng_part_set(void* dst, int i, unsigned long long pos, unsigned long long end, int skip, const int* hdr, int out_row, int out_col,
                      const int* table, unsigned long long rowbuf)
{
    Lj92Part P{};
    P.pos = pos; P.end = end; P.skip = skip;
    P.bits = hdr[0]; P.high = hdr[1]; P.wide = hdr[2]; P.clrs = hdr[3]; P.sraw = hdr[4]; P.psv = hdr[5]; P.restart = hdr[6];
    P.out_row = out_row; P.out_col = out_col;
    for (int c = 0; c < 6; c++) P.table[c] = table[c];
    P.rowbuf = rowbuf;
    ((Lj92Part*)dst)[i] = P;
}

cudaError_t isa_launch_dng(const uint8_t* file, unsigned long long fsize, int compression, const void* parts, int nparts, const uint16_t* tables,
                           uint16_t* rows, const unsigned long long* offs, const unsigned long long* cnts, int rps, int depth, const uint16_t* lin,
                           int nlin, const uint16_t* bh, const uint16_t* bv, int W, int H, int large, uint16_t* out, size_t out_pitch, int* error,
                           cudaStream_t st, int jwide_max, int ntables)
{
    DngArgs A{file, fsize, (const Lj92Part*)parts, nparts, tables, rows, lin, nlin, bh, bv, W, H, large, out, out_pitch, error};
    if (compression == 7) {
        const size_t per_warp = (size_t)DNG_WARPS * (DNG_WIN + 4 * (size_t)jwide_max + 64);
        if (per_warp > 227 * 1024) return cudaErrorInvalidValue;
        // the tables go to shared memory too when they fit beside the warps' buffers
        const int ntab = ((size_t)ntables * 2 + 16 + per_warp <= 200 * 1024) ? ntables : 0;
        const size_t smem = (size_t)(ntab * 2 + 15) / 16 * 16 + per_warp;
        cudaError_t e = cudaFuncSetAttribute(k_dng_lj92, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        k_dng_lj92<<<(nparts + DNG_WARPS - 1) / DNG_WARPS, 32 * DNG_WARPS, smem, st>>>(A, jwide_max, ntab);
    } else {
        dim3 g((W + 255) / 256, H);
        k_dng_plain<<<g, 256, 0, st>>>(A, offs, cnts, rps, depth);
    }
    return cudaGetLastError();
}

// ---- DNG lossless-JPEG parts in parallel ----
//
// The per-part reader above decodes each tile or strip sequentially, so a
// frame of a few hundred tiles keeps only a few hundred lanes busy. Parts
// whose decode is a pure bit-offset recurrence -- predictor 1, no restart
// inside the part, one Huffman table for every component and part,
// categories up to 16 -- are decoded instead with the scheme of the PEF
// decoder:
//   1. each part's bytes go to its own 128-byte-aligned region of one
//      stream with the reader's byte skipping applied (the byte after a data
//      0xFF is dropped, so a byte is dropped exactly when the run of 0xFF
//      bytes before it within the part is odd); the rest of the region is
//      0xFF, which is what the reader sees past a part's end;
//   2. every 1024-bit chunk is decoded from each of its 32 candidate starts
//      (a symbol is at most 16 + 16 bits); a part's first chunk starts at
//      its bit 0 whatever state enters it;
//   3. the start maps are chained in three levels as for PEF, with "stopped"
//      (an empty table entry: the reader no longer advances and every later
//      difference of the part is 0) as a 33rd state;
//   4. each chunk's differences go to its part's sample order, the first
//      column is summed down the rows per component (vpred), each row along
//      itself per component, then the values are checked against the bit
//      depth and converted as above.
// A part whose data runs out inside its region without stopping, or a run
// of more than 64 0xFF bytes, raises a flag, and the host decodes the frame
// with the per-part reader instead.

namespace {

constexpr int DF_K = 32;           // candidate starts per chunk: one lane each
static_assert(DF_K == 32, "a warp holds the candidates of one chunk");
constexpr unsigned DF_STOP = 32;   // state of a stopped reader
constexpr int DF_MS = 40;          // bytes per 33-state map (padded)
constexpr int DF_NT = 256;
constexpr int DF_CB = 1024;        // chunks per block of the map composition
constexpr int DF_FF_RUN = 64;      // longest 0xFF run the byte skipping looks back over
constexpr int DF_MAX_CLRS = 4;

struct DngfPart {
    unsigned long long pos, n;     // the part's entropy bytes in the file
    unsigned long long reg;        // its region of the byte-skipped stream (bytes, a multiple of 128)
    unsigned long long sbase;      // its first sample in the difference buffer
    int cs;                        // its first chunk
    int high, jwide, clrs, bits;
    int out_row, out_col;
    int pad;
};

__device__ __forceinline__ unsigned bswap32(unsigned x) { return __byte_perm(x, 0, 0x0123); }

// Step 1: one CTA per part, 4 bytes per thread per pass; kept bytes placed by a block scan.
__global__ void __launch_bounds__(1024) k_dngf_unstuff(const uint8_t* __restrict__ file, const DngfPart* __restrict__ parts, uint8_t* __restrict__ us,
                                                       uint8_t* __restrict__ first, int* __restrict__ anomaly)
{
    __shared__ unsigned wsum[32];
    __shared__ unsigned long long carry;
    const DngfPart P = parts[blockIdx.x];
    if (threadIdx.x == 0) {
        carry = 0;
        first[P.cs] = 1;
    }
    __syncthreads();
    const uint8_t* src = file + P.pos;
    const long long n = (long long)P.n;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (long long b0 = 0; b0 < n; b0 += 4096) {
        const long long i0 = b0 + 4 * (long long)threadIdx.x;
        uint8_t v[4] = {0, 0, 0, 0};
        unsigned keep = 0;
        if (i0 < n) {
            int run = 0;  // 0xFF bytes just before i0 within the part
            for (long long j = i0 - 1; j >= 0 && run <= DF_FF_RUN; j--) {
                if (__ldg(src + j) != 0xFF) break;
                run++;
            }
            if (run > DF_FF_RUN) atomicExch(anomaly, 1);
#pragma unroll
            for (int k = 0; k < 4; k++) {
                if (i0 + k < n) {
                    v[k] = __ldg(src + i0 + k);
                    if ((run & 1) == 0) keep |= 1u << k;
                    run = v[k] == 0xFF ? run + 1 : 0;
                }
            }
        }
        const unsigned c = __popc(keep);
        unsigned x = c;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) wsum[warp] = x;
        __syncthreads();
        if (warp == 0) {
            unsigned w = wsum[lane];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const unsigned y = __shfl_up_sync(0xffffffffu, w, o);
                if (lane >= o) w += y;
            }
            wsum[lane] = w;
        }
        __syncthreads();
        unsigned long long o = carry + (warp ? wsum[warp - 1] : 0u) + x - c;
#pragma unroll
        for (int k = 0; k < 4; k++)
            if (keep >> k & 1) us[P.reg + o++] = v[k];
        __syncthreads();
        if (threadIdx.x == 0) carry += wsum[31];
        __syncthreads();
    }
}

// Step 2: a warp per chunk (grid-stride), its 34 words staged big-endian in
// shared memory; lane k follows candidate start k (0 for a part's first chunk).
__global__ void __launch_bounds__(DF_NT) k_dngf_map(const unsigned* __restrict__ us, const uint8_t* __restrict__ gadv, int hmax, int adv_smem,
                                                    const uint8_t* __restrict__ first, int nchunks, uint8_t* __restrict__ nextk,
                                                    uint16_t* __restrict__ cntk)
{
    extern __shared__ __align__(16) unsigned char dfm[];
    unsigned* cwall = (unsigned*)dfm;
    uint8_t* sadv = dfm + (DF_NT / 32) * 34 * 4;
    if (adv_smem) {
        const int nw = ((1 << hmax) + 3) / 4;
        for (int i = threadIdx.x; i < nw; i += blockDim.x) ((unsigned*)sadv)[i] = ((const unsigned*)gadv)[i];
    }
    __syncthreads();
    const uint8_t* adv = adv_smem ? sadv : gadv;
    const int warp = threadIdx.x >> 5, k = threadIdx.x & 31, sh = 32 - hmax;
    unsigned* cw = cwall + warp * 34;
    for (int i = blockIdx.x * (DF_NT / 32) + warp; i < nchunks; i += gridDim.x * (DF_NT / 32)) {
        for (int t = k; t < 34; t += 32) cw[t] = bswap32(__ldg(us + (size_t)i * 32 + t));
        __syncwarp();
        unsigned p = first[i] ? 0u : (unsigned)k, c = 0;
        bool stop = false;
        // two symbols per step while both must start inside the chunk (a symbol is at most 32 bits)
        while (p < 1024 - 64) {
            const unsigned w1 = p >> 5;
            const unsigned a1 = adv[__funnelshift_l(cw[w1 + 1], cw[w1], p & 31) >> sh];
            if (a1 == 0) {
                stop = true;
                break;
            }
            p += a1;
            const unsigned w2 = p >> 5;
            const unsigned a2 = adv[__funnelshift_l(cw[w2 + 1], cw[w2], p & 31) >> sh];
            if (a2 == 0) {
                c += 1;
                stop = true;
                break;
            }
            p += a2;
            c += 2;
        }
        while (!stop && p < 1024) {
            const unsigned w = p >> 5;
            const unsigned a = adv[__funnelshift_l(cw[w + 1], cw[w], p & 31) >> sh];
            if (a == 0) {
                stop = true;
                break;
            }
            p += a;
            c++;
        }
        nextk[(size_t)i * 32 + k] = stop ? (uint8_t)DF_STOP : (uint8_t)(p - 1024);
        cntk[(size_t)i * 32 + k] = (uint16_t)c;
        __syncwarp();
    }
}

// Step 3a: per block of DF_CB = 32 x 32 chunks, the 33-state map of each warp's 32 chunks and the block's map.
__global__ void __launch_bounds__(1024) k_dngf_compose(const uint8_t* __restrict__ nextk, const uint8_t* __restrict__ first, int nchunks,
                                                       uint8_t* __restrict__ sub_map, uint8_t* __restrict__ block_map)
{
    __shared__ uint8_t m[DF_CB][33];
    __shared__ uint8_t sm[32][DF_MS];
    const int c0 = blockIdx.x * DF_CB, n = min(DF_CB, nchunks - c0);
    for (int t = threadIdx.x; t < n * 32; t += blockDim.x) m[t >> 5][t & 31] = nextk[(size_t)c0 * 32 + t];
    __syncthreads();
    for (int q = threadIdx.x; q < n; q += blockDim.x) m[q][32] = first[c0 + q] ? m[q][0] : (uint8_t)DF_STOP;
    __syncthreads();
    const int warp = threadIdx.x >> 5, j = threadIdx.x & 31;
    for (int e = j; e < 33; e += 32) {
        unsigned s = (unsigned)e;
        for (int q = warp * 32; q < min(n, warp * 32 + 32); q++) s = m[q][s];
        sm[warp][e] = (uint8_t)s;
        sub_map[((size_t)blockIdx.x * 32 + warp) * DF_MS + e] = (uint8_t)s;
    }
    __syncthreads();
    if (warp == 0) {
        for (int e = j; e < 33; e += 32) {
            unsigned b = (unsigned)e;
            for (int w = 0; w < 32; w++) b = sm[w][b];
            block_map[(size_t)blockIdx.x * DF_MS + e] = (uint8_t)b;
        }
    }
}

// Step 3b: one thread walks the block maps: every block's entry state (chunk 0 starts a part).
__global__ void k_dngf_chain(const uint8_t* __restrict__ block_map, int nblocks, uint8_t* __restrict__ block_in)
{
    extern __shared__ uint8_t dbm[];
    for (int t = threadIdx.x; t < nblocks * DF_MS; t += blockDim.x) dbm[t] = block_map[t];
    __syncthreads();
    if (threadIdx.x != 0) return;
    unsigned s = 0;
    for (int b = 0; b < nblocks; b++) {
        block_in[b] = (uint8_t)s;
        s = dbm[b * DF_MS + s];
    }
}

// Step 3c: warp entry states, then lane 0 of each warp walks its chunks
// (entry state, count); the counts are scanned within the block.
__global__ void __launch_bounds__(1024) k_dngf_walk(const uint8_t* __restrict__ nextk, const uint16_t* __restrict__ cntk,
                                                    const uint8_t* __restrict__ sub_map, const uint8_t* __restrict__ block_in,
                                                    const uint8_t* __restrict__ first, int nchunks, uint8_t* __restrict__ sin,
                                                    unsigned* __restrict__ loc, unsigned* __restrict__ block_total)
{
    __shared__ uint8_t wentry[32];
    __shared__ unsigned wtot[32];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int c0 = blockIdx.x * DF_CB, n = min(DF_CB, nchunks - c0);
    if (threadIdx.x == 0) {
        unsigned s = block_in[blockIdx.x];
        for (int w = 0; w < 32; w++) {
            wentry[w] = (uint8_t)s;
            s = sub_map[((size_t)blockIdx.x * 32 + w) * DF_MS + s];
        }
    }
    __syncthreads();
    if (lane == 0) {
        unsigned s = wentry[warp];
        for (int q = 0; q < 32; q++) {
            const int ci = warp * 32 + q;
            if (ci >= n) break;
            const int i = c0 + ci;
            if (first[i]) s = 0;
            sin[i] = (uint8_t)s;
            if (s == DF_STOP) {
                loc[i] = 0;
                continue;
            }
            loc[i] = cntk[(size_t)i * 32 + s];
            s = nextk[(size_t)i * 32 + s];
        }
    }
    __syncwarp();
    const int ci = warp * 32 + lane;
    const unsigned my = ci < n ? loc[c0 + ci] : 0u;
    unsigned x = my;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) wtot[warp] = x;
    __syncthreads();
    unsigned wpre = 0;
    for (int w = 0; w < warp; w++) wpre += wtot[w];
    if (ci < n) loc[c0 + ci] = wpre + x - my;
    if (threadIdx.x == 0) {
        unsigned tot = 0;
        for (int w = 0; w < 32; w++) tot += wtot[w];
        block_total[blockIdx.x] = tot;
    }
}

__device__ __forceinline__ unsigned long long df_sym(const unsigned long long* __restrict__ boff, const unsigned* __restrict__ loc, int nchunks,
                                                     int nblocks, int i)
{
    return i < nchunks ? boff[i / DF_CB] + loc[i] : boff[nblocks];
}

// Per part: its first symbol's index in the chunk scan; a part that ends
// short of its samples without stopping ran out of its region (flag).
__global__ void k_dngf_parts(const DngfPart* __restrict__ parts, int nparts, int nchunks, int nblocks, const uint8_t* __restrict__ nextk,
                             const uint8_t* __restrict__ sin, const unsigned* __restrict__ loc, const unsigned long long* __restrict__ boff,
                             unsigned long long* __restrict__ g0, int* __restrict__ anomaly)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nparts) return;
    const int a = parts[t].cs, e = t + 1 < nparts ? parts[t + 1].cs : nchunks;
    const unsigned long long ga = df_sym(boff, loc, nchunks, nblocks, a), ge = df_sym(boff, loc, nchunks, nblocks, e);
    g0[t] = ga;
    const unsigned long long S = (unsigned long long)parts[t].high * parts[t].jwide;
    if (ge - ga < S) {
        const unsigned s = sin[e - 1];
        const unsigned exit = s == DF_STOP ? DF_STOP : nextk[(size_t)(e - 1) * 32 + s];
        if (exit != DF_STOP) atomicExch(anomaly, 1);
    }
}

// Step 4a: every chunk's differences (as 16-bit residues) at its part's
// sample offsets; one thread per chunk, the CTA's chunks staged with one
// skew word per 32.
__global__ void __launch_bounds__(DF_NT) k_dngf_emit(const unsigned* __restrict__ us, unsigned long long nwords, const DngfPart* __restrict__ parts,
                                                     const int* __restrict__ cs, int nparts, int nchunks, int nblocks, const uint8_t* __restrict__ sin,
                                                     const unsigned* __restrict__ loc, const unsigned long long* __restrict__ boff,
                                                     const unsigned long long* __restrict__ g0, const uint16_t* __restrict__ gtab, int hmax,
                                                     int tab_smem, int large, uint16_t* __restrict__ diff)
{
    extern __shared__ __align__(16) unsigned char dfe[];
    unsigned* cw = (unsigned*)dfe;
    uint16_t* stab = (uint16_t*)(dfe + (DF_NT * 33 + 4) * 4);
    const int c0 = blockIdx.x * DF_NT;
    for (int j = threadIdx.x; j < DF_NT * 32 + 2; j += DF_NT) {
        const unsigned long long g = (unsigned long long)c0 * 32 + j;
        cw[j + (j >> 5)] = g < nwords ? bswap32(__ldg(us + g)) : 0xffffffffu;
    }
    if (tab_smem)
        for (int i = threadIdx.x; i <= (1 << hmax); i += DF_NT) stab[i] = gtab[i];
    __syncthreads();
    const uint16_t* tab = (tab_smem ? stab : gtab) + 1;
    const int i = c0 + threadIdx.x;
    if (i >= nchunks) return;
    unsigned p = sin[i];
    if (p == DF_STOP) return;
    int lo = 0, hi = nparts - 1;  // the last part whose first chunk is <= i
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(cs + mid) <= i) lo = mid;
        else hi = mid - 1;
    }
    const DngfPart& P = parts[lo];
    const unsigned long long S = (unsigned long long)P.high * P.jwide;
    unsigned long long o = df_sym(boff, loc, nchunks, nblocks, i) - g0[lo];
    if (o >= S) return;
    const unsigned* cb = cw + 33 * threadIdx.x;
    const int sh = 32 - hmax;
    while (p < 1024 && o < S) {
        const unsigned w = p >> 5;
        const unsigned x = __funnelshift_l(cb[w + 1 + ((w + 1) >> 5)], cb[w], p & 31);
        const unsigned e = tab[x >> sh];
        const int clen = (int)(e >> 8), cat = (int)(e & 255);
        if (clen == 0) break;
        int d;
        if (cat == 16 && large) {
            d = -32768;
            p += clen;
        } else {
            d = cat ? (int)((x << clen) >> (32 - cat)) : 0;
            if (cat && ((d >> (cat - 1)) & 1) == 0) d -= (1 << cat) - 1;
            p += clen + cat;
        }
        diff[P.sbase + o++] = (uint16_t)d;
    }
}

// Step 4b: the first column of each component summed down the rows from
// 1 << (bits - 1), written back as values; a warp per (part, component).
__global__ void k_dngf_cols(const DngfPart* __restrict__ parts, int nparts, uint16_t* __restrict__ diff)
{
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    const int t = gw / DF_MAX_CLRS, c = gw % DF_MAX_CLRS;
    if (t >= nparts) return;
    const DngfPart P = parts[t];
    if (c >= P.clrs) return;
    unsigned carry = 1u << (P.bits - 1);
    for (int base = 0; base < P.high; base += 32) {
        const int r = base + lane;
        const size_t at = P.sbase + (size_t)r * P.jwide + c;
        unsigned x = r < P.high ? diff[at] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (r < P.high) diff[at] = (uint16_t)(carry + x);
        carry += __shfl_sync(0xffffffffu, x, 31);
    }
}

// Step 4c: a warp per (part, row): per component the running sum along the
// row, the bit-depth check, the conversion and the store.
__global__ void __launch_bounds__(256) k_dngf_rows(const DngArgs A, const DngfPart* __restrict__ parts, const uint16_t* __restrict__ diff)
{
    const int t = blockIdx.y, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const DngfPart& P = parts[t];
    const int r = blockIdx.x * 8 + warp;
    if (r >= P.high) return;
    const uint16_t* drow = diff + P.sbase + (size_t)r * P.jwide;
    const int orow = P.out_row + r;
    uint16_t* o = orow < A.H ? isa::row_ptr(A.out, A.out_pitch, orow) : nullptr;
    const int clrs = P.clrs, jwide = P.jwide;
    unsigned carry[DF_MAX_CLRS] = {0u, 0u, 0u, 0u};
    bool bad = false;
    for (int base = 0; base < jwide; base += 32 * clrs) {
#pragma unroll
        for (int c = 0; c < DF_MAX_CLRS; c++) {
            if (c >= clrs) break;
            const int j = base + lane * clrs + c;
            unsigned x = j < jwide ? drow[j] : 0u;
#pragma unroll
            for (int q = 1; q < 32; q <<= 1) {
                const unsigned y = __shfl_up_sync(0xffffffffu, x, q);
                if (lane >= q) x += y;
            }
            const uint16_t v = (uint16_t)(carry[c] + x);
            carry[c] += __shfl_sync(0xffffffffu, x, 31);
            if (j < jwide) {
                if (v >> P.bits) bad = true;
                const int ocol = P.out_col + j;
                if (o && ocol < A.W) o[ocol] = dng_value(A, v, orow, ocol);
            }
        }
    }
    if (bad) atomicMin(A.error, t);
}

struct DngfPlan {
    std::vector<DngfPart> parts;
    std::vector<int> cs;
    std::vector<uint8_t> adv;
    const uint16_t* table = nullptr;   // 1 + 2^hmax entries
    int hmax = 0, nchunks = 0, nblocks = 0;
    unsigned long long samples = 0;
    size_t part[20] = {};
    size_t bytes = 0;
};

size_t df_align(size_t v) { return (v + 255) / 256 * 256; }

bool dngf_plan(const Lj92Part* L, int nparts, const uint16_t* tables, size_t ntables, int large, DngfPlan& pl)
{
    if (nparts < 1 || nparts > 65535 || ntables == 0) return false;
    const int tab = L[0].table[0];
    pl.parts.resize(nparts);
    pl.cs.resize(nparts + 1);
    unsigned long long reg = 0, sbase = 0;
    for (int t = 0; t < nparts; t++) {
        const Lj92Part& p = L[t];
        if (p.skip || p.psv != 1 || p.sraw != 0 || p.clrs < 1 || p.clrs > DF_MAX_CLRS || p.bits < 1 || p.bits > 16) return false;
        if ((long long)p.restart < (long long)p.high * p.wide) return false;  // a restart inside the part
        for (int c = 0; c < p.clrs; c++)
            if (p.table[c] != tab) return false;
        DngfPart& q = pl.parts[t];
        q.pos = p.pos;
        q.n = p.end > p.pos ? p.end - p.pos : 0;
        q.reg = reg;
        q.sbase = sbase;
        q.cs = (int)(reg / 128);
        q.high = p.high;
        q.jwide = p.wide * p.clrs;
        q.clrs = p.clrs;
        q.bits = p.bits;
        q.out_row = p.out_row;
        q.out_col = p.out_col;
        pl.cs[t] = q.cs;
        reg += (q.n + 256 + 127) / 128 * 128;
        sbase += (unsigned long long)q.high * q.jwide;
    }
    if (reg / 128 > 0x7fffffffull) return false;
    pl.nchunks = (int)(reg / 128);
    pl.cs[nparts] = pl.nchunks;
    pl.nblocks = (pl.nchunks + DF_CB - 1) / DF_CB;
    if ((size_t)pl.nblocks * DF_MS > 200 * 1024) return false;
    pl.samples = sbase;
    if ((size_t)tab >= ntables) return false;
    pl.hmax = tables[tab];
    if (pl.hmax < 1 || pl.hmax > 16 || (size_t)tab + 1 + ((size_t)1 << pl.hmax) > ntables) return false;
    pl.table = tables + tab;
    pl.adv.assign(std::max<size_t>((size_t)1 << pl.hmax, 4), 0);
    for (int i = 0; i < 1 << pl.hmax; i++) {
        const int e = pl.table[1 + i], clen = e >> 8, cat = e & 255;
        if (clen == 0) continue;
        if (cat > 16) return false;
        pl.adv[i] = (uint8_t)(clen + ((cat == 16 && large) ? 0 : cat));
    }
    // scratch layout
    const size_t sizes[] = {
        (size_t)nparts * sizeof(DngfPart),               // 0 parts
        (size_t)(nparts + 1) * 4,                        // 1 cs
        (size_t)pl.nchunks * 128 + 256,                  // 2 byte-skipped stream (0xFF past each part)
        (size_t)pl.nchunks,                              // 3 first
        (size_t)pl.nchunks * 32,                         // 4 nextk
        (size_t)pl.nchunks * 64,                         // 5 cntk
        (size_t)pl.nchunks,                              // 6 sin
        (size_t)pl.nchunks * 4,                          // 7 loc
        (size_t)pl.nblocks * 32 * DF_MS,                 // 8 sub_map
        (size_t)pl.nblocks * DF_MS,                      // 9 block_map
        (size_t)pl.nblocks,                              // 10 block_in
        (size_t)pl.nblocks * 4,                          // 11 block_total
        (size_t)(pl.nblocks + 1) * 8,                    // 12 boff
        (size_t)nparts * 8,                              // 13 g0
        (size_t)pl.samples * 2 + 16,                     // 14 differences
        ((size_t)1 + ((size_t)1 << pl.hmax)) * 2,        // 15 table
        pl.adv.size(),                                   // 16 advance table
        16,                                              // 17 flag
    };
    size_t o = 0;
    for (int k = 0; k < 18; k++) {
        pl.part[k] = o;
        o += df_align(sizes[k]);
    }
    pl.bytes = o;
    return true;
}

}  // namespace

size_t isa_dngf_scratch(const void* parts, int nparts, const uint16_t* tables, size_t ntables, int large)
{
    DngfPlan pl;
    return dngf_plan((const Lj92Part*)parts, nparts, tables, ntables, large, pl) ? pl.bytes : 0;
}

size_t isa_dngf_flag_offset(const void* parts, int nparts, const uint16_t* tables, size_t ntables, int large)
{
    DngfPlan pl;
    return dngf_plan((const Lj92Part*)parts, nparts, tables, ntables, large, pl) ? pl.part[17] : 0;
}

cudaError_t isa_launch_dngf(const uint8_t* file, unsigned long long fsize, const void* parts_host, int nparts, const uint16_t* tables_host,
                            size_t ntables, const uint16_t* lin, int nlin, const uint16_t* bh, const uint16_t* bv, int W, int H, int large,
                            uint16_t* out, size_t out_pitch, int* error, void* scratch, size_t scratch_bytes, int* anomaly_host, cudaStream_t st)
{
    DngfPlan pl;
    if (!dngf_plan((const Lj92Part*)parts_host, nparts, tables_host, ntables, large, pl) || scratch_bytes < pl.bytes) return cudaErrorInvalidValue;
    char* base = (char*)scratch;
    DngfPart* d_parts = (DngfPart*)(base + pl.part[0]);
    int* d_cs = (int*)(base + pl.part[1]);
    uint8_t* us = (uint8_t*)(base + pl.part[2]);
    uint8_t* first = (uint8_t*)(base + pl.part[3]);
    uint8_t* nextk = (uint8_t*)(base + pl.part[4]);
    uint16_t* cntk = (uint16_t*)(base + pl.part[5]);
    uint8_t* sin = (uint8_t*)(base + pl.part[6]);
    unsigned* loc = (unsigned*)(base + pl.part[7]);
    uint8_t* sub_map = (uint8_t*)(base + pl.part[8]);
    uint8_t* block_map = (uint8_t*)(base + pl.part[9]);
    uint8_t* block_in = (uint8_t*)(base + pl.part[10]);
    unsigned* block_total = (unsigned*)(base + pl.part[11]);
    unsigned long long* boff = (unsigned long long*)(base + pl.part[12]);
    unsigned long long* g0 = (unsigned long long*)(base + pl.part[13]);
    uint16_t* diff = (uint16_t*)(base + pl.part[14]);
    uint16_t* gtab = (uint16_t*)(base + pl.part[15]);
    uint8_t* gadv = (uint8_t*)(base + pl.part[16]);
    int* d_anomaly = (int*)(base + pl.part[17]);
    for (const DngfPart& p : pl.parts)
        if (p.pos + p.n > fsize) return cudaErrorInvalidValue;
    cudaError_t e;
    if ((e = cudaMemcpyAsync(d_parts, pl.parts.data(), pl.parts.size() * sizeof(DngfPart), cudaMemcpyHostToDevice, st)) != cudaSuccess) return e;
    if ((e = cudaMemcpyAsync(d_cs, pl.cs.data(), pl.cs.size() * 4, cudaMemcpyHostToDevice, st)) != cudaSuccess) return e;
    if ((e = cudaMemcpyAsync(gtab, pl.table, ((size_t)1 + ((size_t)1 << pl.hmax)) * 2, cudaMemcpyHostToDevice, st)) != cudaSuccess) return e;
    if ((e = cudaMemcpyAsync(gadv, pl.adv.data(), pl.adv.size(), cudaMemcpyHostToDevice, st)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(us, 0xFF, (size_t)pl.nchunks * 128 + 256, st)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(first, 0, (size_t)pl.nchunks, st)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(diff, 0, (size_t)pl.samples * 2 + 16, st)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(d_anomaly, 0, 16, st)) != cudaSuccess) return e;
    k_dngf_unstuff<<<nparts, 1024, 0, st>>>(file, d_parts, us, first, d_anomaly);
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int adv_smem = (1 << pl.hmax) <= 16384;
    const size_t map_smem = (size_t)(DF_NT / 32) * 34 * 4 + (adv_smem ? pl.adv.size() : 0);
    if ((e = cudaFuncSetAttribute(k_dngf_map, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)map_smem)) != cudaSuccess) return e;
    const unsigned mapg = (unsigned)std::min<long long>((pl.nchunks + DF_NT / 32 - 1) / (DF_NT / 32), (long long)sms * 8);
    k_dngf_map<<<mapg, DF_NT, map_smem, st>>>((const unsigned*)us, gadv, pl.hmax, adv_smem, first, pl.nchunks, nextk, cntk);
    k_dngf_compose<<<pl.nblocks, 1024, 0, st>>>(nextk, first, pl.nchunks, sub_map, block_map);
    const size_t chain_smem = (size_t)pl.nblocks * DF_MS;
    if ((e = cudaFuncSetAttribute(k_dngf_chain, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)chain_smem)) != cudaSuccess) return e;
    k_dngf_chain<<<1, 256, chain_smem, st>>>(block_map, pl.nblocks, block_in);
    k_dngf_walk<<<pl.nblocks, 1024, 0, st>>>(nextk, cntk, sub_map, block_in, first, pl.nchunks, sin, loc, block_total);
    k_pef_scan<<<1, 1024, 0, st>>>(block_total, pl.nblocks, boff);
    k_dngf_parts<<<(nparts + 255) / 256, 256, 0, st>>>(d_parts, nparts, pl.nchunks, pl.nblocks, nextk, sin, loc, boff, g0, d_anomaly);
    const int tab_smem = (1 << pl.hmax) <= 8192;
    const size_t emit_smem = (size_t)(DF_NT * 33 + 4) * 4 + (tab_smem ? ((size_t)1 + ((size_t)1 << pl.hmax)) * 2 : 0);
    if ((e = cudaFuncSetAttribute(k_dngf_emit, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)emit_smem)) != cudaSuccess) return e;
    k_dngf_emit<<<(pl.nchunks + DF_NT - 1) / DF_NT, DF_NT, emit_smem, st>>>((const unsigned*)us, (unsigned long long)pl.nchunks * 32 + 64, d_parts, d_cs,
                                                                          nparts, pl.nchunks, pl.nblocks, sin, loc, boff, g0, gtab, pl.hmax, tab_smem,
                                                                          large, diff);
    k_dngf_cols<<<(nparts * DF_MAX_CLRS * 32 + 255) / 256, 256, 0, st>>>(d_parts, nparts, diff);
    int max_high = 1;
    for (const DngfPart& p : pl.parts) max_high = std::max(max_high, p.high);
    DngArgs A{file, fsize, nullptr, nparts, nullptr, nullptr, lin, nlin, bh, bv, W, H, large, out, out_pitch, error};
    k_dngf_rows<<<dim3((max_high + 7) / 8, nparts), 256, 0, st>>>(A, d_parts, diff);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    return anomaly_host ? cudaMemcpyAsync(anomaly_host, d_anomaly, sizeof(int), cudaMemcpyDeviceToHost, st) : cudaSuccess;
}
