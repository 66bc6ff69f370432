// One-generation streaming kernel: the HBM-bound pass.
//
// What it replaces in the reference: the plain one-generation word kernel
// (src/algorithms/cuda-naive-bitwise/cuda_naive_bitwise_kernel.cu:32-79),
// which loads the 3x3 neighbourhood of every word (9 loads per word, cells
// outside the grid read as 0 through `load`, :24-30) and launches once per
// generation (:58-79).
//
// A single generation does about 12 integer operations per 32-cell word
// against 8 bytes of HBM traffic, so the pass is bound by HBM, not by the
// integer pipe: what matters is bytes in flight, coalescing and no wasted
// traffic. So, unlike the K-stage pipeline of gol_rows_temporal.cuh (one
// barrier per row, a deep register pipeline, two CTAs per SM):
//   * a thread owns WPL consecutive words of a row (one 16/8/4-byte load and
//     store) and walks down a band of `band` rows, reading band + 2 rows;
//   * loads are issued P - 1 rows ahead into a register ring of P rows (P a
//     multiple of 3, the loop unrolled by P, so every ring slot and the
//     3-row ring of horizontal sums are compile-time register names);
//   * no shared memory and no barriers: the word left and right of a lane's
//     span come from its warp neighbours by shuffle, and lanes 0 and 31 load
//     them from global memory (the same 32-byte sectors the neighbouring
//     warps read, so an L1/L2 hit, not extra HBM traffic);
//   * few registers, so many warps per SM keep enough bytes in flight.
// The halo rows (one above and one below each band) are read by both
// neighbouring bands; bands with adjacent blockIdx.y run at the same time,
// so the second read hits L2.
#pragma once

#include <cstdint>

#include "gol_rows_temporal.cuh"
#include "gol_word_ops.cuh"

namespace golb200 {

constexpr int kStreamMaxThreads = 256;
#ifndef GOL_STREAM_AHEAD
// Rows loaded ahead (a multiple of 3). At 32768^2 (128 threads, 4 words per
// lane, 8-row bands) 3 ran at 5.40 TB/s algorithmic against 5.08 for 6;
// fewer registers, more resident warps.
#define GOL_STREAM_AHEAD 3
#endif
constexpr int kStreamAhead = GOL_STREAM_AHEAD;   // rows in flight per thread (multiple of 3)

template <int WPL>
__device__ __forceinline__ void stream_load(const uint32_t* p, bool v, uint32_t (&w)[WPL]) {
    if (v) {
        load_words<WPL>(p, w);
    } else {
#pragma unroll
        for (int i = 0; i < WPL; ++i) w[i] = 0u;
    }
}

// a.band = output rows per thread (any positive value); a.slice = words
// per CTA across the row (blockDim.x lanes of WPL words). The grid is 1-D:
// CTA b takes slice b % nslices of band b / nslices, so CTAs with adjacent
// indices share rows (and their halo rows meet in L2). a.halo is unused (the
// row is never cut with halo lanes: lanes at a CTA boundary read their outer
// words from memory).
// One step of the stream: read-row i (grid row y0 - 1 + i) is in ring slot
// J = i mod P. Its horizontal sums go to ring-of-3 slot i mod 3; then output
// row i - 2 is formed from the sums of read-rows i-2, i-1, i and the centre
// words of read-row i-1, still in slot (J - 1) mod P, which is then free and
// takes read-row i - 1 + P (so P - 1 rows are in flight ahead). FAST: that
// row exists and lies inside the grid (no bounds tests).
template <int WPL, int P, int J, bool FAST>
__device__ __forceinline__ void stream_step(const RowsLaunch& a, int i, int n, int y0, int base,
                                            bool ok, bool load_l, bool load_r, int lane,
                                            const uint32_t*& next, uint32_t (&v)[P][WPL],
                                            uint32_t (&vl)[P], uint32_t (&vr)[P],
                                            uint32_t (&h0)[3][WPL], uint32_t (&h1)[3][WPL]) {
    constexpr int R = J % 3;                 // i mod 3 (i - J is a multiple of P, P of 3)
    constexpr int JP = (J + P - 1) % P;      // slot of read-row i - 1
    uint32_t lw = __shfl_up_sync(0xffffffffu, v[J][WPL - 1], 1);
    uint32_t rw = __shfl_down_sync(0xffffffffu, v[J][0], 1);
    if (lane == 0) lw = vl[J];
    if (lane == 31) rw = vr[J];
#pragma unroll
    for (int w = 0; w < WPL; ++w) {
        const uint32_t l = w == 0 ? lw : v[J][w - 1];
        const uint32_t r = w == WPL - 1 ? rw : v[J][w + 1];
        hsum(l, v[J][w], r, h0[R][w], h1[R][w]);
    }
    if (FAST || i >= 2) {                    // output row y0 + i - 2
        constexpr int RM = (R + 1) % 3;      // (i - 2) mod 3
        constexpr int RC = (R + 2) % 3;      // (i - 1) mod 3
        uint32_t res[WPL];
#pragma unroll
        for (int w = 0; w < WPL; ++w)
            res[w] = next_word(h0[RM][w], h1[RM][w], h0[RC][w], h1[RC][w], h0[R][w], h1[R][w],
                               v[JP][w]);
        if (ok) store_words<WPL>(a.dst + (size_t)(y0 + i - 2) * a.pitch + base, res);
    }
    // slot JP takes read-row i - 1 + P
    if (FAST) {
        if (ok) load_words<WPL>(next, v[JP]);
        vl[JP] = load_l ? __ldg(next - 1) : 0u;
        vr[JP] = load_r ? __ldg(next + WPL) : 0u;
    } else {
        const int ir = i - 1 + P;
        const int y = y0 - 1 + ir;
        const bool rv = ir < n && (unsigned)y < (unsigned)a.Y;
        stream_load<WPL>(next, ok && rv, v[JP]);
        vl[JP] = (load_l && rv) ? __ldg(next - 1) : 0u;
        vr[JP] = (load_r && rv) ? __ldg(next + WPL) : 0u;
    }
    next += a.pitch;
}

template <int WPL, int P, bool FAST, int J = 0>
__device__ __forceinline__ void stream_chunk(const RowsLaunch& a, int i0, int n, int y0, int base,
                                             bool ok, bool load_l, bool load_r, int lane,
                                             const uint32_t*& next, uint32_t (&v)[P][WPL],
                                             uint32_t (&vl)[P], uint32_t (&vr)[P],
                                             uint32_t (&h0)[3][WPL], uint32_t (&h1)[3][WPL]) {
    if constexpr (J < P) {
        if (!FAST && i0 + J >= n) return;   // n is uniform across the CTA
        stream_step<WPL, P, J, FAST>(a, i0 + J, n, y0, base, ok, load_l, load_r, lane, next, v,
                                     vl, vr, h0, h1);
        stream_chunk<WPL, P, FAST, J + 1>(a, i0, n, y0, base, ok, load_l, load_r, lane, next, v,
                                          vl, vr, h0, h1);
    }
}

template <int WPL>
__global__ void __launch_bounds__(kStreamMaxThreads)
rows_stream_kernel(RowsLaunch a) {
    constexpr int P = kStreamAhead;
    static_assert(P % 3 == 0, "the ring of horizontal sums is indexed by row mod 3");
    pdl_trigger_and_wait();
    const int lane = threadIdx.x & 31;
    const int nslices = (a.W + a.slice - 1) / a.slice;
    const int slice = (int)(blockIdx.x % (unsigned)nslices);
    const int band = (int)(blockIdx.x / (unsigned)nslices);
    const int base = slice * a.slice + (int)threadIdx.x * WPL;
    const bool ok = base < a.W;   // W % WPL == 0: a lane is wholly inside or outside
    const bool load_l = ok && lane == 0 && base > 0;
    const bool load_r = ok && lane == 31 && base + WPL < a.W;
    const int y0 = band * a.band;
    const int y1 = min(y0 + a.band, a.Y);
    const int n = y1 - y0 + 2;    // read-rows 0 .. n-1: grid rows y0 - 1 .. y1
    const uint32_t* col = a.src + base;

    uint32_t v[P][WPL], vl[P], vr[P];   // rows in flight: words, outer left / right word
    uint32_t h0[3][WPL], h1[3][WPL];    // horizontal sums by read-row mod 3
#pragma unroll
    for (int s = 0; s < P; ++s) {       // read-rows 0 .. P-2 into slots 0 .. P-2
        const int y = y0 - 1 + s;
        const bool rv = s < P - 1 && s < n && (unsigned)y < (unsigned)a.Y;
        const uint32_t* p = col + (size_t)(rv ? y : 0) * a.pitch;
        stream_load<WPL>(p, ok && rv, v[s]);
        vl[s] = (load_l && rv) ? __ldg(p - 1) : 0u;
        vr[s] = (load_r && rv) ? __ldg(p + WPL) : 0u;
    }
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int w = 0; w < WPL; ++w) h0[r][w] = h1[r][w] = 0u;
    // the next row to issue: read-row P - 1 (a pointer that may point
    // outside the grid; it is dereferenced only for rows inside it)
    const uint32_t* next = col + (long long)(y0 - 2 + P) * a.pitch;
    int i0 = 0;
    // Chunks whose steps all issue rows inside the grid, output rows >= 2
    // in: read-rows up to i0 + 2P - 2 <= n - 2, and i0 >= P.
    if (n >= 2 * P + 2) {
        stream_chunk<WPL, P, false>(a, 0, n, y0, base, ok, load_l, load_r, lane, next, v, vl, vr,
                                    h0, h1);
        for (i0 = P; i0 + 2 * P <= n; i0 += P)
            stream_chunk<WPL, P, true>(a, i0, n, y0, base, ok, load_l, load_r, lane, next, v, vl,
                                       vr, h0, h1);
    }
    for (; i0 < n; i0 += P)
        stream_chunk<WPL, P, false>(a, i0, n, y0, base, ok, load_l, load_r, lane, next, v, vl, vr,
                                    h0, h1);
}

} // namespace golb200
