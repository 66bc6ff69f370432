// Row-band temporal kernel: K generations per launch, streaming in y.
//
// What it replaces in the reference: the one-generation-per-launch word
// kernels (src/algorithms/cuda-naive-bitwise/cuda_naive_bitwise_kernel.cu:32-79,
// cuda-simple-warp-exchange/simple_warp_exchange.cu:33-85) and the shared-
// memory temporal kernel (cuda-temporal-rowed/temporal_rowed.cu:33-229),
// which needs X/64 % 30 == 0 and N % 11 == 0. This one takes any width that
// is a multiple of 32 cells and any K in 1..16, and is bit-exact at every
// grid edge (cells outside the grid are dead).
//
// Work decomposition
//   * One CTA owns a band of output rows [y0, y1) across the full width when
//     it fits (W / WPL <= 256 lanes), so no x-halo is recomputed. Lane t of
//     the CTA holds words [t*WPL, t*WPL + WPL) of every row it touches (one
//     64/128-bit access). Wider grids are cut into x-slices whose CTAs add
//     one halo lane (WPL*32 >= 32 cells >= K) on each side: errors from the
//     unknown cells beyond the halo move one cell per generation, so after
//     K <= 32 generations they have not reached the slice.
//   * The CTA streams down the band. "Stage" 0 loads gen-0 rows; stage g
//     (1..K) turns gen g-1 rows into gen g rows, one row per step, lagging
//     stage g-1 by two rows. So after 3K warm-up steps every step retires
//     one gen-K row; the y-halo costs ~K extra rows per stage per band.
//   * Each stage keeps, in registers, the horizontal 3-cell sums of its last
//     three input rows (a ring of 3) and two raw input rows; it never
//     touches shared memory for row data.
//   * Neighbour bits across lanes come from warp shuffles; across warps from
//     a tiny shared-memory "edge" table (first/last word of each warp's
//     span, per stage, double-buffered by step parity). One __syncthreads
//     per step publishes them.
//   * Warm-up and drain steps test which stages are active and mask rows
//     outside the grid; the steady-state steps between them run a branch-
//     free body, so a step is one basic block whose K stages interleave.
//
// Ring indices depend on the step number mod 3, so the step body is a
// template on that phase and the loop is unrolled by 3: all ring accesses
// are compile-time register names, no moves.
#pragma once

#include <cstdint>

#include "gol_word_ops.cuh"

namespace golb200 {

constexpr int kTemporalMaxThreads = 256;
#ifndef GOL_TEMPORAL_MIN_BLOCKS
#define GOL_TEMPORAL_MIN_BLOCKS 1   // CTAs per SM the register budget is sized for
#endif

struct RowsLaunch {
    const uint32_t* src;   // gen-0 grid, W words per row, Y rows
    uint32_t* dst;         // gen-K grid (must not alias src)
    int W;                 // 32-bit words per row
    int Y;                 // rows
    int band;              // output rows per CTA (blockIdx.x)
    int slice;             // words per x-slice (blockIdx.y); W when unsliced
    int halo;              // words of x-halo each side of a slice (0 or WPL)
};

template <int WPL>
__device__ __forceinline__ void load_words(const uint32_t* p, uint32_t (&v)[WPL]) {
    if constexpr (WPL == 4) {
        const uint4 t = __ldg(reinterpret_cast<const uint4*>(p));
        v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
    } else if constexpr (WPL == 2) {
        const uint2 t = __ldg(reinterpret_cast<const uint2*>(p));
        v[0] = t.x; v[1] = t.y;
    } else {
        v[0] = __ldg(p);
    }
}

template <int WPL>
__device__ __forceinline__ void store_words(uint32_t* p, const uint32_t (&v)[WPL]) {
    if constexpr (WPL == 4) {
        *reinterpret_cast<uint4*>(p) = make_uint4(v[0], v[1], v[2], v[3]);
    } else if constexpr (WPL == 2) {
        *reinterpret_cast<uint2*>(p) = make_uint2(v[0], v[1]);
    } else {
        *p = v[0];
    }
}

template <int WPL, int K>
struct TemporalRegs {
    uint32_t ld[3][WPL];          // stage-0 rows, slot = step % 3
    uint32_t h0[K][3][WPL];       // stage g's horizontal sums, bit plane 0
    uint32_t h1[K][3][WPL];       //                            bit plane 1
    uint32_t o[K][3][WPL];        // stage g's output rows, slot = step % 3
};

// Edge table layout: [EW padded warps][K producer stages][3 step slots]
// [2 sides], then one dummy entry per warp. Every lane's read/write base is
// loop-invariant and each stage/slot offset is a compile-time immediate.
// Padded warps 0 and EW-1 stay zero: the dead cells beyond the CTA's
// outermost words. Lanes 1..30 write their (unused) edge words to their
// warp's dummy entry, so publishing needs no branch.
__host__ __device__ constexpr int edge_off(int g, int slot) { return (g * 3 + slot) * 2; }

struct TemporalCtx {
    const uint32_t* src;
    uint32_t* dst;
    const uint32_t* erd;   // lane 0: left warp's side-1 entry; lane 31: right warp's side-0
    uint32_t* ewr;         // lane 0 / 31: this warp's entry, side 0 / 1; others: dummy word
    bool first_lane, last_lane;
    int W, Y, y0, y1, B;
    int lane, base;
    bool lane_ok;   // this lane's words lie inside the grid
    bool own;       // ... and inside this CTA's slice (not halo): stored
};

// Step body. FAST = steady state: every stage active, every row inside the
// grid, so no activity tests or row masks (the whole step is one basic
// block and the K stages' independent chains interleave). LMASK forces the
// out-of-grid lanes of a partial CTA to stay dead.
template <int WPL, int K, int PH, bool FAST, bool LMASK>
__device__ __forceinline__ void temporal_step(TemporalRegs<WPL, K>& s, const TemporalCtx& c, int i,
                                              uint32_t lane_mask) {
    constexpr int NEW3 = PH % 3;          // ring-of-3 slot written at this step
    constexpr int PREV3 = (PH + 2) % 3;   // ... written one step ago
    constexpr int OLD3 = (PH + 1) % 3;    // ... written two steps ago

    // Stages run high to low so that stage g reads stage g-1's rows from the
    // previous steps before stage g-1 overwrites its ring slot.
#pragma unroll
    for (int g = K; g >= 1; --g) {
        if (FAST || (i >= 3 * g - 2 && i <= c.B + 2 * K + g - 1)) {
            // Intake row P (gen g-1, row r+1) and centre row C (gen g-1, row r).
            uint32_t P[WPL], C[WPL];
#pragma unroll
            for (int w = 0; w < WPL; ++w) {
                if (g == 1) {
                    P[w] = s.ld[PREV3][w];
                    C[w] = s.ld[OLD3][w];
                } else {
                    P[w] = s.o[g - 2][PREV3][w];
                    C[w] = s.o[g - 2][OLD3][w];
                }
            }
            // Words just left and right of this lane's span.
            uint32_t lw = __shfl_up_sync(0xffffffffu, P[WPL - 1], 1);
            uint32_t rw = __shfl_down_sync(0xffffffffu, P[0], 1);
            const uint32_t ev = c.erd[edge_off(g - 1, PREV3)];
            lw = c.first_lane ? ev : lw;
            rw = c.last_lane ? ev : rw;
#pragma unroll
            for (int w = 0; w < WPL; ++w) {
                const uint32_t l = (w == 0) ? lw : P[w - 1];
                const uint32_t r = (w == WPL - 1) ? rw : P[w + 1];
                hsum(l, P[w], r, s.h0[g - 1][NEW3][w], s.h1[g - 1][NEW3][w]);
            }
            // Output row r of gen g (garbage during warm-up, never consumed).
            const int row = c.y0 - K + i - 2 * g;
            uint32_t keep = lane_mask;
            if (!FAST) keep = (c.lane_ok && (unsigned)row < (unsigned)c.Y) ? 0xffffffffu : 0u;
            uint32_t res[WPL];
#pragma unroll
            for (int w = 0; w < WPL; ++w) {
                res[w] = next_word(s.h0[g - 1][OLD3][w], s.h1[g - 1][OLD3][w],
                                   s.h0[g - 1][PREV3][w], s.h1[g - 1][PREV3][w],
                                   s.h0[g - 1][NEW3][w], s.h1[g - 1][NEW3][w], C[w]);
                if (!FAST || LMASK) res[w] &= keep;
            }
            if (g == K) {
                if ((FAST || (row >= c.y0 && row < c.y1)) && c.own)
                    store_words<WPL>(c.dst + (size_t)row * c.W + c.base, res);
            } else {
#pragma unroll
                for (int w = 0; w < WPL; ++w) s.o[g - 1][NEW3][w] = res[w];
                c.ewr[edge_off(g, NEW3)] = c.last_lane ? res[WPL - 1] : res[0];
            }
        }
    }

    // Stage 0: publish this step's loaded row, prefetch the next one.
    if (FAST || i <= c.B + 2 * K - 1) {
        c.ewr[edge_off(0, NEW3)] = c.last_lane ? s.ld[NEW3][WPL - 1] : s.ld[NEW3][0];
        const int nrow = c.y0 - K + i + 1;
        if (FAST) {
            if (!LMASK || c.lane_ok)
                load_words<WPL>(c.src + (size_t)nrow * c.W + c.base, s.ld[(PH + 1) % 3]);
        } else if (i + 1 <= c.B + 2 * K - 1 && c.lane_ok && (unsigned)nrow < (unsigned)c.Y) {
            load_words<WPL>(c.src + (size_t)nrow * c.W + c.base, s.ld[(PH + 1) % 3]);
        } else {
#pragma unroll
            for (int w = 0; w < WPL; ++w) s.ld[(PH + 1) % 3][w] = 0u;
        }
    }
    __syncthreads();
}

template <int WPL, int K, bool FAST, bool LMASK>
__device__ __forceinline__ void temporal_steps(TemporalRegs<WPL, K>& s, const TemporalCtx& c,
                                               int i0, int i1, uint32_t lane_mask) {
    for (int i = i0; i < i1; i += 3) {
        temporal_step<WPL, K, 0, FAST, LMASK>(s, c, i + 0, lane_mask);
        temporal_step<WPL, K, 1, FAST, LMASK>(s, c, i + 1, lane_mask);
        temporal_step<WPL, K, 2, FAST, LMASK>(s, c, i + 2, lane_mask);
    }
}

template <int WPL, int K>
__global__ void __launch_bounds__(kTemporalMaxThreads, GOL_TEMPORAL_MIN_BLOCKS)
rows_temporal_kernel(RowsLaunch a) {
    extern __shared__ uint32_t edges[];
    constexpr int ESTRIDE = K * 6;            // words per padded-warp entry
    TemporalCtx c;
    c.src = a.src;
    c.dst = a.dst;
    c.W = a.W;
    c.Y = a.Y;
    c.y0 = blockIdx.x * a.band;
    c.y1 = min(c.y0 + a.band, a.Y);
    c.B = c.y1 - c.y0;
    c.lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int EW = (blockDim.x >> 5) + 2;
    c.first_lane = c.lane == 0;
    c.last_lane = c.lane == 31;
    c.erd = edges + (c.first_lane ? warp * ESTRIDE + 1 : (warp + 2) * ESTRIDE);
    c.ewr = (c.first_lane || c.last_lane)
                ? edges + (warp + 1) * ESTRIDE + (c.last_lane ? 1 : 0)
                : edges + (EW + warp) * ESTRIDE;
    const int xs = blockIdx.y * a.slice;
    const int x0 = xs - a.halo;
    c.base = x0 + (int)threadIdx.x * WPL;
    c.lane_ok = c.base >= 0 && c.base < a.W;
    c.own = c.lane_ok && c.base >= xs && c.base < xs + a.slice;
    const bool all_lanes_ok = x0 >= 0 && x0 + (int)blockDim.x * WPL <= a.W;
    const uint32_t lane_mask = c.lane_ok ? 0xffffffffu : 0u;

    for (int t = threadIdx.x; t < EW * ESTRIDE; t += blockDim.x) edges[t] = 0u;

    TemporalRegs<WPL, K> s;
#pragma unroll
    for (int w = 0; w < WPL; ++w) {
        s.ld[0][w] = s.ld[1][w] = s.ld[2][w] = 0u;
#pragma unroll
        for (int g = 0; g < K; ++g) {
            s.h0[g][0][w] = s.h0[g][1][w] = s.h0[g][2][w] = 0u;
            s.h1[g][0][w] = s.h1[g][1][w] = s.h1[g][2][w] = 0u;
            s.o[g][0][w] = s.o[g][1][w] = s.o[g][2][w] = 0u;
        }
    }
    const int row0 = c.y0 - K;
    if (c.lane_ok && (unsigned)row0 < (unsigned)c.Y)
        load_words<WPL>(c.src + (size_t)row0 * c.W + c.base, s.ld[0]);
    __syncthreads();

    // Steps [f0, f1) run the steady-state body: all stages active (i >= 3K),
    // the next load row exists (i + 1 <= B + 2K - 1) and lies inside the grid
    // (y0 - K + i + 1 < Y), so no row computed there leaves the grid.
    // Segment bounds are multiples of 3 to keep the ring phases aligned.
    const int nsteps = c.B + 3 * K;
    const int f0 = 3 * K;
    const int f1 = min(c.B + 2 * K - 1, c.Y - c.y0 + K - 1);
    const int fast_end = f1 > f0 ? f0 + (f1 - f0) / 3 * 3 : f0;
    if (fast_end > f0) {
        temporal_steps<WPL, K, false, false>(s, c, 0, f0, lane_mask);
        if (all_lanes_ok)
            temporal_steps<WPL, K, true, false>(s, c, f0, fast_end, lane_mask);
        else
            temporal_steps<WPL, K, true, true>(s, c, f0, fast_end, lane_mask);
        temporal_steps<WPL, K, false, false>(s, c, fast_end, nsteps, lane_mask);
    } else {
        temporal_steps<WPL, K, false, false>(s, c, 0, nsteps, lane_mask);
    }
}

// Shared memory a launch needs: the edge table plus one dummy entry per warp.
__host__ __device__ inline size_t temporal_smem_bytes(int K, int threads) {
    return (size_t)(2 * (threads >> 5) + 2) * K * 6 * sizeof(uint32_t);
}

} // namespace golb200
