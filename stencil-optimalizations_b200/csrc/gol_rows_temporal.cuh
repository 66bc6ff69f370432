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
//   * Neighbour bits across lanes come from a shared-memory "edge" table:
//     every lane publishes the first and last word of each row it produces
//     (per stage, in a ring of 3 step slots) and reads its neighbours'
//     entries of the previous step. One __syncthreads per step separates
//     the two. (Segmented one-warp kernels keep a per-warp table with zero
//     entries at segment ends; one word per lane uses warp shuffles.)
//   * Warm-up and drain steps test which stages are active and mask rows
//     outside the grid; the steady-state steps between them run a branch-
//     free body, so a step is one basic block whose K stages interleave.
//
// Ring indices depend on the step number mod 3, so the step body is a
// template on that phase and the loop is unrolled by 3: all register-ring
// accesses are compile-time register names, no moves, and the shared-
// memory row ring (6 slots = two banks of 3) needs only a bank swap per
// three steps.
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
    int pitch;             // words from one row to the next (>= W)
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

// Rows for stage 0 are staged through a shared-memory ring with cp.async:
// kRowRing slots, kRowsInFlight rows issued ahead of use. Each lane copies
// and later reads back only its own words, so a per-thread
// cp.async.wait_group (a hardware wait, no spin) orders the two. Rows and
// lanes outside the grid are zero-filled by the copy itself (src-size 0).
// Step i's row lives in slot i mod 6, i.e. two banks of three slots: the
// steps are unrolled by three, so within a bank every slot offset is a
// compile-time immediate and only the bank changes (once per three steps).
constexpr int kRowRing = 6;
constexpr int kRowsInFlight = kRowRing - 1;

template <int WPL>
__device__ __forceinline__ void cp_async_words(uint32_t saddr, const uint32_t* g, bool valid) {
    const int bytes = valid ? WPL * 4 : 0;
    if constexpr (WPL == 4) {
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(saddr), "l"(g), "r"(bytes)
                     : "memory");
    } else if constexpr (WPL == 2) {
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(saddr), "l"(g), "r"(bytes)
                     : "memory");
    } else {
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(saddr), "l"(g), "r"(bytes)
                     : "memory");
    }
}

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }

template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

template <int WPL>
__device__ __forceinline__ void lds_words(const uint32_t* p, uint32_t (&v)[WPL]) {
    if constexpr (WPL == 4) {
        const uint4 t = *reinterpret_cast<const uint4*>(p);
        v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
    } else if constexpr (WPL == 2) {
        const uint2 t = *reinterpret_cast<const uint2*>(p);
        v[0] = t.x; v[1] = t.y;
    } else {
        v[0] = *p;
    }
}

template <int WPL, int K>
struct TemporalRegs {
    uint32_t bank_cur, bank_oth;  // shared addresses of this lane's ring banks: steps 3t..3t+2
                                  // keep their rows in bank_cur (slots 3*(t%2) .. +2)
    uint32_t diff;                // change tracking: OR of (new ^ old) over stored words
                                  // (per tile row: bit w = word w of the lane changed)
    int flush_row;                // per tile row: the next row that closes a tile row,
    int flush_ty;                 // ... and its tile row
    uint32_t ld[3][WPL];          // stage-0 rows, slot = step % 3
    uint32_t h0[K][3][WPL];       // stage g's horizontal sums, bit plane 0
    uint32_t h1[K][3][WPL];       //                            bit plane 1
    uint32_t o[K][3][WPL];        // stage g's output rows, slot = step % 3
};

// Edge table: every lane publishes the first and the last word of each row
// it produces (stage g's output, or stage 0's loaded row) and reads its
// neighbours' from the previous step, one barrier per step in between.
// Layout: [2 sides: first words, last words][K producer stages][3 step
// slots][ES entries, lane t at t + 1]; entries 0 and ES - 1 are never
// written and stay zero: the dead cells beyond the CTA's (or a segment's)
// outermost words. Each lane reads through two loop-invariant pointers (its
// left and right neighbour's entry, or a zero entry at a segment end) and
// every stage/slot offset is a compile-time immediate; neighbouring lanes
// touch neighbouring words (no bank conflicts). ES = kEdgeStride for
// CTA-wide tables, kSegEdgeStride for one-warp (segmented) ones.
constexpr int kEdgeStride = kTemporalMaxThreads + 2;
constexpr int kSegEdgeStride = 32 + 2;
template <int ES>
__host__ __device__ constexpr int edge_off(int g, int slot) { return (g * 3 + slot) * ES; }
template <int K, int ES>
__host__ __device__ constexpr int edge_last_side() { return K * 3 * ES; }
// Words of a segmented warp's edge table for depth K.
__host__ __device__ constexpr int seg_edge_words(int K) { return 2 * K * 3 * kSegEdgeStride; }

// Per-tile change bits written by a dense pass (change tracking): tile
// (tx, ty) covers words [tx * words, +words) of rows [ty * rows, +rows) and is
// bit tx % 32 of changed[ty * cw + tx / 32].
struct TileTrack {
    uint32_t* changed;
    int rows, words, cw;
};

struct TemporalCtx {
    const uint32_t* src;
    uint32_t* dst;
    uint32_t* eb;          // edge table + this lane's index (entry of lane t is t + 1)
    const uint32_t* el;    // entry of the left neighbour (eb), or a zero entry
    const uint32_t* er;    // entry of the right neighbour (eb + 2), or a zero entry
    // segmented warps of one word per lane exchange edges by shuffle instead
    bool seg_first, seg_last;   // segment ends (their outer neighbour is dead)
    const uint32_t* ring;  // this lane's words in ring slot 0 (shared memory)
    uint32_t ring_saddr;   // same, as a shared-window address for cp.async
    int ring_stride;       // words per ring slot: ring_slot_words<WPL, SEG>()
    int W, Y, y0, y1, B;
    int pitch;      // words from one row to the next: W, or W rounded up to WPL
                    // (then the words past W are zero and stay zero)
    int lane, base;
    bool lane_ok;   // this lane's first word lies inside the grid
    bool own;       // ... and inside this CTA's slice (not halo): stored
    int src_l, src_r;   // segmented warps: lanes holding the words left / right
    uint32_t wmask[4];  // per word of the lane: all ones inside the grid, else 0
    TileTrack tt;       // per-tile change bits (TRACK == 2):
    uint32_t tbit[4];   // the tile bit of each word of the lane in its change word
    int tfw;            // that change word (-1 for lanes that store nothing)
};

// Word masks of a lane whose words start at `base` in a W-word row.
template <int WPL>
__device__ __forceinline__ void set_word_masks(TemporalCtx& c) {
#pragma unroll
    for (int w = 0; w < 4; ++w)
        c.wmask[w] = (w < WPL && c.lane_ok && c.base + w < c.W) ? 0xffffffffu : 0u;
}

// Words per ring slot: the CTA's widest possible row of lanes (one warp for
// segmented warps), so that slot offsets are compile-time constants.
template <int WPL, bool SEG>
__host__ __device__ constexpr int ring_slot_words() { return (SEG ? 32 : kTemporalMaxThreads) * WPL; }

// Change tracking compares each output row with the same grid row before
// the pass. CTA-wide tracked passes (TRACK 2) stage that row like stage 0's
// rows, in a second ring right after the first (same slot numbering, this
// byte offset): the copy for step j's output row (y0 - 3K + j) travels with
// stage 0's row of step j; so do segmented warps with TRACK 3. (Tile
// warps, TRACK 1, load it when storing:
// their many resident warps hide the latency, and their shared memory
// stays small.)
template <int WPL, bool SEG>
__host__ __device__ constexpr uint32_t old_ring_offset() { return kRowRing * ring_slot_words<WPL, SEG>() * 4u; }

// Copies the row stage 0 consumes at step j (grid row y0 - K + j) to the
// shared address `saddr` (this lane's words of a ring slot), zero-filled
// outside the grid, with TRACK 2 the output row of step j to the old-row
// ring; commits them as one group.
template <int WPL, int K, int TRACK = 0, bool SEG = false>
__device__ __forceinline__ void issue_row_at(const TemporalCtx& c, int j, uint32_t saddr) {
    const int r = c.y0 - K + j;
    const bool v = c.lane_ok && (unsigned)r < (unsigned)c.Y;
    const uint32_t* g = v ? c.src + (size_t)r * c.pitch + c.base : c.src;
    cp_async_words<WPL>(saddr, g, v);
    if (TRACK >= 2) {
        const int ro = r - 2 * K;
        const bool vo = c.lane_ok && (unsigned)ro < (unsigned)c.Y;
        const uint32_t* go = vo ? c.src + (size_t)ro * c.pitch + c.base : c.src;
        cp_async_words<WPL>(saddr + old_ring_offset<WPL, SEG>(), go, vo);
    }
    cp_async_commit();
}

template <int WPL, int K, int TRACK = 0, bool SEG = false>
__device__ __forceinline__ void issue_row(const TemporalCtx& c, int j, int slot) {
    issue_row_at<WPL, K, TRACK, SEG>(c, j, c.ring_saddr + (uint32_t)(slot * c.ring_stride) * 4u);
}

// Reads this lane's words of a ring slot at a shared address.
template <int WPL>
__device__ __forceinline__ void lds_words_at(uint32_t saddr, uint32_t (&v)[WPL]) {
    if constexpr (WPL == 4) {
        asm volatile("ld.shared.v4.u32 {%0, %1, %2, %3}, [%4];"
                     : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]) : "r"(saddr) : "memory");
    } else if constexpr (WPL == 2) {
        asm volatile("ld.shared.v2.u32 {%0, %1}, [%2];" : "=r"(v[0]), "=r"(v[1]) : "r"(saddr) : "memory");
    } else {
        asm volatile("ld.shared.u32 %0, [%1];" : "=r"(v[0]) : "r"(saddr) : "memory");
    }
}

// Tile bits of a lane's words for a per-tile-row tracked pass. A lane's
// words never straddle two change words: they start at a multiple of WPL
// and a change word spans 32 * tt.words words, both powers of two (or
// tt.words = W, one tile column).
template <int WPL>
__device__ __forceinline__ void set_tile_bits(TemporalCtx& c) {
    const int ts = c.tt.words;
#pragma unroll
    for (int w = 0; w < 4; ++w) c.tbit[w] = w < WPL ? 1u << (((c.base + w) / ts) & 31) : 0u;
    c.tfw = c.own ? (c.base / ts) >> 5 : -1;
}

// Closes tile row s.flush_ty of a per-tile-row tracked pass: each lane turns
// its changed-word bits into tile bits of its change word, a segmented OR
// over the runs of lanes sharing a change word (shuffles by doubling: lanes
// are in word order) gathers them, and the first lane of each run sets them
// with one atomic. Every lane of the warp takes part.
template <int WPL, int K>
__device__ __forceinline__ void flush_tile_row(TemporalRegs<WPL, K>& s, const TemporalCtx& c) {
    uint32_t m = 0u;
#pragma unroll
    for (int w = 0; w < WPL; ++w) m |= ((s.diff >> w) & 1u) ? c.tbit[w] : 0u;
    const int fw = c.tfw;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t om = __shfl_down_sync(0xffffffffu, m, o);
        const int ofw = __shfl_down_sync(0xffffffffu, fw, o);
        if (c.lane + o < 32 && ofw == fw) m |= om;
    }
    const int pfw = __shfl_up_sync(0xffffffffu, fw, 1);
    if (fw >= 0 && m != 0u && (c.lane == 0 || pfw != fw))
        atomicOr(c.tt.changed + (size_t)s.flush_ty * c.tt.cw + fw, m);
    s.diff = 0u;
    s.flush_row = min(s.flush_row + c.tt.rows, c.y1 - 1);
    s.flush_ty += 1;
}

// Step body. FAST = steady state: every stage active, every row inside the
// grid, so no activity tests or row masks (the whole step is one basic
// block and the K stages' independent chains interleave). LMASK forces the
// out-of-grid words of a partial CTA (whole lanes, or the tail of the last
// lane of a padded row) to stay dead. SEG = segmented warp: the CTA is
// one warp cut into segments that each span a whole (narrow) grid row for
// their own band; segment ends read zero entries (dead cells), the edge
// table is the warp's own and a step ends with a warp barrier (y0/y1 are
// then per lane, B the common band height). With one word per lane the
// four shared-memory accesses per stage would outweigh the word's own
// work, so those warps shuffle instead (no table, no barrier).
// PART = rows padded to whole lanes: the last lane of a row may hold words
// past W, masked word by word (otherwise a lane is all in or all out).
// TRACK: 0 none; 1 = OR of (new ^ old) over every stored word (s.diff), the
// old word loaded from global memory when storing; 3 = the same with the old
// row staged through the old-row ring (fewer registers in flight);
// 2 = per-tile change bits, closed at each tile row's last row (CTA-wide
// kernels only: every lane of a CTA is on the same row at a step).
template <int WPL, int K, int PH, bool FAST, bool LMASK, int TRACK, bool SEG = false,
          bool PART = false>
__device__ __forceinline__ void temporal_step(TemporalRegs<WPL, K>& s, const TemporalCtx& c, int i) {
    constexpr int ES = SEG ? kSegEdgeStride : kEdgeStride;
    constexpr bool SHFL = SEG && WPL == 1;
    constexpr int NEW3 = PH % 3;          // ring-of-3 slot written at this step
    constexpr int PREV3 = (PH + 2) % 3;   // ... written one step ago
    constexpr int OLD3 = (PH + 1) % 3;    // ... written two steps ago
    constexpr uint32_t SB = ring_slot_words<WPL, SEG>() * 4u;   // bytes per ring slot

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
            uint32_t lw, rw;
            if (SHFL) {
                lw = __shfl_sync(0xffffffffu, P[WPL - 1], c.src_l);
                rw = __shfl_sync(0xffffffffu, P[0], c.src_r);
                lw = c.seg_first ? 0u : lw;
                rw = c.seg_last ? 0u : rw;
            } else {   // published by the neighbour lanes last step
                lw = c.el[edge_last_side<K, ES>() + edge_off<ES>(g - 1, PREV3)];
                rw = c.er[edge_off<ES>(g - 1, PREV3)];
            }
#pragma unroll
            for (int w = 0; w < WPL; ++w) {
                const uint32_t l = (w == 0) ? lw : P[w - 1];
                const uint32_t r = (w == WPL - 1) ? rw : P[w + 1];
                hsum(l, P[w], r, s.h0[g - 1][NEW3][w], s.h1[g - 1][NEW3][w]);
            }
            // Output row r of gen g (garbage during warm-up, never consumed).
            const int row = c.y0 - K + i - 2 * g;
            const bool row_ok = FAST || (unsigned)row < (unsigned)c.Y;
            const uint32_t keep = row_ok ? c.wmask[0] : 0u;   // whole-lane mask
            uint32_t res[WPL];
#pragma unroll
            for (int w = 0; w < WPL; ++w) {
                res[w] = next_word(s.h0[g - 1][OLD3][w], s.h1[g - 1][OLD3][w],
                                   s.h0[g - 1][PREV3][w], s.h1[g - 1][PREV3][w],
                                   s.h0[g - 1][NEW3][w], s.h1[g - 1][NEW3][w], C[w]);
                if (!FAST || LMASK) res[w] &= PART ? (row_ok ? c.wmask[w] : 0u) : keep;
            }
            if (g == K) {
                if ((FAST || (row >= c.y0 && row < c.y1)) && c.own) {
                    store_words<WPL>(c.dst + (size_t)row * c.pitch + c.base, res);
                    if (TRACK) {   // compare with the same row before the pass
                        uint32_t old[WPL];
                        if (TRACK >= 2)   // old-row ring slot i mod 6
                            lds_words_at<WPL>(s.bank_cur + PH * SB + old_ring_offset<WPL, SEG>(), old);
                        else
                            load_words<WPL>(c.src + (size_t)row * c.pitch + c.base, old);
#pragma unroll
                        for (int w = 0; w < WPL; ++w) {
                            if (TRACK != 2)
                                s.diff |= res[w] ^ old[w];
                            else
                                s.diff |= (res[w] != old[w] ? 1u : 0u) << w;
                        }
                    }
                }
            } else {
#pragma unroll
                for (int w = 0; w < WPL; ++w) s.o[g - 1][NEW3][w] = res[w];
                if (!SHFL) {
                    c.eb[1 + edge_off<ES>(g, NEW3)] = res[0];
                    c.eb[1 + edge_last_side<K, ES>() + edge_off<ES>(g, NEW3)] = res[WPL - 1];
                }
            }
        }
    }

    // Stage 0 (every step, so each step commits exactly one copy group):
    // publish this step's row, issue the row kRowsInFlight steps ahead, and
    // read the next step's row out of the ring.
    if (!SHFL) {
        c.eb[1 + edge_off<ES>(0, NEW3)] = s.ld[NEW3][0];
        c.eb[1 + edge_last_side<K, ES>() + edge_off<ES>(0, NEW3)] = s.ld[NEW3][WPL - 1];
    }
    // Step i = 3t + PH reads row i+1 (slot (i+1) mod 6) and issues row i+5
    // (slot (i+5) mod 6, the one read two steps ago): with bank_cur holding
    // slots of steps 3t..3t+2, both are a bank plus a constant.
    const uint32_t rd = PH == 0 ? s.bank_cur + SB : PH == 1 ? s.bank_cur + 2 * SB : s.bank_oth;
    const uint32_t wr = PH == 0 ? s.bank_oth + 2 * SB : PH == 1 ? s.bank_cur : s.bank_cur + SB;
    issue_row_at<WPL, K, TRACK, SEG>(c, i + kRowsInFlight, wr);
    cp_async_wait<kRowsInFlight - 1>();
    lds_words_at<WPL>(rd, s.ld[(PH + 1) % 3]);
    if (PH == 2) {   // steps 3t+3.. use the other bank
        const uint32_t t = s.bank_cur;
        s.bank_cur = s.bank_oth;
        s.bank_oth = t;
    }
    // Tile rows close after the step's stages (a branch there would split
    // the step body, whose stages otherwise interleave as one block).
    if (TRACK == 2 && c.y0 - 3 * K + i == s.flush_row) flush_tile_row<WPL, K>(s, c);
    if (!SEG)
        __syncthreads();
    else if (!SHFL)
        __syncwarp();
}

template <int WPL, int K, bool FAST, bool LMASK, int TRACK, bool SEG = false, bool PART = false>
__device__ __forceinline__ void temporal_steps(TemporalRegs<WPL, K>& s, const TemporalCtx& c,
                                               int i0, int i1) {
    // i0 is a multiple of 3; the bank of steps i0..i0+2 is (i0 / 3) % 2.
    constexpr uint32_t BANK = 3u * ring_slot_words<WPL, SEG>() * 4u;
    const bool odd = (i0 / 3) & 1;
    s.bank_cur = c.ring_saddr + (odd ? BANK : 0u);
    s.bank_oth = c.ring_saddr + (odd ? 0u : BANK);
    for (int i = i0; i < i1; i += 3) {
        temporal_step<WPL, K, 0, FAST, LMASK, TRACK, SEG, PART>(s, c, i + 0);
        temporal_step<WPL, K, 1, FAST, LMASK, TRACK, SEG, PART>(s, c, i + 1);
        temporal_step<WPL, K, 2, FAST, LMASK, TRACK, SEG, PART>(s, c, i + 2);
    }
}

// One tile of one pass: output rows [band*a.band, +a.band) of x-slice
// `slice_idx`, K generations from a.src into a.dst. The CTA's shared memory
// (temporal_smem_bytes) is reused from call to call: every copy is drained
// before returning. With TRACK 1, returns this thread's OR of (new ^ old)
// over the words it stored (0 when its part of the tile did not change);
// with TRACK 2, sets the change bits `tt` of the tiles it changed.
template <int WPL, int K, int TRACK>
__device__ __forceinline__ uint32_t band_tile(const RowsLaunch& a, int band, int slice_idx,
                                              uint32_t* smem, TileTrack tt = {}) {
    uint32_t* ring = smem;                    // kRowRing slots of ring_slot_words words
    // (with TRACK 2, the old-row ring of the same size follows)
    uint32_t* edges = smem + kRowRing * ring_slot_words<WPL, false>() * (TRACK == 2 ? 2 : 1);
    TemporalCtx c;
    c.src = a.src;
    c.dst = a.dst;
    c.W = a.W;
    c.pitch = a.pitch;
    c.Y = a.Y;
    c.y0 = band * a.band;
    c.y1 = min(c.y0 + a.band, a.Y);
    c.B = c.y1 - c.y0;
    c.lane = threadIdx.x & 31;
    c.eb = edges + threadIdx.x;
    c.el = c.eb;
    c.er = c.eb + 2;
    const int xs = slice_idx * a.slice;
    const int x0 = xs - a.halo;
    c.base = x0 + (int)threadIdx.x * WPL;
    c.lane_ok = c.base >= 0 && c.base < a.W;
    c.own = c.lane_ok && c.base >= xs && c.base < xs + a.slice;
    const bool all_lanes_ok = x0 >= 0 && x0 + (int)blockDim.x * WPL <= a.W;
    set_word_masks<WPL>(c);
    c.tt = tt;
    if (TRACK == 2) set_tile_bits<WPL>(c);

    for (int t = threadIdx.x; t < 2 * edge_last_side<K, kEdgeStride>(); t += blockDim.x) edges[t] = 0u;

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
    c.ring = ring + threadIdx.x * WPL;
    c.ring_saddr = (uint32_t)__cvta_generic_to_shared(c.ring);
    c.ring_stride = ring_slot_words<WPL, false>();
    for (int j = 0; j < kRowsInFlight; ++j) issue_row<WPL, K, TRACK>(c, j, j);
    cp_async_wait<kRowsInFlight - 1>();
    lds_words<WPL>(c.ring, s.ld[0]);
    s.diff = 0u;
    if (TRACK == 2) {
        s.flush_ty = c.y0 / tt.rows;
        s.flush_row = min((s.flush_ty + 1) * tt.rows - 1, c.y1 - 1);
    }
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
        temporal_steps<WPL, K, false, false, TRACK>(s, c, 0, f0);
        if (all_lanes_ok)
            temporal_steps<WPL, K, true, false, TRACK>(s, c, f0, fast_end);
        else
            temporal_steps<WPL, K, true, true, TRACK>(s, c, f0, fast_end);
        temporal_steps<WPL, K, false, false, TRACK>(s, c, fast_end, nsteps);
    } else {
        temporal_steps<WPL, K, false, false, TRACK>(s, c, 0, nsteps);
    }
    asm volatile("cp.async.wait_all;\n" ::: "memory");   // no copy outlives the tile
    return s.diff;
}

// Programmatic dependent launch: let the next pass's CTAs be scheduled
// now (they wait below for this grid to finish), then wait for the
// previous pass to complete before the first global access. Both are
// no-ops for an ordinary launch.
__device__ __forceinline__ void pdl_trigger_and_wait() {
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    asm volatile("griddepcontrol.wait;" ::: "memory");
}

template <int WPL, int K>
__global__ void __launch_bounds__(kTemporalMaxThreads, GOL_TEMPORAL_MIN_BLOCKS)
rows_temporal_kernel(RowsLaunch a) {
    extern __shared__ __align__(16) uint32_t smem[];
    pdl_trigger_and_wait();
    band_tile<WPL, K, 0>(a, blockIdx.x, blockIdx.y, smem);
}

// Shared memory a launch needs: the row ring (two with change tracking:
// rows and old rows) and the edge table.
__host__ __device__ inline size_t temporal_smem_bytes(int K, int threads, int wpl, bool track = false) {
    (void)threads;   // the ring is sized for the widest CTA (compile-time slot offsets)
    return ((size_t)kRowRing * kTemporalMaxThreads * wpl * (track ? 2 : 1) +
            (size_t)2 * edge_last_side<1, kEdgeStride>() * K) *
           sizeof(uint32_t);
}

} // namespace golb200
