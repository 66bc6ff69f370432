// Shared-memory-resident run: every generation of a grid that fits in the
// GPU's shared memory, in one cooperative launch.
//
// A grid whose rows fit in the SMs' shared memory (8192^2 bits is 8 MiB;
// 148 SMs hold up to 33 MiB) need not go through HBM or L2 between passes:
// CTA c keeps rows [y0, y1) of the grid (its band) in two shared-memory
// buffers and advances them K generations per epoch. An epoch needs K rows
// above and K below the band (cells within K of the band's edge depend on
// them), which the neighbouring CTAs publish through global memory.
//
// The exchange is overlapped with the band's interior. The first ni
// generations of an epoch (ni = kResidentInterior, at most K) are first
// computed on the rows at least g away from the band's edges (they depend on
// the band only) while the neighbours' rows arrive. Then the CTA waits for
// them (bounded polls: GOL_E_TIMEOUT in *status and the CTA stops), copies
// them into its halo and completes generations g = 1..ni near the two edges:
// rows [K - kk + g, K + g) and the mirror rows at the bottom. Those read
// generation g - 1 rows that the interior pass of generation g + 1 (same
// buffer) left alone, since the interior shrinks by one row per side per
// generation. Generations ni+1..K are then computed whole (the band and the
// K - g halo rows each side that the halo still determines). Rows outside
// the grid are never computed and stay dead (zero).
//
// Epoch e publishes the band's top and bottom K rows into slot e & 1 and
// releases an epoch counter; a CTA rewrites a slot two epochs later, after
// both neighbours have published the epoch in between, i.e. after they read
// it.
//
// Within a pass a thread owns WPL words of a column (the CTA's threads are
// lanes across the row times row groups) and walks a range of rows with
// the horizontal sums of three rows in registers. Shared-memory rows carry
// four zero words of padding each side, so the words just outside a lane's
// span are plain loads from the row (cheaper on the integer pipe, the
// bound here, than shuffles and selects). Columns at or past W exist only
// in the last lanes of a row, which alone run the masked variant.
//
// The band algorithm (resident_band) serves two kernels: one grid, CTA c
// running band c (rows_resident_kernel), and many grids, persistent CTAs
// taking bands of a batch in ticket order (batch_resident_kernel). All
// CTAs of a launch must be resident at once (they wait on each other): the
// launches are cooperative.
#pragma once

#include <cstdint>

#include "gol_internal.h"
#include "gol_rows_temporal.cuh"
#include "gol_word_ops.cuh"

namespace golb200 {

#ifndef GOL_RESIDENT_MAX_THREADS
#define GOL_RESIDENT_MAX_THREADS 512
#endif
constexpr int kResidentMaxThreads = GOL_RESIDENT_MAX_THREADS;
constexpr int kResidentPad = 4;   // zero words each side of a shared-memory row
#ifndef GOL_RESIDENT_INTERIOR
#define GOL_RESIDENT_INTERIOR 1
#endif
// Generations of an epoch computed on the interior alone, before the wait
// for the neighbours' rows.
constexpr int kResidentInterior = GOL_RESIDENT_INTERIOR;

struct ResidentLaunch {   // one grid (rows_resident_kernel)
    const uint32_t* src;   // the grid at generation 0 (W words per row, Y rows)
    uint32_t* dst;         // the grid after `gens` generations (not src)
    uint32_t* pub;         // [nbands][2 parities][2 sides][K rows][W words]
    int* epoch_done;       // [nbands], zero at launch: epochs published
    int* status;           // GOL_E_TIMEOUT if a wait gave up
    int W, Y;
    int K;                 // generations per epoch
    int lanes;             // lanes across a row (ceil(W / WPL), a multiple of 32)
    int groups;            // row groups (blockDim.x = lanes * groups)
    long long gens;
    long long spin_limit;
};

__device__ __forceinline__ int ld_acquire_gpu(const int* p) {
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release_gpu(int* p, int v) {
    asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Words per shared-memory row: the lanes' words plus the padding.
__host__ __device__ inline int resident_stride(int lanes, int wpl) {
    return lanes * wpl + 2 * kResidentPad;
}

// Shared memory of one CTA: two buffers of (band + 2K) rows.
__host__ __device__ inline size_t resident_smem_bytes(int band, int K, int lanes, int wpl) {
    return 2ull * (size_t)(band + 2 * K) * (size_t)resident_stride(lanes, wpl) * sizeof(uint32_t);
}

template <int WPL>
__device__ __forceinline__ void lds_words_gen(const uint32_t* p, uint32_t (&v)[WPL]) {
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

template <int WPL>
__device__ __forceinline__ void sts_words_gen(uint32_t* p, const uint32_t (&v)[WPL]) {
    if constexpr (WPL == 4) {
        *reinterpret_cast<uint4*>(p) = make_uint4(v[0], v[1], v[2], v[3]);
    } else if constexpr (WPL == 2) {
        *reinterpret_cast<uint2*>(p) = make_uint2(v[0], v[1]);
    } else {
        *p = v[0];
    }
}

// A lane's WPL words from global memory through L2 only (the exchange
// slots, which other CTAs rewrite).
template <int WPL>
__device__ __forceinline__ void ldcg_words(const uint32_t* p, uint32_t (&v)[WPL]) {
    if constexpr (WPL == 4) {
        const uint4 t = __ldcg(reinterpret_cast<const uint4*>(p));
        v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
    } else if constexpr (WPL == 2) {
        const uint2 t = __ldcg(reinterpret_cast<const uint2*>(p));
        v[0] = t.x; v[1] = t.y;
    } else {
        v[0] = __ldcg(p);
    }
}

// Horizontal sums of the shared-memory row at p (this lane's words). The
// words just outside the lane's span are plain loads from the row (its
// neighbours' words, or the zero padding at the row's ends): no shuffles,
// selects or divergent loads.
template <int WPL>
__device__ __forceinline__ void resident_hsum(const uint32_t* p, uint32_t (&c)[WPL],
                                              uint32_t (&h0)[WPL], uint32_t (&h1)[WPL]) {
    lds_words_gen<WPL>(p, c);
    const uint32_t lw = p[-1];
    const uint32_t rw = p[WPL];
#pragma unroll
    for (int w = 0; w < WPL; ++w) {
        const uint32_t l = w == 0 ? lw : c[w - 1];
        const uint32_t r = w == WPL - 1 ? rw : c[w + 1];
        hsum(l, c[w], r, h0[w], h1[w]);
    }
}

// One output row from the ring slots M (above), C (the row) and P (below).
template <int WPL, bool RAG, int M, int C, int P>
__device__ __forceinline__ void resident_row(const uint32_t (&h0)[3][WPL],
                                             const uint32_t (&h1)[3][WPL],
                                             const uint32_t (&cw)[3][WPL], uint32_t* d,
                                             const uint32_t (&cm)[WPL]) {
    uint32_t res[WPL];
#pragma unroll
    for (int w = 0; w < WPL; ++w) {
        res[w] = next_word(h0[M][w], h1[M][w], h0[C][w], h1[C][w], h0[P][w], h1[P][w], cw[C][w]);
        if constexpr (RAG) res[w] &= cm[w];
    }
    sts_words_gen<WPL>(d, res);
}

// Rows [r0, r1) of one generation, S -> D (S and D point at this lane's
// first word of row 0). The loop body covers three rows so the ring slots
// are compile-time register names; it has no early exits, so the loads of
// its three rows can be issued together.
template <int WPL, bool RAG>
__device__ __forceinline__ void resident_rows(const uint32_t* S, uint32_t* D, int r0, int r1,
                                              int stride, const uint32_t (&cm)[WPL]) {
    if (r0 >= r1) return;
    uint32_t h0[3][WPL], h1[3][WPL], cw[3][WPL];
    const uint32_t* s = S + (size_t)(r0 - 1) * stride;
    uint32_t* d = D + (size_t)r0 * stride;
    resident_hsum<WPL>(s, cw[0], h0[0], h1[0]);
    s += stride;
    resident_hsum<WPL>(s, cw[1], h0[1], h1[1]);
    s += stride;
    int n = r1 - r0;
    for (; n >= 3; n -= 3) {   // slot 0: row r - 1, slot 1: row r
        resident_hsum<WPL>(s, cw[2], h0[2], h1[2]);
        resident_row<WPL, RAG, 0, 1, 2>(h0, h1, cw, d, cm);
        resident_hsum<WPL>(s + stride, cw[0], h0[0], h1[0]);
        resident_row<WPL, RAG, 1, 2, 0>(h0, h1, cw, d + stride, cm);
        resident_hsum<WPL>(s + 2 * stride, cw[1], h0[1], h1[1]);
        resident_row<WPL, RAG, 2, 0, 1>(h0, h1, cw, d + 2 * stride, cm);
        s += 3 * stride;
        d += 3 * stride;
    }
    if (n >= 1) {
        resident_hsum<WPL>(s, cw[2], h0[2], h1[2]);
        resident_row<WPL, RAG, 0, 1, 2>(h0, h1, cw, d, cm);
    }
    if (n == 2) {
        resident_hsum<WPL>(s + stride, cw[0], h0[0], h1[0]);
        resident_row<WPL, RAG, 1, 2, 0>(h0, h1, cw, d + stride, cm);
    }
}

// Rows [lo, hi) split over groups [g0, g0 + ng) (this thread's group is g).
template <int WPL, bool RAG>
__device__ __forceinline__ void resident_range(const uint32_t* S, uint32_t* D, int lo, int hi,
                                               int g, int g0, int ng, int stride,
                                               const uint32_t (&cm)[WPL]) {
    if (g < g0 || g >= g0 + ng || hi <= lo) return;
    const int per = (hi - lo + ng - 1) / ng;
    const int r0 = lo + (g - g0) * per;
    resident_rows<WPL, RAG>(S, D, r0, min(hi, r0 + per), stride, cm);
}

template <int WPL>
__device__ __forceinline__ void resident_pass(const uint32_t* S, uint32_t* D, int lo, int hi,
                                              int g, int g0, int ng, int stride,
                                              const uint32_t (&cm)[WPL], bool rag) {
    if (rag)   // the same for every lane of a warp
        resident_range<WPL, true>(S, D, lo, hi, g, g0, ng, stride, cm);
    else
        resident_range<WPL, false>(S, D, lo, hi, g, g0, ng, stride, cm);
}

// Global <-> register copies of a lane's words: vector accesses where the
// lane's words are whole and aligned, else word by word up to W.
template <int WPL>
__device__ __forceinline__ void band_load(const uint32_t* p, bool vec, int n, uint32_t (&v)[WPL]) {
    if (vec) {
        load_words<WPL>(p, v);
    } else {
#pragma unroll
        for (int w = 0; w < WPL; ++w) v[w] = w < n ? __ldg(p + w) : 0u;
    }
}

template <int WPL>
__device__ __forceinline__ void band_store(uint32_t* p, bool vec, int n, const uint32_t (&v)[WPL]) {
    if (vec) {
        store_words<WPL>(p, v);
    } else {
#pragma unroll
        for (int w = 0; w < WPL; ++w)
            if (w < n) p[w] = v[w];
    }
}

// Runs band j.b of its grid: returns false if a wait gave up (GOL_E_TIMEOUT
// in *status; the caller ends the CTA). Every thread of the CTA calls it;
// smem holds 2 * (B + 2K) rows of the stride. LANES: the lanes across a row
// when known at compile time (0: j.lanes), so the shared-memory row stride
// is a constant and row addresses are immediate offsets.
template <int WPL, int LANES>
__device__ __forceinline__ bool resident_band(const ResidentBand& j, uint32_t* smem, int* stop,
                                              int* status, long long spin_limit) {
    const int K = j.K;
    const int stride = LANES ? resident_stride(LANES, WPL) : resident_stride(j.lanes, WPL);
    const int lane_in_row = threadIdx.x % j.lanes;
    const int group = threadIdx.x / j.lanes;   // >= j.groups: idle in the passes
    const int col = lane_in_row * WPL;
    const int W = j.W;
    // Warps whose span reaches column W mask their results past it (when
    // lanes is a multiple of 32 a warp lies within one row).
    const bool rag = (j.lanes & 31) ? col + WPL > W : (lane_in_row | 31) * WPL + WPL > W;
    uint32_t cm[WPL];
#pragma unroll
    for (int w = 0; w < WPL; ++w) cm[w] = col + w < W ? 0xffffffffu : 0u;
    const bool top = j.b == 0, bottom = j.b == j.nb - 1;
    // Bands split the rows evenly (sizes differ by at most one row; with
    // several bands every band is at least K rows).
    const int y0 = (int)((long long)j.b * j.Y / j.nb);
    const int B = (int)((long long)(j.b + 1) * j.Y / j.nb) - y0;
    const int rows = B + 2 * K;                 // shared-memory rows: K halo each side
    const size_t side_words = (size_t)K * j.ppitch;
    const int ng_top = j.groups > 1 ? j.groups / 2 : 1;
    const int g_bot = j.groups > 1 ? ng_top : 0;
    const int ng_bot = j.groups > 1 ? j.groups - ng_top : 1;
    const bool mine_lane = col < W && group < j.groups;   // moves words between global and shared
    const int nw = W - col;                             // words of this lane inside the row
    const bool gvec = col + WPL <= W && (j.pitch % WPL) == 0;

    // Buffers zero (halo rows, padding, columns past W), then the band rows
    // into buffer 0 (shared row K + i = grid row y0 + i). Copies between
    // global and shared rows go by row group and lane: each thread moves its
    // lane's WPL words of every groups-th row.
    for (int i = threadIdx.x; i < 2 * rows * stride; i += blockDim.x) smem[i] = 0u;
    __syncthreads();
    uint32_t* const lane0w = smem + kResidentPad + col;   // this lane's words of shared row 0
    if (mine_lane) {
        for (int r = group; r < B; r += j.groups) {
            uint32_t v[WPL];
            band_load<WPL>(j.src + (size_t)(y0 + r) * j.pitch + col, gvec, nw, v);
            sts_words_gen<WPL>(lane0w + (size_t)(K + r) * stride, v);
        }
    }
    if (threadIdx.x == 0) *stop = 0;
    __syncthreads();

    const uint32_t* const lane0 = lane0w;
    int cur = 0;
    long long left = j.gens;
    for (int e = 0; left > 0; ++e) {
        const int kk = (int)min((long long)K, left);
        // Publish the band's top and bottom K rows (the state at epoch start).
        uint32_t* mine = j.pub + ((size_t)j.b * 4 + (e & 1) * 2) * side_words + col;
        const uint32_t* Aw = lane0w + (cur ? (size_t)rows * stride : 0);
        if (mine_lane) {
            for (int r = group; r < K; r += j.groups) {
                uint32_t v[WPL];
                if (!top) {
                    lds_words_gen<WPL>(Aw + (size_t)(K + r) * stride, v);
                    store_words<WPL>(mine + (size_t)r * j.ppitch, v);
                }
                if (!bottom) {
                    lds_words_gen<WPL>(Aw + (size_t)(B + r) * stride, v);
                    store_words<WPL>(mine + side_words + (size_t)r * j.ppitch, v);
                }
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) st_release_gpu(j.done + j.b, e + 1);
        // The interior: generation g's rows at least g from the band's edges,
        // for the first ni generations (enough to cover the exchange).
        const int ni = min(kk, kResidentInterior);
        for (int g = 1; g <= ni; ++g) {
            const int sb = (cur + g - 1) & 1;
            const uint32_t* S = lane0 + (sb ? (size_t)rows * stride : 0);
            uint32_t* D = const_cast<uint32_t*>(lane0) + (sb ? 0 : (size_t)rows * stride);
            resident_pass<WPL>(S, D, K + g, K + B - g, group, 0, j.groups, stride, cm, rag);
            __syncthreads();
        }
        // Wait for the neighbours' rows of this epoch (bounded).
        if (threadIdx.x < 2) {
            const int nb = threadIdx.x == 0 ? j.b - 1 : j.b + 1;
            if (nb >= 0 && nb < j.nb) {
                long long spins = 0;
                while (ld_acquire_gpu(j.done + nb) < e + 1) {
                    if (++spins > spin_limit || *(volatile int*)status != 0) {
                        atomicCAS(status, 0, GOL_E_TIMEOUT);
                        atomicExch(stop, 1);
                        break;
                    }
                    __nanosleep(64);
                }
            }
        }
        __syncthreads();
        if (*(volatile int*)stop) return false;   // the same for every thread of the CTA
        // Halo rows: the upper neighbour's bottom rows, the lower one's top
        // rows, loaded from L2 (a slot is rewritten every other epoch, so no
        // copy of it may linger in L1). At the grid's edges they stay zero
        // (never written).
        if (mine_lane) {
            const uint32_t* up = j.pub + ((size_t)(j.b - 1) * 4 + (e & 1) * 2 + 1) * side_words + col;
            const uint32_t* dn = j.pub + ((size_t)(j.b + 1) * 4 + (e & 1) * 2) * side_words + col;
            uint32_t* Aw2 = lane0w + (cur ? (size_t)rows * stride : 0);
            for (int r = group; r < K; r += j.groups) {
                uint32_t v[WPL];
                if (!top) {
                    ldcg_words<WPL>(up + (size_t)r * j.ppitch, v);
                    sts_words_gen<WPL>(Aw2 + (size_t)r * stride, v);
                }
                if (!bottom) {
                    ldcg_words<WPL>(dn + (size_t)r * j.ppitch, v);
                    sts_words_gen<WPL>(Aw2 + (size_t)(K + B + r) * stride, v);
                }
            }
        }
        __syncthreads();
        // Generations 1..ni near the edges: rows within g of the band's
        // edges, and the halo rows the later generations still need.
        for (int g = 1; g <= ni; ++g) {
            const int sb = (cur + g - 1) & 1;
            const uint32_t* S = lane0 + (sb ? (size_t)rows * stride : 0);
            uint32_t* D = const_cast<uint32_t*>(lane0) + (sb ? 0 : (size_t)rows * stride);
            const int bhi = bottom ? K + B : K + B + kk - g;
            const int tlo = top ? K : K - kk + g, thi = min(K + g, bhi);   // (a band under g rows)
            const int blo = max(K + g, K + B - g);
            resident_pass<WPL>(S, D, tlo, thi, group, 0, ng_top, stride, cm, rag);
            resident_pass<WPL>(S, D, blo, bhi, group, g_bot, ng_bot, stride, cm, rag);
            __syncthreads();
        }
        // Generations ni+1..kk whole: the band and what the halo still
        // determines.
        for (int g = ni + 1; g <= kk; ++g) {
            const int sb = (cur + g - 1) & 1;
            const uint32_t* S = lane0 + (sb ? (size_t)rows * stride : 0);
            uint32_t* D = const_cast<uint32_t*>(lane0) + (sb ? 0 : (size_t)rows * stride);
            const int lo = top ? K : K - kk + g, hi = bottom ? K + B : K + B + kk - g;
            resident_pass<WPL>(S, D, lo, hi, group, 0, j.groups, stride, cm, rag);
            __syncthreads();
        }
        cur = (cur + kk) & 1;
        left -= kk;
    }
    // The band after the last generation.
    if (mine_lane) {
        const uint32_t* Aw = lane0w + (cur ? (size_t)rows * stride : 0);
        for (int r = group; r < B; r += j.groups) {
            uint32_t v[WPL];
            lds_words_gen<WPL>(Aw + (size_t)(K + r) * stride, v);
            band_store<WPL>(j.dst + (size_t)(y0 + r) * j.pitch + col, gvec, nw, v);
        }
    }
    return true;
}

// One grid: CTA c runs band c.
template <int WPL, int LANES>
__global__ void __launch_bounds__(kResidentMaxThreads, 1) rows_resident_kernel(ResidentLaunch a) {
    extern __shared__ __align__(16) uint32_t smem[];
    __shared__ int stop;
    ResidentBand j;
    j.src = a.src;
    j.dst = a.dst;
    j.pub = a.pub;
    j.done = a.epoch_done;
    j.pitch = a.W;
    j.ppitch = a.W;
    j.W = a.W;
    j.Y = a.Y;
    j.K = a.K;
    j.lanes = a.lanes;
    j.groups = a.groups;
    j.b = blockIdx.x;
    j.nb = gridDim.x;
    j.gens = a.gens;
    resident_band<WPL, LANES>(j, smem, &stop, a.status, a.spin_limit);
}

// Many grids: persistent CTAs (all resident: a cooperative launch) take
// bands in ticket order and run each to its last generation. The bands of a
// grid have consecutive tickets, so a band's neighbours are always taken by
// CTAs that are running or will be as soon as one frees up: a grid has at
// most as many bands as there are CTAs, and bands of earlier grids never
// wait on later tickets.
template <int WPL>
__global__ void __launch_bounds__(kResidentMaxThreads, 1)
batch_resident_kernel(const ResidentBand* __restrict__ jobs, int njobs, int* ticket, int* status,
                      long long spin_limit) {
    extern __shared__ __align__(16) uint32_t smem[];
    __shared__ int stop;
    __shared__ int job;
    for (;;) {
        if (threadIdx.x == 0) job = atomicAdd(ticket, 1);
        __syncthreads();
        const int t = job;
        if (t >= njobs) return;
        const ResidentBand j = jobs[t];
        if (!resident_band<WPL, 0>(j, smem, &stop, status, spin_limit)) return;
        __syncthreads();   // shared memory and `job` are reused by the next band
    }
}

} // namespace golb200
