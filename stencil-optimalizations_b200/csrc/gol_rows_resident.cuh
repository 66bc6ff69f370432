// Shared-memory-resident run: every generation of a grid that fits in the
// GPU's shared memory, in one cooperative launch.
//
// A grid whose rows fit in the SMs' shared memory (8192^2 bits is 8 MiB;
// 148 SMs hold up to 33 MiB) need not go through HBM or L2 between passes:
// CTA c keeps rows [y0, y1) of the grid (its band) in two shared-memory
// buffers and advances them K generations per epoch. An epoch needs K rows
// above and K below the band (cells within K of the band's edge depend on
// them): at the start of every epoch each CTA publishes its top and bottom K
// rows to global memory, releases an epoch counter, waits for its two
// neighbours' counters (bounded polls: GOL_E_TIMEOUT in *status and the CTA
// stops), and copies their rows into its halo. Generation g of the epoch
// computes the rows still covered by valid neighbours (the band plus K - g
// rows each side), rows outside the grid stay dead. The publication slots
// alternate by epoch parity: a CTA rewrites a slot only after both
// neighbours have published the next epoch, i.e. after they read it.
//
// Within a generation a thread owns WPL words of a column and walks a range
// of rows (the CTA's threads are lanes across the row times row groups),
// keeping the horizontal sums of three rows in registers like the streaming
// kernel; words beyond its lane come from its warp neighbours by shuffle or
// from shared memory at the warp's edges. One barrier per generation.
//
// All CTAs must be resident at once (they wait on each other): the launch
// is cooperative, one CTA per SM at most.
#pragma once

#include <cstdint>

#include "gol_rows_temporal.cuh"
#include "gol_word_ops.cuh"

namespace golb200 {

constexpr int kResidentMaxThreads = 512;

struct ResidentLaunch {
    const uint32_t* src;   // the grid at generation 0 (W words per row, Y rows)
    uint32_t* dst;         // the grid after `gens` generations (may alias src)
    uint32_t* pub;         // [nbands][2 parities][2 sides][K rows][W words]
    int* epoch_done;       // [nbands], zero at launch: epochs published
    int* status;           // GOL_E_TIMEOUT if a wait gave up
    int W, Y;
    int band;              // rows of the largest band (bands split Y evenly, each >= K)
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

// Shared memory of one CTA: two buffers of (band + 2K) rows of the row's
// lanes * WPL words.
__host__ __device__ inline size_t resident_smem_bytes(int band, int K, int lanes, int wpl) {
    return 2ull * (size_t)(band + 2 * K) * (size_t)lanes * wpl * sizeof(uint32_t);
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

// Horizontal sums of shared-memory row `row` (this lane's WPL words): the
// words just outside the lane come from its warp neighbours, or from shared
// memory at the warp's ends; outside the grid they are zero.
template <int WPL>
__device__ __forceinline__ void resident_hsum(const uint32_t* buf, int row, int pitch, int lane,
                                              int col, int W, uint32_t (&c)[WPL],
                                              uint32_t (&h0)[WPL], uint32_t (&h1)[WPL]) {
    const uint32_t* r = buf + (size_t)row * pitch;
    lds_words_gen<WPL>(r + col, c);
    uint32_t lw = __shfl_up_sync(0xffffffffu, c[WPL - 1], 1);
    uint32_t rw = __shfl_down_sync(0xffffffffu, c[0], 1);
    if (lane == 0) lw = col > 0 ? r[col - 1] : 0u;
    if (lane == 31) rw = col + WPL < pitch ? r[col + WPL] : 0u;
    (void)W;
#pragma unroll
    for (int w = 0; w < WPL; ++w) {
        const uint32_t l = w == 0 ? lw : c[w - 1];
        const uint32_t rr = w == WPL - 1 ? rw : c[w + 1];
        hsum(l, c[w], rr, h0[w], h1[w]);
    }
}

// One output row of a generation: rows of the ring slots M (above), C
// (the row itself) and P (below, just loaded).
template <int WPL, int M, int C, int P>
__device__ __forceinline__ void resident_row(uint32_t (&h0)[3][WPL], uint32_t (&h1)[3][WPL],
                                             uint32_t (&cw)[3][WPL], uint32_t* D, int r, int pitch,
                                             int col, int W, bool in) {
    uint32_t res[WPL];
#pragma unroll
    for (int w = 0; w < WPL; ++w) {
        const uint32_t v = next_word(h0[M][w], h1[M][w], h0[C][w], h1[C][w], h0[P][w], h1[P][w],
                                     cw[C][w]);
        res[w] = (in && col + w < W) ? v : 0u;
    }
    sts_words_gen<WPL>(D + (size_t)r * pitch + col, res);
}

// Rows [r0, r1) of one generation, S -> D: the three-row ring of sums in
// registers, slots named at compile time (the loop is unrolled by three).
template <int WPL>
__device__ __forceinline__ void resident_rows(const uint32_t* S, uint32_t* D, int r0, int r1,
                                              int pitch, int lane, int col, int W, int Y, int gy0) {
    uint32_t h0[3][WPL], h1[3][WPL], cw[3][WPL];
    resident_hsum<WPL>(S, r0 - 1, pitch, lane, col, W, cw[0], h0[0], h1[0]);
    resident_hsum<WPL>(S, r0, pitch, lane, col, W, cw[1], h0[1], h1[1]);
    for (int r = r0; r < r1; r += 3) {
        resident_hsum<WPL>(S, r + 1, pitch, lane, col, W, cw[2], h0[2], h1[2]);
        resident_row<WPL, 0, 1, 2>(h0, h1, cw, D, r, pitch, col, W, (unsigned)(gy0 + r) < (unsigned)Y);
        if (r + 1 >= r1) break;
        resident_hsum<WPL>(S, r + 2, pitch, lane, col, W, cw[0], h0[0], h1[0]);
        resident_row<WPL, 1, 2, 0>(h0, h1, cw, D, r + 1, pitch, col, W,
                                   (unsigned)(gy0 + r + 1) < (unsigned)Y);
        if (r + 2 >= r1) break;
        resident_hsum<WPL>(S, r + 3, pitch, lane, col, W, cw[1], h0[1], h1[1]);
        resident_row<WPL, 2, 0, 1>(h0, h1, cw, D, r + 2, pitch, col, W,
                                   (unsigned)(gy0 + r + 2) < (unsigned)Y);
    }
}

template <int WPL>
__global__ void __launch_bounds__(kResidentMaxThreads, 1) rows_resident_kernel(ResidentLaunch a) {
    extern __shared__ __align__(16) uint32_t smem[];
    __shared__ int stop;
    const int K = a.K;
    const int pitch = a.lanes * WPL;            // words per shared-memory row (zero past W)
    const int rows = a.band + 2 * K;            // shared-memory rows: K halo each side
    uint32_t* const buf0 = smem;
    uint32_t* const buf1 = smem + (size_t)rows * pitch;
    const int lane_in_row = threadIdx.x % a.lanes;
    const int group = threadIdx.x / a.lanes;
    const int lane = threadIdx.x & 31;
    const int col = lane_in_row * WPL;
    const int cta = blockIdx.x;
    const int nbands = gridDim.x;
    // Bands split the rows evenly (sizes differ by at most one row, and the
    // planner makes every band at least K rows).
    const int y0 = (int)((long long)cta * a.Y / nbands);
    const int B = (int)((long long)(cta + 1) * a.Y / nbands) - y0;
    const size_t side_words = (size_t)K * a.W;

    // Band rows into buffer 0 (shared row K + i = grid row y0 + i); halos and
    // columns past W zero.
    for (int i = threadIdx.x; i < rows * pitch; i += blockDim.x) {
        const int r = i / pitch, c = i - r * pitch;
        buf0[i] = (r >= K && r < K + B && c < a.W) ? a.src[(size_t)(y0 - K + r) * a.W + c] : 0u;
        buf1[i] = 0u;
    }
    if (threadIdx.x == 0) stop = 0;
    __syncthreads();

    int cur = 0;
    long long left = a.gens;
    for (int e = 0; left > 0; ++e) {
        const int kk = (int)min((long long)K, left);
        uint32_t* A = cur ? buf1 : buf0;
        // Publish the band's top and bottom K rows (the state at epoch start).
        uint32_t* mine = a.pub + ((size_t)cta * 4 + (e & 1) * 2) * side_words;
        for (int i = threadIdx.x; i < K * a.W; i += blockDim.x) {
            const int r = i / a.W, c = i - r * a.W;
            mine[i] = A[(size_t)(K + r) * pitch + c];                       // top
            mine[side_words + i] = A[(size_t)(K + B - K + r) * pitch + c];   // bottom
        }
        __threadfence();
        __syncthreads();
        if (threadIdx.x == 0) st_release_gpu(a.epoch_done + cta, e + 1);
        // Wait for the neighbours' publications of this epoch (bounded).
        if (threadIdx.x < 2) {
            const int nb = threadIdx.x == 0 ? cta - 1 : cta + 1;
            if (nb >= 0 && nb < nbands) {
                long long spins = 0;
                while (ld_acquire_gpu(a.epoch_done + nb) < e + 1) {
                    if (++spins > a.spin_limit || *(volatile int*)a.status != 0) {
                        atomicCAS(a.status, 0, GOL_E_TIMEOUT);
                        atomicExch(&stop, 1);
                        break;
                    }
                    __nanosleep(128);
                }
            }
        }
        __syncthreads();
        if (stop) return;   // the same for every thread of the CTA
        // Every thread acquires the counters whose data it reads next.
        if (cta > 0) (void)ld_acquire_gpu(a.epoch_done + cta - 1);
        if (cta + 1 < nbands) (void)ld_acquire_gpu(a.epoch_done + cta + 1);
        // Halo rows: the upper neighbour's bottom rows, the lower one's top
        // rows (zero beyond the grid).
        for (int i = threadIdx.x; i < K * a.W; i += blockDim.x) {
            const int r = i / a.W, c = i - r * a.W;
            uint32_t up = 0u, dn = 0u;
            if (cta > 0) up = a.pub[((size_t)(cta - 1) * 4 + (e & 1) * 2 + 1) * side_words + i];
            if (cta + 1 < nbands) dn = a.pub[((size_t)(cta + 1) * 4 + (e & 1) * 2) * side_words + i];
            A[(size_t)r * pitch + c] = up;
            A[(size_t)(K + B + r) * pitch + c] = dn;
        }
        __syncthreads();
        // kk generations in shared memory: generation g computes the shared
        // rows [K - kk + g, K + B + kk - g) (what the halo still determines).
        for (int g = 1; g <= kk; ++g) {
            const int lo = K - kk + g, hi = K + B + kk - g;
            const int per = (hi - lo + a.groups - 1) / a.groups;
            const int r0 = lo + group * per, r1 = min(hi, r0 + per);
            if (r0 < r1)   // the same for every lane of a warp (a warp is in one group)
                resident_rows<WPL>(cur ? buf1 : buf0, cur ? buf0 : buf1, r0, r1, pitch, lane, col, a.W,
                                   a.Y, y0 - K);
            __syncthreads();
            cur ^= 1;
        }
        left -= kk;
    }
    // The band after the last generation.
    const uint32_t* A = cur ? buf1 : buf0;
    for (int i = threadIdx.x; i < B * a.W; i += blockDim.x) {
        const int r = i / a.W, c = i - r * a.W;
        a.dst[(size_t)(y0 + r) * a.W + c] = A[(size_t)(K + r) * pitch + c];
    }
}

} // namespace golb200
