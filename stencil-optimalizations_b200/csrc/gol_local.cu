// Change-tracking tiles: the device side of GOL_ALG_LOCAL.
//
// Reference: cuda-naive-local-one-cell (cuda_local_one_cell.cu:172,
// cuda_local_one_cell.hpp:26-309) and cuda-naive-local
// (cuda_naive_local.cu:125-196, gol_cuda_naive_local.hpp:23-335): a tile is
// recomputed only if it or one of its 8 neighbour tiles changed in the
// previous step; per-block state words record which warp tiles changed.
//
// Here one step is a pass of K generations and a tile is an x-slice (with
// a one-lane halo) times a band of rows, so the skip rule needs tiles at
// least K cells high and wide (a pass reads K cells around each cell). Per
// pass:
//   plan   one CTA reads the previous pass's per-tile `changed` bytes,
//          compacts the tiles whose 3x3 neighbourhood changed into a list
//          (block-wide scan, no atomics), clears this pass's bytes, and
//          appends the list length to a census;
//   tiles  persistent CTAs walk the list, run the K-stage pipeline on each
//          tile (band_tile<.., TRACK>) and set changed[tile] when any of
//          its cells differs after the pass.
// No copies for skipped tiles: a tile skipped at pass p did not change at
// pass p-1 (it is in its own neighbourhood), so the buffer pass p writes —
// the one pass p-1 read — already holds its current state.
#include <algorithm>

#include "gol_internal.h"
#include "gol_rows_temporal.cuh"

namespace golb200 {

namespace {

constexpr int kPlanThreads = 1024;

__device__ __forceinline__ bool tile_active(const uint8_t* prev, int tx, int ty, int tiles_x,
                                            int tiles_y) {
    for (int dy = -1; dy <= 1; ++dy) {
        const int y = ty + dy;
        if (y < 0 || y >= tiles_y) continue;
        for (int dx = -1; dx <= 1; ++dx) {
            const int x = tx + dx;
            if (x < 0 || x >= tiles_x) continue;
            if (prev[y * tiles_x + x]) return true;
        }
    }
    return false;
}

__global__ void __launch_bounds__(kPlanThreads)
plan_tiles_kernel(const uint8_t* __restrict__ prev, uint8_t* __restrict__ clear, int tiles_x,
                  int tiles_y, int* __restrict__ list, int* __restrict__ count,
                  uint32_t* __restrict__ census, uint32_t census_cap, uint32_t* __restrict__ pass_no) {
    __shared__ int warp_sums[kPlanThreads / 32];
    const int ntiles = tiles_x * tiles_y;
    const int per = (ntiles + blockDim.x - 1) / blockDim.x;
    const int t0 = min((int)threadIdx.x * per, ntiles), t1 = min(t0 + per, ntiles);
    int mine = 0;
    for (int t = t0; t < t1; ++t) mine += tile_active(prev, t % tiles_x, t / tiles_x, tiles_x, tiles_y);

    // Block-wide exclusive scan of `mine`.
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int incl = mine;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
    }
    if (lane == 31) warp_sums[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        const int nw = blockDim.x >> 5;
        int w = lane < nw ? warp_sums[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int v = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += v;
        }
        if (lane < nw) warp_sums[lane] = w;   // inclusive over warps
    }
    __syncthreads();
    int pos = incl - mine + (warp > 0 ? warp_sums[warp - 1] : 0);

    for (int t = t0; t < t1; ++t) {
        if (tile_active(prev, t % tiles_x, t / tiles_x, tiles_x, tiles_y)) list[pos++] = t;
        clear[t] = 0;
    }
    if (threadIdx.x == blockDim.x - 1) {
        const int total = pos;   // the last thread's end position is the total
        *count = total;
        const uint32_t p = *pass_no;
        if (census && p < census_cap) census[p] = (uint32_t)total;
        *pass_no = p + 1;
    }
}

template <int WPL, int K>
cudaError_t launch_tiles_one(const RowsLaunch& a, const TileList& t, int threads, int ctas,
                             cudaStream_t stream) {
    const size_t smem = temporal_smem_bytes(K, threads, WPL);
    rows_tiles_kernel<WPL, K><<<ctas, threads, smem, stream>>>(a, t);
    return cudaPeekAtLastError();
}

template <int WPL, int K>
cudaError_t dispatch_tiles(int k, const RowsLaunch& a, const TileList& t, int threads, int ctas,
                           cudaStream_t stream) {
    if constexpr (K > kMaxKForWpl(WPL)) {
        return cudaErrorInvalidValue;
    } else {
        if (k == K) return launch_tiles_one<WPL, K>(a, t, threads, ctas, stream);
        return dispatch_tiles<WPL, K + 1>(k, a, t, threads, ctas, stream);
    }
}

} // namespace

bool plan_local_tiles(int W, int Y, int k, int tile_rows, int wpl, int num_sms, LocalPlan* lp) {
    if (k < 1 || k > kMaxTemporalSteps || W <= 0 || Y <= 0) return false;
    if (wpl == 0) wpl = 1;
    if ((wpl != 1 && wpl != 2 && wpl != 4) || W % wpl || k > kMaxKForWpl(wpl)) return false;
    int band = tile_rows > 0 ? tile_rows : std::max(32, k);
    if (band < k) return false;                         // the 3x3 skip rule needs tiles >= K rows
    RowsPlan& p = lp->rows;
    p.wpl = wpl;
    p.band = band;
    p.nbands = (Y + band - 1) / band;
    p.threads = 32;
    if (W / wpl <= 32) {
        p.slice = W;
        p.halo = 0;
    } else {
        p.slice = 30 * wpl;                              // 30 lanes + a halo lane each side
        p.halo = wpl;
    }
    p.nslices = (W + p.slice - 1) / p.slice;
    lp->tiles_x = p.nslices;
    lp->tiles_y = p.nbands;
    lp->ctas = std::max(1, std::min(lp->tiles_x * lp->tiles_y, num_sms * 16));
    return true;
}

cudaError_t launch_local_pass(const uint32_t* src, uint32_t* dst, int W, int Y, int k,
                              const LocalPlan& lp, const LocalState& st, int parity,
                              cudaStream_t stream) {
    const RowsPlan& p = lp.rows;
    plan_tiles_kernel<<<1, kPlanThreads, 0, stream>>>(st.changed[parity ^ 1], st.changed[parity],
                                                      lp.tiles_x, lp.tiles_y, st.list, st.count,
                                                      st.census, st.census_cap, st.pass_no);
    cudaError_t e = cudaPeekAtLastError();
    if (e != cudaSuccess) return e;
    RowsLaunch a{src, dst, W, Y, p.band, p.slice, p.halo};
    TileList t{st.list, st.count, st.changed[parity], lp.tiles_x};
    switch (p.wpl) {
        case 4: return dispatch_tiles<4, 1>(k, a, t, p.threads, lp.ctas, stream);
        case 2: return dispatch_tiles<2, 1>(k, a, t, p.threads, lp.ctas, stream);
        case 1: return dispatch_tiles<1, 1>(k, a, t, p.threads, lp.ctas, stream);
        default: return cudaErrorInvalidValue;
    }
}

} // namespace golb200
