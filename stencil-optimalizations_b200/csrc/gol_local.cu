// Change-tracking tiles: the device side of GOL_ALG_LOCAL.
//
// Reference: cuda-naive-local-one-cell (cuda_local_one_cell.cu:172,
// cuda_local_one_cell.hpp:26-309) and cuda-naive-local
// (cuda_naive_local.cu:125-196, gol_cuda_naive_local.hpp:23-335): a tile is
// recomputed only if it or one of its 8 neighbour tiles changed in the
// previous step; per-block state words record which warp tiles changed.
//
// Here one step is a pass of K generations and a tile is a narrow x-slice
// (by default one lane of words, 32 cells; a halo lane each side absorbs
// the unknown cells beyond it, whose errors move one cell per generation)
// times a band of rows, so
// the skip rule needs tiles at least K cells high and wide (a pass reads K
// cells around each cell). Per pass:
//   plan   one thread per 32 tiles of a tile row dilates the previous
//          pass's change bits over the 3x3 neighbourhood, active tiles are
//          appended to a list as runs (warp scan + one atomic per warp), this pass's
//          bits are cleared, and the last CTA appends the list length to a
//          census;
//   tiles  persistent one-warp CTAs walk the list in windows of 32 lanes:
//          a run of horizontally adjacent active tiles takes one lane per
//          tile plus a halo lane at each end (neighbouring tiles share their
//          halos: about 1 + 2/run lanes per tile instead of 3), each lane
//          streams its tile's band through the K stages (the segmented-warp
//          form of the pipeline), compares its result with its input and
//          sets the tile's change bit when any of its cells differs after
//          the pass.
// No copies for skipped tiles: a tile skipped at pass p did not change at
// pass p-1 (it is in its own neighbourhood), so the buffer pass p writes —
// the one pass p-1 read — already holds its current state.
//   dense  when the plan finds at least `dense_min` active tiles the tile
//          kernel returns at once and the row-band kernel runs the whole
//          grid instead, comparing each output row with its input and
//          setting the change bits of the tiles that differ. Its bits equal
//          the tile kernel's (same tiles, same comparison), so the two modes
//          hand over from pass to pass either way. Each tile is computed
//          about 6x as fast there as by a tile warp (no halo lanes, no
//          per-tile warm-up), so the dense pass wins above a few percent.
#include <algorithm>
#include <climits>

#include "gol_internal.h"
#include "gol_rows_temporal.cuh"

#ifndef GOL_LOCAL_CARVEOUT
// Shared-memory carveout (percent of the maximum) preferred by all three
// kernels of a pass, so that the SMs keep one L1/shared split from kernel to
// kernel; -1 leaves the CUDA driver's choice. On the sparse 16384^2
// workload (k = 6) the CUDA driver's choice ran at 79 T cell-updates/s, a
// common 100 % at 77.6 T.
#define GOL_LOCAL_CARVEOUT -1
#endif

#ifndef GOL_LOCAL_DENSE_PCT
// Active-tile share (percent) from which a change-tracking pass runs dense.
// On the dense benchmark's 16384^2 random grid at k = 6 (20000 generations,
// a quarter of the tile-passes active on average) 6, 10 and 15 % ran at 49.3,
// 50.3 and 49.5 T cell-updates/s; tiles alone (above 100 %) at 5.2 T over
// the first 4096 generations, against 21.2 T.
#define GOL_LOCAL_DENSE_PCT 10
#endif

namespace golb200 {

namespace {

constexpr int kPlanThreads = 256;

// Change flags are bits: tile (tx, ty) is bit tx % 32 of word
// ty * change_words(tiles_x) + tx / 32.
__host__ __device__ inline int change_words(int tiles_x) { return (tiles_x + 31) / 32; }

// The plan's device words (PlanCounts): active tiles by pass parity, the
// last CTA's ticket, whether the last planned pass had at least dense_min
// active tiles, whether each parity's pass runs dense, and the lane list's
// length by pass parity.
enum PlanCounts { kTiles0 = 0, kTicket = 2, kDenseHint = 3, kDense0 = 4, kLanes0 = 6 };
static_assert(kLanes0 + 2 <= kLocalCountWords, "plan words");

// The lane list: a pass's active tiles in runs of horizontally adjacent
// tiles of one tile row, each run with a halo lane before and after it. An
// entry is tile * 4 + role: the tile of a tile lane, or the first / last
// tile of the run for its left / right halo lane.
enum LaneRole { kRoleTile = 0, kRoleLeft = 1, kRoleRight = 2 };

// One thread per flag word (32 tiles of a tile row). A tile is active if it
// or one of its 8 neighbours changed in the previous pass: the OR of the
// three flag rows around it, each shifted one bit left and right (with the
// carry bits of the neighbouring words). The active tiles are appended to
// the lane list in order, a warp at a time (a scan of the per-thread lane
// counts, one atomic per warp): each run of adjacent active tiles as its
// tiles with a halo lane before and after, so that neighbouring tiles share
// halo lanes. A run continues across flag words of one tile row within a
// warp; at a warp's edge it is cut in two (each part with its halos).
// counts[kTiles0 + parity] / [kLanes0 + parity] are this pass's tile and
// lane counts (zero on entry); the other parity's are zeroed for the next
// pass; the last CTA decides the pass's form and records the census (tiles
// computed: all of them in a dense pass). A pass runs dense when it has at
// least dense_min active tiles, or when the previous one had: then the list
// is not written at all (the counts still are), at the price of one dense
// pass too many when activity drops. This pass's flags are cleared on the way.
__global__ void __launch_bounds__(kPlanThreads)
plan_tiles_kernel(const uint32_t* __restrict__ prev, uint32_t* __restrict__ clear, int tiles_x,
                  int tiles_y, int* __restrict__ list, int* counts, int parity,
                  uint32_t* __restrict__ census, uint32_t census_cap, uint32_t* __restrict__ pass_no,
                  int dense_min) {
    const int wx = change_words(tiles_x);
    const int nw = wx * tiles_y;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31;
    const bool skip_list = counts[kDenseHint] != 0;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        counts[kTiles0 + (parity ^ 1)] = 0;
        counts[kLanes0 + (parity ^ 1)] = 0;
    }
    uint32_t act = 0u;
    int ty = 0, w = 0;
    if (t < nw) {
        ty = t / wx;
        w = t - ty * wx;
        for (int dy = -1; dy <= 1; ++dy) {
            const int y = ty + dy;
            if (y < 0 || y >= tiles_y) continue;
            const uint32_t* row = prev + (size_t)y * wx;
            const uint32_t v = row[w];
            const uint32_t l = w > 0 ? row[w - 1] : 0u;
            const uint32_t r = w + 1 < wx ? row[w + 1] : 0u;
            act |= v | (v << 1) | (l >> 31) | (v >> 1) | (r << 31);
        }
        const int valid = tiles_x - 32 * w;   // tiles in this word
        if (valid < 32) act &= (1u << valid) - 1u;
        clear[t] = 0u;
    }
    // Runs: a run continues from the previous word (same tile row, same
    // warp) when that word's last tile and this word's first are active.
    const uint32_t prev_act = __shfl_up_sync(0xffffffffu, act, 1);
    const uint32_t next_act = __shfl_down_sync(0xffffffffu, act, 1);
    const bool cin = lane > 0 && w > 0 && (prev_act >> 31);
    const bool cout = lane < 31 && w + 1 < wx && (next_act & 1u);
    const uint32_t starts = act & ~((act << 1) | (cin ? 1u : 0u));
    const uint32_t ends = act & ~((act >> 1) | (cout ? 0x80000000u : 0u));
    const int n = __popc(act);
    const int nl = n + __popc(starts) + __popc(ends);
    // scan of (lanes << 16 | tiles): both at most 48 * 32 per warp
    const int packed = (nl << 16) | n;
    int incl = packed;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
    }
    const int wtotal = __shfl_sync(0xffffffffu, incl, 31);
    int base = 0;
    if (lane == 31 && wtotal) {
        atomicAdd(counts + kTiles0 + parity, wtotal & 0xffff);
        base = atomicAdd(counts + kLanes0 + parity, wtotal >> 16);
    }
    base = __shfl_sync(0xffffffffu, base, 31) + ((incl - packed) >> 16);
    // Each lane writes its own runs, all lanes at once.
    if (!skip_list) {
        while (act) {
            const int b = __ffs((int)act) - 1;
            act &= act - 1u;
            const int tile = ty * tiles_x + 32 * w + b;
            if ((starts >> b) & 1u) list[base++] = tile * 4 + kRoleLeft;
            list[base++] = tile * 4 + kRoleTile;
            if ((ends >> b) & 1u) list[base++] = tile * 4 + kRoleRight;
        }
    }

    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned* ticket = reinterpret_cast<unsigned*>(counts + kTicket);
        if (atomicAdd(ticket, 1u) == gridDim.x - 1) {   // every CTA has appended
            __threadfence();
            const int total = atomicAdd(counts + kTiles0 + parity, 0);
            const bool dense = skip_list || total >= dense_min;
            counts[kDense0 + parity] = dense ? 1 : 0;
            counts[kDenseHint] = total >= dense_min ? 1 : 0;
            const uint32_t p = *pass_no;
            // Tiles computed this pass: every tile when the pass runs dense.
            const uint32_t computed = dense ? (uint32_t)tiles_x * tiles_y : (uint32_t)total;
            if (census && p < census_cap) census[p] = computed;
            *pass_no = p + 1;
            *ticket = 0u;
        }
    }
}

struct TileList {
    const int* list;        // the lane list (entries tile * 4 + role)
    const int* lanes;       // number of entries in `list`
    uint32_t* changed;      // change bits of this pass (cleared by the plan kernel)
    int tiles_x;
    const int* dense;       // nonzero: this pass runs dense (the tile kernel returns)
};

#ifndef GOL_TILE_WARPS
// Warps of the tile kernel per CTA (each works alone, with its own shared
// memory). One: with three the compiler gave the (1-word, depth-6) kernel
// 118 registers instead of 96, 15 resident warps per SM instead of 21.
#define GOL_TILE_WARPS 1
#endif
constexpr int kTileWarps = GOL_TILE_WARPS;
constexpr int kWindowOwn = 30;   // lanes of the lane list a warp stores per window

// One warp per window of 32 consecutive entries of the lane list: it owns
// the middle 30 (window w owns entries [30w, 30w + 30)) and computes the two
// outer ones only as context, so a run cut by a window edge still has a
// correct neighbour word beyond each owned lane (an error entering at the
// window's edge moves one cell per generation and stays in the outer lane
// for K <= 32). Each lane streams its own tile's band through the K stages
// (the segmented-warp pipeline, segments = runs: a run's halo lanes and the
// window's edges see dead cells beyond them), compares every stored word
// with its input, and a lane whose tile changed sets the tile's change bit.
// When the dense form is enabled this kernel is launched after it, as a
// programmatic dependent: the two never touch the same data in one pass
// (one of them returns at once), so a tile pass starts without waiting,
// but every CTA waits for the dense kernel before it ends, because later
// work in the stream waits for this kernel only.
template <int WPL, int K>
__global__ void __launch_bounds__(32 * kTileWarps)
seg_tiles_kernel(RowsLaunch a, TileList t) {
    __shared__ __align__(16) uint32_t rings[kTileWarps][kRowRing * 32 * WPL];
    constexpr int kEdgeWords = WPL == 1 ? 1 : seg_edge_words(K);   // one word per lane: shuffles
    __shared__ uint32_t etabs[kTileWarps][kEdgeWords];
    const int dense = *t.dense;
    const int nl = *t.lanes;   // both loads in flight together
    if (dense) {   // a dense pass
        asm volatile("griddepcontrol.wait;" ::: "memory");
        return;
    }
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    uint32_t* ring = rings[warp];
    uint32_t* etab = etabs[warp];
    const int gwarp = blockIdx.x * kTileWarps + warp;
    const int nwarps = gridDim.x * kTileWarps;
    for (int u = lane; u < kEdgeWords; u += 32) etab[u] = 0u;
    __syncwarp();
    for (int win = gwarp; win * kWindowOwn < nl; win += nwarps) {
        const int g = win * kWindowOwn - 1 + lane;
        const int d = (g >= 0 && g < nl) ? t.list[g] : -1;
        const bool valid = d >= 0;
        const int role = valid ? (d & 3) : kRoleTile;
        const int tile = valid ? (d >> 2) : 0;
        const int ty = tile / t.tiles_x, tx = tile - ty * t.tiles_x;
        const int col = tx + (role == kRoleLeft ? -1 : role == kRoleRight ? 1 : 0);
        TemporalCtx c;
        c.src = a.src;
        c.dst = a.dst;
        c.W = a.W;
        c.pitch = a.W;   // change-tracking grids are never padded
        c.Y = a.Y;
        c.B = a.band;
        c.y0 = ty * a.band;
        c.y1 = min(c.y0 + a.band, a.Y);
        c.lane = lane;
        c.base = col * WPL;
        c.lane_ok = valid && c.y0 < a.Y && c.base >= 0 && c.base < a.W;
        c.own = c.lane_ok && role == kRoleTile && lane >= 1 && lane <= kWindowOwn;
        c.seg_first = !valid || role == kRoleLeft || lane == 0;
        c.seg_last = !valid || role == kRoleRight || lane == 31;
        c.eb = etab + lane;
        c.el = c.seg_first ? etab : etab + lane;                      // run ends: zero entries
        c.er = c.seg_last ? etab + kSegEdgeStride - 1 : etab + lane + 2;
        c.src_l = max(lane - 1, 0);
        c.src_r = min(lane + 1, 31);
        c.ring = ring + lane * WPL;
        c.ring_saddr = (uint32_t)__cvta_generic_to_shared(c.ring);
        c.ring_stride = ring_slot_words<WPL, true>();
        set_word_masks<WPL>(c);

        TemporalRegs<WPL, K> s;
#pragma unroll
        for (int w = 0; w < WPL; ++w) {
            s.ld[0][w] = s.ld[1][w] = s.ld[2][w] = 0u;
#pragma unroll
            for (int gg = 0; gg < K; ++gg) {
                s.h0[gg][0][w] = s.h0[gg][1][w] = s.h0[gg][2][w] = 0u;
                s.h1[gg][0][w] = s.h1[gg][1][w] = s.h1[gg][2][w] = 0u;
                s.o[gg][0][w] = s.o[gg][1][w] = s.o[gg][2][w] = 0u;
            }
        }
        for (int j = 0; j < kRowsInFlight; ++j) issue_row<WPL, K, 1, true>(c, j, j);
        cp_async_wait<kRowsInFlight - 1>();
        lds_words<WPL>(c.ring, s.ld[0]);
        s.diff = 0u;

        // Steady state while every lane's rows stay inside the grid: the
        // deepest band among the window's tiles bounds the window.
        const int y0_deep = __reduce_max_sync(0xffffffffu, c.lane_ok ? c.y0 : 0);
        const int nsteps = c.B + 3 * K;
        const int f0 = 3 * K;
        const int f1 = min(c.B + 2 * K - 1, c.Y - y0_deep + K - 1);
        const int fast_end = f1 > f0 ? f0 + (f1 - f0) / 3 * 3 : f0;
        if (fast_end > f0) {
            temporal_steps<WPL, K, false, false, true, true>(s, c, 0, f0);
            temporal_steps<WPL, K, true, true, true, true>(s, c, f0, fast_end);
            temporal_steps<WPL, K, false, false, true, true>(s, c, fast_end, nsteps);
        } else {
            temporal_steps<WPL, K, false, false, true, true>(s, c, 0, nsteps);
        }
        asm volatile("cp.async.wait_all;\n" ::: "memory");
        if (c.own && s.diff != 0u)
            atomicOr(t.changed + ty * change_words(t.tiles_x) + tx / 32, 1u << (tx % 32));
        __syncwarp();
    }
    asm volatile("griddepcontrol.wait;" ::: "memory");
}

// The dense form of a change-tracking pass, launched every pass before the
// tile kernel and returning at once unless the plan chose it; a grid of
// resident CTAs (one wave) walks the row bands. It lets the tile kernel's
// CTAs be scheduled at once: in a dense pass they wait on the SMs' spare
// room, in a tile pass they start while this grid exits.
template <int WPL, int K>
__global__ void __launch_bounds__(kTemporalMaxThreads, GOL_TEMPORAL_MIN_BLOCKS)
rows_tracked_kernel(RowsLaunch a, TileTrack tt, const int* __restrict__ dense, int nbands,
                    int nunits) {
    extern __shared__ __align__(16) uint32_t smem[];
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    if (!*dense) return;
    for (int u = blockIdx.x; u < nunits; u += gridDim.x)
        band_tile<WPL, K, 2>(a, u % nbands, u / nbands, smem, tt);
}

// Lane width of the dense tracked pass for depth k: the widest whose
// register rings fit (one kernel per depth).
constexpr int tracked_wpl(int k) { return k <= kMaxKForWpl(4) ? 4 : (k <= kMaxKForWpl(2) ? 2 : 1); }

// Sets a kernel's preferred carveout once (GOL_LOCAL_CARVEOUT).
template <typename F>
cudaError_t set_carveout(F* kernel) {
    if (GOL_LOCAL_CARVEOUT < 0) return cudaSuccess;
    return cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                                GOL_LOCAL_CARVEOUT);
}

template <int K>
cudaError_t launch_tracked_one(const RowsLaunch& a, const TileTrack& tt, const int* dense,
                               const RowsPlan& p, int num_sms, cudaStream_t stream) {
    constexpr int WPL = tracked_wpl(K);
    static const cudaError_t attr_ok = [] {
        cudaError_t e = cudaFuncSetAttribute(rows_tracked_kernel<WPL, K>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)temporal_smem_bytes(K, kTemporalMaxThreads, WPL, true));
        return e == cudaSuccess ? set_carveout(rows_tracked_kernel<WPL, K>) : e;
    }();
    if (attr_ok != cudaSuccess) return attr_ok;
    const size_t smem = temporal_smem_bytes(K, p.threads, WPL, true);
    int per_sm = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, rows_tracked_kernel<WPL, K>,
                                                                  p.threads, smem);
    if (e != cudaSuccess) return e;
    const int units = p.nbands * p.nslices;
    const int grid = std::max(1, std::min(units, std::max(1, per_sm) * num_sms));
    rows_tracked_kernel<WPL, K><<<grid, p.threads, smem, stream>>>(a, tt, dense, p.nbands, units);
    return cudaPeekAtLastError();
}

template <int K>
cudaError_t dispatch_tracked(int k, const RowsLaunch& a, const TileTrack& tt, const int* dense,
                             const RowsPlan& p, int num_sms, cudaStream_t stream) {
    if constexpr (K > kMaxTemporalSteps) {
        return cudaErrorInvalidValue;
    } else {
        if (k == K) return launch_tracked_one<K>(a, tt, dense, p, num_sms, stream);
        return dispatch_tracked<K + 1>(k, a, tt, dense, p, num_sms, stream);
    }
}

// The tile kernel's grid: lp.ctas, capped at one wave of resident CTAs (it
// walks the list); a programmatic dependent of the dense form when enabled.
template <int WPL, int K>
cudaError_t launch_tiles_one(const RowsLaunch& a, const TileList& t, const LocalPlan& lp,
                             cudaStream_t stream) {
    static const int per_sm = [] {
        int n = 0;
        if (set_carveout(seg_tiles_kernel<WPL, K>) != cudaSuccess) return -1;
        return cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, seg_tiles_kernel<WPL, K>,
                                                             32 * kTileWarps, 0) == cudaSuccess ? n : 0;
    }();
    if (per_sm < 0) return cudaErrorInvalidValue;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(per_sm > 0 ? std::max(1, std::min(lp.ctas, per_sm * lp.num_sms)) : lp.ctas);
    cfg.blockDim = dim3(32 * kTileWarps);
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = lp.dense_min == INT_MAX ? 0 : 1;
    return cudaLaunchKernelEx(&cfg, seg_tiles_kernel<WPL, K>, a, t);
}

template <int WPL, int K>
cudaError_t dispatch_tiles(int k, const RowsLaunch& a, const TileList& t, const LocalPlan& lp,
                           cudaStream_t stream) {
    if constexpr (K > kMaxKForWpl(WPL)) {
        return cudaErrorInvalidValue;
    } else {
        if (k == K) return launch_tiles_one<WPL, K>(a, t, lp, stream);
        return dispatch_tiles<WPL, K + 1>(k, a, t, lp, stream);
    }
}

} // namespace

bool plan_local_tiles(int W, int Y, int k, int tile_rows, int wpl, int num_sms, int dense_pct,
                      LocalPlan* lp) {
    if (k < 1 || k > kMaxTemporalSteps || W <= 0 || Y <= 0) return false;
    if (wpl == 0) wpl = 1;
    if ((wpl != 1 && wpl != 2 && wpl != 4) || W % wpl || k > kMaxKForWpl(wpl)) return false;
    // Default height: the smallest the skip rule allows (k rows), not below 4.
    // Finer tiles skip more: on the sparse 16384^2 workload 8-row tiles ran
    // at 49 T cell-updates/s against 40 T for 32-row ones (k = 8), and 6-row
    // ones at k = 6 at 85 T against 77 T for 8-row ones (32-cell tiles).
    int band = tile_rows > 0 ? tile_rows : std::max(4, k);
    if (band < k) return false;                         // the 3x3 skip rule needs tiles >= K rows
    RowsPlan& p = lp->rows;
    p.wpl = wpl;
    p.band = band;
    p.nbands = (Y + band - 1) / band;
    p.threads = 32;
    // A tile is one lane of words (32 cells at one word per lane); the lane
    // list gives each run of active tiles a halo lane on either side.
    p.slice = wpl;
    p.halo = wpl;
    p.nslices = W / wpl;
    lp->tiles_x = p.nslices;
    lp->tiles_y = p.nbands;
    if ((long long)lp->tiles_x * lp->tiles_y >= (1LL << 29)) return false;   // entries: tile * 4
    const long long lanes = (long long)lp->tiles_x * lp->tiles_y * 3 / 2;
    const long long windows = (lanes + kWindowOwn - 1) / kWindowOwn;
    lp->ctas = (int)std::max(1LL, (std::min<long long>(windows, num_sms * 24LL) + kTileWarps - 1) / kTileWarps);
    lp->num_sms = num_sms;
    // The dense form: the row-band plan at the kernel's lane width. Its
    // lanes start at multiples of that width and tiles are 1, 2 or 4 words
    // wide (or the whole row), so no lane straddles two change words.
    // dense_pct 0 = the default share, above 100 = never.
    const long long ntiles = (long long)lp->tiles_x * lp->tiles_y;
    if (dense_pct == 0) dense_pct = GOL_LOCAL_DENSE_PCT;
    lp->dense_min = INT_MAX;
    if (dense_pct <= 100 && plan_rows(W, Y, k, 0, tracked_wpl(k), num_sms, &lp->dense, false))
        lp->dense_min = (int)std::max(1LL, (ntiles * dense_pct + 99) / 100);
    return true;
}

cudaError_t launch_local_pass(const uint32_t* src, uint32_t* dst, int W, int Y, int k,
                              const LocalPlan& lp, const LocalState& st, int parity,
                              cudaStream_t stream) {
    const RowsPlan& p = lp.rows;
    const int nwords = change_words(lp.tiles_x) * lp.tiles_y;
    static const cudaError_t plan_attr = set_carveout(plan_tiles_kernel);
    if (plan_attr != cudaSuccess) return plan_attr;
    plan_tiles_kernel<<<(nwords + kPlanThreads - 1) / kPlanThreads, kPlanThreads, 0, stream>>>(
        st.changed[parity ^ 1], st.changed[parity], lp.tiles_x, lp.tiles_y, st.list, st.count,
        parity, st.census, st.census_cap, st.pass_no, lp.dense_min);
    cudaError_t e = cudaPeekAtLastError();
    if (e != cudaSuccess) return e;
    if (lp.dense_min != INT_MAX) {
        const RowsPlan& d = lp.dense;
        RowsLaunch da{src, dst, W, Y, d.band, d.slice, d.halo, W};
        TileTrack tt{st.changed[parity], p.band, p.slice, change_words(lp.tiles_x)};
        e = dispatch_tracked<1>(k, da, tt, st.count + kDense0 + parity, d, lp.num_sms, stream);
        if (e != cudaSuccess) return e;
    }
    RowsLaunch a{src, dst, W, Y, p.band, p.slice, p.halo, W};
    TileList t{st.list, st.count + kLanes0 + parity, st.changed[parity], lp.tiles_x,
               st.count + kDense0 + parity};
    switch (p.wpl) {
        case 4: return dispatch_tiles<4, 1>(k, a, t, lp, stream);
        case 2: return dispatch_tiles<2, 1>(k, a, t, lp, stream);
        case 1: return dispatch_tiles<1, 1>(k, a, t, lp, stream);
        default: return cudaErrorInvalidValue;
    }
}

} // namespace golb200
