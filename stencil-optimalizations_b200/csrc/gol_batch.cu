// Batched uneven grids in one persistent launch.
//
// The reference advances one grid per run (ExperimentManager::perform_alg,
// experiment_manager.hpp:365-394). Here many grids of different sizes and
// generation counts advance together:
//
//   work item   (grid, x-slice, band group, pass): one pass of k generations
//               on one warp. Narrow grids (W / WPL <= 32 lanes) have one
//               slice and cut the warp into S segments of L = W / WPL lanes
//               (any L, so narrow grids keep most lanes busy), each segment
//               streaming its own band through the K-stage pipeline
//               (band_tile's step code in segmented mode). Wider grids are
//               cut into slices of 30 lanes plus a halo lane each side
//               (errors from the unknown cells beyond the halo move one cell
//               per generation and stay in the halo for k <= 32).
//   order       items are numbered critical-path first: by descending
//               remaining passes of their grid, so the longest grids start
//               at once and short ones fill in; persistent one-warp CTAs
//               take tickets from an atomic counter, claiming the next one
//               while working on the current one.
//   dependency  (g, s, j, p) needs (g, s-1..s+1, j-1..j+1, p-1) finished:
//               that is every word it reads, and it also ends every read of
//               the buffer it overwrites. A per-group counter holds the
//               passes done; one lane per dependency polls it with
//               ld.acquire, bounded: after kSpinLimit polls the CTA records
//               GOL_E_TIMEOUT and stops. Every dependency has a smaller
//               ticket. The smallest unfinished ticket's dependencies are
//               all finished, and its CTA (resident) holds no smaller
//               unfinished item (a CTA claims tickets in increasing order),
//               so it is running or about to run that item: the wait always
//               ends, and the bound is only a guard.
//   release     each lane fences its stores, the warp syncs, lane 0 stores
//               the new pass count with st.release.
//
// Rows are read through cp.async after the acquire; a weak load ordered
// after an acquire observes the released data (PTX memory model), so L1
// cannot serve a stale line of a buffer rewritten in this same launch.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "gol_b200.h"
#include "gol_internal.h"
#include "gol_rows_resident.cuh"
#include "gol_rows_temporal.cuh"

#ifndef GOL_BATCH_REPLAN
#define GOL_BATCH_REPLAN 4.0   // re-plan grids whose chain exceeds this many work-bound times
#endif
#ifndef GOL_BATCH_MIN_BLOCKS
#define GOL_BATCH_MIN_BLOCKS 1   // resident one-warp CTAs per SM the registers are sized for
#endif
#ifndef GOL_BATCH_TRACK_OLD
// How tracked items read a row before the pass to compare: 3 = through a
// second shared-memory ring beside the row ring, 1 = a global load when
// storing.
#define GOL_BATCH_TRACK_OLD 3
#endif
#ifndef GOL_BATCH_TRACK_CAP
#define GOL_BATCH_TRACK_CAP 0   // 1: hold tracked variants near the untracked registers
#endif

namespace golb200 {

constexpr long long kSpinLimit = 1ll << 24;   // polls of >= 64 ns: a few-second guard

namespace {

__device__ __forceinline__ int ld_acquire(const int* p) {
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release(int* p, int v) {
    asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// One work item: the K-stage pipeline over the item's segments. With TRACK,
// every stored word is compared with the same word before the pass and the
// return value is this lane's OR of the differences (0: its part unchanged).
template <int WPL, int K, bool TRACK>
__device__ __forceinline__ uint32_t seg_group(const BatchGrid& G, int group, int slice_idx,
                                              const uint32_t* src, uint32_t* dst, uint32_t* ring,
                                              uint32_t* etab) {
    const int lane = threadIdx.x & 31;
    const int L = G.seg_lanes;
    const int seg = lane / L, q = lane - seg * L;
    const int xs = slice_idx * G.slice;
    TemporalCtx c;
    c.src = src;
    c.dst = dst;
    c.W = G.W;
    c.pitch = G.pitch;
    c.Y = G.Y;
    c.B = G.band;
    c.y0 = (group * G.segs + seg) * G.band;
    c.y1 = min(c.y0 + G.band, G.Y);
    c.lane = lane;
    c.base = xs - G.halo + q * WPL;
    c.lane_ok = seg < G.segs && c.y0 < G.Y && c.base >= 0 && c.base < G.W;
    c.own = c.lane_ok && c.base >= xs && c.base < xs + G.slice;
    c.eb = etab + lane;
    c.el = q == 0 ? etab : etab + lane;                          // segment ends: zero entries
    c.er = q == L - 1 ? etab + kSegEdgeStride - 1 : etab + lane + 2;
    c.src_l = max(lane - 1, 0);
    c.src_r = min(lane + 1, 31);
    c.seg_first = q == 0;
    c.seg_last = q == L - 1;
    c.ring = ring + lane * WPL;
    c.ring_saddr = (uint32_t)__cvta_generic_to_shared(c.ring);
    c.ring_stride = ring_slot_words<WPL, true>();
    set_word_masks<WPL>(c);

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
    constexpr int TR = TRACK ? GOL_BATCH_TRACK_OLD : 0;
    // (with TRACK the first rows' old-row copies travel with them too)
    for (int j = 0; j < kRowsInFlight; ++j) issue_row<WPL, K, TR, true>(c, j, j);
    cp_async_wait<kRowsInFlight - 1>();
    lds_words<WPL>(c.ring, s.ld[0]);
    s.diff = 0u;

    // Steady state while every active segment's rows stay inside the grid:
    // the deepest active segment bounds the window.
    const int active = min(G.segs, (G.Y - group * G.segs * G.band + G.band - 1) / G.band);
    const int y0_last = (group * G.segs + active - 1) * G.band;
    const int nsteps = G.band + 3 * K;
    const int f0 = 3 * K;
    const int f1 = min(G.band + 2 * K - 1, G.Y - y0_last + K - 1);
    const int fast_end = f1 > f0 ? f0 + (f1 - f0) / 3 * 3 : f0;
    if (fast_end > f0) {
        temporal_steps<WPL, K, false, false, TR, true, true>(s, c, 0, f0);
        temporal_steps<WPL, K, true, true, TR, true, true>(s, c, f0, fast_end);
        temporal_steps<WPL, K, false, false, TR, true, true>(s, c, fast_end, nsteps);
    } else {
        temporal_steps<WPL, K, false, false, TR, true, true>(s, c, 0, nsteps);
    }
    asm volatile("cp.async.wait_all;\n" ::: "memory");
    return s.diff;
}

template <int WPL, bool TRACK>
__device__ __forceinline__ uint32_t seg_dispatch(int k, const BatchGrid& G, int group, int slice,
                                                 const uint32_t* src, uint32_t* dst,
                                                 uint32_t* ring, uint32_t* etab) {
    switch (k) {
        case 1: return seg_group<WPL, 1, TRACK>(G, group, slice, src, dst, ring, etab);
        case 2: return seg_group<WPL, 2, TRACK>(G, group, slice, src, dst, ring, etab);
        case 3: return seg_group<WPL, 3, TRACK>(G, group, slice, src, dst, ring, etab);
        default: return seg_group<WPL, 4, TRACK>(G, group, slice, src, dst, ring, etab);
    }
}

// Loads a descriptor field anew after an item's pipeline (an opaque load
// the compiler cannot merge with the one before it), so the tracking fields
// are not held in registers through the pipeline.
template <typename T>
__device__ __forceinline__ T* ld_ptr_again(T* const* p) {
    unsigned long long v;
    asm volatile("ld.global.nc.u64 %0, [%1];" : "=l"(v) : "l"(p));
    return reinterpret_cast<T*>(v);
}
__device__ __forceinline__ int ld_int_again(const int* p) {
    int v;
    asm volatile("ld.global.nc.s32 %0, [%1];" : "=r"(v) : "l"(p));
    return v;
}

__device__ __forceinline__ void release_max(int* p, int v) {
    // Monotone release: an item of a still grid may finish before the item
    // of the previous pass on the same counter (it does not wait for it).
    asm volatile("red.release.gpu.global.max.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// WPL_ONLY = 1, 2 or 4: every grid of the launch uses that many words per
// lane, so the kernel holds one family of pipeline bodies (its registers
// and instruction footprint are that family's); 0 dispatches on each grid's
// own width. Warps of one SM that run different bodies compete for the
// instruction cache, which halved throughput in measurements, so the
// planner gives a batch one width and one depth.
//
// TRACK: grids with a change-tracking region (G.trk) skip the items whose
// 3x3 neighbour items did not change in the previous pass, the rule of the
// reference's change-tracking kernels (cuda_naive_local.cu:125-161,
// cuda_local_one_cell.cu:172-200). A skipped item needs no copy: it did not
// change in the previous pass (it is its own neighbour), so the buffer it
// would write — the one the previous pass read — already holds its state.
// Computed items compare every stored word with its input and publish a
// change flag before releasing their counter. When every item of a pass is
// done and none changed, the grid is still from the next pass on (the
// "retired" pass): later items of that grid end at once, without waiting for
// their dependencies or touching the grid, and both buffers hold the result.
// census: [0] SM cycles waiting on dependencies, [1] working, [2] items
// computed, [3] items skipped (tracked grids).
// Resident one-warp CTAs per SM the registers are sized for. The tracked
// variants of 1 and 2 words per lane are held near the untracked ones'
// register counts (96 and 136), so tracking costs them little occupancy;
// at 4 words per lane a cap spills heavily, so none is set.
template <int WPL_ONLY, bool TRACK>
constexpr int batch_min_blocks() {
    return !TRACK || !GOL_BATCH_TRACK_CAP
               ? GOL_BATCH_MIN_BLOCKS
               : (WPL_ONLY == 1 ? 19 : WPL_ONLY == 2 ? 15 : GOL_BATCH_MIN_BLOCKS);
}

template <int WPL_ONLY, bool TRACK>
__global__ void __launch_bounds__(32, (batch_min_blocks<WPL_ONLY, TRACK>()))
batch_kernel(const BatchGrid* __restrict__ grids, const BatchItem* __restrict__ items, int nitems,
             int* ticket, int* done, int* status, unsigned long long* census, long long spin_limit) {
    // the row ring, and with TRACK the old-row ring right after it
    __shared__ __align__(16) uint32_t
        ring[kRowRing * 32 * (WPL_ONLY ? WPL_ONLY : 4) * (TRACK && GOL_BATCH_TRACK_OLD == 3 ? 2 : 1)];
    constexpr int kEdgeWords = WPL_ONLY == 1 ? 1 : seg_edge_words(kBatchMaxK);   // 1: shuffles
    __shared__ uint32_t etab[kEdgeWords];
    const int lane = threadIdx.x & 31;
    for (int t = lane; t < kEdgeWords; t += 32) etab[t] = 0u;
    __syncwarp();
    int t = 0;
    if (lane == 0) t = atomicAdd(ticket, 1);
    t = __shfl_sync(0xffffffffu, t, 0);
    while (t < nitems) {
        const BatchItem it = items[t];
        const BatchGrid G = grids[it.grid];
        const int cell = it.group * G.nslices + it.slice;
        int* mine = done + G.done_base + cell;
        const int nper = G.ngroups * G.nslices;   // items per pass
        // A pass shorter than k (the last, when k does not divide the
        // generations) is not covered by the k-generation change flags: an
        // oscillator whose period divides k looks still to them. It computes
        // every item.
        const int k = it.pass == G.passes - 1 ? G.last_k : G.k;
        if (TRACK && G.trk && k == G.k) {
            const unsigned still = *(volatile const uint32_t*)(G.trk + 2 * nper);
            if ((unsigned)(G.pass0 + it.pass) >= still) {   // the grid stopped changing
                int next = 0;
                if (lane == 0) {
                    next = atomicAdd(ticket, 1);
                    // every flag from the still pass on is zero; writing this
                    // pass's keeps a later reader from seeing an older one
                    *(volatile uint32_t*)(G.trk + (((G.parity0 + it.pass) & 1) ? nper : 0) + cell) = 0u;
                    release_max(mine, it.pass + 1);
                    atomicAdd(G.gstat + 1, 1u);
                    if (G.rflag) *(volatile int*)G.rflag = 1;
                    if (census) atomicAdd(census + 3, 1ull);
                }
                t = __shfl_sync(0xffffffffu, next, 0);
                continue;
            }
        }
        // the 3x3 neighbourhood of (group, slice)
        const int jlo = max(it.group - 1, 0), jhi = min(it.group + 1, G.ngroups - 1);
        const int slo = max(it.slice - 1, 0), shi = min(it.slice + 1, G.nslices - 1);
        const int nj = jhi - jlo + 1, ns = shi - slo + 1;
        const int dep = lane < nj * ns ? (jlo + lane / ns) * G.nslices + slo + lane % ns : -1;
        const long long t_wait = clock64();
        if (it.pass > 0) {
            // Lane d polls dependency d until it reached this pass; then every
            // lane acquires every counter (each is already there), so each
            // lane's own copies below are ordered after the producers' releases.
            bool ok = true;
            if (dep >= 0) {
                const int* p = done + G.done_base + dep;
                long long spins = 0;
                while (ld_acquire(p) < it.pass) {
                    if (++spins > spin_limit || *(volatile int*)status != 0) {
                        ok = false;
                        break;
                    }
                    __nanosleep(64);
                }
            }
            if (!__all_sync(0xffffffffu, ok)) {
                if (lane == 0) atomicCAS(status, 0, GOL_E_TIMEOUT);
                return;
            }
            int seen = 0;
            for (int d = 0; d < nj * ns; ++d)
                seen |= ld_acquire(done + G.done_base + (jlo + d / ns) * G.nslices + slo + d % ns);
            asm volatile("" ::"r"(seen));
        }
        // Claim the next item now: the atomic's round trip overlaps the work.
        int next = 0;
        if (lane == 0) next = atomicAdd(ticket, 1);
        const long long t_work = clock64();
        const bool odd = (G.parity0 + it.pass) & 1;
        bool compute = true;
        if (TRACK && G.trk && k == G.k) {   // did the neighbourhood change in the previous pass?
            const uint32_t* prev = G.trk + (odd ? 0 : nper);   // parity of pass - 1
            const uint32_t f = dep >= 0 ? *(volatile const uint32_t*)(prev + dep) : 0u;
            compute = __any_sync(0xffffffffu, f != 0u);
        }
        bool changed = false;
        if (compute) {
            // Selects, not an index: a dynamically indexed descriptor would be
            // kept in local memory for the whole item.
            const uint32_t* src = odd ? G.buf[1] : G.buf[0];
            uint32_t* dst = odd ? G.buf[0] : G.buf[1];
            uint32_t diff;
            if constexpr (WPL_ONLY != 0) {
                diff = seg_dispatch<WPL_ONLY, TRACK>(k, G, it.group, it.slice, src, dst, ring, etab);
            } else {
                switch (G.wpl) {
                    case 4: diff = seg_dispatch<4, TRACK>(k, G, it.group, it.slice, src, dst, ring, etab); break;
                    case 2: diff = seg_dispatch<2, TRACK>(k, G, it.group, it.slice, src, dst, ring, etab); break;
                    default: diff = seg_dispatch<1, TRACK>(k, G, it.group, it.slice, src, dst, ring, etab); break;
                }
            }
            changed = TRACK && __any_sync(0xffffffffu, diff != 0u);
        }
        const BatchGrid* gp = grids + it.grid;
        uint32_t* trk = TRACK ? ld_ptr_again(&gp->trk) : nullptr;
        if (TRACK && trk && lane == 0)   // this pass's flag, read by the next pass
            *(volatile uint32_t*)(trk + (odd ? nper : 0) + cell) = (changed || k != G.k) ? 1u : 0u;
        __threadfence();
        __syncwarp();
        if (lane == 0) {
            if (TRACK && trk)
                release_max(mine, it.pass + 1);
            else
                st_release(mine, it.pass + 1);
            atomicAdd(ld_ptr_again(&gp->gstat) + (compute ? 0 : 1), 1u);
            if (TRACK && trk) {
                // Last item of this pass: if none changed, the grid is still
                // from the next pass on.
                int* pstat = ld_ptr_again(&gp->pstat);
                if (changed || k != G.k) atomicAdd(pstat + 2 * it.pass + 1, 1);
                __threadfence();
                if (atomicAdd(pstat + 2 * it.pass, 1) == nper - 1) {
                    __threadfence();
                    if (atomicAdd(pstat + 2 * it.pass + 1, 0) == 0) {
                        atomicMin(trk + 2 * nper, (unsigned)(ld_int_again(&gp->pass0) + it.pass + 1));
                        int* rflag = ld_ptr_again(&gp->rflag);
                        if (rflag) *(volatile int*)rflag = 1;
                    }
                }
            }
            if (census) {   // SM cycles spent waiting on dependencies / computing
                atomicAdd(census + 0, (unsigned long long)(t_work - t_wait));
                atomicAdd(census + 1, (unsigned long long)(clock64() - t_work));
                atomicAdd(census + (compute ? 2 : 3), 1ull);
            }
        }
        t = __shfl_sync(0xffffffffu, next, 0);
    }
}

} // namespace

// ---------------------------------------------------------------------------
// Autotuner: one (words per lane, depth) for the whole batch, a band height
// per grid.
//
// Model, in units of one word through one stage on a 4-word lane: a work
// item is (band + 3k) pipeline steps of k stages, each step moving WPL words
// per lane at a per-word cost cw[WPL], plus each row's load and store once
// per pass (c_row stage-steps per row) and a fixed start-up and dependency
// cost (c_item):
//     item = ((band + 3k) * k + c_row * band) * WPL * cw[WPL] + c_item.
// The per-pass terms are what make deeper passes pay: on the dense kernel a
// 1-generation pass costs ~1.4x a 4-generation pass per generation, which
// c_row = 0.6 and c_item reproduce. A grid's work is
//     passes * nslices * ngroups * item
// for passes = ceil(gens / k), ngroups = ceil(Y / (S * band)), and its
// dependency chain (one item per pass, in order) is passes * item.
// A batch takes about max(total work / resident warps, longest chain), so a
// first choice minimises work alone; grids whose chain would outlast the
// batch's work-bound time are then re-planned to minimise work / resident
// warps + chain (shorter bands: more, quicker items per pass). Candidates:
// WPL in {1, 2, 4} (rows padded to whole lanes), k in 1..4, band in
// {16, 24, 32, 48} (taller bands measured slower: fewer items per pass
// leave warps waiting on the previous pass)
// with band >= 2k. gol_batch_upload runs this for every (WPL, k) the whole
// batch can use and keeps the pair with the smallest estimated time.
// ---------------------------------------------------------------------------

struct BatchTuning {
    // relative cost per word-stage-step by WPL, measured on uniform batches
    // with every lane busy (per-variant kernels: 21, 15 and 9 resident warps
    // per SM for 1, 2 and 4 words per lane)
    double cw[5] = {0, 1.13, 0.81, 0, 1.0};
    double c_row = 0.6;                        // per row per pass (load + store)
    double c_item = 120.0;                     // per item (start-up, dependency wait, release)
};

static BatchTuning g_tuning;

bool choose_batch_plan(int W, int Y, uint64_t gens, int force_wpl, int force_k, int force_band,
                       GridChoice* out, double parallel, double crit_weight) {
    bool found = false;
    for (int wpl : {1, 2, 4}) {
        if (force_wpl && wpl != force_wpl) continue;
        // A row of W words takes ceil(W / wpl) lanes; rows are padded to a
        // whole number of lanes (the padding words stay zero).
        const int lanes = (W + wpl - 1) / wpl;
        const bool sliced = lanes > 32;
        const int L = sliced ? 32 : lanes;
        const int slice = sliced ? 30 * wpl : W;
        const int nslices = (W + slice - 1) / slice;
        for (int k = 1; k <= kBatchMaxK; ++k) {
            if (force_k && k != force_k) continue;
            for (int band : {16, 24, 32, 48}) {
                if (force_band) band = force_band;
                if (band < 2 * k && !force_band) continue;
                const int S = sliced ? 1 : std::max(1, std::min(32 / L, (Y + band - 1) / band));
                const int ngroups = (Y + S * band - 1) / (S * band);
                const uint64_t passes = (gens + k - 1) / k;
                const double item =
                    ((double)(band + 3 * k) * k + g_tuning.c_row * band) * wpl * g_tuning.cw[wpl] +
                    g_tuning.c_item;
                const double cost = (double)passes * nslices * ngroups * item;
                // one item per pass on the chain of dependent passes
                const double crit = (double)passes * item;
                const double score = cost / std::max(parallel, 1.0) + crit_weight * crit;
                if (!found || score < out->score) {
                    found = true;
                    out->wpl = wpl;
                    out->k = k;
                    out->band = band;
                    out->seg_lanes = L;
                    out->segs = S;
                    out->ngroups = ngroups;
                    out->passes = (int)passes;
                    out->last_k = gens % k ? (int)(gens % k) : k;
                    out->slice = slice;
                    out->nslices = nslices;
                    out->halo = sliced ? wpl : 0;
                    out->cost = cost;
                    out->crit = crit;
                    out->score = score;
                }
                if (force_band) break;
            }
        }
    }
    return found;
}

size_t count_batch_items(const BatchGrid* grids, size_t ngrids) {
    size_t n = 0;
    for (size_t g = 0; g < ngrids; ++g)
        n += (size_t)grids[g].passes * grids[g].ngroups * grids[g].nslices;
    return n;
}

size_t order_batch_items(const BatchGrid* grids, size_t ngrids, BatchItem* out) {
    int max_passes = 0;
    for (size_t g = 0; g < ngrids; ++g) max_passes = std::max(max_passes, grids[g].passes);
    size_t n = 0;
    for (int rem = max_passes; rem >= 1; --rem)
        for (size_t g = 0; g < ngrids; ++g) {
            const BatchGrid& G = grids[g];
            if (G.passes < rem) continue;
            const int p = G.passes - rem;
            for (int j = 0; j < G.ngroups; ++j)
                for (int sl = 0; sl < G.nslices; ++sl) out[n++] = {(int)g, j, sl, p};
        }
    return n;
}

template <int W, bool TR>
static int ctas_per_sm_of() {
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_kernel<W, TR>, 32, 0) !=
        cudaSuccess)
        per_sm = 1;
    return std::max(1, per_sm);
}

int batch_kernel_ctas_per_sm(int wpl_only, bool track) {
    if (track) {
        switch (wpl_only) {
            case 4: return ctas_per_sm_of<4, true>();
            case 2: return ctas_per_sm_of<2, true>();
            case 1: return ctas_per_sm_of<1, true>();
            default: return ctas_per_sm_of<0, true>();
        }
    }
    switch (wpl_only) {
        case 4: return ctas_per_sm_of<4, false>();
        case 2: return ctas_per_sm_of<2, false>();
        case 1: return ctas_per_sm_of<1, false>();
        default: return ctas_per_sm_of<0, false>();
    }
}

int batch_uniform_wpl(const BatchGrid* grids, size_t ngrids) {
    int w = 0;
    for (size_t g = 0; g < ngrids; ++g) {
        if (grids[g].passes == 0) continue;
        if (w && grids[g].wpl != w) return 0;
        w = grids[g].wpl;
    }
    return w;
}

void batch_grid_from_choice(const GridChoice& ch, int W, int Y, BatchGrid* g) {
    g->W = W;
    g->Y = Y;
    g->pitch = (W + ch.wpl - 1) / ch.wpl * ch.wpl;
    g->wpl = ch.wpl;
    g->k = ch.k;
    g->last_k = ch.last_k;
    g->passes = ch.passes;
    g->band = ch.band;
    g->seg_lanes = ch.seg_lanes;
    g->segs = ch.segs;
    g->ngroups = ch.ngroups;
    g->slice = ch.slice;
    g->nslices = ch.nslices;
    g->halo = ch.halo;
}

template <int W, bool TR>
static void launch_batch_variant(int ctas, cudaStream_t stream, const BatchGrid* g,
                                 const BatchItem* items, int nitems, int* ticket, int* done,
                                 int* status, unsigned long long* census, long long spin_limit) {
    batch_kernel<W, TR><<<ctas, 32, 0, stream>>>(g, items, nitems, ticket, done, status, census,
                                                 spin_limit);
}

cudaError_t launch_batch_kernel(const BatchGrid* d_grids, const BatchItem* d_items, int nitems,
                                int* d_ticket, int* d_done, int* d_status, int num_sms,
                                cudaStream_t stream, unsigned long long* d_census, int wpl_only,
                                long long spin_limit, bool track) {
    if (spin_limit <= 0) spin_limit = kSpinLimit;
    if (nitems <= 0) return cudaSuccess;
    // every CTA resident at once (the dependency waits rely on it)
    const int ctas = std::min(nitems, num_sms * batch_kernel_ctas_per_sm(wpl_only, track));
#define GOL_BATCH_ARGS ctas, stream, d_grids, d_items, nitems, d_ticket, d_done, d_status, d_census, \
                       spin_limit
    if (track) {
        switch (wpl_only) {
            case 4: launch_batch_variant<4, true>(GOL_BATCH_ARGS); break;
            case 2: launch_batch_variant<2, true>(GOL_BATCH_ARGS); break;
            case 1: launch_batch_variant<1, true>(GOL_BATCH_ARGS); break;
            default: launch_batch_variant<0, true>(GOL_BATCH_ARGS); break;
        }
    } else {
        switch (wpl_only) {
            case 4: launch_batch_variant<4, false>(GOL_BATCH_ARGS); break;
            case 2: launch_batch_variant<2, false>(GOL_BATCH_ARGS); break;
            case 1: launch_batch_variant<1, false>(GOL_BATCH_ARGS); break;
            default: launch_batch_variant<0, false>(GOL_BATCH_ARGS); break;
        }
    }
#undef GOL_BATCH_ARGS
    return cudaPeekAtLastError();
}

} // namespace golb200

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------

using golb200::BatchGrid;
using golb200::BatchItem;

namespace golb200 {

#ifndef GOL_RBATCH_K
#define GOL_RBATCH_K 8
#endif
#ifndef GOL_RBATCH_ROWS_PER_GROUP
#define GOL_RBATCH_ROWS_PER_GROUP 8
#endif
#ifndef GOL_RBATCH_BANDS_PER_CTA
#define GOL_RBATCH_BANDS_PER_CTA 3
#endif
namespace {
constexpr int kResidentBatchWpl = 2;        // words per lane of the resident batch kernel
constexpr int kResidentBatchThreads = 512;  // threads per CTA
constexpr int kResidentBatchK = GOL_RBATCH_K;   // generations per epoch
constexpr int kResidentBatchRowsPerGroup = GOL_RBATCH_ROWS_PER_GROUP;   // fewer rows per group and
                                                                        // pass cost warm-up
constexpr int kResidentBatchBandsPerCta = GOL_RBATCH_BANDS_PER_CTA;     // about this many bands per
                                                                        // CTA (balance)
} // namespace

// Per grid: lanes of two words across its row and row groups over the CTA's
// threads; as many bands as the shared memory needs, more for grids whose
// work would otherwise make one band a long job (about
// kResidentBatchBandsPerCta bands per CTA over the batch), fewer where a
// band would give a row group under kResidentBatchRowsPerGroup rows; every
// band of a grid at least K rows, at most one band per SM.
namespace {
// Per device: the opt-in shared memory per CTA, with the kernel's dynamic
// shared memory limit raised to it (once), and the resident CTAs per SM by
// shared memory size in 4 KB steps. Serving plans a launch per round, so
// these are looked up once.
struct ResidentDeviceInfo {
    int smem_optin = 0;
    std::map<size_t, int> per_sm;
};
std::mutex g_resident_info_mu;
std::map<int, ResidentDeviceInfo> g_resident_info;

const char* resident_device(int device, size_t smem, int* smem_optin, int* per_sm) {
    std::lock_guard<std::mutex> lock(g_resident_info_mu);
    ResidentDeviceInfo& d = g_resident_info[device];
    if (!d.smem_optin) {
        int v = 0;
        if (cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, device) != cudaSuccess ||
            cudaFuncSetAttribute(batch_resident_kernel<kResidentBatchWpl>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, v - 1024) != cudaSuccess)
            return "device attribute";
        d.smem_optin = v;
    }
    *smem_optin = d.smem_optin;
    if (per_sm) {
        const size_t key = (std::max<size_t>(smem, 1) + 4095) / 4096 * 4096;
        auto it = d.per_sm.find(key);
        if (it == d.per_sm.end()) {
            int n = 0;
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                    &n, batch_resident_kernel<kResidentBatchWpl>, kResidentBatchThreads,
                    std::min<size_t>(key, (size_t)d.smem_optin - 1024)) != cudaSuccess)
                return "resident batch occupancy";
            it = d.per_sm.emplace(key, n).first;
        }
        *per_sm = it->second;
    }
    return nullptr;
}
} // namespace

const char* plan_resident_batch(const ResidentGrid* g, size_t n, int num_sms, int device,
                                ResidentBatchPlan* p) {
    int smem_optin = 0;
    if (const char* why = resident_device(device, 0, &smem_optin, nullptr)) return why;
    const size_t avail = (size_t)smem_optin - 1024;
    double total = 0;
    for (size_t i = 0; i < n; ++i) total += (double)g[i].W * g[i].Y * g[i].gens;
    std::vector<std::pair<double, ResidentBatchPlan::Grid>> order;
    size_t smem = 0;
    for (size_t i = 0; i < n; ++i) {
        const ResidentGrid& e = g[i];
        const int lanes = (e.W + kResidentBatchWpl - 1) / kResidentBatchWpl;
        if (lanes > kResidentBatchThreads) return "a grid is too wide for the resident batch";
        const int groups = kResidentBatchThreads / lanes;
        const int K = (int)std::min<long long>(e.gens, kResidentBatchK);
        const size_t row_bytes = 2ull * resident_stride(lanes, kResidentBatchWpl) * 4;
        const long long fit = (long long)(avail / row_bytes) - 2 * K;   // band rows that fit
        if (fit < 1) return "a grid's rows do not fit in shared memory";
        const int nb_min = (int)((e.Y + fit - 1) / fit);
        const double work = (double)e.W * e.Y * e.gens;
        const int nb_work = (int)std::ceil(work / std::max(1.0, total / ((double)num_sms *
                                                                          kResidentBatchBandsPerCta)));
        const int nb_rows = std::max(1, e.Y / std::max(K, kResidentBatchRowsPerGroup * groups));
        int nb = std::max(nb_min, std::min(nb_work, nb_rows));
        // at most one band per SM (every CTA may hold the largest shared
        // memory), every band at least K rows
        const int nb_cap = std::min(num_sms, std::max(1, e.Y / K));
        if (nb > nb_cap) {
            if (nb_min > nb_cap) return "a grid needs more bands than the GPU runs at once, or bands under K rows";
            nb = nb_cap;
        }
        const int B = (e.Y + nb - 1) / nb;
        smem = std::max(smem, (size_t)(B + 2 * K) * row_bytes);
        ResidentBatchPlan::Grid pg{(int)i, nb, K, lanes, groups, (e.W + 3) / 4 * 4, 0, 0};
        order.push_back({(double)e.W * B * e.gens, pg});
    }
    int per_sm = 0;
    if (const char* why = resident_device(device, smem, &smem_optin, &per_sm)) return why;
    if (per_sm < 1) return "resident batch kernel does not fit on an SM";
    const int ctas = per_sm * num_sms;
    std::stable_sort(order.begin(), order.end(),
                     [](const auto& a, const auto& c) { return a.first > c.first; });
    p->grids.clear();
    p->pub_words = 0;
    p->ndone = 0;
    for (auto& o : order) {
        if (o.second.nb > ctas) return "a grid needs more bands than CTAs";
        o.second.pub_off = p->pub_words;
        o.second.done_off = p->ndone;
        p->pub_words += (size_t)o.second.nb * 4 * o.second.K * o.second.ppitch;
        p->ndone += o.second.nb;
        p->grids.push_back(o.second);
    }
    p->smem = smem;
    p->ctas = ctas;
    return nullptr;
}

bool resident_batch_fits(int W, int Y, int num_sms, int device) {
    int smem_optin = 0;
    if (W <= 0 || Y <= 0 || resident_device(device, 0, &smem_optin, nullptr)) return false;
    const int lanes = (W + kResidentBatchWpl - 1) / kResidentBatchWpl;
    if (lanes > kResidentBatchThreads) return false;
    const size_t row_bytes = 2ull * resident_stride(lanes, kResidentBatchWpl) * 4;
    const long long fit = (long long)(((size_t)smem_optin - 1024) / row_bytes) - 2 * kResidentBatchK;
    if (fit < 1) return false;
    const long long nb_min = (Y + fit - 1) / fit;
    return nb_min <= std::min(num_sms, std::max(1, Y / kResidentBatchK));
}

void fill_resident_jobs(const ResidentBatchPlan& p, const ResidentGrid* g, uint32_t* pub, int* done,
                        ResidentBand* jobs) {
    int t = 0;
    for (const auto& pg : p.grids) {
        const ResidentGrid& e = g[pg.index];
        for (int band = 0; band < pg.nb; ++band) {
            ResidentBand& j = jobs[t++];
            j.src = e.src;
            j.dst = e.dst;
            j.pub = pub + pg.pub_off;
            j.done = done + pg.done_off;
            j.pitch = e.pitch;
            j.ppitch = pg.ppitch;
            j.W = e.W;
            j.Y = e.Y;
            j.K = pg.K;
            j.lanes = pg.lanes;
            j.groups = pg.groups;
            j.b = band;
            j.nb = pg.nb;
            j.gens = e.gens;
        }
    }
}

cudaError_t launch_batch_resident(const ResidentBand* jobs, int njobs, int* ticket, int* status,
                                  const ResidentBatchPlan& p, cudaStream_t stream) {
    // (the kernel's dynamic shared memory limit was raised when p was planned)
    long long spin = 1ll << 24;
    void* args[] = {&jobs, &njobs, &ticket, &status, &spin};
    return cudaLaunchCooperativeKernel((const void*)batch_resident_kernel<kResidentBatchWpl>,
                                       dim3(p.ctas), dim3(kResidentBatchThreads), args, p.smem, stream);
}

} // namespace golb200

struct gol_batch {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int num_sms = 148;

    struct Entry {
        uint64_t x, y, gens;
        int W, Y;
        std::vector<uint32_t> words;      // packed input (host)
        golb200::GridChoice choice{};
        int force_wpl = 0, force_k = 0, force_band = 0;
        size_t offset = 0;                // word offset of buf[0] in the arena
        int pitch = 0;                    // words per row on the device (W padded to wpl)
        size_t stride = 0;                // words from buf[0] to buf[1] (the input region's size)
        int result_buf = 0;               // buffer holding the last run's result
        int track_mode = GOL_TRACK_AUTO;  // gol_batch_set_tracking
        bool tracked = false;             // the uploaded plan tracks changes
        size_t trk_offset = 0;            // words into d_trk (tracked grids)
        size_t pstat_offset = 0;          // ints into d_pstat (tracked grids)
        int tile_rows_hint = 0;           // band height from the last retune (0: the planner's)
        int auto_track = -1;              // the last retune's choice in auto mode (-1: none yet)
    };
    std::vector<Entry> grids;

    // Arena: [every grid's buf[0] | every grid's buf[1] | a copy of the
    // inputs], each region input_words long. A run starts by restoring the
    // buf[0] region from the copy (one device-to-device copy).
    uint32_t* arena = nullptr;
    size_t arena_words = 0;
    size_t input_words = 0;
    BatchGrid* d_grids = nullptr;
    BatchItem* d_items = nullptr;
    int* d_done = nullptr;
    int* d_ticket = nullptr;
    int* d_status = nullptr;
    unsigned long long* d_census = nullptr;   // wait / work SM cycles, items computed / skipped
    uint32_t* d_trk = nullptr;            // change flags and still pass of the tracked grids
    size_t trk_words = 0;
    int* d_pstat = nullptr;               // per pass of each tracked grid: items done, changed
    size_t pstat_words = 0;
    uint32_t* d_gstat = nullptr;          // per grid: items computed, skipped
    bool track_any = false;
    int nitems = 0, ngroups_total = 0;
    int wpl_only = 0;                     // lane width shared by every grid (0: mixed)
    bool uploaded = false, ran = false;
    cudaGraphExec_t graph = nullptr;
    // Resident runs (gol_batch_run_resident): bands of every grid, their
    // exchange slots and epoch counters; built on the first such run after
    // an upload.
    golb200::ResidentBand* d_rjobs = nullptr;
    uint32_t* d_rpub = nullptr;
    int* d_rdone = nullptr;
    int rjobs = 0, rdone = 0, rctas = 0;
    size_t rsmem = 0;
    golb200::ResidentBatchPlan rplan;
    double last_ms = 0;
    std::string err;

    int fail(int code, const std::string& m) {
        err = m;
        return code;
    }
    int cuda_fail(cudaError_t e, const char* what) {
        err = std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
        return GOL_E_CUDA;
    }
};

namespace {

// Grids of at least this many passes track changes unless told otherwise
// (a short run has little time to settle).
constexpr int kTrackMinPasses = 8;
constexpr double kRetuneMinSkip = 0.05;    // skipped share below which a grid runs dense
constexpr double kRetuneFineSkip = 0.5;    // skipped share from which it gets the finest tiles
constexpr int kRetuneFineRows = 16;        // the planner's smallest band
// Time of an item under the tracked kernel over the untracked one (the
// settling variant of the 512-grid workload: 65.2 ms for 3.51 M computed
// items against 52.5 ms for 3.56 M untracked ones).
constexpr double kTrackItemCost = 1.25;

int forced_band(const gol_batch::Entry& e) { return e.force_band ? e.force_band : e.tile_rows_hint; }

void batch_free_device(gol_batch* b) {
    if (b->graph) cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
    for (void* p : {(void*)b->d_rjobs, (void*)b->d_rpub, (void*)b->d_rdone})
        if (p) cudaFree(p);
    b->d_rjobs = nullptr;
    b->d_rpub = nullptr;
    b->d_rdone = nullptr;
    b->rjobs = b->rdone = b->rctas = 0;
    b->rsmem = 0;
    for (void* p : {(void*)b->arena, (void*)b->d_grids, (void*)b->d_items, (void*)b->d_done,
                    (void*)b->d_ticket, (void*)b->d_status, (void*)b->d_census, (void*)b->d_trk,
                    (void*)b->d_pstat, (void*)b->d_gstat})
        if (p) cudaFree(p);
    b->d_trk = nullptr;
    b->d_pstat = nullptr;
    b->d_gstat = nullptr;
    b->arena = nullptr;
    b->d_grids = nullptr;
    b->d_items = nullptr;
    b->d_done = nullptr;
    b->d_ticket = nullptr;
    b->d_status = nullptr;
    b->d_census = nullptr;
    b->uploaded = false;
}

} // namespace

extern "C" {

int gol_batch_create(gol_batch** out, int32_t device, void* stream) {
    if (!out) return GOL_E_INVALID;
    gol_batch* b = new (std::nothrow) gol_batch();
    if (!b) return GOL_E_NOMEM;
    b->device = device;
    cudaError_t ce = cudaSetDevice(device);
    if (ce == cudaSuccess) {
        if (stream) {
            b->stream = static_cast<cudaStream_t>(stream);
        } else {
            ce = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
            b->own_stream = ce == cudaSuccess;
        }
    }
    if (ce != cudaSuccess) {
        delete b;
        return GOL_E_CUDA;
    }
    b->num_sms = golb200::device_sm_count(device);
    *out = b;
    return GOL_OK;
}

int gol_batch_add(gol_batch* b, const uint8_t* cells, uint64_t x, uint64_t y, uint64_t generations,
                  int32_t* grid_id) {
    if (!b) return GOL_E_INVALID;
    if (x == 0 || y == 0 || x % 32) return b->fail(GOL_E_INVALID, "x must be a positive multiple of 32");
    if (y > (1u << 30) || generations > (1ull << 31))
        return b->fail(GOL_E_INVALID, "grid or generation count too large");
    if (!cells) return b->fail(GOL_E_INVALID, "null cells");
    gol_batch::Entry e;
    e.x = x;
    e.y = y;
    e.gens = generations;
    e.W = (int)(x / 32);
    e.Y = (int)y;
    e.words.resize((size_t)e.W * e.Y);
    golb200::host_pack_u8(cells, x, y, e.words.data());
    b->grids.push_back(std::move(e));
    b->uploaded = false;
    if (grid_id) *grid_id = (int32_t)b->grids.size() - 1;
    return GOL_OK;
}

int gol_batch_set_plan(gol_batch* b, int32_t grid_id, uint32_t lane_words, uint32_t temporal_steps,
                       uint32_t band_rows) {
    if (!b || grid_id < 0 || grid_id >= (int)b->grids.size()) return GOL_E_INVALID;
    if (temporal_steps > golb200::kBatchMaxK) return b->fail(GOL_E_INVALID, "temporal_steps > 4");
    auto& e = b->grids[grid_id];
    e.force_wpl = (int)lane_words;
    e.force_k = (int)temporal_steps;
    e.force_band = (int)band_rows;
    b->uploaded = false;
    return GOL_OK;
}

int gol_batch_plan(const gol_batch* b, int32_t grid_id, uint32_t* lane_words,
                   uint32_t* temporal_steps, uint32_t* band_rows, uint32_t* segments) {
    if (!b || grid_id < 0 || grid_id >= (int)b->grids.size()) return GOL_E_INVALID;
    const auto& e = b->grids[grid_id];
    golb200::GridChoice ch = e.choice;   // the uploaded batch's plan
    if (!b->uploaded &&
        !golb200::choose_batch_plan(e.W, e.Y, e.gens, e.force_wpl, e.force_k, e.force_band, &ch))
        return GOL_E_UNSUPPORTED;
    if (lane_words) *lane_words = ch.wpl;
    if (temporal_steps) *temporal_steps = ch.k;
    if (band_rows) *band_rows = ch.band;
    if (segments) *segments = ch.segs;
    return GOL_OK;
}

// Plans every grid, uploads inputs and the work list (host -> device).
int gol_batch_upload(gol_batch* b) {
    if (!b) return GOL_E_INVALID;
    cudaError_t ce = cudaSetDevice(b->device);
    if (ce != cudaSuccess) return b->cuda_fail(ce, "cudaSetDevice");
    batch_free_device(b);
    std::vector<BatchGrid> hg;
    size_t words = 0;
    int groups = 0, max_passes = 0;
    // Plans: for every (words per lane, depth) all grids can use, each grid
    // takes its least-work band, then grids whose chain would outlast the
    // work-bound time of the whole batch take shorter chains; the pair with
    // the smallest max(work / resident warps, longest chain) wins. Grids with
    // a plan forced by gol_batch_set_plan keep it.
    // Units: a work item's cost is warp time at the variant's occupancy
    // (per-word costs are calibrated on whole batches), so a batch needs
    // about max(total / num_sms, longest chain * warps per SM) SM time.
    double best_est = -1, parallel = 1;
    std::vector<golb200::GridChoice> best;
    for (int wpl : {4, 2, 1}) {
        const double wps = golb200::batch_kernel_ctas_per_sm(wpl);
        const double par = (double)b->num_sms * wps;
        for (int k = golb200::kBatchMaxK; k >= 1; --k) {
            std::vector<golb200::GridChoice> ch(b->grids.size());
            double total_work = 0;
            bool ok = true;
            for (size_t i = 0; i < b->grids.size() && ok; ++i) {
                const auto& e = b->grids[i];
                ok = golb200::choose_batch_plan(e.W, e.Y, std::max<uint64_t>(e.gens, 1),
                                                e.force_wpl ? e.force_wpl : wpl,
                                                e.force_k ? e.force_k : k, forced_band(e), &ch[i]);
                total_work += ok && e.gens ? ch[i].cost : 0;
            }
            if (!ok) continue;
            const double work_time = total_work / par;
            double chain = 0;
            for (size_t i = 0; i < b->grids.size(); ++i) {
                const auto& e = b->grids[i];
                if (ch[i].crit > GOL_BATCH_REPLAN * work_time && !forced_band(e))
                    golb200::choose_batch_plan(e.W, e.Y, std::max<uint64_t>(e.gens, 1),
                                               e.force_wpl ? e.force_wpl : wpl,
                                               e.force_k ? e.force_k : k, forced_band(e), &ch[i],
                                               par, 1.0);
                if (e.gens) chain = std::max(chain, ch[i].crit);
            }
            double total2 = 0;
            for (size_t i = 0; i < b->grids.size(); ++i)
                if (b->grids[i].gens) total2 += ch[i].cost;
            const double est = wps * std::max(total2 / par, chain);
            if (best_est < 0 || est < best_est) {
                best_est = est;
                parallel = par;
                best = std::move(ch);
            }
        }
    }
    if (best_est < 0) return b->fail(GOL_E_UNSUPPORTED, "no batched plan for a grid");
    for (size_t i = 0; i < b->grids.size(); ++i) b->grids[i].choice = best[i];
    // A first pass with fewer items than about two per resident warp leaves
    // SMs idle on every pass: halve the tallest bands (not below 16 rows)
    // until it has enough items.
    for (int round = 0; round < 3; ++round) {
        double first_pass = 0;
        int tallest = 0;
        for (const auto& e : b->grids) {
            if (e.gens == 0) continue;
            first_pass += (double)e.choice.ngroups * e.choice.nslices;
            tallest = std::max(tallest, e.choice.band);
        }
        if (first_pass >= 2 * parallel || tallest <= 16) break;
        for (auto& e : b->grids) {
            if (e.gens == 0 || forced_band(e) || e.choice.band != tallest) continue;
            golb200::GridChoice c2;
            if (golb200::choose_batch_plan(e.W, e.Y, std::max<uint64_t>(e.gens, 1), e.choice.wpl,
                                           e.choice.k, std::max(16, tallest / 2), &c2))
                e.choice = c2;
        }
    }
    size_t trk_words = 0, pstat_words = 0;
    b->track_any = false;
    for (auto& e : b->grids) {
        if (e.gens == 0) e.choice.passes = 0;
        // Every buffer starts on a 256-byte boundary: lanes move up to 16
        // bytes at once (uint4 / 16-byte cp.async), whatever the grid sizes.
        BatchGrid g{};
        golb200::batch_grid_from_choice(e.choice, e.W, e.Y, &g);
        e.pitch = g.pitch;
        e.offset = words;
        words += ((size_t)g.pitch * e.Y + 63) / 64 * 64;
        g.parity0 = 0;
        g.done_base = groups;
        groups += g.ngroups * g.nslices;
        max_passes = std::max(max_passes, g.passes);
        // Change tracking: on or off as set, else (auto) the last retune's
        // choice, else on for grids of at least kTrackMinPasses passes.
        e.tracked = g.passes > 0 &&
                    (e.track_mode == GOL_TRACK_ON ||
                     (e.track_mode == GOL_TRACK_AUTO &&
                      (e.auto_track >= 0 ? e.auto_track == 1 : g.passes >= kTrackMinPasses)));
        if (e.tracked) {
            e.trk_offset = trk_words;
            trk_words += golb200::batch_trk_words(g.ngroups, g.nslices);
            e.pstat_offset = pstat_words;
            pstat_words += 2 * (size_t)g.passes;
            b->track_any = true;
        }
        hg.push_back(g);
    }
    b->trk_words = trk_words;
    b->pstat_words = pstat_words;
    std::vector<BatchItem> items(golb200::count_batch_items(hg.data(), hg.size()));
    golb200::order_batch_items(hg.data(), hg.size(), items.data());
    b->nitems = (int)items.size();
    b->ngroups_total = groups;
    b->wpl_only = golb200::batch_uniform_wpl(hg.data(), hg.size());
    b->input_words = words;
    b->arena_words = 3 * words;
    for (auto& e : b->grids) e.stride = words;
    ce = cudaMalloc(&b->arena, std::max<size_t>(b->arena_words, 1) * sizeof(uint32_t));
    if (ce == cudaSuccess) ce = cudaMalloc(&b->d_grids, std::max<size_t>(hg.size(), 1) * sizeof(BatchGrid));
    if (ce == cudaSuccess) ce = cudaMalloc(&b->d_items, std::max<size_t>(items.size(), 1) * sizeof(BatchItem));
    if (ce == cudaSuccess) ce = cudaMalloc(&b->d_done, std::max(groups, 1) * sizeof(int));
    if (ce == cudaSuccess) ce = cudaMalloc(&b->d_ticket, sizeof(int));
    if (ce == cudaSuccess) ce = cudaMalloc(&b->d_status, sizeof(int));
    if (ce == cudaSuccess) ce = cudaMalloc(&b->d_census, 4 * sizeof(unsigned long long));
    if (ce == cudaSuccess) ce = cudaMalloc(&b->d_trk, std::max<size_t>(trk_words, 1) * sizeof(uint32_t));
    if (ce == cudaSuccess) ce = cudaMalloc(&b->d_pstat, std::max<size_t>(pstat_words, 1) * sizeof(int));
    if (ce == cudaSuccess) ce = cudaMalloc(&b->d_gstat, std::max<size_t>(2 * hg.size(), 1) * sizeof(uint32_t));
    if (ce != cudaSuccess) {
        batch_free_device(b);
        return ce == cudaErrorMemoryAllocation ? b->fail(GOL_E_NOMEM, "device allocation failed")
                                               : b->cuda_fail(ce, "cudaMalloc");
    }
    // Padding words past W must read as dead: the arena starts zeroed.
    ce = cudaMemsetAsync(b->arena, 0, std::max<size_t>(b->arena_words, 1) * sizeof(uint32_t), b->stream);
    for (size_t gi = 0; gi < hg.size() && ce == cudaSuccess; ++gi) {
        auto& e = b->grids[gi];
        hg[gi].buf[0] = b->arena + e.offset;
        hg[gi].buf[1] = b->arena + e.offset + e.stride;
        hg[gi].gstat = b->d_gstat + 2 * gi;
        if (e.tracked) {
            hg[gi].trk = b->d_trk + e.trk_offset;
            hg[gi].pstat = b->d_pstat + e.pstat_offset;
        }
        if (e.W == 0 || e.Y == 0) continue;
        ce = cudaMemcpy2DAsync(hg[gi].buf[0], (size_t)e.pitch * sizeof(uint32_t), e.words.data(),
                               (size_t)e.W * sizeof(uint32_t), (size_t)e.W * sizeof(uint32_t), e.Y,
                               cudaMemcpyHostToDevice, b->stream);
    }
    if (ce == cudaSuccess && words)
        ce = cudaMemcpyAsync(b->arena + 2 * words, b->arena, words * sizeof(uint32_t),
                             cudaMemcpyDeviceToDevice, b->stream);
    if (ce == cudaSuccess)
        ce = cudaMemcpyAsync(b->d_grids, hg.data(), hg.size() * sizeof(BatchGrid),
                             cudaMemcpyHostToDevice, b->stream);
    if (ce == cudaSuccess && !items.empty())
        ce = cudaMemcpyAsync(b->d_items, items.data(), items.size() * sizeof(BatchItem),
                             cudaMemcpyHostToDevice, b->stream);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(b->stream);
    if (ce != cudaSuccess) {
        batch_free_device(b);
        return b->cuda_fail(ce, "batch upload");
    }
    b->uploaded = true;
    b->ran = false;
    return GOL_OK;
}

// Restores every grid's buf[0] from the device copy of the inputs.
static cudaError_t batch_restore_inputs(gol_batch* b, cudaStream_t s) {
    if (!b->input_words) return cudaSuccess;
    return cudaMemcpyAsync(b->arena, b->arena + 2 * b->input_words,
                           b->input_words * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s);
}

static int batch_reset_inputs(gol_batch* b) {
    cudaError_t ce = batch_restore_inputs(b, b->stream);
    return ce == cudaSuccess ? GOL_OK : b->cuda_fail(ce, "batch input restore");
}

// All grids, all generations: one persistent launch, captured once as a
// CUDA graph together with the input restore (device-to-device) and the
// counter resets. Asynchronous; gol_batch_sync waits and reports a timeout
// recorded by the kernel.
int gol_batch_run(gol_batch* b) {
    if (!b) return GOL_E_INVALID;
    int rc;
    if (!b->uploaded && (rc = gol_batch_upload(b))) return rc;
    if (!b->graph) {
        cudaStream_t cs = nullptr;
        cudaError_t ce = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
        if (ce != cudaSuccess) return b->cuda_fail(ce, "capture stream");
        ce = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
        if (ce == cudaSuccess) ce = batch_restore_inputs(b, cs);
        if (ce == cudaSuccess) ce = cudaMemsetAsync(b->d_done, 0, std::max(b->ngroups_total, 1) * sizeof(int), cs);
        if (ce == cudaSuccess) ce = cudaMemsetAsync(b->d_ticket, 0, sizeof(int), cs);
        if (ce == cudaSuccess) ce = cudaMemsetAsync(b->d_status, 0, sizeof(int), cs);
        if (ce == cudaSuccess) ce = cudaMemsetAsync(b->d_census, 0, 4 * sizeof(unsigned long long), cs);
        // change tracking: every flag "changed" (the first pass computes
        // everything), no still pass, counters zero
        if (ce == cudaSuccess && b->trk_words)
            ce = cudaMemsetAsync(b->d_trk, 0xff, b->trk_words * sizeof(uint32_t), cs);
        if (ce == cudaSuccess && b->pstat_words)
            ce = cudaMemsetAsync(b->d_pstat, 0, b->pstat_words * sizeof(int), cs);
        if (ce == cudaSuccess)
            ce = cudaMemsetAsync(b->d_gstat, 0, std::max<size_t>(2 * b->grids.size(), 1) * sizeof(uint32_t), cs);
        if (ce == cudaSuccess)
            ce = golb200::launch_batch_kernel(b->d_grids, b->d_items, b->nitems, b->d_ticket,
                                              b->d_done, b->d_status, b->num_sms, cs, b->d_census,
                                              b->wpl_only, 0, b->track_any);
        cudaGraph_t g = nullptr;
        cudaError_t ce2 = cudaStreamEndCapture(cs, &g);
        if (ce == cudaSuccess) ce = ce2;
        if (ce == cudaSuccess) ce = cudaGraphInstantiate(&b->graph, g, 0);
        if (g) cudaGraphDestroy(g);
        cudaStreamDestroy(cs);
        if (ce != cudaSuccess) return b->cuda_fail(ce, "batch graph");
    }
    cudaError_t ce = cudaGraphLaunch(b->graph, b->stream);
    if (ce != cudaSuccess) return b->cuda_fail(ce, "batch launch");
    for (auto& e : b->grids) e.result_buf = e.choice.passes & 1;
    b->ran = true;
    return GOL_OK;
}

int gol_batch_sync(gol_batch* b) {
    if (!b) return GOL_E_INVALID;
    cudaError_t ce = cudaStreamSynchronize(b->stream);
    if (ce != cudaSuccess) return b->cuda_fail(ce, "batch synchronize");
    if (b->d_status) {
        int st = 0;
        ce = cudaMemcpy(&st, b->d_status, sizeof(int), cudaMemcpyDeviceToHost);
        if (ce != cudaSuccess) return b->cuda_fail(ce, "batch status");
        if (st != 0) return b->fail(st, "batched kernel gave up waiting on a dependency");
    }
    return GOL_OK;
}

// Baseline: the same grids with the single-grid path, one after another:
// every grid gets its own kernel launches (one per k-generation pass), as a
// caller of the one-grid contract would run them.
int gol_batch_run_plain(gol_batch* b, uint32_t temporal_steps) {
    if (!b) return GOL_E_INVALID;
    int rc;
    if (!b->uploaded && (rc = gol_batch_upload(b))) return rc;
    if ((rc = batch_reset_inputs(b))) return rc;
    const int k0 = temporal_steps ? (int)temporal_steps : 4;
    for (auto& e : b->grids) {
        uint32_t* buf[2] = {b->arena + e.offset, b->arena + e.offset + e.stride};
        int cur = 0;
        uint64_t left = e.gens;
        while (left > 0) {
            const int k = (int)std::min<uint64_t>(left, (uint64_t)k0);
            golb200::RowsPlan p;
            if (!golb200::plan_rows(e.W, e.Y, k, 0, 0, b->num_sms, &p))
                return b->fail(GOL_E_UNSUPPORTED, "no plan");
            cudaError_t ce = golb200::launch_rows_pass(buf[cur], buf[cur ^ 1], e.W, e.Y, k, p,
                                                       b->stream, e.pitch);
            if (ce != cudaSuccess) return b->cuda_fail(ce, "plain launch");
            cur ^= 1;
            left -= k;
        }
        e.result_buf = cur;
    }
    b->ran = true;
    return GOL_OK;
}

// Every grid's bands kept in shared memory for all their generations (the
// single-grid resident run's algorithm), persistent CTAs taking bands in
// ticket order. Asynchronous like gol_batch_run; results in buf[1].
int gol_batch_run_resident(gol_batch* b) {
    if (!b) return GOL_E_INVALID;
    int rc;
    if (!b->uploaded && (rc = gol_batch_upload(b))) return rc;
    if (!b->d_rjobs) {   // plan the bands once per upload
        std::vector<golb200::ResidentGrid> rg;
        for (const auto& e : b->grids)
            if (e.gens && e.W && e.Y)
                rg.push_back({b->arena + e.offset, b->arena + e.offset + e.stride, e.pitch, e.W, e.Y,
                              (long long)e.gens});
        golb200::ResidentBatchPlan plan;
        if (const char* why = golb200::plan_resident_batch(rg.data(), rg.size(), b->num_sms,
                                                           b->device, &plan))
            return b->fail(GOL_E_UNSUPPORTED, why);
        cudaError_t ce = cudaMalloc(&b->d_rpub, std::max<size_t>(plan.pub_words, 1) * sizeof(uint32_t));
        if (ce == cudaSuccess) ce = cudaMalloc(&b->d_rdone, std::max(plan.ndone, 1) * sizeof(int));
        if (ce == cudaSuccess)
            ce = cudaMalloc(&b->d_rjobs, std::max(plan.ndone, 1) * sizeof(golb200::ResidentBand));
        if (ce != cudaSuccess) return b->cuda_fail(ce, "resident batch scratch");
        std::vector<golb200::ResidentBand> jobs(plan.ndone);
        golb200::fill_resident_jobs(plan, rg.data(), b->d_rpub, b->d_rdone, jobs.data());
        ce = cudaMemcpyAsync(b->d_rjobs, jobs.data(), jobs.size() * sizeof(golb200::ResidentBand),
                             cudaMemcpyHostToDevice, b->stream);
        if (ce == cudaSuccess) ce = cudaStreamSynchronize(b->stream);
        if (ce != cudaSuccess) return b->cuda_fail(ce, "resident batch bands");
        b->rplan = plan;
        b->rjobs = plan.ndone;
        b->rdone = plan.ndone;
        b->rctas = plan.ctas;
        b->rsmem = plan.smem;
    }
    cudaError_t ce = batch_restore_inputs(b, b->stream);
    // grids with no generations: the result is the input
    for (auto& e : b->grids)
        if (ce == cudaSuccess && e.gens == 0 && e.W && e.Y)
            ce = cudaMemcpyAsync(b->arena + e.offset + e.stride, b->arena + e.offset,
                                 (size_t)e.pitch * e.Y * sizeof(uint32_t), cudaMemcpyDeviceToDevice,
                                 b->stream);
    if (ce == cudaSuccess) ce = cudaMemsetAsync(b->d_rdone, 0, std::max(b->rdone, 1) * sizeof(int), b->stream);
    if (ce == cudaSuccess) ce = cudaMemsetAsync(b->d_ticket, 0, sizeof(int), b->stream);
    if (ce == cudaSuccess) ce = cudaMemsetAsync(b->d_status, 0, sizeof(int), b->stream);
    if (ce == cudaSuccess && b->rjobs)
        ce = golb200::launch_batch_resident(b->d_rjobs, b->rjobs, b->d_ticket, b->d_status, b->rplan,
                                            b->stream);
    if (ce != cudaSuccess) return b->cuda_fail(ce, "resident batch launch");
    for (auto& e : b->grids) e.result_buf = 1;
    b->ran = true;
    return GOL_OK;
}

int gol_batch_resident_info(const gol_batch* b, uint64_t* bands, uint32_t* ctas, uint64_t* smem_bytes) {
    if (!b) return GOL_E_INVALID;
    if (bands) *bands = (uint64_t)b->rjobs;
    if (ctas) *ctas = (uint32_t)b->rctas;
    if (smem_bytes) *smem_bytes = (uint64_t)b->rsmem;
    return GOL_OK;
}

int gol_batch_fetch(gol_batch* b, int32_t grid_id, uint8_t* cells) {
    if (!b || grid_id < 0 || grid_id >= (int)b->grids.size() || !cells) return GOL_E_INVALID;
    if (!b->uploaded) return b->fail(GOL_E_STATE, "fetch before run");
    auto& e = b->grids[grid_id];
    const int which = e.result_buf;
    std::vector<uint32_t> words((size_t)e.W * e.Y);
    cudaError_t ce = cudaSuccess;
    if (!words.empty())
        ce = cudaMemcpy2DAsync(words.data(), (size_t)e.W * sizeof(uint32_t),
                               b->arena + e.offset + (size_t)which * e.stride,
                               (size_t)e.pitch * sizeof(uint32_t), (size_t)e.W * sizeof(uint32_t),
                               e.Y, cudaMemcpyDeviceToHost, b->stream);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(b->stream);
    if (ce != cudaSuccess) return b->cuda_fail(ce, "batch fetch");
    golb200::host_unpack_u8(words.data(), e.x, e.y, cells);
    return GOL_OK;
}

int gol_batch_info(const gol_batch* b, uint64_t* grids, uint64_t* items, uint64_t* cell_updates) {
    if (!b) return GOL_E_INVALID;
    uint64_t cu = 0;
    for (const auto& e : b->grids) cu += e.x * e.y * e.gens;
    if (grids) *grids = b->grids.size();
    if (items) *items = (uint64_t)b->nitems;
    if (cell_updates) *cell_updates = cu;
    return GOL_OK;
}

// Exercises the dependency-wait guard without a fault: a work list whose
// only item (pass 1 of a one-word grid) depends on pass 0, which is not in
// the list, so its wait must give up after spin_limit polls, record
// GOL_E_TIMEOUT in the status word and end the launch normally.
int gol_batch_probe_timeout(int32_t device, uint64_t spin_limit, int32_t* status_out) {
    if (!status_out || spin_limit == 0 || spin_limit > (1ull << 24)) return GOL_E_INVALID;
    *status_out = 0;
    if (cudaSetDevice(device) != cudaSuccess) return GOL_E_CUDA;
    golb200::GridChoice ch;
    if (!golb200::choose_batch_plan(1, 32, 2, 1, 1, 16, &ch)) return GOL_E_UNSUPPORTED;
    BatchGrid g{};
    golb200::batch_grid_from_choice(ch, 1, 32, &g);
    const BatchItem item{0, 0, 0, 1};
    const int ncount = g.ngroups * g.nslices;
    uint32_t* bufs = nullptr;
    BatchGrid* d_grid = nullptr;
    BatchItem* d_item = nullptr;
    int* d_ints = nullptr;   // done[ncount], ticket, status
    cudaStream_t s = nullptr;
    cudaError_t ce = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    if (ce == cudaSuccess) ce = cudaMalloc(&bufs, 2 * 32 * sizeof(uint32_t));
    if (ce == cudaSuccess) ce = cudaMalloc(&d_grid, sizeof(BatchGrid));
    if (ce == cudaSuccess) ce = cudaMalloc(&d_item, sizeof(BatchItem));
    if (ce == cudaSuccess) ce = cudaMalloc(&d_ints, (ncount + 2) * sizeof(int));
    if (ce == cudaSuccess) {
        g.buf[0] = bufs;
        g.buf[1] = bufs + 32;
        ce = cudaMemsetAsync(bufs, 0, 2 * 32 * sizeof(uint32_t), s);
    }
    if (ce == cudaSuccess) ce = cudaMemsetAsync(d_ints, 0, (ncount + 2) * sizeof(int), s);
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(d_grid, &g, sizeof(g), cudaMemcpyHostToDevice, s);
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(d_item, &item, sizeof(item), cudaMemcpyHostToDevice, s);
    if (ce == cudaSuccess)
        ce = golb200::launch_batch_kernel(d_grid, d_item, 1, d_ints + ncount, d_ints, d_ints + ncount + 1,
                                          1, s, nullptr, g.wpl, (long long)spin_limit);
    int st = 0;
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(&st, d_ints + ncount + 1, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(s);
    for (void* p : {(void*)bufs, (void*)d_grid, (void*)d_item, (void*)d_ints})
        if (p) cudaFree(p);
    if (s) cudaStreamDestroy(s);
    if (ce != cudaSuccess) return GOL_E_CUDA;
    *status_out = st;
    return GOL_OK;
}

// Cycles the last run's work items spent waiting on their dependencies and
// computing, summed over items (SM clock cycles).
int gol_batch_census(gol_batch* b, uint64_t* wait_cycles, uint64_t* work_cycles) {
    if (!b || !b->d_census) return GOL_E_INVALID;
    unsigned long long c[2] = {0, 0};
    cudaError_t ce = cudaStreamSynchronize(b->stream);
    if (ce == cudaSuccess) ce = cudaMemcpy(c, b->d_census, sizeof(c), cudaMemcpyDeviceToHost);
    if (ce != cudaSuccess) return b->cuda_fail(ce, "batch census");
    if (wait_cycles) *wait_cycles = c[0];
    if (work_cycles) *work_cycles = c[1];
    return GOL_OK;
}

int gol_batch_set_tracking(gol_batch* b, int32_t grid_id, int32_t mode) {
    if (!b || grid_id < 0 || grid_id >= (int)b->grids.size()) return GOL_E_INVALID;
    if (mode != GOL_TRACK_AUTO && mode != GOL_TRACK_OFF && mode != GOL_TRACK_ON)
        return b->fail(GOL_E_INVALID, "tracking mode must be GOL_TRACK_AUTO, _OFF or _ON");
    b->grids[grid_id].track_mode = mode;
    b->uploaded = false;
    return GOL_OK;
}

// The autotuner's second look: each grid in auto mode keeps change tracking
// if the last run skipped a useful share of its items (at least
// kRetuneMinSkip; below that the comparisons cost more than they save),
// and a grid that skipped most of its items gets the finest tiles
// (kRetuneFineRows-row bands). The next run re-plans and re-uploads.
int gol_batch_retune(gol_batch* b) {
    if (!b) return GOL_E_INVALID;
    if (!b->uploaded || !b->ran) return b->fail(GOL_E_STATE, "retune needs a batched run first");
    std::vector<uint32_t> st(2 * b->grids.size());
    cudaError_t ce = cudaStreamSynchronize(b->stream);
    if (ce == cudaSuccess && !st.empty())
        ce = cudaMemcpy(st.data(), b->d_gstat, st.size() * sizeof(uint32_t), cudaMemcpyDeviceToHost);
    if (ce != cudaSuccess) return b->cuda_fail(ce, "batch retune");
    // Per grid: keep tracking where it skipped enough of the grid's items.
    // Then for the batch: a launch with any tracked grid runs the tracked
    // kernel for every item, at kTrackItemCost times an untracked item's
    // time, so tracking stays on only if the items it skips pay for that.
    double with_tracking = 0, without = 0;
    bool forced = false;
    for (size_t i = 0; i < b->grids.size(); ++i) {
        auto& e = b->grids[i];
        const double computed = st[2 * i], total = (double)st[2 * i] + st[2 * i + 1];
        without += total;
        forced |= e.track_mode == GOL_TRACK_ON && e.choice.passes > 0;
        if (e.track_mode != GOL_TRACK_AUTO || !e.tracked || total <= 0) {
            with_tracking += kTrackItemCost * (e.tracked ? computed : total);
            continue;
        }
        const double skip = st[2 * i + 1] / total;
        e.auto_track = skip >= kRetuneMinSkip ? 1 : 0;
        e.tile_rows_hint = (e.auto_track == 1 && skip >= kRetuneFineSkip) ? kRetuneFineRows : 0;
        with_tracking += kTrackItemCost * (e.auto_track ? computed : total);
    }
    if (!forced && with_tracking >= without)
        for (auto& e : b->grids)
            if (e.track_mode == GOL_TRACK_AUTO) {
                e.auto_track = 0;
                e.tile_rows_hint = 0;
            }
    b->uploaded = false;
    return GOL_OK;
}

int gol_batch_tiles(gol_batch* b, uint64_t* computed, uint64_t* skipped) {
    if (!b || !b->d_census) return GOL_E_INVALID;
    unsigned long long c[4] = {0, 0, 0, 0};
    cudaError_t ce = cudaStreamSynchronize(b->stream);
    if (ce == cudaSuccess) ce = cudaMemcpy(c, b->d_census, sizeof(c), cudaMemcpyDeviceToHost);
    if (ce != cudaSuccess) return b->cuda_fail(ce, "batch census");
    if (computed) *computed = c[2];
    if (skipped) *skipped = c[3];
    return GOL_OK;
}

int gol_batch_grid_stats(gol_batch* b, int32_t grid_id, uint32_t* tracked, uint32_t* computed,
                         uint32_t* skipped, uint32_t* still_pass) {
    if (!b || grid_id < 0 || grid_id >= (int)b->grids.size()) return GOL_E_INVALID;
    if (!b->uploaded || !b->ran) return b->fail(GOL_E_STATE, "no batched run yet");
    const auto& e = b->grids[grid_id];
    uint32_t st[2] = {0, 0}, still = 0xffffffffu;
    cudaError_t ce = cudaStreamSynchronize(b->stream);
    if (ce == cudaSuccess)
        ce = cudaMemcpy(st, b->d_gstat + 2 * (size_t)grid_id, sizeof(st), cudaMemcpyDeviceToHost);
    if (ce == cudaSuccess && e.tracked)
        ce = cudaMemcpy(&still, b->d_trk + e.trk_offset + 2 * (size_t)e.choice.ngroups * e.choice.nslices,
                        sizeof(still), cudaMemcpyDeviceToHost);
    if (ce != cudaSuccess) return b->cuda_fail(ce, "batch grid stats");
    if (tracked) *tracked = e.tracked ? 1u : 0u;
    if (computed) *computed = st[0];
    if (skipped) *skipped = st[1];
    if (still_pass) *still_pass = still;
    return GOL_OK;
}

void* gol_batch_stream(gol_batch* b) { return b ? static_cast<void*>(b->stream) : nullptr; }

const char* gol_batch_last_error(const gol_batch* b) { return b ? b->err.c_str() : "null batch"; }

void gol_batch_destroy(gol_batch* b) {
    if (!b) return;
    if (b->stream) cudaStreamSynchronize(b->stream);
    batch_free_device(b);
    if (b->own_stream && b->stream) cudaStreamDestroy(b->stream);
    delete b;
}

} // extern "C"
