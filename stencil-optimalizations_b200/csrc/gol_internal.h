// Internal declarations shared by the engine's translation units.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <vector>

namespace golb200 {

// Largest temporal depth instantiated for a given words-per-lane width.
// The register rings grow as 8 * K * WPL words per thread, so K * WPL <= 16
// keeps them well inside 255 registers.
constexpr int kMaxKForWpl(int wpl) { return wpl == 4 ? 4 : (wpl == 2 ? 8 : 16); }
constexpr int kMaxTemporalSteps = 16;

struct RowsPlan {
    int wpl = 0;       // 32-bit words per lane: 4, 2 or 1
    int threads = 0;   // CTA size
    int band = 0;      // output rows per CTA
    int nbands = 0;    // CTAs along y
    int slice = 0;     // words per x-slice (= W when one CTA spans the row)
    int nslices = 0;   // CTAs along x
    int halo = 0;      // x-halo words each side of a slice (0 when unsliced)
    bool stream = false;   // k = 1 streaming kernel (gol_rows_stream.cuh): band = rows
                           // per thread, nslices = CTAs across the row, no halo
};

// Picks words-per-lane and CTA shape for a W-word by Y-row grid and depth k.
// wpl = 0 chooses the widest lane access whose rings fit k; 1, 2 or 4 forces
// it. Returns false for k outside 1..16 or a wpl that W or k rules out.
// k = 1 plans the streaming kernel (band_rows = rows per thread, 0 = auto)
// unless allow_stream is false (callers that need the K-stage geometry).
bool plan_rows(int W, int Y, int k, int band_rows, int wpl, int num_sms, RowsPlan* plan,
               bool allow_stream = true);

// Shared-memory-resident run (gol_rows_resident.cuh): every generation of
// a grid whose bands fit in the SMs' shared memory, in one cooperative
// launch of one CTA per band.
// One band of one grid, all generations, in one CTA's shared memory
// (resident_band in gol_rows_resident.cuh).
struct ResidentBand {
    const uint32_t* src;   // the grid at generation 0 (row r at src + r * pitch)
    uint32_t* dst;         // the grid after `gens` generations (not src)
    uint32_t* pub;         // the grid's exchange slots: band b's at (b * 4 + parity * 2 + side)
                           // * K * ppitch words (side 0: its top K rows, 1: its bottom K rows)
    int* done;             // the grid's epoch counters, one per band, zero at start
    int pitch;             // words from one grid row to the next (>= W)
    int ppitch;            // words per row in the exchange slots (>= W, a multiple of 4)
    int W, Y;              // words per row, rows
    int K;                 // generations per epoch
    int lanes, groups;     // threads: lanes across a row x row groups
    int b, nb;             // this band, bands of the grid (rows split evenly)
    long long gens;
};

// A grid of a resident batch launch (batch_resident_kernel).
struct ResidentGrid {
    const uint32_t* src;
    uint32_t* dst;
    int pitch, W, Y;
    long long gens;        // > 0
};

// The bands of a resident batch: per grid its band count, epoch length,
// lanes and row groups, in launch order (longest band first, a grid's bands
// consecutive); the exchange slots, counters and shared memory they need and
// the CTAs the launch runs.
struct ResidentBatchPlan {
    struct Grid {
        int index;             // into the ResidentGrid list
        int nb, K, lanes, groups, ppitch;
        size_t pub_off;        // words into the exchange slots
        int done_off;          // ints into the counters
    };
    std::vector<Grid> grids;
    size_t smem = 0, pub_words = 0;
    int ndone = 0;             // bands in all
    int ctas = 0;
};
// Plans grids g[0..n) (every gens > 0); nullptr or why they cannot run.
const char* plan_resident_batch(const ResidentGrid* g, size_t n, int num_sms, int device,
                                ResidentBatchPlan* p);
// Whether a W x Y grid can run in a resident batch (whatever its generations).
bool resident_batch_fits(int W, int Y, int num_sms, int device);
// The band list (p.ndone entries, launch order) given the slots and counters.
void fill_resident_jobs(const ResidentBatchPlan& p, const ResidentGrid* g, uint32_t* pub, int* done,
                        ResidentBand* jobs);
// One persistent cooperative launch over the bands; ticket, status and the
// counters must be zero.
cudaError_t launch_batch_resident(const ResidentBand* jobs, int njobs, int* ticket, int* status,
                                  const ResidentBatchPlan& p, cudaStream_t stream);

struct ResidentPlan {
    int wpl = 0, lanes = 0, groups = 0;   // lanes of wpl words across a row, row groups
    int K = 0;                            // generations per epoch (halo rows)
    int band = 0, nbands = 0;             // largest band, CTAs
    size_t smem = 0;                      // dynamic shared memory per CTA
    size_t pub_words = 0;                 // words of the publication slots
};
// False when the grid does not fit (or k_epoch is out of range). k_epoch = 0
// picks the default.
bool plan_resident(int W, int Y, int k_epoch, int device, ResidentPlan* p);
// gens generations src -> dst. pub (p.pub_words), epoch_done (p.nbands ints)
// and status are device scratch; epoch_done and status are cleared here.
cudaError_t launch_resident(const uint32_t* src, uint32_t* dst, int W, int Y, long long gens,
                            const ResidentPlan& p, uint32_t* pub, int* epoch_done, int* status,
                            cudaStream_t stream, long long spin_limit = 0);

// One pass of k generations (1 <= k <= kMaxKForWpl(plan.wpl)). pitch: words
// from one row to the next (0 = W).
cudaError_t launch_rows_pass(const uint32_t* src, uint32_t* dst, int W, int Y, int k,
                             const RowsPlan& plan, cudaStream_t stream, int pitch = 0);

// Change-tracking tiles (GOL_ALG_LOCAL): tile = x-slice x row band.
struct LocalPlan {
    RowsPlan rows;     // slice/band geometry of one tile (one lane of words)
    int tiles_x = 0, tiles_y = 0;
    int ctas = 0;      // persistent CTAs of the tile kernel (capped at one wave)
    int num_sms = 0;
    RowsPlan dense;    // the dense form of a pass (row bands over the whole grid)
    int dense_min = 0; // active tiles from which a pass runs dense (INT_MAX = never)
};

// Word layouts (gol_layouts.cu): X_BITS x Y_BITS cells per word.
bool layout_geom(int layout, uint32_t wb, uint32_t* xb, uint32_t* yb);
void host_cells_to_layout(const uint8_t* cells, size_t x, size_t y, int layout, uint32_t wb,
                          uint32_t xb, uint32_t yb, void* words);
void host_layout_to_cells(const void* words, size_t x, size_t y, int layout, uint32_t wb,
                          uint32_t xb, uint32_t yb, uint8_t* cells);
void host_layout_to_rows(const void* words, size_t x, size_t y, int layout, uint32_t wb,
                         uint32_t xb, uint32_t yb, uint32_t* rows);
void host_rows_to_layout(const uint32_t* rows, size_t x, size_t y, int layout, uint32_t wb,
                         uint32_t xb, uint32_t yb, void* words);

// Bytes of one pass's change bits: a bit per tile, rows of
// ceil(tiles_x / 32) words.
inline size_t local_change_bytes(const LocalPlan& lp) {
    return (size_t)lp.tiles_y * ((lp.tiles_x + 31) / 32) * sizeof(uint32_t);
}

constexpr int kLocalCountWords = 8;

// Entries of the lane list a pass's plan writes: one per active tile and
// one halo lane at each end of every run of active tiles. At most 48 per 32
// tiles of a tile row (16 runs of one tile).
inline size_t local_list_ints(const LocalPlan& lp) {
    return (size_t)lp.tiles_y * ((lp.tiles_x + 31) / 32) * 48 + 64;
}

struct LocalState {
    uint32_t* changed[2] = {nullptr, nullptr};  // change bits per tile, by pass parity
    int* list = nullptr;                        // active tiles of the current pass
    int* count = nullptr;                       // kLocalCountWords plan words: tile counts
                                                // by pass parity, CTA ticket, dense choice
    uint32_t* census = nullptr;                 // active tiles per pass
    uint32_t census_cap = 0;
    uint32_t* pass_no = nullptr;                // passes recorded so far
};

// dense_pct: active-tile share (percent) from which a pass runs dense;
// 0 = the default, above 100 = never.
bool plan_local_tiles(int W, int Y, int k, int tile_rows, int wpl, int num_sms, int dense_pct,
                      LocalPlan* lp);

// One change-tracking pass: plan (reads changed[parity ^ 1], clears
// changed[parity]) then the tile kernel or, from dense_min active tiles, the
// dense tracked kernel (either writes changed[parity]).
cudaError_t launch_local_pass(const uint32_t* src, uint32_t* dst, int W, int Y, int k,
                              const LocalPlan& lp, const LocalState& st, int parity,
                              cudaStream_t stream);

// Batched uneven grids (one persistent launch over a work list).
struct BatchGrid {
    uint32_t* buf[2];      // ping-pong device grids (W words per row)
    int W, Y;              // words per row, rows
    int pitch;             // words from one row to the next: W rounded up to wpl
    int wpl;               // words per lane
    int k;                 // depth of full passes
    int last_k;            // depth of the final pass
    int passes;            // passes to run (0 = nothing to do)
    int band;              // rows per segment
    int seg_lanes;         // L lanes per segment (W / wpl, or 32 when sliced)
    int segs;              // S segments per warp (1 when sliced)
    int ngroups;           // band groups
    int slice;             // words per x-slice (W when unsliced)
    int nslices;
    int halo;              // halo words each side of a slice (0 when unsliced)
    int done_base;         // offset of this grid's (group, slice) counters
    int parity0;           // buffer holding the grid at the start of the launch
    // Change tracking (trk null: every item is computed). An item is a tile:
    // it is recomputed only if it or one of its 3x3 neighbour items changed
    // in the previous pass.
    uint32_t* trk;         // [2][ngroups * nslices] change flags by absolute pass
                           // parity (parity0 + pass) & 1, nonzero = changed; then one
                           // word: the pass from which nothing changes (0xFFFFFFFF: none)
    int* pstat;            // per pass of this launch: [items done, items changed]
    uint32_t* gstat;       // items computed, items skipped (accumulated)
    int* rflag;            // set to 1 once the grid is known to be still (may be null)
    int pass0;             // passes this grid ran in earlier launches (the still pass
                           // in trk counts from the grid's first launch)
};

// Words of a grid's change-tracking region (trk).
inline size_t batch_trk_words(int ngroups, int nslices) {
    return 2 * (size_t)ngroups * nslices + 1;
}

struct BatchItem {
    int grid, group, slice, pass;
};

constexpr int kBatchMaxK = 4;

struct GridChoice {
    int wpl, k, band, seg_lanes, segs, ngroups, passes, last_k, slice, nslices, halo;
    double cost;    // total work
    double crit;    // dependency chain
    double score;   // what the autotuner minimised
};

// The batched autotuner: words per lane, depth and band height for one grid.
// Minimises work / parallel + crit_weight * (the grid's dependency chain).
bool choose_batch_plan(int W, int Y, uint64_t gens, int force_wpl, int force_k, int force_band,
                       GridChoice* out, double parallel = 1.0, double crit_weight = 0.0);

// Emits the work items of `grids` in critical-path-first order: descending
// remaining passes (passes - pass), so long grids start first and every
// dependency (same grid, previous pass) has a smaller ticket. Returns the count.
size_t order_batch_items(const BatchGrid* grids, size_t ngrids, BatchItem* out);
size_t count_batch_items(const BatchGrid* grids, size_t ngrids);

// Resident one-warp CTAs per SM of the batch kernel built for one lane
// width (1, 2, 4) or for any (0), without or with change tracking.
int batch_kernel_ctas_per_sm(int wpl_only = 0, bool track = false);

// The lane width every grid with work shares, or 0 when they differ.
int batch_uniform_wpl(const BatchGrid* grids, size_t ngrids);

// Fills a descriptor from a plan (buffers, progress base and parity set by the caller).
void batch_grid_from_choice(const GridChoice& ch, int W, int Y, BatchGrid* g);

// Launches the persistent batch kernel over `nitems` items (pass-major
// order); done[] and *ticket, *status must be zero. All CTAs fit at once.
// wpl_only: the lane width all grids share (batch_uniform_wpl), or 0.
// spin_limit: polls before a dependency wait gives up (0 = the default guard).
// track: some grid has change tracking (the kernel variant that compares
// every stored word with its input).
cudaError_t launch_batch_kernel(const BatchGrid* d_grids, const BatchItem* d_items, int nitems,
                                int* d_ticket, int* d_done, int* d_status, int num_sms,
                                cudaStream_t stream, unsigned long long* d_census = nullptr,
                                int wpl_only = 0, long long spin_limit = 0, bool track = false);

cudaError_t launch_pack_cells(const uint8_t* cells, uint32_t* words, size_t x, size_t y,
                              cudaStream_t stream);
// Counter-based Bernoulli grid written straight into device row words, and
// the same cells on the host (mix64 hash of the seed and the cell index).
cudaError_t launch_hash_bernoulli(uint32_t* words, size_t x, size_t y, uint64_t seed,
                                  double density, cudaStream_t stream);
void host_hash_bernoulli(uint8_t* cells, size_t n, uint64_t seed, double density);
cudaError_t launch_unpack_cells(const uint32_t* words, uint8_t* cells, size_t x, size_t y,
                                cudaStream_t stream);

// Host packing between a cell grid and 32-bit row words (multi-threaded).
void host_pack_u8(const uint8_t* cells, size_t x, size_t y, uint32_t* words);
void host_pack_i32(const int32_t* cells, size_t x, size_t y, uint32_t* words);
void host_unpack_u8(const uint32_t* words, size_t x, size_t y, uint8_t* cells);
void host_unpack_i32(const uint32_t* words, size_t x, size_t y, int32_t* cells);

void host_random_ones_zeros(uint8_t* cells, size_t n, uint64_t seed);
void host_workload_uneven(uint64_t seed, uint32_t n, uint32_t lo, uint32_t hi, uint32_t mult,
                          double dlo, double dhi, uint64_t glo, uint64_t ghi, uint64_t* xs,
                          uint64_t* ys, double* dens, uint64_t* gens, uint64_t* cell_seeds);
void host_bernoulli(uint8_t* cells, size_t n, uint64_t seed, double density);
void host_poisson_arrivals(uint64_t seed, uint32_t n, double rate, double* t);
int host_sparse_patches(uint8_t* cells, size_t x, size_t y, uint64_t seed, size_t patch,
                        double fraction, double density);

int device_sm_count(int device);

// Host threads this process may run on (its CPU affinity).
unsigned usable_cpus();

// Measured LOP3 throughput of the device (32-bit lane-ops per second).
cudaError_t probe_lop3_rate(int device, cudaStream_t stream, double* lane_ops_per_s);

} // namespace golb200
