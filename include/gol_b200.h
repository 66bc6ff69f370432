/*
 * gol_b200.h — C ABI of the B200 Game of Life engine (libgolb200.so).
 *
 * A drop-in for the reference's algorithm contract
 *   infrastructure::Algorithm<2, cell_t>   (src/infrastructure/algorithm.hpp:17-87)
 * as driven by ExperimentManager::perform_alg
 *   (src/infrastructure/experiment_manager.hpp:365-394):
 *
 *   reference virtual                              entry point here
 *   --------------------------------------------   ------------------------------
 *   set_params(const ExperimentParams&)  :76-78    gol_create (gol_config)
 *   set_and_format_input_data(grid)      :37       gol_set_input_u8 / _i32 / _words
 *   initialize_data_structures()         :42       gol_init
 *   run(iterations)                      :49       gol_run
 *   finalize_data_structures()           :54       gol_finalize
 *   fetch_result()                       :61       gol_fetch_u8 / _i32 / _words
 *   actually_performed_iterations()      :69       gol_performed
 *   (destructor)                                   gol_destroy
 *
 * Semantics follow the reference: Conway B3/S23, cells outside the grid are
 * dead, `iterations` generations are advanced (0 leaves the grid as it
 * is, like GoLCpuNaive, gol_cpu_naive.hpp:26-78), a nonzero cell is alive
 * when packing (general_bit_grid.hpp:217-246), results unpack to 0/1, and
 * run() stops early once `max_runtime_seconds` of wall time have passed,
 * reporting the generations actually done (timer.hpp:29-52).
 *
 * The grid lives on one GPU in the reference's fully-packed rows layout
 * (bit_modes.hpp:127-148): bit i of row word xw is cell (xw*W + i, y), words
 * row-major. On a little-endian device 32- and 64-bit words give the same
 * bytes, so `word_bits` only fixes the width granularity (X % word_bits == 0).
 *
 * Errors: every int-returning call returns GOL_OK (0) or a negative
 * GOL_E_* code and never throws; gol_last_error() describes the last
 * failure of that engine. (The reference throws std::runtime_error /
 * CudaError instead, cuch.hpp:42-52; the C++ adapter in
 * stencil-optimalizations_b200/host/gol_b200_algorithm.hpp maps codes back
 * to exceptions.) There is no CPU fallback: without a usable CUDA device
 * gol_init fails with GOL_E_CUDA.
 */
#ifndef GOL_B200_H
#define GOL_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GOL_B200_ABI_VERSION 1

enum gol_status {
    GOL_OK = 0,
    GOL_E_INVALID = -1,      /* bad argument or shape                           */
    GOL_E_STATE = -2,        /* call out of the contract's phase order          */
    GOL_E_CUDA = -3,         /* CUDA runtime error (message in gol_last_error)  */
    GOL_E_NOMEM = -4,        /* host or device allocation failed                */
    GOL_E_UNSUPPORTED = -5,  /* shape/parameters outside what the kernels cover */
    GOL_E_TIMEOUT = -6       /* a device-side wait gave up (bounded spin)       */
};

/* Which kernel family gol_run uses. */
enum gol_algorithm {
    GOL_ALG_AUTO = 0,        /* temporal rows, depth picked by the engine       */
    GOL_ALG_ROWS = 1,        /* temporal rows with temporal_steps = k           */
    GOL_ALG_LOCAL = 2,       /* change-tracking tiles (skips stable tiles)      */
    GOL_ALG_RESIDENT = 3     /* the whole run in one cooperative launch, bands
                                kept in shared memory (grids that fit in the
                                SMs' shared memory, e.g. 8192 x 8192, else
                                gol_init returns GOL_E_UNSUPPORTED);
                                temporal_steps = generations between halo
                                exchanges (0 = 8); with a run budget the run
                                goes in launches of 64, 128, ... generations,
                                the budget checked before each; a band that waits too
                                long for a neighbour stops the run with
                                GOL_E_TIMEOUT (from gol_sync / gol_finalize) */
};

/* Mirrors the ExperimentParams fields the hot path reads
 * (src/infrastructure/experiment_params.hpp:21-116). Zero = engine default. */
typedef struct gol_config {
    uint32_t struct_size;           /* sizeof(gol_config), for ABI checks        */
    uint32_t algorithm;             /* enum gol_algorithm                        */
    uint64_t x, y;                  /* grid_dimensions (cells)                   */
    uint32_t word_bits;             /* 32 or 64 (state width of the layout)      */
    uint32_t temporal_steps;        /* k generations per pass (0 = auto)         */
    uint32_t thread_block_size;     /* rows per band (0 = auto; k = 1: per thread) */
    uint32_t tile_rows;             /* change-tracking tile height (0 = auto)    */
    uint64_t max_runtime_seconds;   /* 0 = unlimited                             */
    int32_t device;                 /* CUDA device ordinal                       */
    uint32_t lane_words;            /* 32-bit words per lane: 1, 2, 4 (0 = auto) */
    void* stream;                   /* cudaStream_t to use; NULL = own stream    */
    uint32_t dense_pct;             /* change tracking: a pass with at least this
                                       percentage of its tiles active runs the
                                       dense kernel instead of the tile kernel
                                       (0 = auto, 10; above 100 = never)        */
    uint32_t reserved;              /* zero                                      */
} gol_config;

typedef struct gol_engine gol_engine;

/* Fills *cfg with defaults for an x-by-y grid. */
void gol_config_init(gol_config* cfg, uint64_t x, uint64_t y);

/* Creates an engine (no device work yet). */
int gol_create(gol_engine** out, const gol_config* cfg);

/* set_and_format_input_data: copies and packs a host cell grid (row-major,
 * x fastest: cell (cx, cy) at cells[cy*x + cx]). x, y must match the config. */
int gol_set_input_u8(gol_engine* e, const uint8_t* cells, uint64_t x, uint64_t y);
int gol_set_input_i32(gol_engine* e, const int32_t* cells, uint64_t x, uint64_t y);
/* Already packed rows (word_bits 32 or 64, x/word_bits words per row). */
int gol_set_input_words(gol_engine* e, const void* words, uint64_t x, uint64_t y,
                        uint32_t word_bits);

/* Word layouts of the reference's GeneralBitGrid modes
 * (src/algorithms/_shared/bitwise/bit_modes.hpp:10-177):
 *   GOL_LAYOUT_ROWS    FullyPackedRows: cell (cx, cy) is bit cx % W of word
 *                      cy * (x / W) + cx / W (the engine's own layout);
 *   GOL_LAYOUT_COLUMNS BitColumns: bit cy % W of word (cy / W) * x + cx;
 *   GOL_LAYOUT_TILES   BitTile: 4x4 cells per 16-bit word, 8x4 per 32-bit,
 *                      8x8 per 64-bit; bit W-1 - ((cy % YB) * XB + cx % XB)
 *                      of word (cy / YB) * (x / XB) + cx / XB.
 * Word bits 16, 32 or 64; x and y multiples of the word's cell block. */
enum gol_layout { GOL_LAYOUT_ROWS = 0, GOL_LAYOUT_COLUMNS = 1, GOL_LAYOUT_TILES = 2 };

/* set_and_format_input_data from words in any layout (converted to rows on
 * the host; x must also be a multiple of 32). */
int gol_set_input_layout(gol_engine* e, const void* words, int layout, uint32_t word_bits);

/* initialize_data_structures: allocates the device grids, copies input in. */
int gol_init(gol_engine* e);

/* run: advances n generations on the device (asynchronous on the engine's
 * stream; gol_finalize or gol_sync waits). */
int gol_run(gol_engine* e, uint64_t n);

/* Waits for the engine's queued device work. */
int gol_sync(gol_engine* e);

/* finalize_data_structures: waits and copies the grid back. The engine keeps
 * its two device grids (and captured graphs) for the next round; gol_destroy
 * frees them. */
int gol_finalize(gol_engine* e);

/* fetch_result: unpacks the finalized grid into the caller's buffer. */
int gol_fetch_u8(gol_engine* e, uint8_t* cells);
int gol_fetch_i32(gol_engine* e, int32_t* cells);
int gol_fetch_words(gol_engine* e, void* words, uint32_t word_bits);

/* fetch_result as words in any layout (see gol_set_input_layout). */
int gol_fetch_layout(gol_engine* e, void* words, int layout, uint32_t word_bits);

/* actually_performed_iterations of the last gol_run. */
uint64_t gol_performed(const gol_engine* e);

void gol_destroy(gol_engine* e);

/* Last failure of this engine (or of gol_create when e is NULL). */
const char* gol_last_error(const gol_engine* e);

/* --- Input generation ----------------------------------------------------- */

/* The reference's RandomOnesZerosDataLoader
 * (src/infrastructure/data_loader.hpp:57-75): one
 * std::uniform_int_distribution<int>(0, 1) draw from std::mt19937(seed) per
 * cell, raster order (cells[cy*x + cx]). Host only. */
int gol_load_random_ones_zeros(uint8_t* cells, uint64_t x, uint64_t y, uint64_t seed);

/* Sparse/settling input: all dead except floor(S * fraction) of the S
 * aligned patch-by-patch slots, filled with Bernoulli(density) cells. The
 * draw order is fixed (std::mt19937_64(seed); Fisher-Yates over slot
 * indices, j = rng() % (i+1) from the back; chosen slots sorted; cells of
 * each chosen slot row by row, alive iff (rng() >> 11) * 2^-53 < density).
 * x, y multiples of patch. Returns the number of filled slots (>= 0) or
 * GOL_E_INVALID. Host only. */
int gol_load_sparse_patches(uint8_t* cells, uint64_t x, uint64_t y, uint64_t seed, uint32_t patch,
                            double fraction, double density);

/* The reference's other input loaders (src/infrastructure/data_loader.hpp:
 * 77-152, registered in experiment_manager.hpp:396-410). Host only; cells
 * are raster order (cells[cy*x + cx]), 0 dead / 1 alive.
 *   zeros            : every cell dead (ZerosLoader).
 *   always-changing  : a blinker (three live cells in a row) with its left
 *                      cell at every (cx, cy) with cx % 4 == 0 and
 *                      cy % 4 == 0, on a dead grid (AlwaysChangingSpaceLoader).
 * A pattern cell that lands past the right edge continues on the next row
 * (the reference's flat indexing); one past the end of the raster is
 * dropped. */
int gol_load_zeros(uint8_t* cells, uint64_t x, uint64_t y);
int gol_load_always_changing(uint8_t* cells, uint64_t x, uint64_t y);

/* Lexicon loader (LexiconLoader<2,T>, data_loader.hpp:77-99, and
 * lexicon::Lexicon, gol-lexicon/lexicon.hpp:118-186). A gol_lexicon is a
 * pattern dictionary read at run time from text in the format of the
 * reference's gol-lexicon/patterns.cpp (entries {"name", {{_, X, ...}, ...}},
 * `_` dead, `X` alive, one brace group per row; only the part between the
 * LEXICON_START and LEXICON_END marker comments when both are present; the
 * first entry of a repeated name wins). It starts with "blinker" only.
 *   gol_lexicon_add_text / _add_file : add entries (later calls override
 *       earlier names); returns the number of entries read, or GOL_E_INVALID
 *       with gol_lexicon_last_error set.
 *   gol_lexicon_insert : place the patterns of an expression such as
 *       "glider[10,20]; block[3,4]" (whitespace and ';' are ignored; each
 *       record is name[x,y] with (x, y) the pattern's top-left cell). Pattern
 *       cells overwrite the grid, dead ones included; unknown names place
 *       nothing. Returns the number of records placed, or GOL_E_INVALID for a
 *       coordinate that is not a non-negative integer.
 *   gol_lexicon_insert_repeating : the named pattern at every multiple of
 *       (x_jump, y_jump) (Lexicon::insert_repeating, lexicon.hpp:137-145). */
typedef struct gol_lexicon gol_lexicon;
int gol_lexicon_create(gol_lexicon** out);
int gol_lexicon_add_text(gol_lexicon* lx, const char* text);
int gol_lexicon_add_file(gol_lexicon* lx, const char* path);
int gol_lexicon_count(const gol_lexicon* lx);
int gol_lexicon_pattern_size(const gol_lexicon* lx, const char* name, uint64_t* width,
                             uint64_t* height);
int gol_lexicon_insert(gol_lexicon* lx, const char* expression, uint8_t* cells, uint64_t x,
                       uint64_t y);
int gol_lexicon_insert_repeating(gol_lexicon* lx, const char* name, uint64_t x_jump,
                                 uint64_t y_jump, uint8_t* cells, uint64_t x, uint64_t y);
const char* gol_lexicon_last_error(const gol_lexicon* lx);
void gol_lexicon_destroy(gol_lexicon* lx);

/* Uneven multi-grid workloads (batched and serving configurations), drawn
 * from one std::mt19937_64(seed) stream with u = (rng() >> 11) * 2^-53, per
 * grid in order: x = multiple * llround(exp(ln min + u (ln max - ln min)) /
 * multiple) clamped to [min, max]; y likewise; density = lo + u (hi - lo);
 * gens = llround(exp(ln glo + u (ln ghi - ln glo))); cell_seed = rng(). */
int gol_workload_uneven(uint64_t seed, uint32_t n, uint32_t min_side, uint32_t max_side,
                        uint32_t multiple, double density_lo, double density_hi, uint64_t gens_lo,
                        uint64_t gens_hi, uint64_t* xs, uint64_t* ys, double* densities,
                        uint64_t* gens, uint64_t* cell_seeds);
/* Bernoulli(density) cells, raster order, alive iff (rng() >> 11) * 2^-53 <
 * density for std::mt19937_64(seed). */
int gol_load_bernoulli(uint8_t* cells, uint64_t x, uint64_t y, uint64_t seed, double density);
/* Counter-based Bernoulli cells (the serving loop's device-generated inputs):
 * cell i alive iff (mix64(seed + (i + 1) * 0x9E3779B97F4A7C15) >> 11) * 2^-53
 * < density. Host only. */
int gol_load_hash_bernoulli(uint8_t* cells, uint64_t x, uint64_t y, uint64_t seed, double density);
/* Poisson arrival times (seconds): exponential gaps -ln(1 - u) / rate. */
int gol_poisson_arrivals(uint64_t seed, uint32_t n, double rate, double* times);

/* --- Device-resident access (between gol_init and gol_finalize) ---------- */

/* Device pointer to the current grid (x/32 uint32 words per row). */
void* gol_device_grid(gol_engine* e);
/* The engine's cudaStream_t. */
void* gol_stream(gol_engine* e);
/* Temporal depth and band height gol_run uses (after gol_init). For
 * GOL_ALG_RESIDENT: generations per epoch and the largest CTA band. */
int gol_plan(const gol_engine* e, uint32_t* temporal_steps, uint32_t* band_rows,
             uint32_t* words_per_lane);

/* Change-tracking census of the last gol_run with GOL_ALG_LOCAL (the
 * reference's --collect-touched-tiles-stats, cuda_local_one_cell.hpp:61-71,
 * 186-289): passes run, tiles per pass, tiles computed over all passes, and
 * up to max_entries per-pass computed-tile counts (the rest untouched: this
 * engine never copies skipped tiles). Synchronizes the engine's stream. */
int gol_local_stats(gol_engine* e, uint64_t* passes, uint64_t* tiles_per_pass,
                    uint64_t* computed_total, uint32_t* per_pass, uint64_t max_entries);

/* --- Stateless device entry points -------------------------------------- */

/* One pass of k generations, d_src -> d_dst (device row grids, x/32 words
 * per row, 16-byte aligned, must not overlap). k in 1..16. k = 1 runs the
 * HBM-streaming one-generation kernel (band_rows: rows each thread walks),
 * k >= 2 the K-stage row-band kernel (band_rows: output rows per CTA);
 * band_rows = 0 picks a default. Asynchronous on `stream`. */
int gol_rows_pass(const void* d_src, void* d_dst, uint64_t x, uint64_t y, uint32_t k,
                  uint32_t band_rows, void* stream);
/* Same with the lane width forced (lane_words 1, 2 or 4; 0 = auto). */
int gol_rows_pass_ex(const void* d_src, void* d_dst, uint64_t x, uint64_t y, uint32_t k,
                     uint32_t band_rows, uint32_t lane_words, void* stream);

/* No counterpart in the reference (its algorithms always cudaMalloc their own
 * grids in initialize_data_structures). For callers that cannot allocate
 * device memory (a framework that owns all memory through its own pool, a
 * real-time loop that cannot absorb the synchronisation cudaMalloc/cudaFree
 * can cause, a plugin host that forbids foreign allocations): advances n
 * generations from d_in into d_out (device row grids, x/32 uint32 words per
 * row, 16-byte aligned, distinct, not overlapping) and calls no cudaMalloc,
 * cudaFree or allocating library routine. The passes' ping-pong partner is
 * a fixed 32 MiB array inside the library (GOL_NOALLOC_MAX_BYTES): grids of
 * more than that many bytes (x*y/8, e.g. above 16384 x 16384) are rejected
 * with GOL_E_UNSUPPORTED. Every GPU that loads the library holds that array
 * until the process exits. The first call on a device looks up the array's
 * device address (cudaGetSymbolAddress, with that device current); make that
 * first call before any stream capture. That address is cached for the life
 * of the process: it becomes stale if the caller resets the device
 * (cudaDeviceReset), after which this entry point must not be called on that
 * device again. All calls share the one array:
 * calls that overlap on the GPU (other streams, other threads) race and must
 * be serialised by the caller. k = 0 picks 4. Asynchronous on `stream`. */
#define GOL_NOALLOC_MAX_BYTES (32u << 20)
int gol_rows_run_noalloc(const void* d_in, void* d_out, uint64_t x, uint64_t y, uint64_t n,
                         uint32_t k, void* stream);

/* Packs / unpacks a device cell grid (uint8, nonzero = alive, 16-byte
 * aligned) to / from device row words. x % 32 == 0. */
int gol_pack_cells_device(const uint8_t* d_cells, void* d_words, uint64_t x, uint64_t y,
                          void* stream);
int gol_unpack_cells_device(const void* d_words, uint8_t* d_cells, uint64_t x, uint64_t y,
                            void* stream);

/* Host cells (uint8, nonzero = alive) <-> words in a layout
 * (GeneralBitGrid fill_grid / to_grid, general_bit_grid.hpp:171-246). */
int gol_pack_layout(const uint8_t* cells, uint64_t x, uint64_t y, int layout, uint32_t word_bits,
                    void* words);
int gol_unpack_layout(const void* words, uint64_t x, uint64_t y, int layout, uint32_t word_bits,
                      uint8_t* cells);

/* Device words in the column or tile layout <-> device rows (32-bit
 * words), stream-ordered. x % 32 == 0, y a multiple of the layout's block
 * height, both at most 2^30; pointers aligned to their word size (and 4). */
int gol_layout_to_rows_device(const void* d_src, void* d_rows, uint64_t x, uint64_t y, int layout,
                              uint32_t word_bits, void* stream);
int gol_rows_to_layout_device(const void* d_rows, void* d_dst, uint64_t x, uint64_t y, int layout,
                              uint32_t word_bits, void* stream);

/* Measures the device's 32-bit LOP3 throughput (lane-ops/s) with a short
 * register-only kernel: the integer-pipe roofline of the bit-sliced passes.
 * Synchronizes `stream`. */
int gol_probe_int_peak(double* lane_ops_per_s, void* stream);

/* --- Batched uneven grids (one persistent launch) ------------------------ */

/* Many independent grids, each with its own size and generation count,
 * advanced together by one persistent kernel launch (captured as a CUDA
 * graph). An autotuner picks one words-per-lane width and temporal depth for
 * the whole batch (one pipeline body per launch) and a band height per grid;
 * gol_batch_set_plan overrides a grid's plan (mixed widths then run the
 * general kernel). gol_batch_plan reports the plan of the uploaded batch, or
 * the grid's own best plan before gol_batch_upload. No reference
 * counterpart: the reference runs one grid per invocation
 * (experiment_manager.hpp:365-394). */
typedef struct gol_batch gol_batch;

int gol_batch_create(gol_batch** out, int32_t device, void* stream);
/* Adds a host cell grid (x % 32 == 0) to run `generations`. */
int gol_batch_add(gol_batch* b, const uint8_t* cells, uint64_t x, uint64_t y, uint64_t generations,
                  int32_t* grid_id);
int gol_batch_set_plan(gol_batch* b, int32_t grid_id, uint32_t lane_words, uint32_t temporal_steps,
                       uint32_t band_rows);
int gol_batch_plan(const gol_batch* b, int32_t grid_id, uint32_t* lane_words,
                   uint32_t* temporal_steps, uint32_t* band_rows, uint32_t* segments);
/* Plans all grids and copies inputs and the work list to the device. */
int gol_batch_upload(gol_batch* b);
/* Runs every grid to its generation count in one persistent launch
 * (asynchronous; gol_batch_sync waits). Every run restarts from the inputs,
 * restored from a device copy made at upload. */
int gol_batch_run(gol_batch* b);
/* Baseline: the same grids one after another through the single-grid pass
 * kernel, one launch per k-generation pass per grid. */
int gol_batch_run_plain(gol_batch* b, uint32_t temporal_steps);
/* Every grid in shared memory: each grid is cut into bands, and one
 * persistent cooperative launch runs every band to its grid's last generation
 * in one CTA's shared memory (the GOL_ALG_RESIDENT algorithm; neighbouring
 * bands exchange halo rows every 8 generations). CTAs take bands in order of
 * their work, a grid's bands consecutively. Asynchronous; restarts from the
 * inputs; gol_batch_sync reports GOL_E_TIMEOUT if a band waited too long for
 * a neighbour. GOL_E_UNSUPPORTED if a grid is wider than 32768 cells or
 * needs more bands than the GPU has SMs. No change tracking. */
int gol_batch_run_resident(gol_batch* b);
/* The last resident plan: bands, CTAs, shared memory per CTA. */
int gol_batch_resident_info(const gol_batch* b, uint64_t* bands, uint32_t* ctas,
                            uint64_t* smem_bytes);
/* Waits; GOL_E_TIMEOUT if the persistent kernel gave up a dependency wait. */
int gol_batch_sync(gol_batch* b);
int gol_batch_fetch(gol_batch* b, int32_t grid_id, uint8_t* cells);
int gol_batch_info(const gol_batch* b, uint64_t* grids, uint64_t* items, uint64_t* cell_updates);
/* Exercises the persistent kernel's dependency-wait guard without a fault:
 * launches a work list whose only item waits on a pass that never runs;
 * the wait gives up after spin_limit polls (1 .. 2^24, each >= 64 ns) and
 * *status = GOL_E_TIMEOUT is expected; the context stays usable. */
int gol_batch_probe_timeout(int32_t device, uint64_t spin_limit, int32_t* status);
/* Census of the last gol_batch_run: SM clock cycles its work items spent
 * waiting on dependencies and computing, summed over items. */
int gol_batch_census(gol_batch* b, uint64_t* wait_cycles, uint64_t* work_cycles);

/* Change tracking in the batch (the rule of the reference's change-tracking
 * kernels, cuda_naive_local.cu:125-161 and cuda_local_one_cell.cu:172-200,
 * on the batch's work items as tiles): an item of pass p is computed only if
 * it or one of its 8 neighbour items changed in pass p-1; a grid whose pass
 * changed nothing is still from then on, and its remaining items end at
 * once. GOL_TRACK_AUTO (default) tracks grids of at least 8 passes until
 * gol_batch_retune has seen a run; gol_batch_retune then keeps tracking per
 * grid where the run skipped at least 5 % of its items (finest tiles, 16-row
 * bands, from 50 %) and runs the others dense, and turns tracking off for
 * the whole batch when the items it would skip do not pay for the tracked
 * kernel's extra time on every item (about 25 %). Both take effect at the
 * next upload/run. */
enum gol_track_mode { GOL_TRACK_AUTO = 0, GOL_TRACK_OFF = 1, GOL_TRACK_ON = 2 };
int gol_batch_set_tracking(gol_batch* b, int32_t grid_id, int32_t mode);
int gol_batch_retune(gol_batch* b);
/* Work items of the last run computed and skipped (skipped: tracked grids). */
int gol_batch_tiles(gol_batch* b, uint64_t* computed, uint64_t* skipped);
/* One grid of the last run: whether it tracked changes, its items computed
 * and skipped, and the pass from which it was still (0xFFFFFFFF: never). */
int gol_batch_grid_stats(gol_batch* b, int32_t grid_id, uint32_t* tracked, uint32_t* computed,
                         uint32_t* skipped, uint32_t* still_pass);
void* gol_batch_stream(gol_batch* b);
const char* gol_batch_last_error(const gol_batch* b);
void gol_batch_destroy(gol_batch* b);

/* --- Serving: continuous batching of simulations --------------------------- */

/* No reference counterpart. A server owns a device arena (arena_bytes; 0 =
 * half the free HBM at creation) in which admitted requests keep their two
 * grid buffers until fetched. gol_serve_step admits queued requests that fit
 * (arrival order, first fit) and queues one persistent batch launch that
 * advances every admitted request by up to `quantum` generations (0 = 64);
 * up to three rounds are queued at once, so requests arriving meanwhile join
 * the next round while the GPU keeps working. */
typedef struct gol_server gol_server;

int gol_serve_create(gol_server** out, int32_t device, uint64_t arena_bytes, uint32_t quantum,
                     void* stream);
/* Queues a request (host cells, x % 32 == 0); *id identifies it. */
int gol_serve_submit(gol_server* s, const uint8_t* cells, uint64_t x, uint64_t y,
                     uint64_t generations, uint64_t* id);
/* Queues a request whose input is generated on the device at admission:
 * cell i (raster order) alive iff (mix64(seed + (i + 1) * 0x9E3779B97F4A7C15)
 * >> 11) * 2^-53 < density, mix64 the SplitMix64 finaliser; the same cells
 * on the host: gol_load_hash_bernoulli. */
int gol_serve_submit_random(gol_server* s, uint64_t x, uint64_t y, uint64_t generations,
                            uint64_t seed, double density, uint64_t* id);
int gol_serve_step(gol_server* s);
/* Ids of requests finished since the last call (results ready). */
int gol_serve_finished(gol_server* s, uint64_t* ids, uint32_t max_ids, uint32_t* count);
/* Copies a finished request's cells out and frees its arena slot. */
int gol_serve_fetch(gol_server* s, uint64_t id, uint8_t* cells);
/* The packed result (x/32 uint32 words per row); frees the slot. */
int gol_serve_fetch_words(gol_server* s, uint64_t id, void* words);
/* Drops a finished request without copying it out. */
int gol_serve_release(gol_server* s, uint64_t id);
int gol_serve_stats(const gol_server* s, uint64_t* queued, uint64_t* running, uint64_t* rounds,
                    uint64_t* cell_updates, uint64_t* arena_free_bytes);
/* Waits for every queued round. */
int gol_serve_drain(gol_server* s);
/* Admission policy: GOL_SERVE_FIFO (default) admits queued requests in
 * arrival order, GOL_SERVE_SRPT the one with the least work (cells x
 * generations) first, when the arena cannot take them all. Either way every
 * running request advances `quantum` generations per round. */
enum gol_serve_policy { GOL_SERVE_FIFO = 0, GOL_SERVE_SRPT = 1 };
int gol_serve_set_policy(gol_server* s, int32_t policy);
/* Change tracking for requests submitted from then on (GOL_TRACK_AUTO: those
 * of at least 8 passes; _ON, _OFF). A tracked request keeps its change flags
 * resident in its slot between rounds and skips the tiles (work items) whose
 * 3x3 neighbourhood did not change in the previous pass; once a whole pass
 * changes nothing the request is finished at the end of that round, before
 * its remaining generations (they could not change it). */
int gol_serve_set_tracking(gol_server* s, int32_t mode);
/* How a round runs: GOL_SERVE_PASSES (default) as one persistent launch of
 * dependent k-generation work items (change tracking as set above);
 * GOL_SERVE_RESIDENT with every running request's grid cut into bands held
 * in shared memory for the round's generations (gol_batch_run_resident's
 * kernel; no change tracking, requests finish when their generations are
 * done; in this mode gol_serve_submit rejects, GOL_E_UNSUPPORTED, a request
 * whose bands cannot all be resident at once: rows wider than 32768 cells, or
 * taller than the SMs' shared memory holds). Changes only while no request is
 * queued or running (GOL_E_STATE). */
enum gol_serve_mode { GOL_SERVE_PASSES = 0, GOL_SERVE_RESIDENT = 1 };
int gol_serve_set_mode(gol_server* s, int32_t mode);
/* Work items computed and skipped over all rounds so far, and the number of
 * requests finished early because they became still. */
int gol_serve_tiles(gol_server* s, uint64_t* computed, uint64_t* skipped, uint64_t* early_finished);
const char* gol_serve_last_error(const gol_server* s);
void* gol_serve_stream(gol_server* s);
void gol_serve_destroy(gol_server* s);

/* Library identification: ABI version and the sm arch it was built for. */
int gol_abi_version(void);
const char* gol_build_info(void);

#ifdef __cplusplus
}
#endif

#endif /* GOL_B200_H */
