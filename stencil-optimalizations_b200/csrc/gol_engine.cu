// The engine behind include/gol_b200.h: the reference's Algorithm phase
// contract (src/infrastructure/algorithm.hpp:17-87) over device-resident,
// row-packed grids, advanced by the temporal row-band kernel.
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>

#include "gol_b200.h"
#include "gol_internal.h"

#define GOL_STR_(v) #v
#define GOL_STR(v) GOL_STR_(v)

using golb200::RowsPlan;

namespace {

thread_local std::string g_create_error;

// Passes per captured CUDA graph (even, so a chunk ends on the same buffer
// parity it started from and one executable graph per parity suffices).
constexpr int kGraphPasses = 16;

} // namespace

struct gol_engine {
    gol_config cfg{};
    uint64_t x = 0, y = 0;
    int W = 0, Y = 0;              // 32-bit words per row, rows

    uint32_t* h_words = nullptr;   // host copy of the grid (input, then result)
    size_t h_bytes = 0;
    bool h_pinned = false;
    bool has_host_grid = false;

    bool initialized = false;
    uint32_t* d[2] = {nullptr, nullptr};
    int cur = 0;                   // buffer holding the current generation
    uint64_t performed = 0;

    cudaStream_t stream = nullptr;
    bool own_stream = false;
    cudaStream_t capture_stream = nullptr;
    cudaGraphExec_t chunk[2] = {nullptr, nullptr};

    int k = 1;
    RowsPlan plan{};

    // shared-memory-resident run (GOL_ALG_RESIDENT)
    bool resident = false;
    golb200::ResidentPlan rplan{};
    uint32_t* r_pub = nullptr;
    int* r_ints = nullptr;                 // epoch counters, then the status word

    // change tracking (GOL_ALG_LOCAL)
    bool local = false;
    golb200::LocalPlan lplan{};
    golb200::LocalState lst{};
    int lparity = 0;                       // pass parity of the change flags
    cudaGraphExec_t lchunk[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};   // [cur][lparity]

    std::string err;

    int fail(int code, const std::string& msg) {
        err = msg;
        return code;
    }
    int cuda_fail(cudaError_t e, const char* what) {
        err = std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
        return GOL_E_CUDA;
    }
};

namespace {

void release_graphs(gol_engine* e) {
    for (auto& g : e->chunk) {
        if (g) cudaGraphExecDestroy(g);
        g = nullptr;
    }
    for (auto& row : e->lchunk)
        for (auto& g : row) {
            if (g) cudaGraphExecDestroy(g);
            g = nullptr;
        }
}

void release_local(gol_engine* e) {
    golb200::LocalState& s = e->lst;
    for (auto& p : s.changed) {
        if (p) cudaFree(p);
        p = nullptr;
    }
    if (s.list) cudaFree(s.list);
    if (s.count) cudaFree(s.count);
    if (s.census) cudaFree(s.census);
    if (s.pass_no) cudaFree(s.pass_no);
    s = golb200::LocalState{};
}

void release_device(gol_engine* e) {
    release_graphs(e);
    release_local(e);
    if (e->r_pub) cudaFree(e->r_pub);
    if (e->r_ints) cudaFree(e->r_ints);
    e->r_pub = nullptr;
    e->r_ints = nullptr;
    for (auto& p : e->d) {
        if (p) cudaFree(p);
        p = nullptr;
    }
    e->initialized = false;
}

constexpr uint32_t kCensusCap = 1u << 20;   // passes recorded per run (4 MiB)

int alloc_local(gol_engine* e) {
    golb200::LocalState& s = e->lst;
    cudaError_t ce = cudaSuccess;
    if (!s.list) {
        for (auto& p : s.changed)
            if (ce == cudaSuccess) ce = cudaMalloc(&p, golb200::local_change_bytes(e->lplan));
        if (ce == cudaSuccess) ce = cudaMalloc(&s.list, golb200::local_list_ints(e->lplan) * sizeof(int));
        if (ce == cudaSuccess) ce = cudaMalloc(&s.count, golb200::kLocalCountWords * sizeof(int));
        if (ce == cudaSuccess) ce = cudaMalloc(&s.census, kCensusCap * sizeof(uint32_t));
        if (ce == cudaSuccess) ce = cudaMalloc(&s.pass_no, sizeof(uint32_t));
        s.census_cap = kCensusCap;
        if (ce != cudaSuccess) {
            release_local(e);
            return e->cuda_fail(ce, "change-tracking allocation");
        }
    }
    // First pass of a round: every tile counts as changed.
    const size_t cb = golb200::local_change_bytes(e->lplan);
    ce = cudaMemsetAsync(s.changed[1], 0xff, cb, e->stream);
    if (ce == cudaSuccess) ce = cudaMemsetAsync(s.changed[0], 0, cb, e->stream);
    if (ce == cudaSuccess) ce = cudaMemsetAsync(s.pass_no, 0, sizeof(uint32_t), e->stream);
    if (ce == cudaSuccess) ce = cudaMemsetAsync(s.count, 0, golb200::kLocalCountWords * sizeof(int), e->stream);
    if (ce != cudaSuccess) return e->cuda_fail(ce, "change-tracking reset");
    e->lparity = 0;
    return GOL_OK;
}

void release_host(gol_engine* e) {
    if (e->h_words) {
        if (e->h_pinned)
            cudaFreeHost(e->h_words);
        else
            std::free(e->h_words);
    }
    e->h_words = nullptr;
    e->h_bytes = 0;
    e->h_pinned = false;
    e->has_host_grid = false;
}

int check_shape(gol_engine* e, uint64_t x, uint64_t y) {
    if (x != e->x || y != e->y)
        return e->fail(GOL_E_INVALID, "grid dimensions differ from the engine's configuration");
    return GOL_OK;
}

// Host grid buffer, pinned when a device is available so H2D/D2H run at
// full link speed; pageable otherwise (packing needs no device).
int ensure_host(gol_engine* e) {
    const size_t bytes = (size_t)e->W * (size_t)e->Y * sizeof(uint32_t);
    if (e->h_words && e->h_bytes == bytes) return GOL_OK;
    release_host(e);
    void* p = nullptr;
    if (bytes && cudaSetDevice(e->cfg.device) == cudaSuccess &&
        cudaMallocHost(&p, bytes) == cudaSuccess) {
        e->h_pinned = true;
    } else {
        cudaGetLastError();
        p = std::malloc(bytes ? bytes : 4);
        e->h_pinned = false;
        if (!p) return e->fail(GOL_E_NOMEM, "host allocation failed");
    }
    e->h_words = static_cast<uint32_t*>(p);
    e->h_bytes = bytes;
    return GOL_OK;
}

int launch_pass(gol_engine* e, int k, cudaStream_t s, int from) {
    RowsPlan p = e->plan;
    if (k != e->k) {
        if (!golb200::plan_rows(e->W, e->Y, k, (int)e->cfg.thread_block_size, 0,
                                golb200::device_sm_count(e->cfg.device), &p))
            return e->fail(GOL_E_UNSUPPORTED, "no kernel plan for this width and depth");
    }
    cudaError_t ce = golb200::launch_rows_pass(e->d[from], e->d[from ^ 1], e->W, e->Y, k, p, s);
    if (ce != cudaSuccess) return e->cuda_fail(ce, "rows pass launch");
    return GOL_OK;
}

int launch_local(gol_engine* e, cudaStream_t s, int from, int parity) {
    cudaError_t ce = golb200::launch_local_pass(e->d[from], e->d[from ^ 1], e->W, e->Y, e->k,
                                                e->lplan, e->lst, parity, s);
    if (ce != cudaSuccess) return e->cuda_fail(ce, "change-tracking pass launch");
    return GOL_OK;
}

int build_local_graph(gol_engine* e, int cur, int parity) {
    if (!e->capture_stream) {
        cudaError_t ce = cudaStreamCreateWithFlags(&e->capture_stream, cudaStreamNonBlocking);
        if (ce != cudaSuccess) return e->cuda_fail(ce, "capture stream");
    }
    cudaError_t ce = cudaStreamBeginCapture(e->capture_stream, cudaStreamCaptureModeThreadLocal);
    if (ce != cudaSuccess) return e->cuda_fail(ce, "begin capture");
    int rc = GOL_OK;
    for (int i = 0; i < kGraphPasses && rc == GOL_OK; ++i) {
        rc = launch_local(e, e->capture_stream, cur, parity);
        cur ^= 1;
        parity ^= 1;
    }
    cudaGraph_t graph = nullptr;
    ce = cudaStreamEndCapture(e->capture_stream, &graph);
    if (rc != GOL_OK) {
        if (graph) cudaGraphDestroy(graph);
        return rc;
    }
    if (ce != cudaSuccess) return e->cuda_fail(ce, "end capture");
    ce = cudaGraphInstantiate(&e->lchunk[cur][parity], graph, 0);
    cudaGraphDestroy(graph);
    if (ce != cudaSuccess) return e->cuda_fail(ce, "graph instantiate");
    return GOL_OK;
}

int build_chunk_graph(gol_engine* e, int parity) {
    if (!e->capture_stream) {
        cudaError_t ce = cudaStreamCreateWithFlags(&e->capture_stream, cudaStreamNonBlocking);
        if (ce != cudaSuccess) return e->cuda_fail(ce, "capture stream");
    }
    cudaError_t ce = cudaStreamBeginCapture(e->capture_stream, cudaStreamCaptureModeThreadLocal);
    if (ce != cudaSuccess) return e->cuda_fail(ce, "begin capture");
    int from = parity;
    int rc = GOL_OK;
    for (int i = 0; i < kGraphPasses && rc == GOL_OK; ++i) {
        rc = launch_pass(e, e->k, e->capture_stream, from);
        from ^= 1;
    }
    cudaGraph_t graph = nullptr;
    ce = cudaStreamEndCapture(e->capture_stream, &graph);
    if (rc != GOL_OK) {
        if (graph) cudaGraphDestroy(graph);
        return rc;
    }
    if (ce != cudaSuccess) return e->cuda_fail(ce, "end capture");
    ce = cudaGraphInstantiate(&e->chunk[parity], graph, 0);
    cudaGraphDestroy(graph);
    if (ce != cudaSuccess) return e->cuda_fail(ce, "graph instantiate");
    return GOL_OK;
}

} // namespace

extern "C" {

void gol_config_init(gol_config* cfg, uint64_t x, uint64_t y) {
    if (!cfg) return;
    std::memset(cfg, 0, sizeof(*cfg));
    cfg->struct_size = sizeof(gol_config);
    cfg->algorithm = GOL_ALG_AUTO;
    cfg->x = x;
    cfg->y = y;
    cfg->word_bits = 64;
}

int gol_create(gol_engine** out, const gol_config* cfg) {
    if (!out || !cfg) {
        g_create_error = "null argument";
        return GOL_E_INVALID;
    }
    *out = nullptr;
    if (cfg->struct_size != sizeof(gol_config)) {
        g_create_error = "gol_config.struct_size does not match this library's ABI";
        return GOL_E_INVALID;
    }
    if (cfg->word_bits != 32 && cfg->word_bits != 64) {
        g_create_error = "word_bits must be 32 or 64";
        return GOL_E_INVALID;
    }
    if (cfg->x % cfg->word_bits != 0) {
        g_create_error = "grid dimension x must be a multiple of word_bits";
        return GOL_E_INVALID;
    }
    if (cfg->x / 32 > (uint64_t)1 << 30 || cfg->y > (uint64_t)1 << 30) {
        g_create_error = "grid too large";
        return GOL_E_INVALID;
    }
    if (cfg->temporal_steps > (uint32_t)golb200::kMaxTemporalSteps) {
        g_create_error = "temporal_steps must be at most 16";
        return GOL_E_INVALID;
    }
    if (cfg->lane_words != 0 && cfg->lane_words != 1 && cfg->lane_words != 2 &&
        cfg->lane_words != 4) {
        g_create_error = "lane_words must be 0, 1, 2 or 4";
        return GOL_E_INVALID;
    }
    if (cfg->algorithm > GOL_ALG_RESIDENT) {
        g_create_error = "unknown algorithm";
        return GOL_E_INVALID;
    }
    gol_engine* e = new (std::nothrow) gol_engine();
    if (!e) {
        g_create_error = "out of host memory";
        return GOL_E_NOMEM;
    }
    e->cfg = *cfg;
    e->x = cfg->x;
    e->y = cfg->y;
    e->W = (int)(cfg->x / 32);
    e->Y = (int)cfg->y;
    *out = e;
    return GOL_OK;
}

int gol_set_input_u8(gol_engine* e, const uint8_t* cells, uint64_t x, uint64_t y) {
    if (!e) return GOL_E_INVALID;
    if (!cells && x * y) return e->fail(GOL_E_INVALID, "null cells");
    if (e->initialized) return e->fail(GOL_E_STATE, "set_input while device data is live");
    int rc = check_shape(e, x, y);
    if (rc) return rc;
    if ((rc = ensure_host(e))) return rc;
    golb200::host_pack_u8(cells, x, y, e->h_words);
    e->has_host_grid = true;
    e->performed = 0;
    return GOL_OK;
}

int gol_set_input_i32(gol_engine* e, const int32_t* cells, uint64_t x, uint64_t y) {
    if (!e) return GOL_E_INVALID;
    if (!cells && x * y) return e->fail(GOL_E_INVALID, "null cells");
    if (e->initialized) return e->fail(GOL_E_STATE, "set_input while device data is live");
    int rc = check_shape(e, x, y);
    if (rc) return rc;
    if ((rc = ensure_host(e))) return rc;
    golb200::host_pack_i32(cells, x, y, e->h_words);
    e->has_host_grid = true;
    e->performed = 0;
    return GOL_OK;
}

int gol_set_input_words(gol_engine* e, const void* words, uint64_t x, uint64_t y,
                        uint32_t word_bits) {
    if (!e) return GOL_E_INVALID;
    if (word_bits != 32 && word_bits != 64) return e->fail(GOL_E_INVALID, "word_bits must be 32 or 64");
    if (x % word_bits) return e->fail(GOL_E_INVALID, "x must be a multiple of word_bits");
    if (!words && x * y) return e->fail(GOL_E_INVALID, "null words");
    if (e->initialized) return e->fail(GOL_E_STATE, "set_input while device data is live");
    int rc = check_shape(e, x, y);
    if (rc) return rc;
    if ((rc = ensure_host(e))) return rc;
    std::memcpy(e->h_words, words, e->h_bytes);   // same bytes for 32- and 64-bit rows
    e->has_host_grid = true;
    e->performed = 0;
    return GOL_OK;
}

int gol_set_input_layout(gol_engine* e, const void* words, int layout, uint32_t word_bits) {
    if (!e) return GOL_E_INVALID;
    uint32_t xb, yb;
    if (!golb200::layout_geom(layout, word_bits, &xb, &yb))
        return e->fail(GOL_E_INVALID, "unknown layout or word_bits not 16, 32 or 64");
    if (e->x % xb || e->y % yb) return e->fail(GOL_E_INVALID, "grid is not a whole number of layout words");
    if (!words && e->x * e->y) return e->fail(GOL_E_INVALID, "null words");
    if (e->initialized) return e->fail(GOL_E_STATE, "set_input while device data is live");
    int rc = ensure_host(e);
    if (rc) return rc;
    golb200::host_layout_to_rows(words, e->x, e->y, layout, word_bits, xb, yb, e->h_words);
    e->has_host_grid = true;
    e->performed = 0;
    return GOL_OK;
}

int gol_init(gol_engine* e) {
    if (!e) return GOL_E_INVALID;
    if (!e->has_host_grid) return e->fail(GOL_E_STATE, "initialize before set_input");
    if (e->initialized) return e->fail(GOL_E_STATE, "already initialized");
    cudaError_t ce = cudaSetDevice(e->cfg.device);
    if (ce != cudaSuccess) return e->cuda_fail(ce, "cudaSetDevice");
    if (!e->stream) {
        if (e->cfg.stream) {
            e->stream = static_cast<cudaStream_t>(e->cfg.stream);
            e->own_stream = false;
        } else {
            ce = cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking);
            if (ce != cudaSuccess) return e->cuda_fail(ce, "stream create");
            e->own_stream = true;
        }
    }
    int k = (int)e->cfg.temporal_steps;
    // Auto depth: 4 (the dense optimum on B200); 6 with change tracking,
    // where a pass of k generations sees oscillators whose period divides k
    // as still (period 2 blinkers and period 3 pulsars are most of the ash
    // a random grid settles into).
    if (k <= 0) k = e->cfg.algorithm == GOL_ALG_LOCAL ? 6 : 4;
    const int sms = golb200::device_sm_count(e->cfg.device);
    if (!golb200::plan_rows(e->W, e->Y, k, (int)e->cfg.thread_block_size,
                            (int)e->cfg.lane_words, sms, &e->plan))
        return e->fail(GOL_E_UNSUPPORTED, "no kernel plan for this width and depth");
    e->local = e->cfg.algorithm == GOL_ALG_LOCAL;
    e->resident = e->cfg.algorithm == GOL_ALG_RESIDENT;
    if (e->resident &&
        !golb200::plan_resident(e->W, e->Y, (int)e->cfg.temporal_steps, e->cfg.device, &e->rplan))
        return e->fail(GOL_E_UNSUPPORTED,
                       "grid does not fit in the SMs' shared memory for a resident run");
    if (e->local && !golb200::plan_local_tiles(e->W, e->Y, k, (int)e->cfg.tile_rows,
                                               (int)e->cfg.lane_words, sms,
                                               (int)std::min<uint32_t>(e->cfg.dense_pct, 101u),
                                               &e->lplan))
        return e->fail(GOL_E_UNSUPPORTED,
                       "no change-tracking tile plan (tile_rows must be >= temporal_steps)");
    e->k = k;
    // The two device grids live from the first init to gol_destroy, so an
    // instance reused round after round (as ExperimentManager reuses its
    // algorithms) allocates once and keeps its captured graphs valid.
    const size_t bytes = (size_t)e->W * e->Y * sizeof(uint32_t);
    for (auto& p : e->d) {
        if (p) continue;
        ce = cudaMalloc(&p, bytes ? bytes : 4);
        if (ce != cudaSuccess) {
            release_device(e);
            return ce == cudaErrorMemoryAllocation ? e->fail(GOL_E_NOMEM, "device allocation failed")
                                                   : e->cuda_fail(ce, "cudaMalloc");
        }
    }
    e->cur = 0;
    ce = cudaMemcpyAsync(e->d[0], e->h_words, bytes, cudaMemcpyHostToDevice, e->stream);
    if (ce != cudaSuccess) {
        release_device(e);
        return e->cuda_fail(ce, "H2D copy");
    }
    if (e->local) {
        int rc = alloc_local(e);
        if (rc) return rc;
    }
    if (e->resident && !e->r_pub) {
        ce = cudaMalloc(&e->r_pub, std::max<size_t>(e->rplan.pub_words, 1) * sizeof(uint32_t));
        if (ce == cudaSuccess) ce = cudaMalloc(&e->r_ints, (e->rplan.nbands + 1) * sizeof(int));
        if (ce != cudaSuccess) {
            release_device(e);
            return e->cuda_fail(ce, "resident-run scratch");
        }
    }
    e->initialized = true;
    e->performed = 0;
    return GOL_OK;
}

static int resident_status(gol_engine* e);

int gol_run(gol_engine* e, uint64_t n) {
    if (!e) return GOL_E_INVALID;
    if (!e->initialized) return e->fail(GOL_E_STATE, "run before initialize");
    e->performed = 0;
    if (n == 0 || e->W == 0 || e->Y == 0) {
        e->performed = n;
        return GOL_OK;
    }
    const uint64_t budget = e->cfg.max_runtime_seconds;
    const auto t0 = std::chrono::steady_clock::now();
    auto time_is_up = [&]() {
        if (budget == 0) return false;
        auto s = std::chrono::duration_cast<std::chrono::seconds>(std::chrono::steady_clock::now() - t0);
        return (uint64_t)s.count() >= budget;
    };
    if (e->resident) {   // every generation in one cooperative launch
        // Runs longer than 2^30 generations take several launches (the
        // kernel's epoch counters stay within int). With a time budget the
        // run goes in launches of 64, 128, 256, ... generations, each waited
        // for, and stops before the first launch past the budget (so it ends
        // within about twice the budget).
        uint64_t step = 64;
        for (uint64_t done = 0; done < n;) {
            if (time_is_up()) return GOL_OK;
            const uint64_t chunk = std::min<uint64_t>(n - done, budget ? step : (1ull << 30));
            cudaError_t ce = golb200::launch_resident(e->d[e->cur], e->d[e->cur ^ 1], e->W, e->Y,
                                                      (long long)chunk, e->rplan, e->r_pub, e->r_ints,
                                                      e->r_ints + e->rplan.nbands, e->stream);
            if (ce == cudaSuccess && budget) ce = cudaStreamSynchronize(e->stream);
            if (ce != cudaSuccess) return e->cuda_fail(ce, "resident run launch");
            e->cur ^= 1;
            done += chunk;
            e->performed = done;
            if (budget) {
                if (int st = resident_status(e)) return st;
                step = std::min<uint64_t>(step * 2, 1ull << 30);
            }
        }
        return GOL_OK;
    }
    const int k = e->k;
    uint64_t passes = n / (uint64_t)k;
    const int rem = (int)(n % (uint64_t)k);
    int rc;
    if (e->local) {
        if (budget == 0) {
            while (passes >= (uint64_t)kGraphPasses) {
                auto& g = e->lchunk[e->cur][e->lparity];
                if (!g && (rc = build_local_graph(e, e->cur, e->lparity))) return rc;
                cudaError_t ce = cudaGraphLaunch(g, e->stream);
                if (ce != cudaSuccess) return e->cuda_fail(ce, "graph launch");
                passes -= kGraphPasses;          // even: cur and lparity come back
                e->performed += (uint64_t)kGraphPasses * k;
            }
        }
        for (; passes > 0; --passes) {
            if (time_is_up()) return GOL_OK;
            if ((rc = launch_local(e, e->stream, e->cur, e->lparity))) return rc;
            e->cur ^= 1;
            e->lparity ^= 1;
            e->performed += k;
        }
        if (rem > 0) {
            // A shorter pass is not covered by the k-generation change flags:
            // advance every tile, then let the next pass start from "all changed".
            if (time_is_up()) return GOL_OK;
            if ((rc = launch_pass(e, rem, e->stream, e->cur))) return rc;
            e->cur ^= 1;
            e->performed += rem;
            cudaError_t ce = cudaMemsetAsync(e->lst.changed[e->lparity ^ 1], 0xff,
                                             golb200::local_change_bytes(e->lplan), e->stream);
            if (ce != cudaSuccess) return e->cuda_fail(ce, "change-flag reset");
        }
        return GOL_OK;
    }
    if (budget == 0 && passes >= 2 * (uint64_t)kGraphPasses) {
        while (passes >= (uint64_t)kGraphPasses) {
            if (!e->chunk[e->cur] && (rc = build_chunk_graph(e, e->cur))) return rc;
            cudaError_t ce = cudaGraphLaunch(e->chunk[e->cur], e->stream);
            if (ce != cudaSuccess) return e->cuda_fail(ce, "graph launch");
            passes -= kGraphPasses;
            e->performed += (uint64_t)kGraphPasses * k;
        }
    }
    for (; passes > 0; --passes) {
        if (time_is_up()) return GOL_OK;
        if ((rc = launch_pass(e, k, e->stream, e->cur))) return rc;
        e->cur ^= 1;
        e->performed += k;
    }
    if (rem > 0) {
        if (time_is_up()) return GOL_OK;
        if ((rc = launch_pass(e, rem, e->stream, e->cur))) return rc;
        e->cur ^= 1;
        e->performed += rem;
    }
    return GOL_OK;
}

// A resident run records GOL_E_TIMEOUT in its status word when a CTA gave
// up waiting for a neighbour (bounded polls); reported after a sync.
static int resident_status(gol_engine* e) {
    if (!e->resident || !e->r_ints) return GOL_OK;
    int st = 0;
    cudaError_t ce = cudaMemcpy(&st, e->r_ints + e->rplan.nbands, sizeof(int), cudaMemcpyDeviceToHost);
    if (ce != cudaSuccess) return e->cuda_fail(ce, "resident status");
    return st ? e->fail(st, "a resident-run CTA gave up waiting for a neighbour") : GOL_OK;
}

int gol_sync(gol_engine* e) {
    if (!e) return GOL_E_INVALID;
    if (!e->stream) return GOL_OK;
    cudaError_t ce = cudaStreamSynchronize(e->stream);
    if (ce != cudaSuccess) return e->cuda_fail(ce, "stream synchronize");
    return resident_status(e);
}

int gol_finalize(gol_engine* e) {
    if (!e) return GOL_E_INVALID;
    if (!e->initialized) return e->fail(GOL_E_STATE, "finalize before initialize");
    cudaError_t ce = cudaMemcpyAsync(e->h_words, e->d[e->cur], e->h_bytes, cudaMemcpyDeviceToHost,
                                     e->stream);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(e->stream);
    e->initialized = false;
    if (ce != cudaSuccess) {
        release_device(e);
        return e->cuda_fail(ce, "D2H copy");
    }
    return resident_status(e);
}

int gol_fetch_u8(gol_engine* e, uint8_t* cells) {
    if (!e) return GOL_E_INVALID;
    if (!e->has_host_grid || e->initialized) return e->fail(GOL_E_STATE, "fetch before finalize");
    if (!cells && e->x * e->y) return e->fail(GOL_E_INVALID, "null cells");
    golb200::host_unpack_u8(e->h_words, e->x, e->y, cells);
    return GOL_OK;
}

int gol_fetch_i32(gol_engine* e, int32_t* cells) {
    if (!e) return GOL_E_INVALID;
    if (!e->has_host_grid || e->initialized) return e->fail(GOL_E_STATE, "fetch before finalize");
    if (!cells && e->x * e->y) return e->fail(GOL_E_INVALID, "null cells");
    golb200::host_unpack_i32(e->h_words, e->x, e->y, cells);
    return GOL_OK;
}

int gol_fetch_words(gol_engine* e, void* words, uint32_t word_bits) {
    if (!e) return GOL_E_INVALID;
    if (word_bits != 32 && word_bits != 64) return e->fail(GOL_E_INVALID, "word_bits must be 32 or 64");
    if (e->x % word_bits) return e->fail(GOL_E_INVALID, "x must be a multiple of word_bits");
    if (!e->has_host_grid || e->initialized) return e->fail(GOL_E_STATE, "fetch before finalize");
    if (!words && e->h_bytes) return e->fail(GOL_E_INVALID, "null words");
    std::memcpy(words, e->h_words, e->h_bytes);
    return GOL_OK;
}

int gol_fetch_layout(gol_engine* e, void* words, int layout, uint32_t word_bits) {
    if (!e) return GOL_E_INVALID;
    uint32_t xb, yb;
    if (!golb200::layout_geom(layout, word_bits, &xb, &yb))
        return e->fail(GOL_E_INVALID, "unknown layout or word_bits not 16, 32 or 64");
    if (e->x % xb || e->y % yb) return e->fail(GOL_E_INVALID, "grid is not a whole number of layout words");
    if (!e->has_host_grid || e->initialized) return e->fail(GOL_E_STATE, "fetch before finalize");
    if (!words && e->h_bytes) return e->fail(GOL_E_INVALID, "null words");
    golb200::host_rows_to_layout(e->h_words, e->x, e->y, layout, word_bits, xb, yb, words);
    return GOL_OK;
}

uint64_t gol_performed(const gol_engine* e) { return e ? e->performed : 0; }

void gol_destroy(gol_engine* e) {
    if (!e) return;
    if (e->stream) cudaStreamSynchronize(e->stream);
    release_device(e);
    release_host(e);
    if (e->capture_stream) cudaStreamDestroy(e->capture_stream);
    if (e->own_stream && e->stream) cudaStreamDestroy(e->stream);
    delete e;
}

const char* gol_last_error(const gol_engine* e) {
    return e ? e->err.c_str() : g_create_error.c_str();
}

void* gol_device_grid(gol_engine* e) {
    return (e && e->initialized) ? static_cast<void*>(e->d[e->cur]) : nullptr;
}

void* gol_stream(gol_engine* e) { return e ? static_cast<void*>(e->stream) : nullptr; }

int gol_plan(const gol_engine* e, uint32_t* temporal_steps, uint32_t* band_rows,
             uint32_t* words_per_lane) {
    if (!e) return GOL_E_INVALID;
    if (!e->initialized) return GOL_E_STATE;
    if (e->resident) {   // generations per epoch, the largest CTA band
        if (temporal_steps) *temporal_steps = (uint32_t)e->rplan.K;
        if (band_rows) *band_rows = (uint32_t)e->rplan.band;
        if (words_per_lane) *words_per_lane = (uint32_t)e->rplan.wpl;
        return GOL_OK;
    }
    if (temporal_steps) *temporal_steps = (uint32_t)e->k;
    if (band_rows) *band_rows = (uint32_t)e->plan.band;
    if (words_per_lane) *words_per_lane = (uint32_t)e->plan.wpl;
    return GOL_OK;
}

int gol_rows_pass(const void* d_src, void* d_dst, uint64_t x, uint64_t y, uint32_t k,
                  uint32_t band_rows, void* stream) {
    return gol_rows_pass_ex(d_src, d_dst, x, y, k, band_rows, 0, stream);
}

int gol_rows_pass_ex(const void* d_src, void* d_dst, uint64_t x, uint64_t y, uint32_t k,
                     uint32_t band_rows, uint32_t lane_words, void* stream) {
    if (!d_src || !d_dst || x % 32 || k < 1 || k > (uint32_t)golb200::kMaxTemporalSteps)
        return GOL_E_INVALID;
    if (((uintptr_t)d_src | (uintptr_t)d_dst) & 15u) return GOL_E_INVALID;   // 16-byte lane accesses
    if (x / 32 > (uint64_t)1 << 30 || y > (uint64_t)1 << 30) return GOL_E_INVALID;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return GOL_E_CUDA;
    RowsPlan p;
    if (!golb200::plan_rows((int)(x / 32), (int)y, (int)k, (int)band_rows, (int)lane_words,
                            golb200::device_sm_count(dev), &p))
        return GOL_E_UNSUPPORTED;
    cudaError_t ce = golb200::launch_rows_pass(static_cast<const uint32_t*>(d_src),
                                               static_cast<uint32_t*>(d_dst), (int)(x / 32), (int)y,
                                               (int)k, p, static_cast<cudaStream_t>(stream));
    return ce == cudaSuccess ? GOL_OK : GOL_E_CUDA;
}

int gol_pack_cells_device(const uint8_t* d_cells, void* d_words, uint64_t x, uint64_t y,
                          void* stream) {
    if ((!d_cells || !d_words) && x * y) return GOL_E_INVALID;
    if (x % 32 || ((uintptr_t)d_cells & 15u) || ((uintptr_t)d_words & 3u)) return GOL_E_INVALID;
    cudaError_t ce = golb200::launch_pack_cells(d_cells, static_cast<uint32_t*>(d_words), x, y,
                                                static_cast<cudaStream_t>(stream));
    return ce == cudaSuccess ? GOL_OK : GOL_E_CUDA;
}

int gol_unpack_cells_device(const void* d_words, uint8_t* d_cells, uint64_t x, uint64_t y,
                            void* stream) {
    if ((!d_cells || !d_words) && x * y) return GOL_E_INVALID;
    if (x % 32 || ((uintptr_t)d_cells & 15u) || ((uintptr_t)d_words & 3u)) return GOL_E_INVALID;
    cudaError_t ce = golb200::launch_unpack_cells(static_cast<const uint32_t*>(d_words), d_cells, x,
                                                  y, static_cast<cudaStream_t>(stream));
    return ce == cudaSuccess ? GOL_OK : GOL_E_CUDA;
}

int gol_load_random_ones_zeros(uint8_t* cells, uint64_t x, uint64_t y, uint64_t seed) {
    if (!cells && x * y) return GOL_E_INVALID;
    golb200::host_random_ones_zeros(cells, (size_t)(x * y), seed);
    return GOL_OK;
}

int gol_local_stats(gol_engine* e, uint64_t* passes, uint64_t* tiles_per_pass,
                    uint64_t* computed_total, uint32_t* per_pass, uint64_t max_entries) {
    if (!e) return GOL_E_INVALID;
    if (!e->local || !e->lst.pass_no) return e->fail(GOL_E_STATE, "no change-tracking run");
    uint32_t n = 0;
    cudaError_t ce = cudaStreamSynchronize(e->stream);
    if (ce == cudaSuccess) ce = cudaMemcpy(&n, e->lst.pass_no, sizeof(n), cudaMemcpyDeviceToHost);
    if (ce != cudaSuccess) return e->cuda_fail(ce, "census read");
    const uint32_t rec = n < e->lst.census_cap ? n : e->lst.census_cap;
    uint64_t sum = 0;
    if (rec) {
        uint32_t* tmp = static_cast<uint32_t*>(std::malloc(rec * sizeof(uint32_t)));
        if (!tmp) return e->fail(GOL_E_NOMEM, "host allocation failed");
        ce = cudaMemcpy(tmp, e->lst.census, rec * sizeof(uint32_t), cudaMemcpyDeviceToHost);
        if (ce != cudaSuccess) {
            std::free(tmp);
            return e->cuda_fail(ce, "census read");
        }
        for (uint32_t i = 0; i < rec; ++i) sum += tmp[i];
        if (per_pass) std::memcpy(per_pass, tmp, (size_t)std::min<uint64_t>(rec, max_entries) * 4);
        std::free(tmp);
    }
    if (passes) *passes = n;
    if (tiles_per_pass) *tiles_per_pass = (uint64_t)e->lplan.tiles_x * e->lplan.tiles_y;
    if (computed_total) *computed_total = sum;
    return GOL_OK;
}

int gol_load_sparse_patches(uint8_t* cells, uint64_t x, uint64_t y, uint64_t seed, uint32_t patch,
                            double fraction, double density) {
    if (!cells && x * y) return GOL_E_INVALID;
    const int n = golb200::host_sparse_patches(cells, x, y, seed, patch, fraction, density);
    return n < 0 ? GOL_E_INVALID : n;
}

int gol_workload_uneven(uint64_t seed, uint32_t n, uint32_t min_side, uint32_t max_side,
                        uint32_t multiple, double density_lo, double density_hi, uint64_t gens_lo,
                        uint64_t gens_hi, uint64_t* xs, uint64_t* ys, double* densities,
                        uint64_t* gens, uint64_t* cell_seeds) {
    if (!xs || !ys || !densities || !gens || !cell_seeds || multiple == 0 || min_side == 0 ||
        min_side > max_side || gens_lo == 0 || gens_lo > gens_hi)
        return GOL_E_INVALID;
    golb200::host_workload_uneven(seed, n, min_side, max_side, multiple, density_lo, density_hi,
                                  gens_lo, gens_hi, xs, ys, densities, gens, cell_seeds);
    return GOL_OK;
}

int gol_load_bernoulli(uint8_t* cells, uint64_t x, uint64_t y, uint64_t seed, double density) {
    if (!cells && x * y) return GOL_E_INVALID;
    golb200::host_bernoulli(cells, (size_t)(x * y), seed, density);
    return GOL_OK;
}

int gol_poisson_arrivals(uint64_t seed, uint32_t n, double rate, double* times) {
    if (!times || !(rate > 0)) return GOL_E_INVALID;
    golb200::host_poisson_arrivals(seed, n, rate, times);
    return GOL_OK;
}

int gol_load_hash_bernoulli(uint8_t* cells, uint64_t x, uint64_t y, uint64_t seed, double density) {
    if (!cells && x * y) return GOL_E_INVALID;
    golb200::host_hash_bernoulli(cells, (size_t)(x * y), seed, density);
    return GOL_OK;
}

int gol_probe_int_peak(double* lane_ops_per_s, void* stream) {
    if (!lane_ops_per_s) return GOL_E_INVALID;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return GOL_E_CUDA;
    cudaError_t ce = golb200::probe_lop3_rate(dev, static_cast<cudaStream_t>(stream), lane_ops_per_s);
    return ce == cudaSuccess ? GOL_OK : GOL_E_CUDA;
}

int gol_abi_version(void) { return GOL_B200_ABI_VERSION; }

const char* gol_build_info(void) {
    return "golb200: sm_100a row-band temporal Game of Life engine, CUDA runtime " GOL_STR(CUDART_VERSION);
}

} // extern "C"
