// Serving: continuous batching of Game of Life simulations on one GPU.
//
// No counterpart in the reference (it runs one grid per invocation,
// experiment_manager.hpp:365-394). Requests (grid + generation count) are
// queued on the host; each round the server
//   1. admits queued requests, in arrival order, whose two grid buffers fit
//      in the free space of a device arena sized from free HBM (first fit,
//      coalescing free list) and copies their packed input in;
//   2. advances every admitted, unfinished request by up to `quantum`
//      generations in ONE persistent launch of the batch kernel (the same
//      dependency-driven work list as gol_batch_run, built for this round,
//      each grid starting from whichever buffer holds its state);
//   3. keeps grids resident between rounds; a request that reaches its
//      generation count is finished once its round's event completes, and
//      its slot returns to the arena when the caller fetches the result.
// The state after a round is known in advance (every request advances a
// fixed number of generations), so round r+1 is planned and queued while
// round r still runs: up to kRoundsInFlight launches are queued back to
// back and the GPU does not wait for the host between rounds. Requests
// arriving meanwhile join the next round planned.
#include <algorithm>
#include <cstring>
#include <deque>
#include <map>
#include <new>
#include <string>
#include <unordered_map>
#include <vector>

#include "gol_b200.h"
#include "gol_internal.h"

namespace {

constexpr int kRoundsInFlight = 3;
constexpr uint64_t kServeTrackMinPasses = 8;   // auto: requests this long track changes
constexpr size_t kStageBytes = (size_t)256 << 20;   // pinned staging ring for host inputs

struct Request {
    uint64_t id = 0;
    uint64_t x = 0, y = 0;
    int W = 0, Y = 0;
    uint64_t gens = 0;          // requested
    uint64_t planned = 0;       // generations covered by rounds queued so far
    std::vector<uint32_t> words;
    bool device_input = false;  // generated on the device at admission (hash Bernoulli)
    uint64_t input_seed = 0;
    double input_density = 0;
    size_t offset = 0, stride = 0;
    size_t slot_words = 0;      // 2 * stride + the change-tracking region, rounded up
    bool tracked = false;       // skips still tiles (its flags live in its slot)
    bool early = false;         // finished before its last planned round: it became still
    int parity = 0;             // buffer holding the state after the rounds queued so far
    golb200::GridChoice plan{};
    int state = 0;              // 0 queued, 1 admitted, 2 finished (after its last round), 3 fetched
    int last_round_slot = -1;   // round buffer slot of its final round
    uint64_t last_round_seq = 0;
};

struct RoundBuffers {
    golb200::BatchGrid* d_grids = nullptr;
    golb200::BatchItem* d_items = nullptr;
    int* d_done = nullptr;
    int* d_ticket = nullptr;
    int* d_status = nullptr;
    int* h_status = nullptr;                 // pinned copy, written by the round's stream
    int* d_pstat = nullptr;                  // per pass of each tracked request
    int* d_still = nullptr;                  // per request of the round: it is still
    int* h_still = nullptr;                  // pinned copy
    size_t cap_grids = 0, cap_items = 0, cap_done = 0, cap_pstat = 0, cap_still = 0;
    // resident rounds (GOL_SERVE_RESIDENT): bands, exchange slots, counters
    golb200::ResidentBand* d_rjobs = nullptr;
    golb200::ResidentBand* h_rjobs = nullptr;   // pinned staging
    uint32_t* d_rpub = nullptr;
    int* d_rdone = nullptr;
    size_t cap_rjobs = 0, cap_rpub = 0, cap_rdone = 0;
    std::vector<uint64_t> ids;               // request of each grid of the round
    golb200::BatchGrid* h_grids = nullptr;   // pinned staging
    golb200::BatchItem* h_items = nullptr;
    cudaEvent_t done_event = nullptr;
    bool in_flight = false;
    uint64_t seq = 0;
    std::vector<uint64_t> finishing;        // requests whose last round this is
};

} // namespace

struct gol_server {
    int device = 0;
    cudaStream_t stream = nullptr;         // uploads and rounds, in order
    bool own_stream = false;
    cudaStream_t copy_stream = nullptr;    // result copies, overlapping later rounds
    // Host inputs reach the device through a pinned staging ring on their
    // own stream (a copy from pageable memory would first wait for every
    // round queued on the round stream); the round stream waits for each
    // upload's event before the round that first uses it.
    cudaStream_t upload_stream = nullptr;
    uint8_t* stage = nullptr;
    size_t stage_bytes = 0, stage_head = 0;
    struct StageUse {
        size_t pos, len;
        cudaEvent_t done;
    };
    std::deque<StageUse> stage_uses;       // uploads whose staging bytes may still be read
    std::vector<cudaEvent_t> free_events;
    int num_sms = 148;
    uint32_t* arena = nullptr;
    size_t arena_words = 0;
    std::map<size_t, size_t> free_blocks;   // offset -> length (words)
    uint64_t quantum = 64;
    int policy = GOL_SERVE_FIFO;
    int track_mode = GOL_TRACK_AUTO;
    int mode = GOL_SERVE_PASSES;           // how a round runs (gol_serve_set_mode)
    unsigned long long* d_census = nullptr;   // wait / work cycles, items computed / skipped
    uint64_t early_finished = 0;
    uint64_t next_id = 1;
    std::unordered_map<uint64_t, Request> reqs;
    std::deque<uint64_t> queue;             // waiting for memory
    std::vector<uint64_t> running;          // admitted, generations left to plan
    std::vector<uint64_t> finished;         // completed, not yet reported
    RoundBuffers rounds[kRoundsInFlight];
    int next_slot = 0;
    uint64_t round_seq = 0;
    uint64_t rounds_launched = 0, admitted = 0, cell_updates_done = 0;
    int status = 0;
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

bool arena_alloc(gol_server* s, size_t words, size_t* off) {
    for (auto it = s->free_blocks.begin(); it != s->free_blocks.end(); ++it) {
        if (it->second >= words) {
            *off = it->first;
            const size_t rest = it->second - words;
            const size_t at = it->first + words;
            s->free_blocks.erase(it);
            if (rest) s->free_blocks[at] = rest;
            return true;
        }
    }
    return false;
}

void arena_free(gol_server* s, size_t off, size_t words) {
    auto it = s->free_blocks.emplace(off, words).first;
    auto next = std::next(it);
    if (next != s->free_blocks.end() && it->first + it->second == next->first) {
        it->second += next->second;
        s->free_blocks.erase(next);
    }
    if (it != s->free_blocks.begin()) {
        auto prev = std::prev(it);
        if (prev->first + prev->second == it->first) {
            prev->second += it->second;
            s->free_blocks.erase(it);
        }
    }
}

int ensure_round_capacity(gol_server* s, RoundBuffers& r, size_t grids, size_t items, size_t done,
                          size_t pstat) {
    cudaError_t ce = cudaSuccess;
    auto grow = [&](size_t need, size_t& cap, auto** dptr, auto** hptr) {
        if (need <= cap || ce != cudaSuccess) return;
        size_t n = std::max<size_t>(need, cap * 2);
        if (*dptr) cudaFree(*dptr);
        if (hptr && *hptr) cudaFreeHost(*hptr);
        *dptr = nullptr;
        ce = cudaMalloc(reinterpret_cast<void**>(dptr), n * sizeof(**dptr));
        if (ce == cudaSuccess && hptr) ce = cudaMallocHost(reinterpret_cast<void**>(hptr), n * sizeof(**hptr));
        cap = ce == cudaSuccess ? n : 0;
    };
    grow(std::max<size_t>(grids, 1), r.cap_grids, &r.d_grids, &r.h_grids);
    grow(std::max<size_t>(items, 1), r.cap_items, &r.d_items, &r.h_items);
    grow(std::max<size_t>(done, 1), r.cap_done, &r.d_done, static_cast<int**>(nullptr));
    grow(std::max<size_t>(pstat, 1), r.cap_pstat, &r.d_pstat, static_cast<int**>(nullptr));
    grow(std::max<size_t>(grids, 1), r.cap_still, &r.d_still, &r.h_still);
    if (ce == cudaSuccess && !r.d_ticket) ce = cudaMalloc(&r.d_ticket, sizeof(int));
    if (ce == cudaSuccess && !r.d_status) ce = cudaMalloc(&r.d_status, sizeof(int));
    if (ce == cudaSuccess && !r.h_status) ce = cudaMallocHost(&r.h_status, sizeof(int));
    if (ce == cudaSuccess && !r.done_event) ce = cudaEventCreateWithFlags(&r.done_event, cudaEventDisableTiming);
    if (ce != cudaSuccess) return s->cuda_fail(ce, "round buffers");
    return GOL_OK;
}

int ensure_resident_capacity(gol_server* s, RoundBuffers& r, size_t jobs, size_t pub, size_t done) {
    cudaError_t ce = cudaSuccess;
    auto grow = [&](size_t need, size_t& cap, auto** dptr, auto** hptr) {
        if (need <= cap || ce != cudaSuccess) return;
        size_t n = std::max<size_t>(need, cap * 2);
        if (*dptr) cudaFree(*dptr);
        if (hptr && *hptr) cudaFreeHost(*hptr);
        *dptr = nullptr;
        ce = cudaMalloc(reinterpret_cast<void**>(dptr), n * sizeof(**dptr));
        if (ce == cudaSuccess && hptr) ce = cudaMallocHost(reinterpret_cast<void**>(hptr), n * sizeof(**hptr));
        cap = ce == cudaSuccess ? n : 0;
    };
    grow(std::max<size_t>(jobs, 1), r.cap_rjobs, &r.d_rjobs, &r.h_rjobs);
    grow(std::max<size_t>(pub, 1), r.cap_rpub, &r.d_rpub, static_cast<uint32_t**>(nullptr));
    grow(std::max<size_t>(done, 1), r.cap_rdone, &r.d_rdone, static_cast<int**>(nullptr));
    if (ce != cudaSuccess) return s->cuda_fail(ce, "resident round buffers");
    return GOL_OK;
}

// Copies a request's packed host input into its slot: through the pinned
// staging ring on the upload stream, the round stream waiting for it (an
// input larger than the ring goes straight from pageable memory).
cudaError_t upload_words(gol_server* s, uint32_t* dst, const std::vector<uint32_t>& words) {
    const size_t len = words.size() * sizeof(uint32_t);
    if (len == 0) return cudaSuccess;
    if (len > s->stage_bytes)
        return cudaMemcpyAsync(dst, words.data(), len, cudaMemcpyHostToDevice, s->stream);
    size_t pos = (s->stage_head + 255) / 256 * 256;
    if (pos + len > s->stage_bytes) pos = 0;
    // wait for the uploads still reading bytes we are about to overwrite
    while (!s->stage_uses.empty()) {
        const auto& u = s->stage_uses.front();
        const bool overlap = u.pos < pos + len && pos < u.pos + u.len;
        if (!overlap && cudaEventQuery(u.done) != cudaSuccess) break;
        cudaError_t ce = cudaEventSynchronize(u.done);
        if (ce != cudaSuccess) return ce;
        s->free_events.push_back(u.done);
        s->stage_uses.pop_front();
    }
    for (const auto& u : s->stage_uses)   // (an older one left overlapping: wait for it too)
        if (u.pos < pos + len && pos < u.pos + u.len) {
            cudaError_t ce = cudaEventSynchronize(u.done);
            if (ce != cudaSuccess) return ce;
        }
    std::memcpy(s->stage + pos, words.data(), len);
    cudaEvent_t ev = nullptr;
    if (!s->free_events.empty()) {
        ev = s->free_events.back();
        s->free_events.pop_back();
    } else {
        cudaError_t ce = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
        if (ce != cudaSuccess) return ce;
    }
    cudaError_t ce = cudaMemcpyAsync(dst, s->stage + pos, len, cudaMemcpyHostToDevice, s->upload_stream);
    if (ce == cudaSuccess) ce = cudaEventRecord(ev, s->upload_stream);
    if (ce == cudaSuccess) ce = cudaStreamWaitEvent(s->stream, ev, 0);
    if (ce != cudaSuccess) {
        s->free_events.push_back(ev);
        return ce;
    }
    s->stage_uses.push_back({pos, len, ev});
    s->stage_head = pos + len;
    return cudaSuccess;
}

// Marks the requests of a completed round finished and checks its status.
int retire_round(gol_server* s, RoundBuffers& r) {
    const int st = *r.h_status;           // copied before the round's event was recorded
    r.in_flight = false;
    if (st != 0) {
        s->status = st;
        return s->fail(st, "a serving round gave up waiting on a dependency");
    }
    for (uint64_t id : r.finishing) {
        auto it = s->reqs.find(id);
        if (it != s->reqs.end() && it->second.state == 1) {
            it->second.state = 2;
            s->finished.push_back(id);
        }
    }
    r.finishing.clear();
    // A request found still in this round (a whole k-generation pass changed
    // nothing, so its state repeats every k generations and both of its
    // buffers hold it): if k divides its generation count it is done now,
    // whatever rounds are still queued for it (their passes end at once). If
    // not, only the remainder (fewer than k generations) is left to plan;
    // rounds already queued for it end at once until that last short pass.
    for (size_t i = 0; i < r.ids.size(); ++i) {
        if (!r.h_still[i]) continue;
        auto it = s->reqs.find(r.ids[i]);
        if (it == s->reqs.end() || it->second.state != 1) continue;
        Request& q = it->second;
        const uint64_t k = (uint64_t)q.plan.k;
        auto run = std::find(s->running.begin(), s->running.end(), r.ids[i]);
        if (q.gens % k == 0) {
            q.state = 2;
            q.early = true;
            s->finished.push_back(r.ids[i]);
            if (run != s->running.end()) s->running.erase(run);
            ++s->early_finished;
        } else if (run != s->running.end()) {
            q.planned = std::max(q.planned, q.gens - q.gens % k);
        }
    }
    r.ids.clear();
    return GOL_OK;
}

// Retires every round whose event has completed (wait = block on the oldest).
int harvest(gol_server* s, bool wait_oldest) {
    for (;;) {
        RoundBuffers* oldest = nullptr;
        for (auto& r : s->rounds)
            if (r.in_flight && (!oldest || r.seq < oldest->seq)) oldest = &r;
        if (!oldest) return GOL_OK;
        cudaError_t q = wait_oldest ? cudaEventSynchronize(oldest->done_event)
                                    : cudaEventQuery(oldest->done_event);
        if (q == cudaErrorNotReady) return GOL_OK;
        if (q != cudaSuccess) return s->cuda_fail(q, "round event");
        int rc = retire_round(s, *oldest);
        if (rc) return rc;
        wait_oldest = false;
    }
}

} // namespace

extern "C" {

int gol_serve_create(gol_server** out, int32_t device, uint64_t arena_bytes, uint32_t quantum,
                     void* stream) {
    if (!out) return GOL_E_INVALID;
    *out = nullptr;
    gol_server* s = new (std::nothrow) gol_server();
    if (!s) return GOL_E_NOMEM;
    s->device = device;
    s->quantum = quantum ? quantum : 64;
    cudaError_t ce = cudaSetDevice(device);
    if (ce == cudaSuccess) {
        if (stream) {
            s->stream = static_cast<cudaStream_t>(stream);
        } else {
            ce = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
            s->own_stream = ce == cudaSuccess;
        }
    }
    if (ce == cudaSuccess) ce = cudaStreamCreateWithFlags(&s->copy_stream, cudaStreamNonBlocking);
    if (ce == cudaSuccess) ce = cudaStreamCreateWithFlags(&s->upload_stream, cudaStreamNonBlocking);
    if (ce == cudaSuccess) {
        s->stage_bytes = kStageBytes;
        ce = cudaMallocHost(&s->stage, s->stage_bytes);
    }
    if (ce == cudaSuccess && arena_bytes == 0) {
        // Admission is bounded by the HBM free when the server starts:
        // half of it goes to resident grids.
        size_t fr = 0, tot = 0;
        ce = cudaMemGetInfo(&fr, &tot);
        arena_bytes = fr / 2;
    }
    if (ce == cudaSuccess) {
        s->arena_words = arena_bytes / sizeof(uint32_t) / 64 * 64;
        ce = cudaMalloc(&s->arena, std::max<size_t>(s->arena_words, 64) * sizeof(uint32_t));
    }
    if (ce == cudaSuccess) ce = cudaMalloc(&s->d_census, 4 * sizeof(unsigned long long));
    if (ce == cudaSuccess) ce = cudaMemsetAsync(s->d_census, 0, 4 * sizeof(unsigned long long), s->stream);
    if (ce != cudaSuccess) {
        if (s->arena) cudaFree(s->arena);
        if (s->d_census) cudaFree(s->d_census);
        if (s->own_stream) cudaStreamDestroy(s->stream);
        if (s->copy_stream) cudaStreamDestroy(s->copy_stream);
        if (s->upload_stream) cudaStreamDestroy(s->upload_stream);
        if (s->stage) cudaFreeHost(s->stage);
        delete s;
        return ce == cudaErrorMemoryAllocation ? GOL_E_NOMEM : GOL_E_CUDA;
    }
    s->free_blocks[0] = s->arena_words;
    s->num_sms = golb200::device_sm_count(device);
    *out = s;
    return GOL_OK;
}

// Every request runs 2 words per lane (1 for an odd word count) at depth
// 4 with its own band height, so a round's launch holds one pipeline family
// (mixed families on one SM compete for the instruction cache). Its slot in
// the arena: the two grid buffers, two counters (items computed / skipped)
// and, when it tracks changes, its change flags and still pass (the
// batch kernel's tracking region), kept for the request's whole life.
static bool plan_request(gol_server* s, Request& r, uint64_t generations) {
    if (!golb200::choose_batch_plan(r.W, r.Y, std::max<uint64_t>(generations, 1), r.W % 2 ? 1 : 2,
                                    golb200::kBatchMaxK, 0, &r.plan))
        return false;
    const uint64_t passes = (generations + r.plan.k - 1) / r.plan.k;
    r.tracked = s->track_mode == GOL_TRACK_ON ||
                (s->track_mode == GOL_TRACK_AUTO && passes >= kServeTrackMinPasses);
    r.stride = ((size_t)r.W * r.Y + 63) / 64 * 64;
    const size_t extra = 2 + (r.tracked ? golb200::batch_trk_words(r.plan.ngroups, r.plan.nslices) : 0);
    r.slot_words = 2 * r.stride + (extra + 63) / 64 * 64;
    return true;
}

static uint32_t* slot_gstat(gol_server* s, const Request& r) { return s->arena + r.offset + 2 * r.stride; }
static uint32_t* slot_trk(gol_server* s, const Request& r) { return slot_gstat(s, r) + 2; }

// Generations a request advances in one round: the quantum. Every round
// but a request's last advances a multiple of its depth k, so its change
// flags (which speak of k-generation passes) stay valid from round to
// round; only the last round may end with a shorter pass. (Giving small
// grids more generations per round, 2^20 / cells quanta, at most 64 or at
// most 4, made rounds as long as those grids' chains of dependent passes:
// on the 2000 req/s stream p50 rose from 9.7 to 36-57 ms and p99 from 94 to
// 430-600 ms, so both policies use the quantum.)
static uint64_t round_generations(const gol_server* s, const Request& r) {
    const uint64_t left = r.gens - r.planned;
    const uint64_t k = (uint64_t)r.plan.k;
    const uint64_t q = std::max(k, s->quantum / k * k);
    return left <= q ? left : q;
}

// A resident round: every running request advances up to the quantum of
// generations with its grid cut into bands held in shared memory (one
// persistent cooperative launch, gol_batch_run_resident's kernel), from its
// current buffer into the other. No change flags: requests finish when their
// generations are done.
static int queue_resident_round(gol_server* s, RoundBuffers& rb) {
    // the round's grids first (requests change state only once it is planned)
    std::vector<golb200::ResidentGrid> grids;
    for (uint64_t id : s->running) {
        const Request& r = s->reqs[id];
        const uint64_t g = std::min<uint64_t>(r.gens - r.planned, s->quantum);
        uint32_t* cur = s->arena + r.offset + (size_t)r.parity * r.stride;
        uint32_t* nxt = s->arena + r.offset + (size_t)(r.parity ^ 1) * r.stride;
        grids.push_back({cur, nxt, r.W, r.W, r.Y, (long long)g});
    }
    golb200::ResidentBatchPlan plan;
    if (const char* why = golb200::plan_resident_batch(grids.data(), grids.size(), s->num_sms,
                                                       s->device, &plan))
        return s->fail(GOL_E_UNSUPPORTED, why);
    std::vector<uint64_t> still;
    rb.ids.clear();
    for (size_t i = 0; i < s->running.size(); ++i) {
        const uint64_t id = s->running[i];
        Request& r = s->reqs[id];
        const uint64_t g = (uint64_t)grids[i].gens;
        rb.ids.push_back(id);
        r.planned += g;
        r.parity ^= 1;
        s->cell_updates_done += r.x * r.y * g;
        if (r.planned >= r.gens)
            rb.finishing.push_back(id);
        else
            still.push_back(id);
    }
    s->running.swap(still);
    int rc = ensure_round_capacity(s, rb, grids.size(), 1, 1, 1);
    if (rc) return rc;
    if ((rc = ensure_resident_capacity(s, rb, (size_t)plan.ndone, plan.pub_words, (size_t)plan.ndone)))
        return rc;
    golb200::fill_resident_jobs(plan, grids.data(), rb.d_rpub, rb.d_rdone, rb.h_rjobs);
    cudaError_t ce = cudaMemcpyAsync(rb.d_rjobs, rb.h_rjobs, (size_t)plan.ndone * sizeof(golb200::ResidentBand),
                                     cudaMemcpyHostToDevice, s->stream);
    if (ce == cudaSuccess) ce = cudaMemsetAsync(rb.d_rdone, 0, (size_t)std::max(plan.ndone, 1) * sizeof(int), s->stream);
    if (ce == cudaSuccess) ce = cudaMemsetAsync(rb.d_ticket, 0, sizeof(int), s->stream);
    if (ce == cudaSuccess) ce = cudaMemsetAsync(rb.d_status, 0, sizeof(int), s->stream);
    if (ce == cudaSuccess) ce = cudaMemsetAsync(rb.d_still, 0, grids.size() * sizeof(int), s->stream);
    if (ce == cudaSuccess && plan.ndone)
        ce = golb200::launch_batch_resident(rb.d_rjobs, plan.ndone, rb.d_ticket, rb.d_status, plan, s->stream);
    if (ce == cudaSuccess)
        ce = cudaMemcpyAsync(rb.h_status, rb.d_status, sizeof(int), cudaMemcpyDeviceToHost, s->stream);
    if (ce == cudaSuccess)
        ce = cudaMemcpyAsync(rb.h_still, rb.d_still, grids.size() * sizeof(int), cudaMemcpyDeviceToHost,
                             s->stream);
    if (ce == cudaSuccess) ce = cudaEventRecord(rb.done_event, s->stream);
    if (ce != cudaSuccess) return s->cuda_fail(ce, "resident round launch");
    rb.in_flight = true;
    rb.seq = ++s->round_seq;
    for (uint64_t id : rb.finishing) {
        s->reqs[id].last_round_slot = s->next_slot;
        s->reqs[id].last_round_seq = rb.seq;
    }
    ++s->rounds_launched;
    s->next_slot = (s->next_slot + 1) % kRoundsInFlight;
    return GOL_OK;
}

int gol_serve_submit(gol_server* s, const uint8_t* cells, uint64_t x, uint64_t y,
                     uint64_t generations, uint64_t* id) {
    if (!s) return GOL_E_INVALID;
    if (!cells || x == 0 || y == 0 || x % 32) return s->fail(GOL_E_INVALID, "x must be a positive multiple of 32");
    if (y > (1u << 30) || generations > (1ull << 40)) return s->fail(GOL_E_INVALID, "request too large");
    Request r;
    r.id = s->next_id++;
    r.x = x;
    r.y = y;
    r.W = (int)(x / 32);
    r.Y = (int)y;
    r.gens = generations;
    if (!plan_request(s, r, generations)) return s->fail(GOL_E_UNSUPPORTED, "no plan for this request");
    if (s->mode == GOL_SERVE_RESIDENT && !golb200::resident_batch_fits(r.W, r.Y, s->num_sms, s->device))
        return s->fail(GOL_E_UNSUPPORTED, "request does not fit a resident round");
    if (r.slot_words > s->arena_words) return s->fail(GOL_E_NOMEM, "request larger than the device arena");
    r.words.resize((size_t)r.W * r.Y);
    golb200::host_pack_u8(cells, x, y, r.words.data());
    if (id) *id = r.id;
    s->queue.push_back(r.id);
    s->reqs.emplace(r.id, std::move(r));
    return GOL_OK;
}

// A request whose input is generated on the device when it is admitted:
// cell i is alive iff (mix64(seed + (i+1) * 0x9E3779B97F4A7C15) >> 11) * 2^-53
// < density (gol_load_hash_bernoulli gives the same cells on the host).
int gol_serve_submit_random(gol_server* s, uint64_t x, uint64_t y, uint64_t generations,
                            uint64_t seed, double density, uint64_t* id) {
    if (!s) return GOL_E_INVALID;
    if (x == 0 || y == 0 || x % 32) return s->fail(GOL_E_INVALID, "x must be a positive multiple of 32");
    if (y > (1u << 30) || generations > (1ull << 40)) return s->fail(GOL_E_INVALID, "request too large");
    Request r;
    r.id = s->next_id++;
    r.x = x;
    r.y = y;
    r.W = (int)(x / 32);
    r.Y = (int)y;
    r.gens = generations;
    r.device_input = true;
    r.input_seed = seed;
    r.input_density = density;
    if (!plan_request(s, r, generations)) return s->fail(GOL_E_UNSUPPORTED, "no plan for this request");
    if (s->mode == GOL_SERVE_RESIDENT && !golb200::resident_batch_fits(r.W, r.Y, s->num_sms, s->device))
        return s->fail(GOL_E_UNSUPPORTED, "request does not fit a resident round");
    if (r.slot_words > s->arena_words) return s->fail(GOL_E_NOMEM, "request larger than the device arena");
    if (id) *id = r.id;
    s->queue.push_back(r.id);
    s->reqs.emplace(r.id, std::move(r));
    return GOL_OK;
}

// One scheduling step: retire completed rounds, admit what fits, and queue
// the next round if any admitted request has generations left. Returns
// without waiting unless kRoundsInFlight rounds are already queued.
int gol_serve_step(gol_server* s) {
    if (!s) return GOL_E_INVALID;
    if (s->status) return s->fail(s->status, "server stopped after a device-side timeout");
    cudaError_t ce = cudaSetDevice(s->device);
    if (ce != cudaSuccess) return s->cuda_fail(ce, "cudaSetDevice");
    int rc = harvest(s, false);
    if (rc) return rc;

    // Admission: arrival order (FIFO) or least work first (SRPT: cells x
    // generations); a request that does not fit lets later ones through.
    if (s->policy == GOL_SERVE_SRPT && s->queue.size() > 1)
        std::stable_sort(s->queue.begin(), s->queue.end(), [s](uint64_t a, uint64_t b) {
            const Request& ra = s->reqs[a];
            const Request& rb = s->reqs[b];
            return (double)ra.x * ra.y * ra.gens < (double)rb.x * rb.y * rb.gens;
        });
    for (auto it = s->queue.begin(); it != s->queue.end();) {
        Request& r = s->reqs[*it];
        size_t off = 0;
        if (!arena_alloc(s, r.slot_words, &off)) {
            ++it;
            continue;
        }
        r.offset = off;
        r.parity = 0;
        r.state = 1;
        if (r.device_input) {
            ce = golb200::launch_hash_bernoulli(s->arena + off, r.x, r.y, r.input_seed,
                                                r.input_density, s->stream);
        } else {
            ce = upload_words(s, s->arena + off, r.words);
        }
        // counters zero; change flags "changed" (the first pass computes
        // every tile) and no still pass
        if (ce == cudaSuccess) ce = cudaMemsetAsync(slot_gstat(s, r), 0, 2 * sizeof(uint32_t), s->stream);
        if (ce == cudaSuccess && r.tracked)
            ce = cudaMemsetAsync(slot_trk(s, r), 0xff,
                                 golb200::batch_trk_words(r.plan.ngroups, r.plan.nslices) * sizeof(uint32_t),
                                 s->stream);
        if (ce != cudaSuccess) return s->cuda_fail(ce, "request upload");
        std::vector<uint32_t>().swap(r.words);   // a pageable source is staged before the call returns
        if (r.gens == 0) {               // nothing to run: finished at once
            r.state = 2;
            s->finished.push_back(r.id);
        } else {
            s->running.push_back(r.id);
        }
        ++s->admitted;
        it = s->queue.erase(it);
    }
    if (s->running.empty()) return GOL_OK;

    RoundBuffers& rb = s->rounds[s->next_slot];
    if (rb.in_flight) {                   // all round slots queued: wait for the oldest
        rc = harvest(s, true);
        if (rc) return rc;
    }
    if (s->mode == GOL_SERVE_RESIDENT) return queue_resident_round(s, rb);
    // Plan this round: every running request advances its round's
    // generations (round_generations).
    std::vector<golb200::BatchGrid> grids;
    int done = 0, max_passes = 0;
    size_t pstat = 0;
    bool track_any = false;
    std::vector<size_t> pstat_off;   // per grid: its pass counters in rb.d_pstat (tracked grids)
    std::vector<uint64_t> still;
    rb.ids.clear();
    for (uint64_t id : s->running) {
        Request& r = s->reqs[id];
        const uint64_t g = round_generations(s, r);
        golb200::GridChoice ch = r.plan;
        ch.passes = (int)((g + ch.k - 1) / ch.k);
        ch.last_k = g % ch.k ? (int)(g % ch.k) : ch.k;
        golb200::BatchGrid bg{};
        golb200::batch_grid_from_choice(ch, r.W, r.Y, &bg);
        bg.buf[0] = s->arena + r.offset;
        bg.buf[1] = s->arena + r.offset + r.stride;
        bg.parity0 = r.parity;
        bg.pass0 = (int)std::min<uint64_t>(r.planned / (uint64_t)ch.k, 0x3fffffff);
        bg.done_base = done;
        done += bg.ngroups * bg.nslices;
        max_passes = std::max(max_passes, bg.passes);
        bg.gstat = slot_gstat(s, r);
        pstat_off.push_back(pstat);
        if (r.tracked) {   // flags and still pass stay in the slot between rounds
            bg.trk = slot_trk(s, r);
            pstat += 2 * (size_t)bg.passes;
            track_any = true;
        }
        rb.ids.push_back(id);
        grids.push_back(bg);
        r.planned += g;
        r.parity = (r.parity + ch.passes) & 1;
        s->cell_updates_done += r.x * r.y * g;
        if (r.planned >= r.gens) {
            rb.finishing.push_back(id);
        } else {
            still.push_back(id);
        }
    }
    s->running.swap(still);
    const size_t nitems = golb200::count_batch_items(grids.data(), grids.size());
    if ((rc = ensure_round_capacity(s, rb, grids.size(), nitems, (size_t)done, pstat))) return rc;
    for (size_t i = 0; i < grids.size(); ++i) {
        grids[i].rflag = rb.d_still + i;
        if (grids[i].trk) grids[i].pstat = rb.d_pstat + pstat_off[i];
    }
    golb200::order_batch_items(grids.data(), grids.size(), rb.h_items);
    (void)max_passes;
    std::memcpy(rb.h_grids, grids.data(), grids.size() * sizeof(golb200::BatchGrid));
    ce = cudaMemcpyAsync(rb.d_grids, rb.h_grids, grids.size() * sizeof(golb200::BatchGrid),
                         cudaMemcpyHostToDevice, s->stream);
    if (ce == cudaSuccess)
        ce = cudaMemcpyAsync(rb.d_items, rb.h_items, nitems * sizeof(golb200::BatchItem),
                             cudaMemcpyHostToDevice, s->stream);
    if (ce == cudaSuccess) ce = cudaMemsetAsync(rb.d_done, 0, (size_t)std::max(done, 1) * sizeof(int), s->stream);
    if (ce == cudaSuccess) ce = cudaMemsetAsync(rb.d_ticket, 0, sizeof(int), s->stream);
    if (ce == cudaSuccess) ce = cudaMemsetAsync(rb.d_status, 0, sizeof(int), s->stream);
    if (ce == cudaSuccess && pstat) ce = cudaMemsetAsync(rb.d_pstat, 0, pstat * sizeof(int), s->stream);
    if (ce == cudaSuccess) ce = cudaMemsetAsync(rb.d_still, 0, grids.size() * sizeof(int), s->stream);
    if (ce == cudaSuccess)
        ce = golb200::launch_batch_kernel(rb.d_grids, rb.d_items, (int)nitems, rb.d_ticket, rb.d_done,
                                          rb.d_status, s->num_sms, s->stream, s->d_census,
                                          golb200::batch_uniform_wpl(grids.data(), grids.size()), 0,
                                          track_any);
    if (ce == cudaSuccess)
        ce = cudaMemcpyAsync(rb.h_status, rb.d_status, sizeof(int), cudaMemcpyDeviceToHost, s->stream);
    if (ce == cudaSuccess)
        ce = cudaMemcpyAsync(rb.h_still, rb.d_still, grids.size() * sizeof(int), cudaMemcpyDeviceToHost,
                             s->stream);
    if (ce == cudaSuccess) ce = cudaEventRecord(rb.done_event, s->stream);
    if (ce != cudaSuccess) return s->cuda_fail(ce, "round launch");
    rb.in_flight = true;
    rb.seq = ++s->round_seq;
    for (uint64_t id : rb.finishing) {
        s->reqs[id].last_round_slot = s->next_slot;
        s->reqs[id].last_round_seq = rb.seq;
    }
    ++s->rounds_launched;
    s->next_slot = (s->next_slot + 1) % kRoundsInFlight;
    return GOL_OK;
}

// Ids finished since the last call (their results are ready to fetch).
int gol_serve_finished(gol_server* s, uint64_t* ids, uint32_t max_ids, uint32_t* count) {
    if (!s || !count) return GOL_E_INVALID;
    int rc = harvest(s, false);
    if (rc) return rc;
    const uint32_t n = (uint32_t)std::min<size_t>(s->finished.size(), max_ids);
    for (uint32_t i = 0; i < n; ++i) ids[i] = s->finished[i];
    s->finished.erase(s->finished.begin(), s->finished.begin() + n);
    *count = n;
    return GOL_OK;
}

// Copies a finished request's grid out and returns its slot to the arena.
int gol_serve_fetch(gol_server* s, uint64_t id, uint8_t* cells) {
    if (!s || !cells) return GOL_E_INVALID;
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return s->fail(GOL_E_INVALID, "unknown request");
    Request& r = it->second;
    if (r.state != 2) return s->fail(GOL_E_STATE, "request not finished");
    // Its last round has completed and no later round writes its grid (a
    // request finished early is still: rounds still queued for it end at
    // once), so the copy runs on its own stream, beside the rounds still
    // queued. A request with no generations never ran: wait for its upload.
    cudaError_t ce = cudaSuccess;
    if (r.gens == 0) ce = cudaStreamSynchronize(s->stream);
    std::vector<uint32_t> words((size_t)r.W * r.Y);
    if (ce == cudaSuccess)
        ce = cudaMemcpyAsync(words.data(), s->arena + r.offset + (size_t)r.parity * r.stride,
                             words.size() * sizeof(uint32_t), cudaMemcpyDeviceToHost, s->copy_stream);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(s->copy_stream);
    if (ce != cudaSuccess) return s->cuda_fail(ce, "result copy");
    golb200::host_unpack_u8(words.data(), r.x, r.y, cells);
    arena_free(s, r.offset, r.slot_words);
    s->reqs.erase(it);
    return GOL_OK;
}

// Packed result (x/32 uint32 words per row) of a finished request; frees its slot.
int gol_serve_fetch_words(gol_server* s, uint64_t id, void* words) {
    if (!s || !words) return GOL_E_INVALID;
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return s->fail(GOL_E_INVALID, "unknown request");
    Request& r = it->second;
    if (r.state != 2) return s->fail(GOL_E_STATE, "request not finished");
    cudaError_t ce = cudaSuccess;
    if (r.gens == 0) ce = cudaStreamSynchronize(s->stream);
    if (ce == cudaSuccess)
        ce = cudaMemcpyAsync(words, s->arena + r.offset + (size_t)r.parity * r.stride,
                             (size_t)r.W * r.Y * sizeof(uint32_t), cudaMemcpyDeviceToHost, s->copy_stream);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(s->copy_stream);
    if (ce != cudaSuccess) return s->cuda_fail(ce, "result copy");
    arena_free(s, r.offset, r.slot_words);
    s->reqs.erase(it);
    return GOL_OK;
}

// Drops a finished request without copying it out.
int gol_serve_release(gol_server* s, uint64_t id) {
    if (!s) return GOL_E_INVALID;
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return s->fail(GOL_E_INVALID, "unknown request");
    if (it->second.state != 2) return s->fail(GOL_E_STATE, "request not finished");
    arena_free(s, it->second.offset, it->second.slot_words);
    s->reqs.erase(it);
    return GOL_OK;
}

// Queued (waiting for memory), running, and finished-but-unfetched counts.
int gol_serve_stats(const gol_server* s, uint64_t* queued, uint64_t* running, uint64_t* rounds,
                    uint64_t* cell_updates, uint64_t* arena_free_bytes) {
    if (!s) return GOL_E_INVALID;
    size_t fr = 0;
    for (const auto& b : s->free_blocks) fr += b.second;
    if (queued) *queued = s->queue.size();
    if (running) *running = s->running.size();
    if (rounds) *rounds = s->rounds_launched;
    if (cell_updates) *cell_updates = s->cell_updates_done;
    if (arena_free_bytes) *arena_free_bytes = fr * sizeof(uint32_t);
    return GOL_OK;
}

// Waits for every queued round.
int gol_serve_drain(gol_server* s) {
    if (!s) return GOL_E_INVALID;
    for (int i = 0; i < kRoundsInFlight; ++i) {
        int rc = harvest(s, true);
        if (rc) return rc;
    }
    return GOL_OK;
}

int gol_serve_set_policy(gol_server* s, int32_t policy) {
    if (!s) return GOL_E_INVALID;
    if (policy != GOL_SERVE_FIFO && policy != GOL_SERVE_SRPT)
        return s->fail(GOL_E_INVALID, "policy must be GOL_SERVE_FIFO or GOL_SERVE_SRPT");
    s->policy = policy;
    return GOL_OK;
}

int gol_serve_set_tracking(gol_server* s, int32_t mode) {
    if (!s) return GOL_E_INVALID;
    if (mode != GOL_TRACK_AUTO && mode != GOL_TRACK_OFF && mode != GOL_TRACK_ON)
        return s->fail(GOL_E_INVALID, "tracking mode must be GOL_TRACK_AUTO, _OFF or _ON");
    s->track_mode = mode;
    return GOL_OK;
}

int gol_serve_set_mode(gol_server* s, int32_t mode) {
    if (!s) return GOL_E_INVALID;
    if (mode != GOL_SERVE_PASSES && mode != GOL_SERVE_RESIDENT)
        return s->fail(GOL_E_INVALID, "mode must be GOL_SERVE_PASSES or GOL_SERVE_RESIDENT");
    if (!s->running.empty() || !s->queue.empty())
        return s->fail(GOL_E_STATE, "the round mode changes only while no request is queued or running");
    s->mode = mode;
    return GOL_OK;
}

int gol_serve_tiles(gol_server* s, uint64_t* computed, uint64_t* skipped, uint64_t* early_finished) {
    if (!s) return GOL_E_INVALID;
    unsigned long long c[4] = {0, 0, 0, 0};
    cudaError_t ce = cudaMemcpy(c, s->d_census, sizeof(c), cudaMemcpyDeviceToHost);
    if (ce != cudaSuccess) return s->cuda_fail(ce, "serving census");
    if (computed) *computed = c[2];
    if (skipped) *skipped = c[3];
    if (early_finished) *early_finished = s->early_finished;
    return GOL_OK;
}

const char* gol_serve_last_error(const gol_server* s) { return s ? s->err.c_str() : "null server"; }

void* gol_serve_stream(gol_server* s) { return s ? static_cast<void*>(s->stream) : nullptr; }

void gol_serve_destroy(gol_server* s) {
    if (!s) return;
    if (s->stream) cudaStreamSynchronize(s->stream);
    for (auto& r : s->rounds) {
        if (r.d_grids) cudaFree(r.d_grids);
        if (r.d_items) cudaFree(r.d_items);
        if (r.d_done) cudaFree(r.d_done);
        if (r.d_ticket) cudaFree(r.d_ticket);
        if (r.d_status) cudaFree(r.d_status);
        if (r.h_grids) cudaFreeHost(r.h_grids);
        if (r.h_status) cudaFreeHost(r.h_status);
        if (r.h_items) cudaFreeHost(r.h_items);
        if (r.d_pstat) cudaFree(r.d_pstat);
        if (r.d_still) cudaFree(r.d_still);
        if (r.h_still) cudaFreeHost(r.h_still);
        if (r.d_rjobs) cudaFree(r.d_rjobs);
        if (r.h_rjobs) cudaFreeHost(r.h_rjobs);
        if (r.d_rpub) cudaFree(r.d_rpub);
        if (r.d_rdone) cudaFree(r.d_rdone);
        if (r.done_event) cudaEventDestroy(r.done_event);
    }
    if (s->arena) cudaFree(s->arena);
    if (s->d_census) cudaFree(s->d_census);
    if (s->copy_stream) cudaStreamDestroy(s->copy_stream);
    if (s->upload_stream) cudaStreamSynchronize(s->upload_stream);
    for (auto& u : s->stage_uses) cudaEventDestroy(u.done);
    for (auto ev : s->free_events) cudaEventDestroy(ev);
    if (s->upload_stream) cudaStreamDestroy(s->upload_stream);
    if (s->stage) cudaFreeHost(s->stage);
    if (s->own_stream && s->stream) cudaStreamDestroy(s->stream);
    delete s;
}

} // extern "C"
