// Host packing between a cell grid and 32-bit row words, the host side of
// the reference's set_and_format_input_data / fetch_result phases
// (GeneralBitGrid::fill_grid / to_grid, general_bit_grid.hpp:171-246):
// cell (cx, cy) at cells[cy*x + cx] maps to bit cx % 32 of word
// cy*(x/32) + cx/32; a nonzero cell is alive; unpacked cells are 0/1.
//
// Packing takes thirty-two cells per AVX2 compare + movemask where the CPU
// has AVX2 (checked at run time), else eight per 64-bit operation (a
// byte-to-bit multiply gather); unpacking expands eight cells per 64-bit
// multiply and streams them out (it is bound by the memory writes); rows
// are split across hardware threads.
#include <sched.h>
#include <unistd.h>

#include <algorithm>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <functional>
#include <mutex>
#include <random>
#include <thread>
#include <vector>

#include "gol_internal.h"

#if defined(__x86_64__) || defined(_M_X64)
#include <immintrin.h>
#define GOL_HAVE_STREAM_STORES 1
#define GOL_HAVE_AVX2_PATH 1
#endif

namespace golb200 {

// Threads this process may run on: its CPU affinity (a container may allow
// fewer CPUs than the machine has).
unsigned usable_cpus() {
    cpu_set_t set;
    if (sched_getaffinity(0, sizeof(set), &set) == 0) {
        const int n = CPU_COUNT(&set);
        if (n > 0) return (unsigned)n;
    }
    const unsigned hw = std::thread::hardware_concurrency();
    return hw ? hw : 1;
}

namespace {

inline uint32_t pack8(uint64_t v) {
    v |= v >> 4;
    v |= v >> 2;
    v |= v >> 1;
    v &= 0x0101010101010101ull;
    return (uint32_t)((v * 0x0102040810204080ull) >> 56);
}

inline uint64_t unpack8(uint32_t b) {
    uint64_t v = (uint64_t)(b & 0xffu) * 0x0101010101010101ull;
    v &= 0x8040201008040201ull;
    return ((v + 0x7f7f7f7f7f7f7f7full) >> 7) & 0x0101010101010101ull;
}

#ifdef GOL_HAVE_AVX2_PATH
bool cpu_has_avx2() {
    static const bool yes = __builtin_cpu_supports("avx2");
    return yes;
}

// Rows [y0, y1): 32 cells (bytes) -> one word, bit i = (cell i != 0).
__attribute__((target("avx2"))) void pack_rows_avx2(const uint8_t* cells, size_t x, size_t y0,
                                                     size_t y1, uint32_t* words) {
    const size_t W = x / 32;
    const __m256i zero = _mm256_setzero_si256();
    for (size_t r = y0; r < y1; ++r) {
        const uint8_t* row = cells + r * x;
        uint32_t* out = words + r * W;
        for (size_t w = 0; w < W; ++w) {
            const __m256i v = _mm256_loadu_si256(reinterpret_cast<const __m256i*>(row + w * 32));
            out[w] = ~(uint32_t)_mm256_movemask_epi8(_mm256_cmpeq_epi8(v, zero));
        }
    }
}

#endif

// Worker threads kept for the life of the process (starting a thread per
// call cost more than packing a few MiB), shared by every caller. A process
// forked from one that started them has no workers (fork copies only the
// calling thread), so there parallel_rows starts threads per call instead.
class RowPool {
  public:
    static RowPool& get() {
        static RowPool* pool = new RowPool();   // never destroyed: workers outlive statics
        return *pool;
    }
    size_t workers() const { return threads_.size(); }
    bool usable() const { return getpid() == pid_; }
    void submit(std::function<void()> job) {
        {
            std::lock_guard<std::mutex> lk(mu_);
            jobs_.push_back(std::move(job));
        }
        cv_.notify_one();
    }

  private:
    RowPool() : pid_(getpid()) {
        const unsigned hw = usable_cpus();
        const size_t n = std::min<size_t>(hw > 1 ? hw - 1 : 0, 63);
        for (size_t i = 0; i < n; ++i) threads_.emplace_back([this] { loop(); });
        for (auto& t : threads_) t.detach();
    }
    void loop() {
        for (;;) {
            std::function<void()> job;
            {
                std::unique_lock<std::mutex> lk(mu_);
                cv_.wait(lk, [this] { return !jobs_.empty(); });
                job = std::move(jobs_.front());
                jobs_.pop_front();
            }
            job();
        }
    }
    pid_t pid_;
    std::mutex mu_;
    std::condition_variable cv_;
    std::deque<std::function<void()>> jobs_;
    std::vector<std::thread> threads_;
};

template <typename F>
void parallel_rows(size_t y, size_t bytes_per_row, F&& body) {
    const size_t total = y * bytes_per_row;
    const unsigned hw = usable_cpus();
    size_t nt = std::max<size_t>(1, std::min<size_t>(hw, 64));
    // One thread per 256 KiB: below that handing out the work costs more
    // than it saves.
    nt = std::min(nt, std::max<size_t>(1, total >> 18));
    nt = std::min(nt, std::max<size_t>(y, 1));
    if (nt <= 1) {
        body(0, y);
        return;
    }
    const size_t per = (y + nt - 1) / nt;
    RowPool& pool = RowPool::get();
    if (!pool.usable() || pool.workers() == 0) {
        std::vector<std::thread> ts;
        for (size_t t = 1; t < nt; ++t) {
            const size_t y0 = t * per, y1 = std::min(y, y0 + per);
            if (y0 >= y1) break;
            ts.emplace_back([&body, y0, y1] { body(y0, y1); });
        }
        body(0, std::min(y, per));
        for (auto& th : ts) th.join();
        return;
    }
    // The count of outstanding ranges is set before the first is handed
    // out: workers decrement it (under mu) while later ranges are still
    // being submitted.
    size_t tasks = 0;
    for (size_t t = 1; t < nt && t * per < y; ++t) ++tasks;
    std::mutex mu;
    std::condition_variable cv;
    size_t left = tasks;
    for (size_t t = 1; t <= tasks; ++t) {
        const size_t y0 = t * per, y1 = std::min(y, y0 + per);
        pool.submit([&, y0, y1] {
            body(y0, y1);
            std::lock_guard<std::mutex> lk(mu);
            if (--left == 0) cv.notify_one();
        });
    }
    body(0, std::min(y, per));
    std::unique_lock<std::mutex> lk(mu);
    cv.wait(lk, [&] { return left == 0; });
}

} // namespace

void host_pack_u8(const uint8_t* cells, size_t x, size_t y, uint32_t* words) {
    const size_t W = x / 32;
#ifdef GOL_HAVE_AVX2_PATH
    if (cpu_has_avx2()) {
        parallel_rows(y, x, [=](size_t y0, size_t y1) { pack_rows_avx2(cells, x, y0, y1, words); });
        return;
    }
#endif
    parallel_rows(y, x, [=](size_t y0, size_t y1) {
        for (size_t r = y0; r < y1; ++r) {
            const uint8_t* row = cells + r * x;
            uint32_t* out = words + r * W;
            for (size_t w = 0; w < W; ++w) {
                uint64_t q[4];
                std::memcpy(q, row + w * 32, 32);
                out[w] = pack8(q[0]) | (pack8(q[1]) << 8) | (pack8(q[2]) << 16) |
                         (pack8(q[3]) << 24);
            }
        }
    });
}

void host_pack_i32(const int32_t* cells, size_t x, size_t y, uint32_t* words) {
    const size_t W = x / 32;
    parallel_rows(y, x * 4, [=](size_t y0, size_t y1) {
        for (size_t r = y0; r < y1; ++r) {
            const int32_t* row = cells + r * x;
            uint32_t* out = words + r * W;
            for (size_t w = 0; w < W; ++w) {
                uint32_t v = 0;
                for (int b = 0; b < 32; ++b) v |= (uint32_t)(row[w * 32 + b] != 0) << b;
                out[w] = v;
            }
        }
    });
}

void host_unpack_u8(const uint32_t* words, size_t x, size_t y, uint8_t* cells) {
    const size_t W = x / 32;
    parallel_rows(y, x, [=](size_t y0, size_t y1) {
#ifdef GOL_HAVE_STREAM_STORES
        // The output is written once and not read back here: stream it past
        // the caches (no read-for-ownership of every line).
        if ((reinterpret_cast<uintptr_t>(cells) & 15u) == 0) {
            for (size_t r = y0; r < y1; ++r) {
                const uint32_t* in = words + r * W;
                __m128i* row = reinterpret_cast<__m128i*>(cells + r * x);
                for (size_t w = 0; w < W; ++w) {
                    const uint32_t v = in[w];
                    _mm_stream_si128(row + 2 * w, _mm_set_epi64x((long long)unpack8(v >> 8),
                                                                 (long long)unpack8(v)));
                    _mm_stream_si128(row + 2 * w + 1, _mm_set_epi64x((long long)unpack8(v >> 24),
                                                                     (long long)unpack8(v >> 16)));
                }
            }
            _mm_sfence();
            return;
        }
#endif
        for (size_t r = y0; r < y1; ++r) {
            const uint32_t* in = words + r * W;
            uint8_t* row = cells + r * x;
            for (size_t w = 0; w < W; ++w) {
                const uint32_t v = in[w];
                uint64_t q[4] = {unpack8(v), unpack8(v >> 8), unpack8(v >> 16), unpack8(v >> 24)};
                std::memcpy(row + w * 32, q, 32);
            }
        }
    });
}

void host_unpack_i32(const uint32_t* words, size_t x, size_t y, int32_t* cells) {
    const size_t W = x / 32;
    parallel_rows(y, x * 4, [=](size_t y0, size_t y1) {
        for (size_t r = y0; r < y1; ++r) {
            const uint32_t* in = words + r * W;
            int32_t* row = cells + r * x;
            for (size_t w = 0; w < W; ++w) {
                const uint32_t v = in[w];
                for (int b = 0; b < 32; ++b) row[w * 32 + b] = (int32_t)((v >> b) & 1u);
            }
        }
    });
}

// RandomOnesZerosDataLoader::load_data (src/infrastructure/data_loader.hpp:57-75):
// std::mt19937 seeded with the seed reduced to the engine's result_type,
// one std::uniform_int_distribution<int>(0, 1) draw per cell in raster
// order. Same standard-library algorithms, so the same grid for a seed.
void host_random_ones_zeros(uint8_t* cells, size_t n, uint64_t seed) {
    std::mt19937 rng(static_cast<std::mt19937::result_type>(seed));
    std::uniform_int_distribution<int> dist(0, 1);
    for (size_t i = 0; i < n; ++i) cells[i] = static_cast<uint8_t>(dist(rng));
}

// Sparse/settling workload: an all-dead grid whose aligned patch x patch
// tile slots are chosen at random and filled with Bernoulli(density) cells.
// Fully specified so any implementation can reproduce it:
//   rng = std::mt19937_64(seed);
//   slots = 0 .. S-1 (row-major over the (x/patch) x (y/patch) slots),
//   Fisher-Yates from the back: for i = S-1 .. 1: j = rng() % (i + 1), swap;
//   the first floor(S * fraction) slots are chosen, then sorted ascending;
//   each chosen slot's cells, row by row, x fastest: alive iff
//   (rng() >> 11) * 2^-53 < density.
int host_sparse_patches(uint8_t* cells, size_t x, size_t y, uint64_t seed, size_t patch,
                        double fraction, double density) {
    if (patch == 0 || x % patch || y % patch || fraction < 0 || fraction > 1) return -1;
    std::memset(cells, 0, x * y);
    const size_t sx = x / patch, sy = y / patch, S = sx * sy;
    std::vector<uint32_t> slots(S);
    for (size_t i = 0; i < S; ++i) slots[i] = (uint32_t)i;
    std::mt19937_64 rng(seed);
    for (size_t i = S; i > 1; --i) {
        const size_t j = (size_t)(rng() % (uint64_t)i);
        std::swap(slots[i - 1], slots[j]);
    }
    const size_t chosen = (size_t)((double)S * fraction);
    std::sort(slots.begin(), slots.begin() + chosen);
    for (size_t c = 0; c < chosen; ++c) {
        const size_t ox = slots[c] % sx * patch, oy = slots[c] / sx * patch;
        for (size_t r = 0; r < patch; ++r)
            for (size_t q = 0; q < patch; ++q)
                cells[(oy + r) * x + ox + q] =
                    (double)(rng() >> 11) * 0x1.0p-53 < density ? 1 : 0;
    }
    return (int)chosen;
}

// Uneven multi-grid workloads (batched and serving configurations). One
// std::mt19937_64(seed) stream, u = (rng() >> 11) * 2^-53, per grid in order:
//   x = mult * llround(exp(ln lo + u * (ln hi - ln lo)) / mult), clamped to [lo, hi]
//   y likewise (next draw), density = dlo + u * (dhi - dlo),
//   gens = llround(exp(ln glo + u * (ln ghi - ln glo))), cell_seed = rng().
static inline double unit(std::mt19937_64& r) { return (double)(r() >> 11) * 0x1.0p-53; }

void host_workload_uneven(uint64_t seed, uint32_t n, uint32_t lo, uint32_t hi, uint32_t mult,
                          double dlo, double dhi, uint64_t glo, uint64_t ghi, uint64_t* xs,
                          uint64_t* ys, double* dens, uint64_t* gens, uint64_t* cell_seeds) {
    std::mt19937_64 rng(seed);
    auto side = [&](double u) {
        const double v = std::exp(std::log((double)lo) + u * (std::log((double)hi) - std::log((double)lo)));
        long long s = std::llround(v / mult) * (long long)mult;
        return (uint64_t)std::min<long long>(std::max<long long>(s, lo), hi);
    };
    for (uint32_t i = 0; i < n; ++i) {
        xs[i] = side(unit(rng));
        ys[i] = side(unit(rng));
        dens[i] = dlo + unit(rng) * (dhi - dlo);
        const double g = std::exp(std::log((double)glo) + unit(rng) * (std::log((double)ghi) - std::log((double)glo)));
        gens[i] = (uint64_t)std::llround(g);
        cell_seeds[i] = rng();
    }
}

// Bernoulli(density) cells in raster order from std::mt19937_64(seed):
// alive iff (rng() >> 11) * 2^-53 < density.
void host_bernoulli(uint8_t* cells, size_t n, uint64_t seed, double density) {
    std::mt19937_64 rng(seed);
    for (size_t i = 0; i < n; ++i) cells[i] = unit(rng) < density ? 1 : 0;
}

// Poisson arrivals: t_0 = 0-based exponential gaps of mean 1/rate from
// std::mt19937_64(seed): t_i = t_{i-1} - ln(1 - u) / rate.
void host_poisson_arrivals(uint64_t seed, uint32_t n, double rate, double* t) {
    std::mt19937_64 rng(seed);
    double now = 0.0;
    for (uint32_t i = 0; i < n; ++i) {
        now += -std::log(1.0 - unit(rng)) / rate;
        t[i] = now;
    }
}

} // namespace golb200
