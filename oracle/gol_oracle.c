#define _GNU_SOURCE
/*
 * ORACLE — test infrastructure, not product code.
 *
 * A plain-C restatement of the reference's CPU path for bit-packed Conway
 * Game of Life (B3/S23, cells outside the grid dead), used only as the
 * checker by tests/, __graft_entry__.smoke() and bench.py's cpu_baseline
 * leg. Nothing in the product links or calls this file.
 *
 * Parity pin: every function here is checked against the reference itself
 * (oracle/_ref/libgolref.so, built from the reference sources by
 * oracle/Makefile) in tests/test_oracle.py, and the golden fixtures under
 * tests/golden/ were produced by the reference build
 * (tests/golden/make_golden.py).
 *
 * Functions and the reference code each one restates:
 *   gor_random_ones_zeros  RandomOnesZerosDataLoader::load_data
 *                          (src/infrastructure/data_loader.hpp:57-75):
 *                          std::mt19937(seed) feeding
 *                          std::uniform_int_distribution<int>(0, 1) over the
 *                          cells in raster order i = y*X + x. MT19937 is the
 *                          published Matsumoto-Nishimura generator; libstdc++
 *                          maps a 32-bit engine onto {0,1} with Lemire's
 *                          multiply-shift, (u * 2) >> 32, i.e. the top bit.
 *   gor_life_naive         GoLCpuNaive::run / count_alive_neighbours
 *                          (src/algorithms/cpu-naive/gol_cpu_naive.hpp:26-117)
 *   gor_pack_rows,         GeneralBitGrid<uintW_t, FullyPackedRows> fill_grid /
 *   gor_unpack_rows        to_grid (src/algorithms/_shared/bitwise/
 *                          general_bit_grid.hpp:171-246, bit_modes.hpp:127-148):
 *                          bit i of word (xw, y) is cell (xw*W + i, y), words
 *                          stored row-major at y*(X/W) + xw.
 *   gor_pack_layout,       GeneralBitGrid<uintW_t, BitColumnsMode | BitTileMode>
 *   gor_unpack_layout      fill_grid / to_grid (general_bit_grid.hpp:171-246,
 *                          bit_modes.hpp:10-125, 165-177): words hold
 *                          X_BITS x Y_BITS cell blocks, stored row-major at
 *                          (y / Y_BITS) * (X / X_BITS) + x / X_BITS.
 *   gor_life_rows          GoLCpuBitwise<char, W, AdderOps>::run
 *                          (src/algorithms/cpu-bitwise-general/
 *                          gol_cpu_bitwise_general.hpp:32-120) with the
 *                          per-word adder of
 *                          src/algorithms/_shared/bitwise/bitwise-ops/adder.cuh:17-104.
 *
 * Build: oracle/Makefile (gcc -O3 -pthread -shared).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <pthread.h>
#include <sched.h>
#include <unistd.h>

/* ---------------------------------------------------------------------- */
/* MT19937 + uniform {0,1}  (data_loader.hpp:60-74)                        */
/* ---------------------------------------------------------------------- */

typedef struct {
    uint32_t mt[624];
    int idx;
} gor_mt19937;

static void gor_mt_seed(gor_mt19937* s, uint32_t seed) {
    s->mt[0] = seed;
    for (int i = 1; i < 624; ++i)
        s->mt[i] = 1812433253u * (s->mt[i - 1] ^ (s->mt[i - 1] >> 30)) + (uint32_t)i;
    s->idx = 624;
}

static uint32_t gor_mt_next(gor_mt19937* s) {
    if (s->idx >= 624) {
        for (int i = 0; i < 624; ++i) {
            uint32_t y = (s->mt[i] & 0x80000000u) | (s->mt[(i + 1) % 624] & 0x7fffffffu);
            s->mt[i] = s->mt[(i + 397) % 624] ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
        }
        s->idx = 0;
    }
    uint32_t y = s->mt[s->idx++];
    y ^= y >> 11;
    y ^= (y << 7) & 0x9d2c5680u;
    y ^= (y << 15) & 0xefc60000u;
    y ^= y >> 18;
    return y;
}

/* std::mt19937 seeds from result_type (uint_fast32_t) reduced mod 2^32. */
int gor_random_ones_zeros(uint64_t x, uint64_t y, uint64_t seed, uint8_t* out) {
    gor_mt19937 s;
    gor_mt_seed(&s, (uint32_t)seed);
    uint64_t n = x * y;
    for (uint64_t i = 0; i < n; ++i) {
        uint64_t product = (uint64_t)gor_mt_next(&s) * 2u;
        out[i] = (uint8_t)(product >> 32);
    }
    return 0;
}

/* ---------------------------------------------------------------------- */
/* Naive cell grid  (gol_cpu_naive.hpp:26-117)                             */
/* ---------------------------------------------------------------------- */

/* Centre alive iff the byte is 1 (gol_cpu_naive.hpp:55); a neighbour counts
 * iff the byte, read as char, is > 0 (:114); out-of-grid neighbours are
 * skipped (:108-111). Generations ping-pong between two grids (:75). */
int gor_life_naive(const uint8_t* in, uint64_t x, uint64_t y, uint64_t iters, uint8_t* out) {
    uint64_t n = x * y;
    uint8_t* a = (uint8_t*)malloc(n ? n : 1);
    uint8_t* b = (uint8_t*)malloc(n ? n : 1);
    if (!a || !b) {
        free(a);
        free(b);
        return -1;
    }
    memcpy(a, in, n);
    uint8_t* src = a;
    uint8_t* dst = b;
    for (uint64_t it = 0; it < iters; ++it) {
        for (uint64_t yy = 0; yy < y; ++yy) {
            for (uint64_t xx = 0; xx < x; ++xx) {
                int alive_nei = 0;
                for (int i = -1; i <= 1; ++i) {
                    for (int j = -1; j <= 1; ++j) {
                        if (i == 0 && j == 0) continue;
                        uint64_t nx = xx + (uint64_t)(int64_t)i;
                        uint64_t ny = yy + (uint64_t)(int64_t)j;
                        if (nx >= x || ny >= y) continue;
                        alive_nei += ((signed char)src[ny * x + nx] > 0) ? 1 : 0;
                    }
                }
                uint8_t c = src[yy * x + xx];
                uint8_t next;
                if (c == 1)
                    next = (alive_nei < 2 || alive_nei > 3) ? 0 : 1;
                else
                    next = (alive_nei == 3) ? 1 : 0;
                dst[yy * x + xx] = next;
            }
        }
        uint8_t* t = src;
        src = dst;
        dst = t;
    }
    memcpy(out, src, n);
    free(a);
    free(b);
    return 0;
}

/* ---------------------------------------------------------------------- */
/* Row packing  (general_bit_grid.hpp:171-246, bit_modes.hpp:127-148)      */
/* ---------------------------------------------------------------------- */

int gor_pack_rows(int word_bits, const uint8_t* cells, uint64_t x, uint64_t y, void* words) {
    if (word_bits != 32 && word_bits != 64) return -2;
    if (x % (uint64_t)word_bits) return -3;
    uint64_t wx = x / (uint64_t)word_bits;
    for (uint64_t yy = 0; yy < y; ++yy) {
        for (uint64_t xw = 0; xw < wx; ++xw) {
            uint64_t w = 0;
            for (int bit = 0; bit < word_bits; ++bit)
                if (cells[yy * x + xw * (uint64_t)word_bits + (uint64_t)bit]) w |= (uint64_t)1 << bit;
            if (word_bits == 64)
                ((uint64_t*)words)[yy * wx + xw] = w;
            else
                ((uint32_t*)words)[yy * wx + xw] = (uint32_t)w;
        }
    }
    return 0;
}

int gor_unpack_rows(int word_bits, const void* words, uint64_t x, uint64_t y, uint8_t* cells) {
    if (word_bits != 32 && word_bits != 64) return -2;
    if (x % (uint64_t)word_bits) return -3;
    uint64_t wx = x / (uint64_t)word_bits;
    for (uint64_t yy = 0; yy < y; ++yy) {
        for (uint64_t xw = 0; xw < wx; ++xw) {
            uint64_t w = (word_bits == 64) ? ((const uint64_t*)words)[yy * wx + xw]
                                           : (uint64_t)((const uint32_t*)words)[yy * wx + xw];
            for (int bit = 0; bit < word_bits; ++bit)
                cells[yy * x + xw * (uint64_t)word_bits + (uint64_t)bit] = (uint8_t)((w >> bit) & 1u);
        }
    }
    return 0;
}

/* ---------------------------------------------------------------------- */
/* Column and tile layouts  (bit_modes.hpp:10-125)                          */
/* ---------------------------------------------------------------------- */

/* layout 1 = BitColumns<uintW>: X_BITS 1, Y_BITS W; the first mask is bit 0
 *            and each next cell (down the column) moves it one bit up.
 * layout 2 = BitTile<uintW>: 4x4 (16-bit), 8x4 (32-bit), 8x8 (64-bit); the
 *            first mask is the top bit and each next cell (x fastest, then y)
 *            moves it one bit down. */
static int gor_layout_geom(int layout, int word_bits, uint64_t* xb, uint64_t* yb) {
    if (word_bits != 16 && word_bits != 32 && word_bits != 64) return -2;
    if (layout == 1) {
        *xb = 1;
        *yb = (uint64_t)word_bits;
        return 0;
    }
    if (layout == 2) {
        *xb = word_bits == 16 ? 4 : 8;
        *yb = word_bits == 64 ? 8 : 4;
        return 0;
    }
    return -2;
}

static uint64_t gor_get_word(const void* words, int word_bits, uint64_t i) {
    if (word_bits == 64) return ((const uint64_t*)words)[i];
    if (word_bits == 32) return ((const uint32_t*)words)[i];
    return ((const uint16_t*)words)[i];
}

static void gor_set_word(void* words, int word_bits, uint64_t i, uint64_t w) {
    if (word_bits == 64) ((uint64_t*)words)[i] = w;
    else if (word_bits == 32) ((uint32_t*)words)[i] = (uint32_t)w;
    else ((uint16_t*)words)[i] = (uint16_t)w;
}

/* Walks the cells of one word in the reference's order, yielding each
 * cell's mask. */
static uint64_t gor_first_mask(int layout, int word_bits) {
    return layout == 1 ? 1u : (uint64_t)1 << (word_bits - 1);
}

static uint64_t gor_next_mask(int layout, uint64_t m) { return layout == 1 ? m << 1 : m >> 1; }

int gor_pack_layout(int layout, int word_bits, const uint8_t* cells, uint64_t x, uint64_t y,
                    void* words) {
    uint64_t xb, yb;
    if (gor_layout_geom(layout, word_bits, &xb, &yb)) return -2;
    if (x % xb || y % yb) return -3;
    const uint64_t wx = x / xb;
    for (uint64_t cy = 0; cy < y; cy += yb) {
        for (uint64_t cx = 0; cx < x; cx += xb) {
            uint64_t w = 0, m = gor_first_mask(layout, word_bits);
            for (uint64_t by = 0; by < yb; ++by)
                for (uint64_t bx = 0; bx < xb; ++bx) {
                    if (cells[(cy + by) * x + cx + bx]) w |= m;
                    m = gor_next_mask(layout, m);
                }
            gor_set_word(words, word_bits, (cy / yb) * wx + cx / xb, w);
        }
    }
    return 0;
}

int gor_unpack_layout(int layout, int word_bits, const void* words, uint64_t x, uint64_t y,
                      uint8_t* cells) {
    uint64_t xb, yb;
    if (gor_layout_geom(layout, word_bits, &xb, &yb)) return -2;
    if (x % xb || y % yb) return -3;
    const uint64_t wx = x / xb;
    for (uint64_t cy = 0; cy < y; cy += yb) {
        for (uint64_t cx = 0; cx < x; cx += xb) {
            const uint64_t w = gor_get_word(words, word_bits, (cy / yb) * wx + cx / xb);
            uint64_t m = gor_first_mask(layout, word_bits);
            for (uint64_t by = 0; by < yb; ++by)
                for (uint64_t bx = 0; bx < xb; ++bx) {
                    cells[(cy + by) * x + cx + bx] = (w & m) ? 1 : 0;
                    m = gor_next_mask(layout, m);
                }
        }
    }
    return 0;
}

/* ---------------------------------------------------------------------- */
/* Bit-sliced rows  (adder.cuh:17-104, gol_cpu_bitwise_general.hpp:32-120) */
/* ---------------------------------------------------------------------- */

/* One generated word from its 3x3 word neighbourhood, following the
 * reference adder step by step:
 *   1. vertical: the centre column count (ct + cc + cb, 0..3) as two bit
 *      planes (adder.cuh:23-27, add :67-77);
 *   2. the columns just left and right of the word come from the MSBs of
 *      lt/lc/lb and the LSBs of rt/rc/rb (:29-33, :106-160);
 *   3. the centre planes, shifted by one cell each way with those edge
 *      columns shifted in, are added with a 2-bit + 3-bit adder (:35-47,
 *      add_two :80-104), giving the 3x3 count including the centre (0..9)
 *      in three planes r0, r1, r2 (r2 = weight 4 mod 8; a count of 8 or 9
 *      wraps to 0/1 there, which neither rule below accepts);
 *   4. alive iff count == 3, or count == 4 and the centre is alive
 *      (GOL :56-65).                                                     */
#define GOR_DEFINE_ROWS(WT, BITS)                                                            \
    static inline void gor_add_##BITS(WT a, WT* p0, WT* p1) {                                \
        WT r0 = a ^ *p0;                                                                     \
        WT c0 = a & *p0;                                                                     \
        *p1 = c0 ^ *p1;                                                                      \
        *p0 = r0;                                                                            \
    }                                                                                        \
    static inline void gor_add_two_##BITS(WT a0, WT a1, WT* p0, WT* p1, WT* p2) {            \
        WT x1 = *p1 ^ a1;                                                                    \
        WT r0 = a0 ^ *p0;                                                                    \
        WT c0 = a0 & *p0;                                                                    \
        WT r1 = x1 ^ c0;                                                                     \
        WT c1 = (*p1 & a1) | (c0 & x1);                                                      \
        *p2 = *p2 ^ c1;                                                                      \
        *p0 = r0;                                                                            \
        *p1 = r1;                                                                            \
    }                                                                                        \
    static inline WT gor_word_##BITS(WT lt, WT ct, WT rt, WT lc, WT cc, WT rc, WT lb, WT cb, \
                                     WT rb) {                                                \
        const int S = BITS - 1;                                                              \
        WT v0 = cc, v1 = 0;                                                                  \
        gor_add_##BITS(ct, &v0, &v1);                                                        \
        gor_add_##BITS(cb, &v0, &v1);                                                        \
        unsigned lcount = (unsigned)(lt >> S) + (unsigned)(lc >> S) + (unsigned)(lb >> S);   \
        unsigned rcount = (unsigned)(rt & 1u) + (unsigned)(rc & 1u) + (unsigned)(rb & 1u);   \
        WT l0 = (WT)(lcount & 1u), l1 = (WT)(lcount >> 1);                                   \
        WT r0e = (WT)(rcount & 1u) << S, r1e = (WT)(rcount >> 1) << S;                       \
        WT s0 = v0, s1 = v1, s2 = 0;                                                         \
        gor_add_two_##BITS((WT)(v0 << 1) | l0, (WT)(v1 << 1) | l1, &s0, &s1, &s2);           \
        gor_add_two_##BITS((WT)(v0 >> 1) | r0e, (WT)(v1 >> 1) | r1e, &s0, &s1, &s2);         \
        WT is3 = s0 & s1 & (WT)~s2;                                                          \
        WT is4 = (WT)~s0 & (WT)~s1 & s2;                                                     \
        return is3 | (is4 & cc);                                                             \
    }                                                                                        \
    /* Rows [y0, y1): words outside the grid read as 0. `zero` is a row of  \
     * wx zero words standing in for the rows above and below the grid, so   \
     * the inner words need no bounds tests (only the first and last word of  \
     * a row look past its ends).                                            */ \
    __attribute__((target_clones("avx2", "default")))                                      \
    static void gor_rows_##BITS(const WT* src, WT* dst, const WT* zero, int64_t wx, int64_t y, \
                                int64_t y0, int64_t y1) {                                    \
        for (int64_t yy = y0; yy < y1; ++yy) {                                               \
            const WT* up = (yy > 0) ? src + (yy - 1) * wx : zero;                            \
            const WT* mid = src + yy * wx;                                                   \
            const WT* dn = (yy + 1 < y) ? src + (yy + 1) * wx : zero;                        \
            WT* out = dst + yy * wx;                                                         \
            if (wx == 1) {                                                                   \
                out[0] = gor_word_##BITS(0, up[0], 0, 0, mid[0], 0, 0, dn[0], 0);            \
                continue;                                                                    \
            }                                                                                \
            out[0] = gor_word_##BITS(0, up[0], up[1], 0, mid[0], mid[1], 0, dn[0], dn[1]);   \
            for (int64_t xw = 1; xw + 1 < wx; ++xw)                                          \
                out[xw] = gor_word_##BITS(up[xw - 1], up[xw], up[xw + 1], mid[xw - 1],       \
                                          mid[xw], mid[xw + 1], dn[xw - 1], dn[xw],          \
                                          dn[xw + 1]);                                       \
            const int64_t e = wx - 1;                                                        \
            out[e] = gor_word_##BITS(up[e - 1], up[e], 0, mid[e - 1], mid[e], 0, dn[e - 1],  \
                                     dn[e], 0);                                              \
        }                                                                                    \
    }

GOR_DEFINE_ROWS(uint64_t, 64)
GOR_DEFINE_ROWS(uint32_t, 32)

/* Worker team: the rows are split into `threads` contiguous ranges, one per
 * thread, for the whole run; a barrier separates the generations (every
 * thread reads the previous generation's buffer, then writes its own rows of
 * the next one). Started threads wait at a gate until the whole team exists
 * (or give up with it, if a thread could not be created). */
typedef struct {
    pthread_mutex_t mu;
    pthread_cond_t cv;
    int state; /* 0 wait, 1 go, -1 abandon */
} gor_gate;

typedef struct {
    int word_bits;
    void* buf[2];
    const void* zero; /* a row of wx zero words */
    int64_t wx, y, y0, y1;
    uint64_t iters;
    pthread_barrier_t* bar;
    gor_gate* gate;
} gor_job;

static void* gor_job_run(void* arg) {
    gor_job* j = (gor_job*)arg;
    if (j->gate) {
        pthread_mutex_lock(&j->gate->mu);
        while (j->gate->state == 0) pthread_cond_wait(&j->gate->cv, &j->gate->mu);
        const int go = j->gate->state == 1;
        pthread_mutex_unlock(&j->gate->mu);
        if (!go) return NULL;
    }
    for (uint64_t it = 0; it < j->iters; ++it) {
        const void* src = j->buf[it & 1];
        void* dst = j->buf[(it & 1) ^ 1];
        if (j->word_bits == 64)
            gor_rows_64((const uint64_t*)src, (uint64_t*)dst, (const uint64_t*)j->zero, j->wx,
                        j->y, j->y0, j->y1);
        else
            gor_rows_32((const uint32_t*)src, (uint32_t*)dst, (const uint32_t*)j->zero, j->wx,
                        j->y, j->y0, j->y1);
        if (j->bar) pthread_barrier_wait(j->bar);
    }
    return NULL;
}

/* Threads this process may run on: its CPU affinity (a container may allow
 * fewer CPUs than the machine has online). */
int gor_max_threads(void) {
    cpu_set_t set;
    if (sched_getaffinity(0, sizeof(set), &set) == 0) {
        const int n = CPU_COUNT(&set);
        if (n > 0) return n;
    }
    long n = sysconf(_SC_NPROCESSORS_ONLN);
    return n > 0 ? (int)n : 1;
}

/* Advances `iters` generations of a row-packed grid (x cells wide, x a
 * multiple of word_bits). `threads` <= 0 uses every online core. */
int gor_life_rows(int word_bits, const void* in, uint64_t x, uint64_t y, uint64_t iters,
                  void* out, int threads) {
    if (word_bits != 32 && word_bits != 64) return -2;
    if (x % (uint64_t)word_bits) return -3;
    uint64_t wx = x / (uint64_t)word_bits;
    size_t bytes = (size_t)(wx * y * (uint64_t)(word_bits / 8));
    if (threads <= 0) threads = gor_max_threads();
    if ((uint64_t)threads > y) threads = y ? (int)y : 1;
    if (threads > 512) threads = 512;
    void* tmp = malloc(bytes ? bytes : 8);
    void* zero = calloc(wx ? wx : 1, 8);
    if (!tmp || !zero) {
        free(tmp);
        free(zero);
        return -1;
    }
    memcpy(out, in, bytes);
    if (y == 0 || iters == 0 || wx == 0) {
        free(tmp);
        free(zero);
        return 0;
    }
    int64_t per = ((int64_t)y + threads - 1) / threads;
    int n = (int)(((int64_t)y + per - 1) / per); /* ranges that hold rows */
    pthread_barrier_t bar;
    if (n > 1 && pthread_barrier_init(&bar, NULL, (unsigned)n) != 0) n = 1;
    if (n == 1) per = (int64_t)y;
    gor_gate gate = {PTHREAD_MUTEX_INITIALIZER, PTHREAD_COND_INITIALIZER, 0};
    gor_job jobs[512];
    pthread_t tids[512];
    for (int t = 0; t < n; ++t) {
        int64_t y0 = t * per, y1 = y0 + per;
        if (y1 > (int64_t)y) y1 = (int64_t)y;
        jobs[t] = (gor_job){word_bits, {out, tmp}, zero, (int64_t)wx, (int64_t)y, y0, y1, iters,
                            n > 1 ? &bar : NULL, n > 1 ? &gate : NULL};
    }
    int started = 0;
    for (int t = 1; t < n; ++t) {
        if (pthread_create(&tids[t], NULL, gor_job_run, &jobs[t]) != 0) break;
        started = t;
    }
    const int whole = started == n - 1;
    if (n > 1) {
        pthread_mutex_lock(&gate.mu);
        gate.state = whole ? 1 : -1;
        pthread_cond_broadcast(&gate.cv);
        pthread_mutex_unlock(&gate.mu);
    }
    if (whole) {
        jobs[0].gate = NULL;
        gor_job_run(&jobs[0]);
    }
    for (int t = 1; t <= started; ++t) pthread_join(tids[t], NULL);
    if (n > 1) pthread_barrier_destroy(&bar);
    if (!whole) { /* no team: one thread, all rows */
        jobs[0] = (gor_job){word_bits, {out, tmp}, zero, (int64_t)wx, (int64_t)y, 0, (int64_t)y,
                            iters, NULL, NULL};
        gor_job_run(&jobs[0]);
    }
    if (iters & 1) memcpy(out, tmp, bytes);
    free(tmp);
    free(zero);
    return 0;
}

/* FNV-1a 64 over a byte buffer: compact fingerprints for golden fixtures. */
uint64_t gor_fnv1a64(const void* data, uint64_t n) {
    const uint8_t* p = (const uint8_t*)data;
    uint64_t h = 0xcbf29ce484222325ull;
    for (uint64_t i = 0; i < n; ++i) {
        h ^= p[i];
        h *= 0x100000001b3ull;
    }
    return h;
}
