// Host packing between a cell grid and 32-bit row words, the host side of
// the reference's set_and_format_input_data / fetch_result phases
// (GeneralBitGrid::fill_grid / to_grid, general_bit_grid.hpp:171-246):
// cell (cx, cy) at cells[cy*x + cx] maps to bit cx % 32 of word
// cy*(x/32) + cx/32; a nonzero cell is alive; unpacked cells are 0/1.
//
// Eight cells are handled per 64-bit operation (a byte-to-bit multiply
// gather), and rows are split across hardware threads.
#include <algorithm>
#include <cstring>
#include <random>
#include <thread>
#include <vector>

#include "gol_internal.h"

namespace golb200 {

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

template <typename F>
void parallel_rows(size_t y, size_t bytes_per_row, F&& body) {
    const size_t total = y * bytes_per_row;
    unsigned hw = std::thread::hardware_concurrency();
    size_t nt = std::max<size_t>(1, std::min<size_t>(hw ? hw : 1, 32));
    // Below ~4 MiB threads cost more than they save.
    nt = std::min(nt, std::max<size_t>(1, total >> 22));
    nt = std::min(nt, std::max<size_t>(y, 1));
    if (nt <= 1) {
        body(0, y);
        return;
    }
    std::vector<std::thread> ts;
    const size_t per = (y + nt - 1) / nt;
    for (size_t t = 1; t < nt; ++t) {
        const size_t y0 = t * per, y1 = std::min(y, y0 + per);
        if (y0 >= y1) break;
        ts.emplace_back([&body, y0, y1] { body(y0, y1); });
    }
    body(0, std::min(y, per));
    for (auto& th : ts) th.join();
}

} // namespace

void host_pack_u8(const uint8_t* cells, size_t x, size_t y, uint32_t* words) {
    const size_t W = x / 32;
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

} // namespace golb200
