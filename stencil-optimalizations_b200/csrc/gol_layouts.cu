// Column and tile word layouts as input / output formats beside the rows
// layout the engine computes in: GeneralBitGrid<uintW_t, BitColumnsMode |
// BitTileMode> (src/algorithms/_shared/bitwise/general_bit_grid.hpp:171-246,
// bit_modes.hpp:10-125, 165-177), the layouts of the reference's
// columns-based (Fujita) and tiled ("Core Tiled 64") kernels.
//
//   columns (W = 16/32/64): a word holds W cells of one column; cell (x, y)
//     is bit y % W (lowest bit = top cell) of word (y / W) * X + x.
//   tiles: 4x4 cells in 16-bit words, 8x4 in 32-bit, 8x8 in 64-bit; cell
//     (x, y) is bit W-1 - ((y % YB) * XB + x % XB) (top-left cell in the
//     highest bit, x fastest) of word (y / YB) * (X / XB) + x / XB.
//   rows (W = 16/32/64): cell (x, y) is bit x % W of word y * (X / W) + x / W;
//     the same bytes for every W on a little-endian host.
//
// Host conversions (cells <-> any layout; layout words <-> the engine's
// rows) run over row bands on all host threads. Device conversions between
// rows and the other layouts, for grids kept on the device:
//   columns: one warp per 32-column x 32- (or 64-) row block, a bit
//            transpose by ballot: lane i holds row y0+i's word, and the
//            ballot of bit j across lanes is column x0+j's word (and back).
//   tiles:   one thread per 8-cell byte column of a tile row: it reads the
//            rows' bytes (or nibbles), reverses their bit order and
//            assembles the tile word(s) (and back).
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "gol_b200.h"
#include "gol_internal.h"

namespace golb200 {

bool layout_geom(int layout, uint32_t wb, uint32_t* xb, uint32_t* yb) {
    if (wb != 16 && wb != 32 && wb != 64) return false;
    switch (layout) {
        case GOL_LAYOUT_ROWS: *xb = wb; *yb = 1; return true;
        case GOL_LAYOUT_COLUMNS: *xb = 1; *yb = wb; return true;
        case GOL_LAYOUT_TILES:
            *xb = wb == 16 ? 4 : 8;
            *yb = wb == 64 ? 8 : 4;
            return true;
        default: return false;
    }
}

namespace {

// Bit position of cell (bx, by) inside its word.
inline uint32_t bit_of(int layout, uint32_t wb, uint32_t xb, uint32_t bx, uint32_t by) {
    switch (layout) {
        case GOL_LAYOUT_ROWS: return bx;
        case GOL_LAYOUT_COLUMNS: return by;
        default: return wb - 1 - (by * xb + bx);
    }
}

inline uint64_t get_word(const void* w, uint32_t wb, size_t i) {
    if (wb == 64) return static_cast<const uint64_t*>(w)[i];
    if (wb == 32) return static_cast<const uint32_t*>(w)[i];
    return static_cast<const uint16_t*>(w)[i];
}

inline void set_word(void* w, uint32_t wb, size_t i, uint64_t v) {
    if (wb == 64) static_cast<uint64_t*>(w)[i] = v;
    else if (wb == 32) static_cast<uint32_t*>(w)[i] = static_cast<uint32_t>(v);
    else static_cast<uint16_t*>(w)[i] = static_cast<uint16_t>(v);
}

// Runs body(r0, r1) over word rows [0, n) split across host threads.
template <typename F>
void parallel_word_rows(size_t n, size_t cells_per_row, F&& body) {
    unsigned hw = std::max(1u, usable_cpus());
    size_t nt = std::min<size_t>(hw, std::max<size_t>(1, n * cells_per_row / (1u << 20)));
    nt = std::min(nt, n ? n : 1);
    if (nt <= 1) {
        body(size_t(0), n);
        return;
    }
    std::vector<std::thread> ts;
    const size_t per = (n + nt - 1) / nt;
    for (size_t t = 0; t < nt; ++t) {
        const size_t r0 = t * per, r1 = std::min(n, r0 + per);
        if (r0 >= r1) break;
        ts.emplace_back([=, &body] { body(r0, r1); });
    }
    for (auto& th : ts) th.join();
}

} // namespace

void host_cells_to_layout(const uint8_t* cells, size_t x, size_t y, int layout, uint32_t wb,
                          uint32_t xb, uint32_t yb, void* words) {
    const size_t wx = x / xb;
    parallel_word_rows(y / yb, x * yb, [=](size_t r0, size_t r1) {
        for (size_t wy = r0; wy < r1; ++wy)
            for (size_t i = 0; i < wx; ++i) {
                uint64_t w = 0;
                for (uint32_t by = 0; by < yb; ++by) {
                    const uint8_t* row = cells + (wy * yb + by) * x + i * xb;
                    for (uint32_t bx = 0; bx < xb; ++bx)
                        if (row[bx]) w |= uint64_t(1) << bit_of(layout, wb, xb, bx, by);
                }
                set_word(words, wb, wy * wx + i, w);
            }
    });
}

void host_layout_to_cells(const void* words, size_t x, size_t y, int layout, uint32_t wb,
                          uint32_t xb, uint32_t yb, uint8_t* cells) {
    const size_t wx = x / xb;
    parallel_word_rows(y / yb, x * yb, [=](size_t r0, size_t r1) {
        for (size_t wy = r0; wy < r1; ++wy)
            for (size_t i = 0; i < wx; ++i) {
                const uint64_t w = get_word(words, wb, wy * wx + i);
                for (uint32_t by = 0; by < yb; ++by) {
                    uint8_t* row = cells + (wy * yb + by) * x + i * xb;
                    for (uint32_t bx = 0; bx < xb; ++bx)
                        row[bx] = (w >> bit_of(layout, wb, xb, bx, by)) & 1u;
                }
            }
    });
}

// Layout words -> rows words (32-bit, x % 32 == 0) and back, without a cell
// buffer: each rows word gathers its 32 cells from the layout words.
void host_layout_to_rows(const void* words, size_t x, size_t y, int layout, uint32_t wb,
                         uint32_t xb, uint32_t yb, uint32_t* rows) {
    const size_t wx = x / xb, rw = x / 32;
    parallel_word_rows(y, x, [=](size_t r0, size_t r1) {
        for (size_t cy = r0; cy < r1; ++cy) {
            const size_t wy = cy / yb;
            const uint32_t by = static_cast<uint32_t>(cy % yb);
            for (size_t j = 0; j < rw; ++j) {
                uint32_t out = 0;
                for (uint32_t b = 0; b < 32; ++b) {
                    const size_t cx = j * 32 + b;
                    const uint64_t w = get_word(words, wb, wy * wx + cx / xb);
                    out |= static_cast<uint32_t>((w >> bit_of(layout, wb, xb, cx % xb, by)) & 1u) << b;
                }
                rows[cy * rw + j] = out;
            }
        }
    });
}

void host_rows_to_layout(const uint32_t* rows, size_t x, size_t y, int layout, uint32_t wb,
                         uint32_t xb, uint32_t yb, void* words) {
    const size_t wx = x / xb, rw = x / 32;
    parallel_word_rows(y / yb, x * yb, [=](size_t r0, size_t r1) {
        for (size_t wy = r0; wy < r1; ++wy)
            for (size_t i = 0; i < wx; ++i) {
                uint64_t w = 0;
                for (uint32_t by = 0; by < yb; ++by) {
                    const uint32_t* row = rows + (wy * yb + by) * rw;
                    for (uint32_t bx = 0; bx < xb; ++bx) {
                        const size_t cx = i * xb + bx;
                        if ((row[cx / 32] >> (cx % 32)) & 1u)
                            w |= uint64_t(1) << bit_of(layout, wb, xb, bx, by);
                    }
                }
                set_word(words, wb, wy * wx + i, w);
            }
    });
}

namespace {

constexpr int kLayoutThreads = 256;

// Rows -> columns. Warp w takes word column wx = w % Wx and the row group
// g = w / Wx of R = max(W, 32) rows; lane j ends with column 32*wx + j.
template <int WB>
__global__ void __launch_bounds__(kLayoutThreads)
rows_to_columns_kernel(const uint32_t* __restrict__ rows, void* __restrict__ cols, int X, int Y) {
    constexpr int R = WB > 32 ? WB : 32;
    const int Wx = X / 32;
    const long long w = (long long)blockIdx.x * (kLayoutThreads / 32) + (threadIdx.x >> 5);
    const int groups = (Y + R - 1) / R;
    if (w >= (long long)Wx * groups) return;   // whole warp
    const int lane = threadIdx.x & 31;
    const int wx = (int)(w % Wx), y0 = (int)(w / Wx) * R;
    uint32_t mine[R / 32];
#pragma unroll
    for (int h = 0; h < R / 32; ++h) {
        const int r = y0 + 32 * h + lane;
        const uint32_t v = r < Y ? rows[(size_t)r * Wx + wx] : 0u;
        uint32_t m = 0;
#pragma unroll
        for (int j = 0; j < 32; ++j) {
            const uint32_t b = __ballot_sync(0xffffffffu, (v >> j) & 1u);
            m = lane == j ? b : m;
        }
        mine[h] = m;
    }
    const size_t x = (size_t)wx * 32 + lane;
    if (WB == 64) {
        static_cast<uint64_t*>(cols)[(size_t)(y0 / 64) * X + x] =
            (uint64_t)mine[0] | ((uint64_t)mine[R / 32 - 1] << 32);
    } else if (WB == 32) {
        static_cast<uint32_t*>(cols)[(size_t)(y0 / 32) * X + x] = mine[0];
    } else {
        uint16_t* c = static_cast<uint16_t*>(cols);
        c[(size_t)(y0 / 16) * X + x] = (uint16_t)mine[0];
        if (y0 + 16 < Y) c[(size_t)(y0 / 16 + 1) * X + x] = (uint16_t)(mine[0] >> 16);
    }
}

template <int WB>
__global__ void __launch_bounds__(kLayoutThreads)
columns_to_rows_kernel(const void* __restrict__ cols, uint32_t* __restrict__ rows, int X, int Y) {
    constexpr int R = WB > 32 ? WB : 32;
    const int Wx = X / 32;
    const long long w = (long long)blockIdx.x * (kLayoutThreads / 32) + (threadIdx.x >> 5);
    const int groups = (Y + R - 1) / R;
    if (w >= (long long)Wx * groups) return;
    const int lane = threadIdx.x & 31;
    const int wx = (int)(w % Wx), y0 = (int)(w / Wx) * R;
    const size_t x = (size_t)wx * 32 + lane;
    uint32_t src[R / 32];
    if (WB == 64) {
        const uint64_t c = static_cast<const uint64_t*>(cols)[(size_t)(y0 / 64) * X + x];
        src[0] = (uint32_t)c;
        src[R / 32 - 1] = (uint32_t)(c >> 32);
    } else if (WB == 32) {
        src[0] = static_cast<const uint32_t*>(cols)[(size_t)(y0 / 32) * X + x];
    } else {
        const uint16_t* c = static_cast<const uint16_t*>(cols);
        uint32_t v = c[(size_t)(y0 / 16) * X + x];
        if (y0 + 16 < Y) v |= (uint32_t)c[(size_t)(y0 / 16 + 1) * X + x] << 16;
        src[0] = v;
    }
#pragma unroll
    for (int h = 0; h < R / 32; ++h) {
        uint32_t m = 0;
#pragma unroll
        for (int i = 0; i < 32; ++i) {
            const uint32_t b = __ballot_sync(0xffffffffu, (src[h] >> i) & 1u);
            m = lane == i ? b : m;
        }
        const int r = y0 + 32 * h + lane;
        if (r < Y) rows[(size_t)r * Wx + wx] = m;
    }
}

__device__ __forceinline__ uint32_t brev8(uint32_t v) { return __brev(v) >> 24; }
__device__ __forceinline__ uint32_t brev4(uint32_t v) { return __brev(v) >> 28; }

// Rows <-> tiles, one thread per (8-cell byte column, tile row): the 8
// cells of a row byte are one tile row (8-wide tiles) or two (4-wide).
template <int WB>
__global__ void __launch_bounds__(kLayoutThreads)
rows_to_tiles_kernel(const uint8_t* __restrict__ rows, void* __restrict__ tiles, int X, int Y) {
    constexpr int XB = WB == 16 ? 4 : 8, YB = WB == 64 ? 8 : 4;
    const int bx = X / 8;                                   // bytes per row
    const long long t = (long long)blockIdx.x * kLayoutThreads + threadIdx.x;
    if (t >= (long long)bx * (Y / YB)) return;
    const int c = (int)(t % bx), ty = (int)(t / bx);
    uint64_t w0 = 0, w1 = 0;
#pragma unroll
    for (int yb = 0; yb < YB; ++yb) {
        const uint32_t v = rows[(size_t)(ty * YB + yb) * bx + c];
        const int shift = WB - XB * (yb + 1);
        if (XB == 8) {
            w0 |= (uint64_t)brev8(v) << shift;
        } else {
            w0 |= (uint64_t)brev4(v & 15u) << shift;
            w1 |= (uint64_t)brev4(v >> 4) << shift;
        }
    }
    const size_t wx = (size_t)(X / XB);
    if (WB == 64) {
        static_cast<uint64_t*>(tiles)[(size_t)ty * wx + c] = w0;
    } else if (WB == 32) {
        static_cast<uint32_t*>(tiles)[(size_t)ty * wx + c] = (uint32_t)w0;
    } else {
        uint16_t* p = static_cast<uint16_t*>(tiles) + (size_t)ty * wx + 2 * (size_t)c;
        p[0] = (uint16_t)w0;
        p[1] = (uint16_t)w1;
    }
}

template <int WB>
__global__ void __launch_bounds__(kLayoutThreads)
tiles_to_rows_kernel(const void* __restrict__ tiles, uint8_t* __restrict__ rows, int X, int Y) {
    constexpr int XB = WB == 16 ? 4 : 8, YB = WB == 64 ? 8 : 4;
    const int bx = X / 8;
    const long long t = (long long)blockIdx.x * kLayoutThreads + threadIdx.x;
    if (t >= (long long)bx * (Y / YB)) return;
    const int c = (int)(t % bx), ty = (int)(t / bx);
    const size_t wx = (size_t)(X / XB);
    uint64_t w0, w1 = 0;
    if (WB == 64) {
        w0 = static_cast<const uint64_t*>(tiles)[(size_t)ty * wx + c];
    } else if (WB == 32) {
        w0 = static_cast<const uint32_t*>(tiles)[(size_t)ty * wx + c];
    } else {
        const uint16_t* p = static_cast<const uint16_t*>(tiles) + (size_t)ty * wx + 2 * (size_t)c;
        w0 = p[0];
        w1 = p[1];
    }
#pragma unroll
    for (int yb = 0; yb < YB; ++yb) {
        const int shift = WB - XB * (yb + 1);
        uint32_t v;
        if (XB == 8) {
            v = brev8((uint32_t)(w0 >> shift) & 255u);
        } else {
            v = brev4((uint32_t)(w0 >> shift) & 15u) | (brev4((uint32_t)(w1 >> shift) & 15u) << 4);
        }
        rows[(size_t)(ty * YB + yb) * bx + c] = (uint8_t)v;
    }
}

template <int WB>
cudaError_t launch_convert(bool to_rows, int layout, const void* src, void* dst, int X, int Y,
                           cudaStream_t s) {
    if (layout == GOL_LAYOUT_COLUMNS) {
        constexpr int R = WB > 32 ? WB : 32;
        const long long warps = (long long)(X / 32) * ((Y + R - 1) / R);
        const long long blocks = (warps + kLayoutThreads / 32 - 1) / (kLayoutThreads / 32);
        if (to_rows)
            columns_to_rows_kernel<WB><<<(unsigned)blocks, kLayoutThreads, 0, s>>>(
                src, static_cast<uint32_t*>(dst), X, Y);
        else
            rows_to_columns_kernel<WB><<<(unsigned)blocks, kLayoutThreads, 0, s>>>(
                static_cast<const uint32_t*>(src), dst, X, Y);
    } else {
        constexpr int YB = WB == 64 ? 8 : 4;
        const long long threads = (long long)(X / 8) * (Y / YB);
        const long long blocks = (threads + kLayoutThreads - 1) / kLayoutThreads;
        if (to_rows)
            tiles_to_rows_kernel<WB><<<(unsigned)blocks, kLayoutThreads, 0, s>>>(
                src, static_cast<uint8_t*>(dst), X, Y);
        else
            rows_to_tiles_kernel<WB><<<(unsigned)blocks, kLayoutThreads, 0, s>>>(
                static_cast<const uint8_t*>(src), dst, X, Y);
    }
    return cudaPeekAtLastError();
}

int device_convert(bool to_rows, const void* src, void* dst, uint64_t x, uint64_t y, int layout,
                   uint32_t wb, void* stream) {
    uint32_t xb, yb;
    if (!layout_geom(layout, wb, &xb, &yb) || layout == GOL_LAYOUT_ROWS) return GOL_E_INVALID;
    if ((!src || !dst) && x * y) return GOL_E_INVALID;
    if (x % 32 || y % yb || x > (1u << 30) || y > (1u << 30)) return GOL_E_INVALID;
    if (((uintptr_t)src | (uintptr_t)dst) & (wb / 8 - 1) || ((uintptr_t)src | (uintptr_t)dst) & 3u)
        return GOL_E_INVALID;
    if (x * y == 0) return GOL_OK;
    auto s = static_cast<cudaStream_t>(stream);
    cudaError_t ce;
    switch (wb) {
        case 64: ce = launch_convert<64>(to_rows, layout, src, dst, (int)x, (int)y, s); break;
        case 32: ce = launch_convert<32>(to_rows, layout, src, dst, (int)x, (int)y, s); break;
        default: ce = launch_convert<16>(to_rows, layout, src, dst, (int)x, (int)y, s); break;
    }
    return ce == cudaSuccess ? GOL_OK : GOL_E_CUDA;
}

} // namespace
} // namespace golb200

extern "C" {

int gol_pack_layout(const uint8_t* cells, uint64_t x, uint64_t y, int layout, uint32_t word_bits,
                    void* words) {
    uint32_t xb, yb;
    if (!golb200::layout_geom(layout, word_bits, &xb, &yb)) return GOL_E_INVALID;
    if (x % xb || y % yb || ((!cells || !words) && x * y)) return GOL_E_INVALID;
    golb200::host_cells_to_layout(cells, x, y, layout, word_bits, xb, yb, words);
    return GOL_OK;
}

int gol_unpack_layout(const void* words, uint64_t x, uint64_t y, int layout, uint32_t word_bits,
                      uint8_t* cells) {
    uint32_t xb, yb;
    if (!golb200::layout_geom(layout, word_bits, &xb, &yb)) return GOL_E_INVALID;
    if (x % xb || y % yb || ((!cells || !words) && x * y)) return GOL_E_INVALID;
    golb200::host_layout_to_cells(words, x, y, layout, word_bits, xb, yb, cells);
    return GOL_OK;
}

int gol_layout_to_rows_device(const void* d_src, void* d_rows, uint64_t x, uint64_t y, int layout,
                              uint32_t word_bits, void* stream) {
    return golb200::device_convert(true, d_src, d_rows, x, y, layout, word_bits, stream);
}

int gol_rows_to_layout_device(const void* d_rows, void* d_dst, uint64_t x, uint64_t y, int layout,
                              uint32_t word_bits, void* stream) {
    return golb200::device_convert(false, d_rows, d_dst, x, y, layout, word_bits, stream);
}

} // extern "C"
