// Bit-sliced Game of Life arithmetic on 32-bit row words (sm_100a).
//
// Layout: a row of X cells is X/32 consecutive uint32 words, bit i of word
// xw holding cell xw*32 + i (LSB = smallest x). On a little-endian device
// this is byte-for-byte the reference's FullyPackedRows layout for both 32-
// and 64-bit words (src/algorithms/_shared/bitwise/bit_modes.hpp:127-148,
// general_bit_grid.hpp:224-243,257-259), so one kernel serves both widths.
//
// The neighbour count is formed the way the reference's adder does it
// (src/algorithms/_shared/bitwise/bitwise-ops/adder.cuh:17-65): bit planes
// of partial counts added with full adders, then "alive iff the 3x3 count
// including the centre is 3, or 4 with the centre alive". The order is
// changed for a streaming kernel: each row is first summed horizontally
// (left + centre + right, a 2-bit count per cell), once, and the three row
// sums of a 3-row window are then added vertically. Every step is a single
// LOP3 (three-input boolean, immediate truth table) or a funnel shift.
#pragma once

#include <cstdint>

namespace golb200 {

// lop3.b32 with an immediate truth table: LUT bit (a<<2 | b<<1 | c) gives
// the output for inputs (a, b, c); a = 0xF0, b = 0xCC, c = 0xAA.
template <unsigned LUT>
__device__ __forceinline__ uint32_t lop3(uint32_t a, uint32_t b, uint32_t c) {
    uint32_t r;
    asm("lop3.b32 %0, %1, %2, %3, %4;" : "=r"(r) : "r"(a), "r"(b), "r"(c), "n"(LUT));
    return r;
}

constexpr unsigned LUT_XOR3 = 0x96;        // a ^ b ^ c
constexpr unsigned LUT_MAJ = 0xE8;         // majority(a, b, c): carry of a full adder
constexpr unsigned LUT_EQ1 = 0x14;         // (a ^ b) & ~c
constexpr unsigned LUT_EQ2 = 0x42;         // (~a & ~b & c) | (a & b & ~c)
constexpr unsigned LUT_ANDN_AND = 0x08;    // ~a & b & c
constexpr unsigned LUT_AND_OR = 0xEA;      // (a & b) | c

// Horizontal 3-cell sum of one row word: (left + centre + right) per cell as
// two bit planes. `lw` is the word to the left (its bit 31 is the cell just
// left of bit 0), `rw` the word to the right (its bit 0 follows bit 31).

__device__ __forceinline__ void hsum(uint32_t lw, uint32_t c, uint32_t rw, uint32_t& h0,
                                     uint32_t& h1) {
    const uint32_t l = __funnelshift_l(lw, c, 1);   // cell x-1 aligned to x
    const uint32_t r = __funnelshift_r(c, rw, 1);   // cell x+1 aligned to x
    h0 = lop3<LUT_XOR3>(l, c, r);
    h1 = lop3<LUT_MAJ>(l, c, r);
}

// Next state of one word from the horizontal sums of rows y-1 (a), y (b) and
// y+1 (p) and the current centre word. T = a + b + p is the 3x3 count with
// the centre: T = t0 + 2*(c0 + u0) + 4*u1. Alive next iff T == 3, or T == 4
// with the centre alive (adder.cuh:56-65).
__device__ __forceinline__ uint32_t next_word(uint32_t a0, uint32_t a1, uint32_t b0, uint32_t b1,
                                              uint32_t p0, uint32_t p1, uint32_t alive) {
    const uint32_t t0 = lop3<LUT_XOR3>(a0, b0, p0);
    const uint32_t c0 = lop3<LUT_MAJ>(a0, b0, p0);
    const uint32_t u0 = lop3<LUT_XOR3>(a1, b1, p1);
    const uint32_t u1 = lop3<LUT_MAJ>(a1, b1, p1);
    const uint32_t eq1 = lop3<LUT_EQ1>(c0, u0, u1);          // c0 + u0 + 2*u1 == 1
    const uint32_t eq2 = lop3<LUT_EQ2>(c0, u0, u1);          // c0 + u0 + 2*u1 == 2
    const uint32_t born4 = lop3<LUT_ANDN_AND>(t0, eq2, alive);  // T == 4 and alive
    return lop3<LUT_AND_OR>(t0, eq1, born4);                 // T == 3, or the above
}

} // namespace golb200
