// Test infrastructure, not product code.
//
// Builds the reference's own CPU path for bit-packed Game of Life into
// oracle/_ref/libgolref.so, straight from the reference sources (compiled
// where they lie, never copied), so tests can check the C restatement in
// gol_oracle.c and the CUDA engine against the reference itself.
//
// Exposed (extern "C", plain pointers):
//   ref_load_random_ones_zeros : RandomOnesZerosDataLoader<2,char>::load_data
//                                (src/infrastructure/data_loader.hpp:57-75)
//   ref_run_cpu_naive          : algorithms::GoLCpuNaive<char>, the
//                                reference's default validator
//                                (src/algorithms/cpu-naive/gol_cpu_naive.hpp:26-117,
//                                src/infrastructure/experiment_params.hpp:43)
//   ref_run_cpu_bitwise_adder  : algorithms::GoLCpuBitwise<char, 32|64, AdderOps>
//                                (src/algorithms/cpu-bitwise-general/gol_cpu_bitwise_general.hpp:32-120)
//   ref_bitwise_create / _run / _finish : the same 64-bit algorithm with its
//                                phases apart, so run() can be timed alone
//   ref_pack_rows / ref_unpack_rows : GeneralBitGrid<uintW_t, AdderMode>
//                                fill_grid / to_grid
//                                (src/algorithms/_shared/bitwise/general_bit_grid.hpp:171-246)
//   ref_pack_layout / ref_unpack_layout : the same for BitColumnsMode and
//                                BitTileMode (bit_modes.hpp:10-125, 165-177)
//   ref_load_zeros             : ZerosLoader<2,char> (data_loader.hpp:128-146)
// (the pattern loaders, which need the reference's compiled pattern
// dictionary, are in ref_lexicon.cpp)
//
// The algorithm phases are called directly in the order the reference's
// ExperimentManager::perform_alg uses (experiment_manager.hpp:365-394);
// TimedAlgorithm is skipped because its Timer synchronises a CUDA device
// (timer.hpp:15-26) and this harness must run without one.
#include <cstdint>
#include <cstring>
#include <exception>
#include <limits>
#include <vector>

#include "algorithms/_shared/bitwise/bitwise-ops/cpu-ops-interface.hpp"
#include "algorithms/_shared/bitwise/general_bit_grid.hpp"
#include "algorithms/cpu-bitwise-general/gol_cpu_bitwise_general.hpp"
#include "algorithms/cpu-naive/gol_cpu_naive.hpp"
#include "infrastructure/data_loader.hpp"
#include "infrastructure/experiment_params.hpp"
#include "infrastructure/grid.hpp"

namespace {

using CharGrid = infrastructure::Grid<2, char>;

infrastructure::ExperimentParams make_params(std::size_t x, std::size_t y, std::size_t iters,
                                             std::size_t seed) {
    infrastructure::ExperimentParams p;
    p.grid_dimensions = {x, y};
    p.iterations = iters;
    p.random_seed = seed;
    p.animate_output = false;
    p.max_runtime_seconds = infrastructure::StopWatch::MAX_TIME;
    return p;
}

CharGrid grid_from(const uint8_t* cells, std::size_t x, std::size_t y) {
    CharGrid g(x, y);
    std::memcpy(g.data(), cells, x * y);
    return g;
}

void grid_to(const CharGrid& g, uint8_t* out) {
    std::memcpy(out, g.data(), g.size());
}

template <typename Alg>
void run_phases(Alg& alg, const uint8_t* in, std::size_t x, std::size_t y, std::size_t iters,
                uint8_t* out) {
    alg.set_params(make_params(x, y, iters, 0));
    alg.set_and_format_input_data(grid_from(in, x, y));
    alg.initialize_data_structures();
    alg.run(iters);
    alg.finalize_data_structures();
    grid_to(alg.fetch_result(), out);
}

template <typename word_t>
using RowBitGrid = algorithms::GeneralBitGrid<word_t, algorithms::AdderMode>;

// layout 1 = BitColumnsMode, 2 = BitTileMode.
template <typename word_t, typename mode>
int pack_as(const uint8_t* cells, uint64_t x, uint64_t y, void* words) {
    algorithms::GeneralBitGrid<word_t, mode> bg(grid_from(cells, x, y));
    std::memcpy(words, bg.data(), bg.size() * sizeof(word_t));
    return 0;
}

template <typename word_t, typename mode>
int unpack_as(const void* words, uint64_t x, uint64_t y, uint8_t* cells) {
    algorithms::GeneralBitGrid<word_t, mode> bg(x, y);
    std::memcpy(bg.data(), words, bg.size() * sizeof(word_t));
    grid_to(bg.template to_grid<char>(), cells);
    return 0;
}

template <typename mode>
int pack_bits(int word_bits, const uint8_t* cells, uint64_t x, uint64_t y, void* words) {
    switch (word_bits) {
        case 16: return pack_as<uint16_t, mode>(cells, x, y, words);
        case 32: return pack_as<uint32_t, mode>(cells, x, y, words);
        case 64: return pack_as<uint64_t, mode>(cells, x, y, words);
        default: return -2;
    }
}

template <typename mode>
int unpack_bits(int word_bits, const void* words, uint64_t x, uint64_t y, uint8_t* cells) {
    switch (word_bits) {
        case 16: return unpack_as<uint16_t, mode>(words, x, y, cells);
        case 32: return unpack_as<uint32_t, mode>(words, x, y, cells);
        case 64: return unpack_as<uint64_t, mode>(words, x, y, cells);
        default: return -2;
    }
}

} // namespace

extern "C" {

int ref_load_random_ones_zeros(uint64_t x, uint64_t y, uint64_t seed, uint8_t* out) {
    try {
        infrastructure::RandomOnesZerosDataLoader<2, char> loader;
        auto g = loader.load_data(make_params(x, y, 0, seed));
        grid_to(g, out);
        return 0;
    } catch (const std::exception&) {
        return -1;
    }
}

int ref_run_cpu_naive(const uint8_t* in, uint64_t x, uint64_t y, uint64_t iters, uint8_t* out) {
    try {
        algorithms::GoLCpuNaive<char> alg;
        run_phases(alg, in, x, y, iters, out);
        return 0;
    } catch (const std::exception&) {
        return -1;
    }
}

int ref_run_cpu_bitwise_adder(int word_bits, const uint8_t* in, uint64_t x, uint64_t y,
                              uint64_t iters, uint8_t* out) {
    try {
        if (word_bits == 64) {
            algorithms::GoLCpuBitwise<char, 64, algorithms::AdderOps> alg;
            run_phases(alg, in, x, y, iters, out);
        } else if (word_bits == 32) {
            algorithms::GoLCpuBitwise<char, 32, algorithms::AdderOps> alg;
            run_phases(alg, in, x, y, iters, out);
        } else {
            return -2;
        }
        return 0;
    } catch (const std::exception&) {
        return -1;
    }
}

// GoLCpuBitwise<char, 64, AdderOps> split into its phases so a caller can
// time run() alone: create = set_params + set_and_format_input_data +
// initialize_data_structures; run = run(iters), continuing from the
// instance's current state; finish = finalize_data_structures +
// fetch_result, then the instance is freed.
void* ref_bitwise_create(const uint8_t* in, uint64_t x, uint64_t y) {
    try {
        auto* alg = new algorithms::GoLCpuBitwise<char, 64, algorithms::AdderOps>();
        alg->set_params(make_params(x, y, 0, 0));
        alg->set_and_format_input_data(grid_from(in, x, y));
        alg->initialize_data_structures();
        return alg;
    } catch (const std::exception&) {
        return nullptr;
    }
}

int ref_bitwise_run(void* h, uint64_t iters) {
    try {
        static_cast<algorithms::GoLCpuBitwise<char, 64, algorithms::AdderOps>*>(h)->run(iters);
        return 0;
    } catch (const std::exception&) {
        return -1;
    }
}

int ref_bitwise_finish(void* h, uint8_t* out) {
    auto* alg = static_cast<algorithms::GoLCpuBitwise<char, 64, algorithms::AdderOps>*>(h);
    int rc = 0;
    try {
        alg->finalize_data_structures();
        if (out) grid_to(alg->fetch_result(), out);
    } catch (const std::exception&) {
        rc = -1;
    }
    delete alg;
    return rc;
}

int ref_pack_rows(int word_bits, const uint8_t* cells, uint64_t x, uint64_t y, void* words) {
    try {
        auto g = grid_from(cells, x, y);
        if (word_bits == 64) {
            RowBitGrid<uint64_t> bg(g);
            std::memcpy(words, bg.data(), bg.size() * sizeof(uint64_t));
        } else if (word_bits == 32) {
            RowBitGrid<uint32_t> bg(g);
            std::memcpy(words, bg.data(), bg.size() * sizeof(uint32_t));
        } else {
            return -2;
        }
        return 0;
    } catch (const std::exception&) {
        return -1;
    }
}

int ref_unpack_rows(int word_bits, const void* words, uint64_t x, uint64_t y, uint8_t* cells) {
    try {
        if (word_bits == 64) {
            RowBitGrid<uint64_t> bg(x, y);
            std::memcpy(bg.data(), words, bg.size() * sizeof(uint64_t));
            grid_to(bg.template to_grid<char>(), cells);
        } else if (word_bits == 32) {
            RowBitGrid<uint32_t> bg(x, y);
            std::memcpy(bg.data(), words, bg.size() * sizeof(uint32_t));
            grid_to(bg.template to_grid<char>(), cells);
        } else {
            return -2;
        }
        return 0;
    } catch (const std::exception&) {
        return -1;
    }
}

int ref_pack_layout(int layout, int word_bits, const uint8_t* cells, uint64_t x, uint64_t y,
                    void* words) {
    try {
        if (layout == 1) return pack_bits<algorithms::BitColumnsMode>(word_bits, cells, x, y, words);
        if (layout == 2) return pack_bits<algorithms::BitTileMode>(word_bits, cells, x, y, words);
        return -2;
    } catch (const std::exception&) {
        return -1;
    }
}

int ref_unpack_layout(int layout, int word_bits, const void* words, uint64_t x, uint64_t y,
                      uint8_t* cells) {
    try {
        if (layout == 1) return unpack_bits<algorithms::BitColumnsMode>(word_bits, words, x, y, cells);
        if (layout == 2) return unpack_bits<algorithms::BitTileMode>(word_bits, words, x, y, cells);
        return -2;
    } catch (const std::exception&) {
        return -1;
    }
}

int ref_load_zeros(uint64_t x, uint64_t y, uint8_t* out) {
    try {
        infrastructure::ZerosLoader<2, char> loader;
        grid_to(loader.load_data(make_params(x, y, 0, 0)), out);
        return 0;
    } catch (const std::exception&) {
        return -1;
    }
}

} // extern "C"
