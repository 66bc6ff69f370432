// Test infrastructure, not product code.
//
// The reference's pattern loaders, compiled from the reference sources in
// place into oracle/_ref/libgollexref.so together with its generated pattern
// dictionary (gol-lexicon/patterns.cpp, a large initializer list that takes
// minutes to compile, so it is a separate make target), for the loader
// parity tests:
//   ref_load_always_changing : AlwaysChangingSpaceLoader<2,char>
//                              (src/infrastructure/data_loader.hpp:102-125)
//   ref_load_lexicon         : LexiconLoader<2,char> (data_loader.hpp:77-99)
//   ref_lexicon_count / ref_lexicon_pattern : lexicon::PatternDict
//                              (gol-lexicon/patterns.hpp:10-18)
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <exception>
#include <iterator>

#include "infrastructure/data_loader.hpp"
#include "infrastructure/experiment_params.hpp"
#include "infrastructure/grid.hpp"

namespace {

infrastructure::ExperimentParams make_params(std::size_t x, std::size_t y) {
    infrastructure::ExperimentParams p;
    p.grid_dimensions = {x, y};
    p.iterations = 0;
    p.random_seed = 0;
    p.animate_output = false;
    p.max_runtime_seconds = infrastructure::StopWatch::MAX_TIME;
    return p;
}

void grid_to(const infrastructure::Grid<2, char>& g, uint8_t* out) {
    std::memcpy(out, g.data(), g.size());
}

} // namespace

extern "C" {

int ref_load_always_changing(uint64_t x, uint64_t y, uint8_t* out) {
    try {
        infrastructure::AlwaysChangingSpaceLoader<2, char> loader;
        grid_to(loader.load_data(make_params(x, y)), out);
        return 0;
    } catch (const std::exception&) {
        return -1;
    }
}

int ref_load_lexicon(const char* expression, uint64_t x, uint64_t y, uint8_t* out) {
    try {
        infrastructure::LexiconLoader<2, char> loader;
        auto p = make_params(x, y);
        p.pattern_expression = expression;
        grid_to(loader.load_data(p), out);
        return 0;
    } catch (const std::exception&) {
        return -1;
    }
}

int64_t ref_lexicon_count() {
    return (int64_t)lexicon::PatternDict().all_patterns().size();
}

// Name of entry `index` (map order) into name_out (NUL-terminated, at most
// cap bytes); its height and widest row into *h, *w; cells row-major into
// cells (w * h bytes, short rows padded dead) when cells is non-null.
int ref_lexicon_pattern(int64_t index, char* name_out, uint64_t cap, uint64_t* w, uint64_t* h,
                        uint8_t* cells) {
    static const auto dict = lexicon::PatternDict().all_patterns();
    if (index < 0 || index >= (int64_t)dict.size()) return -2;
    auto it = dict.begin();
    std::advance(it, index);
    std::snprintf(name_out, cap, "%s", it->first.c_str());
    uint64_t width = 0;
    for (const auto& row : it->second) width = row.size() > width ? row.size() : width;
    *w = width;
    *h = it->second.size();
    if (cells) {
        std::memset(cells, 0, width * it->second.size());
        for (size_t r = 0; r < it->second.size(); ++r)
            for (size_t c = 0; c < it->second[r].size(); ++c) cells[r * width + c] = it->second[r][c];
    }
    return 0;
}

} // extern "C"
