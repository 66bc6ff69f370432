// Input loaders beside random-ones-zeros: "zeros", "always-changing" and
// "lexicon" (pattern expressions), host only, as the reference registers
// them (src/infrastructure/experiment_manager.hpp:396-410,
// src/infrastructure/data_loader.hpp:77-152).
//
// Pattern dictionaries are read at run time from text in the format of the
// reference's generated dictionary (gol-lexicon/patterns.cpp): entries
// {"name", {{_, X, ...}, {...}}} with `_` dead and `X` alive, row by row; when
// the text has the /* LEXICON_START */ and /* LEXICON_END */ markers only the
// part between them is read. No pattern data is compiled in except the
// blinker (three live cells in a row), which the always-changing loader
// needs.
//
// Placement follows Grid<2,T>::operator[] (src/infrastructure/grid.hpp:
// 80-101): cell (x, y) of a pattern at offset (ox, oy) is element
// (oy + y) * X + (ox + x) of the raster, so a pattern running past the right
// edge continues on the next row. Dead pattern cells are written too (a
// pattern overwrites what is under it). Writes past the end of the raster,
// which the reference leaves undefined, are dropped here.
#include <cctype>
#include <cerrno>
#include <climits>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <new>
#include <sstream>
#include <string>
#include <vector>

#include "gol_b200.h"

struct gol_lexicon {
    std::map<std::string, std::vector<std::vector<uint8_t>>> patterns;
    std::string err;

    int fail(int code, std::string msg) {
        err = std::move(msg);
        return code;
    }
};

namespace {

using Pattern = std::vector<std::vector<uint8_t>>;

Pattern blinker() { return Pattern{{1, 1, 1}}; }

void put_pattern(const Pattern& p, uint64_t ox, uint64_t oy, uint8_t* cells, uint64_t x,
                 uint64_t y) {
    const uint64_t n = x * y;
    for (uint64_t py = 0; py < p.size(); ++py) {
        const auto& row = p[py];
        for (uint64_t px = 0; px < row.size(); ++px) {
            const uint64_t i = (oy + py) * x + (ox + px);
            if (i < n) cells[i] = row[px];
        }
    }
}

// Expression separators: whitespace and ';' are removed before parsing
// (lexicon.hpp:12-33, 104-117).
bool is_sep(char c) { return std::isspace(static_cast<unsigned char>(c)) || c == ';'; }

// A coordinate string as std::stoi reads it (optional sign, digits, rest
// ignored), kept to non-negative values that fit an int.
bool parse_coord(const std::string& s, uint64_t* v) {
    const char* p = s.c_str();
    errno = 0;
    char* end = nullptr;
    const long long r = std::strtoll(p, &end, 10);
    if (end == p || errno == ERANGE || r > INT_MAX || r < INT_MIN) return false;
    if (r < 0) return false;
    *v = static_cast<uint64_t>(r);
    return true;
}

struct Record {
    std::string name, xs, ys;
};

// Records name[x,y] one after another in the separator-free expression
// (PatternExpresionRecord::from, lexicon.hpp:42-95): the name runs to '[',
// x to ',' or ']', y to ',' or ']', and the next record starts one past
// where y stopped.
std::vector<Record> parse_expression(const std::string& expr) {
    std::string t;
    for (char c : expr)
        if (!is_sep(c)) t.push_back(c);
    std::vector<Record> out;
    size_t i = 0;
    while (i < t.size()) {
        Record r;
        while (i < t.size() && t[i] != '[') r.name.push_back(t[i++]);
        ++i;
        while (i < t.size() && t[i] != ',' && t[i] != ']') r.xs.push_back(t[i++]);
        ++i;
        while (i < t.size() && t[i] != ',' && t[i] != ']') r.ys.push_back(t[i++]);
        out.push_back(std::move(r));
        i += 1;
    }
    return out;
}

// Dictionary text -> patterns. Returns the number of entries read, or -1
// with *err set on malformed text.
long parse_dictionary(const std::string& all, std::map<std::string, Pattern>* dict,
                      std::string* err) {
    std::string text = all;
    const size_t a = all.find("/* LEXICON_START */");
    const size_t b = all.find("/* LEXICON_END */");
    if (a != std::string::npos && b != std::string::npos && b > a)
        text = all.substr(a, b - a);
    long count = 0;
    size_t i = 0;
    const size_t n = text.size();
    auto skip = [&](void) {
        while (i < n && (std::isspace(static_cast<unsigned char>(text[i])) || text[i] == ','))
            ++i;
    };
    while (true) {
        const size_t q = text.find("{\"", i);
        if (q == std::string::npos) break;
        i = q + 2;
        const size_t e = text.find('"', i);
        if (e == std::string::npos) return *err = "unterminated pattern name", -1;
        std::string name = text.substr(i, e - i);
        i = e + 1;
        skip();
        if (i >= n || text[i] != '{') return *err = "pattern '" + name + "': expected '{'", -1;
        ++i;
        Pattern p;
        while (true) {
            skip();
            if (i >= n) return *err = "pattern '" + name + "': unterminated", -1;
            if (text[i] == '}') {
                ++i;
                break;
            }
            if (text[i] != '{') return *err = "pattern '" + name + "': expected a row", -1;
            ++i;
            std::vector<uint8_t> row;
            while (true) {
                skip();
                if (i >= n) return *err = "pattern '" + name + "': unterminated row", -1;
                const char c = text[i];
                if (c == '}') {
                    ++i;
                    break;
                }
                if (c == 'X') row.push_back(1);
                else if (c == '_') row.push_back(0);
                else return *err = "pattern '" + name + "': unexpected '" + std::string(1, c) + "'", -1;
                ++i;
            }
            p.push_back(std::move(row));
        }
        dict->emplace(name, std::move(p));   // first entry of a name wins, as in a std::map
        ++count;                             // built from an initializer list
    }
    return count;
}

} // namespace

extern "C" {

int gol_load_zeros(uint8_t* cells, uint64_t x, uint64_t y) {
    if (!cells && x * y) return GOL_E_INVALID;
    if (x * y) std::memset(cells, 0, x * y);
    return GOL_OK;
}

// AlwaysChangingSpaceLoader<2,T> (data_loader.hpp:102-125): a blinker at
// every (x, y) with x % 4 == 0 and y % 4 == 0 (Lexicon::insert_repeating,
// lexicon.hpp:137-145), on a dead grid.
int gol_load_always_changing(uint8_t* cells, uint64_t x, uint64_t y) {
    if (!cells && x * y) return GOL_E_INVALID;
    if (x * y == 0) return GOL_OK;
    std::memset(cells, 0, x * y);
    const Pattern p = blinker();
    for (uint64_t ox = 0; ox < x; ox += 4)
        for (uint64_t oy = 0; oy < y; oy += 4) put_pattern(p, ox, oy, cells, x, y);
    return GOL_OK;
}

int gol_lexicon_create(gol_lexicon** out) {
    if (!out) return GOL_E_INVALID;
    *out = nullptr;
    auto* lx = new (std::nothrow) gol_lexicon();
    if (!lx) return GOL_E_NOMEM;
    lx->patterns["blinker"] = blinker();
    *out = lx;
    return GOL_OK;
}

int gol_lexicon_add_text(gol_lexicon* lx, const char* text) {
    if (!lx) return GOL_E_INVALID;
    if (!text) return lx->fail(GOL_E_INVALID, "null dictionary text");
    std::map<std::string, Pattern> dict;
    std::string err;
    const long n = parse_dictionary(text, &dict, &err);
    if (n < 0) return lx->fail(GOL_E_INVALID, err);
    for (auto& kv : dict) lx->patterns[kv.first] = std::move(kv.second);
    return static_cast<int>(n);
}

int gol_lexicon_add_file(gol_lexicon* lx, const char* path) {
    if (!lx) return GOL_E_INVALID;
    if (!path) return lx->fail(GOL_E_INVALID, "null dictionary path");
    std::ifstream f(path, std::ios::binary);
    if (!f) return lx->fail(GOL_E_INVALID, std::string("cannot open ") + path);
    std::ostringstream ss;
    ss << f.rdbuf();
    return gol_lexicon_add_text(lx, ss.str().c_str());
}

int gol_lexicon_count(const gol_lexicon* lx) {
    return lx ? static_cast<int>(lx->patterns.size()) : GOL_E_INVALID;
}

int gol_lexicon_pattern_size(const gol_lexicon* lx, const char* name, uint64_t* width,
                             uint64_t* height) {
    if (!lx || !name || !width || !height) return GOL_E_INVALID;
    auto it = lx->patterns.find(name);
    if (it == lx->patterns.end()) return GOL_E_INVALID;
    uint64_t w = 0;
    for (const auto& r : it->second) w = r.size() > w ? r.size() : w;
    *width = w;
    *height = it->second.size();
    return GOL_OK;
}

// LexiconLoader<2,T> (data_loader.hpp:88-99, Lexicon::insert_patters,
// lexicon.hpp:123-130): each record name[x,y] of the expression places the
// named pattern with its top-left cell at (x, y); unknown names place
// nothing (the empty pattern, lexicon.hpp:174-179). Returns the number of
// records placed, or GOL_E_INVALID for a coordinate std::stoi would reject
// (or a negative one).
int gol_lexicon_insert(gol_lexicon* lx, const char* expression, uint8_t* cells, uint64_t x,
                       uint64_t y) {
    if (!lx) return GOL_E_INVALID;
    if (!expression || (!cells && x * y)) return lx->fail(GOL_E_INVALID, "null argument");
    const auto recs = parse_expression(expression);
    std::vector<std::pair<const Pattern*, std::pair<uint64_t, uint64_t>>> place;
    for (const auto& r : recs) {
        uint64_t ox, oy;
        if (!parse_coord(r.xs, &ox) || !parse_coord(r.ys, &oy))
            return lx->fail(GOL_E_INVALID, "bad coordinates in record '" + r.name + "[" + r.xs +
                                               "," + r.ys + "]'");
        auto it = lx->patterns.find(r.name);
        place.push_back({it == lx->patterns.end() ? nullptr : &it->second, {ox, oy}});
    }
    int placed = 0;
    for (const auto& pl : place) {
        if (!pl.first) continue;
        put_pattern(*pl.first, pl.second.first, pl.second.second, cells, x, y);
        ++placed;
    }
    return placed;
}

int gol_lexicon_insert_repeating(gol_lexicon* lx, const char* name, uint64_t x_jump,
                                 uint64_t y_jump, uint8_t* cells, uint64_t x, uint64_t y) {
    if (!lx) return GOL_E_INVALID;
    if (!name || !x_jump || !y_jump || (!cells && x * y))
        return lx->fail(GOL_E_INVALID, "bad argument");
    auto it = lx->patterns.find(name);
    if (it == lx->patterns.end()) return GOL_OK;
    for (uint64_t ox = 0; ox < x; ox += x_jump)
        for (uint64_t oy = 0; oy < y; oy += y_jump) put_pattern(it->second, ox, oy, cells, x, y);
    return GOL_OK;
}

const char* gol_lexicon_last_error(const gol_lexicon* lx) {
    return lx ? lx->err.c_str() : "null lexicon";
}

void gol_lexicon_destroy(gol_lexicon* lx) { delete lx; }

} // extern "C"
