"""ORACLE — test infrastructure, not product code.

ctypes front end for the two checkers of bit-packed Game of Life:

* ``liboracle`` — oracle/libgoloracle.so, the plain-C restatement of the
  reference's CPU path (oracle/gol_oracle.c; each function there cites the
  reference file:line it follows);
* ``libref`` — oracle/_ref/libgolref.so, the reference's own CPU code
  (GoLCpuNaive, GoLCpuBitwise<AdderOps>, RandomOnesZerosDataLoader,
  GeneralBitGrid) compiled from the reference sources by oracle/Makefile.
  It exists only where the reference sources were present at build time;
  ``ref_available()`` says whether it loaded.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module, and only as the checker or the timed CPU baseline.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "libgoloracle.so")
REF_SO = os.path.join(HERE, "_ref", "libgolref.so")
LEX_SO = os.path.join(HERE, "_ref", "libgollexref.so")

# Where the reference's sources are read from when the checkers are built
# (one environment variable; the default is where this build's recipe finds
# them). Nothing at run time reads them.
REFERENCE_SRC = os.environ.get("GOL_REFERENCE_SRC", "/root/reference/src")

LAYOUT_COLUMNS = 1
LAYOUT_TILES = 2

_u8p = ctypes.POINTER(ctypes.c_uint8)
_vp = ctypes.c_void_p
_u64 = ctypes.c_uint64

_oracle = None
_ref = None
_ref_tried = False
_lex = None
_lex_tried = False


def build(with_ref: bool | None = None) -> None:
    """Compiles the oracle (and the reference harness when its sources exist)."""
    targets = ["all"]
    if with_ref is None:
        with_ref = os.path.isdir(REFERENCE_SRC)
    if with_ref:
        targets.append("ref")
    subprocess.run(["make", "-s", "-C", HERE, *targets, f"REF_SRC={REFERENCE_SRC}"], check=True)


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_vp)


def liboracle():
    global _oracle
    if _oracle is None:
        if not os.path.exists(ORACLE_SO):
            build(with_ref=False)
        lib = ctypes.CDLL(ORACLE_SO)
        lib.gor_random_ones_zeros.argtypes = [_u64, _u64, _u64, _vp]
        lib.gor_life_naive.argtypes = [_vp, _u64, _u64, _u64, _vp]
        lib.gor_pack_rows.argtypes = [ctypes.c_int, _vp, _u64, _u64, _vp]
        lib.gor_unpack_rows.argtypes = [ctypes.c_int, _vp, _u64, _u64, _vp]
        lib.gor_life_rows.argtypes = [ctypes.c_int, _vp, _u64, _u64, _u64, _vp, ctypes.c_int]
        lib.gor_pack_layout.argtypes = [ctypes.c_int, ctypes.c_int, _vp, _u64, _u64, _vp]
        lib.gor_unpack_layout.argtypes = [ctypes.c_int, ctypes.c_int, _vp, _u64, _u64, _vp]
        lib.gor_fnv1a64.argtypes = [_vp, _u64]
        lib.gor_fnv1a64.restype = _u64
        lib.gor_max_threads.restype = ctypes.c_int
        _oracle = lib
    return _oracle


def libref():
    """The reference's own CPU path, or None when it was not built here."""
    global _ref, _ref_tried
    if not _ref_tried:
        _ref_tried = True
        if os.path.exists(REF_SO):
            lib = ctypes.CDLL(REF_SO)
            lib.ref_load_random_ones_zeros.argtypes = [_u64, _u64, _u64, _vp]
            lib.ref_run_cpu_naive.argtypes = [_vp, _u64, _u64, _u64, _vp]
            lib.ref_run_cpu_bitwise_adder.argtypes = [ctypes.c_int, _vp, _u64, _u64, _u64, _vp]
            lib.ref_pack_rows.argtypes = [ctypes.c_int, _vp, _u64, _u64, _vp]
            lib.ref_unpack_rows.argtypes = [ctypes.c_int, _vp, _u64, _u64, _vp]
            lib.ref_pack_layout.argtypes = [ctypes.c_int, ctypes.c_int, _vp, _u64, _u64, _vp]
            lib.ref_unpack_layout.argtypes = [ctypes.c_int, ctypes.c_int, _vp, _u64, _u64, _vp]
            lib.ref_load_zeros.argtypes = [_u64, _u64, _vp]
            lib.ref_bitwise_create.argtypes = [_vp, _u64, _u64]
            lib.ref_bitwise_create.restype = _vp
            lib.ref_bitwise_run.argtypes = [_vp, _u64]
            lib.ref_bitwise_finish.argtypes = [_vp, _vp]
            _ref = lib
    return _ref


def liblexref():
    """The reference's pattern loaders and compiled dictionary
    (oracle/_ref/libgollexref.so, `make -C oracle lexicon`), or None."""
    global _lex, _lex_tried
    if not _lex_tried:
        _lex_tried = True
        if os.path.exists(LEX_SO):
            lib = ctypes.CDLL(LEX_SO)
            lib.ref_load_always_changing.argtypes = [_u64, _u64, _vp]
            lib.ref_load_lexicon.argtypes = [ctypes.c_char_p, _u64, _u64, _vp]
            lib.ref_lexicon_count.restype = ctypes.c_int64
            lib.ref_lexicon_pattern.argtypes = [ctypes.c_int64, ctypes.c_char_p, _u64,
                                                ctypes.POINTER(_u64), ctypes.POINTER(_u64), _vp]
            _lex = lib
    return _lex


def ref_available() -> bool:
    return libref() is not None


def _check(rc: int, what: str) -> None:
    if rc != 0:
        raise RuntimeError(f"oracle call {what} failed with status {rc}")


# --------------------------------------------------------------------------
# restatement (oracle/gol_oracle.c)
# --------------------------------------------------------------------------

def random_ones_zeros(x: int, y: int, seed: int) -> np.ndarray:
    """uint8[y, x] of 0/1 cells as RandomOnesZerosDataLoader draws them."""
    out = np.empty((y, x), dtype=np.uint8)
    _check(liboracle().gor_random_ones_zeros(x, y, seed, _ptr(out)), "random_ones_zeros")
    return out


def life_naive(cells: np.ndarray, iters: int) -> np.ndarray:
    """GoLCpuNaive restated: uint8[y, x] in, uint8[y, x] out."""
    cells = np.ascontiguousarray(cells, dtype=np.uint8)
    y, x = cells.shape
    out = np.empty_like(cells)
    _check(liboracle().gor_life_naive(_ptr(cells), x, y, iters, _ptr(out)), "life_naive")
    return out


def pack_rows(cells: np.ndarray, word_bits: int = 64) -> np.ndarray:
    cells = np.ascontiguousarray(cells, dtype=np.uint8)
    y, x = cells.shape
    dt = np.uint64 if word_bits == 64 else np.uint32
    out = np.empty((y, x // word_bits), dtype=dt)
    _check(liboracle().gor_pack_rows(word_bits, _ptr(cells), x, y, _ptr(out)), "pack_rows")
    return out


def unpack_rows(words: np.ndarray, x: int, word_bits: int = 64) -> np.ndarray:
    words = np.ascontiguousarray(words)
    y = words.shape[0]
    out = np.empty((y, x), dtype=np.uint8)
    _check(liboracle().gor_unpack_rows(word_bits, _ptr(words), x, y, _ptr(out)), "unpack_rows")
    return out


_WORD_DTYPES = {16: np.uint16, 32: np.uint32, 64: np.uint64}


def layout_geom(layout: int, word_bits: int) -> tuple:
    """(X_BITS, Y_BITS) of BitColumns / BitTile (bit_modes.hpp:10-125)."""
    if layout == LAYOUT_COLUMNS:
        return 1, word_bits
    if layout == LAYOUT_TILES:
        return {16: (4, 4), 32: (8, 4), 64: (8, 8)}[word_bits]
    raise ValueError(layout)


def pack_layout(cells: np.ndarray, layout: int, word_bits: int) -> np.ndarray:
    cells = np.ascontiguousarray(cells, dtype=np.uint8)
    y, x = cells.shape
    xb, yb = layout_geom(layout, word_bits)
    out = np.empty((y // yb, x // xb), dtype=_WORD_DTYPES[word_bits])
    _check(liboracle().gor_pack_layout(layout, word_bits, _ptr(cells), x, y, _ptr(out)),
           "pack_layout")
    return out


def unpack_layout(words: np.ndarray, x: int, y: int, layout: int, word_bits: int) -> np.ndarray:
    words = np.ascontiguousarray(words)
    out = np.empty((y, x), dtype=np.uint8)
    _check(liboracle().gor_unpack_layout(layout, word_bits, _ptr(words), x, y, _ptr(out)),
           "unpack_layout")
    return out


# Pattern loaders, restated in Python for small grids
# (src/infrastructure/data_loader.hpp:77-146, gol-lexicon/lexicon.hpp:11-186).

def parse_pattern_dictionary(text: str) -> dict:
    """Entries {"name", {{_, X, ...}, ...}} of a patterns.cpp-style text
    (only between the LEXICON_START / LEXICON_END markers when both are
    present); the first entry of a repeated name wins, as in a std::map
    built from an initializer list."""
    a, b = text.find("/* LEXICON_START */"), text.find("/* LEXICON_END */")
    if a >= 0 and b > a:
        text = text[a:b]
    out: dict = {}
    i = 0
    while True:
        q = text.find('{"', i)
        if q < 0:
            return out
        e = text.index('"', q + 2)
        name = text[q + 2:e]
        depth, j, rows, row = 0, e + 1, [], None
        while True:
            c = text[j]
            j += 1
            if c == "{":
                depth += 1
                if depth == 2:
                    row = []
            elif c == "}":
                if depth == 2:
                    rows.append(row)
                depth -= 1
                if depth == 0:
                    break
            elif c in "X_" and depth == 2:
                row.append(1 if c == "X" else 0)
        out.setdefault(name, rows)
        i = j


def parse_pattern_expression(expr: str) -> list:
    """[(name, x_str, y_str)] of "name[x,y]; ..." with whitespace and ';'
    dropped first (PatterExpression::from, lexicon.hpp:97-116)."""
    t = "".join(c for c in expr if not (c.isspace() or c == ";"))
    recs, i = [], 0
    while i < len(t):
        j = i
        while j < len(t) and t[j] != "[":
            j += 1
        name = t[i:j]
        k = j + 1
        while k < len(t) and t[k] not in ",]":
            k += 1
        xs = t[j + 1:k]
        m = k + 1
        while m < len(t) and t[m] not in ",]":
            m += 1
        ys = t[k + 1:m]
        recs.append((name, xs, ys))
        i = m + 1
    return recs


def place_pattern(cells: np.ndarray, rows: list, ox: int, oy: int) -> None:
    """Lexicon::insert_pattern_at (lexicon.hpp:160-172) on a flat raster:
    cell (px, py) goes to element (oy + py) * X + ox + px; past the end is
    dropped."""
    y, x = cells.shape
    flat = cells.reshape(-1)
    for py, row in enumerate(rows):
        for px, v in enumerate(row):
            i = (oy + py) * x + ox + px
            if i < flat.size:
                flat[i] = v


def load_always_changing(x: int, y: int) -> np.ndarray:
    """AlwaysChangingSpaceLoader: a blinker at every multiple of (4, 4)."""
    g = np.zeros((y, x), dtype=np.uint8)
    for ox in range(0, x, 4):
        for oy in range(0, y, 4):
            place_pattern(g, [[1, 1, 1]], ox, oy)
    return g


def load_lexicon(patterns: dict, expr: str, x: int, y: int) -> np.ndarray:
    """LexiconLoader::load_data with the given dictionary; unknown names
    place nothing."""
    g = np.zeros((y, x), dtype=np.uint8)
    for name, xs, ys in parse_pattern_expression(expr):
        ox, oy = int(xs), int(ys)
        if name in patterns:
            place_pattern(g, patterns[name], ox, oy)
    return g


def life_rows(words: np.ndarray, x: int, iters: int, word_bits: int = 64,
              threads: int = 0) -> np.ndarray:
    """GoLCpuBitwise<AdderOps> restated on row-packed words (multi-threaded)."""
    words = np.ascontiguousarray(words)
    y = words.shape[0]
    out = np.empty_like(words)
    _check(liboracle().gor_life_rows(word_bits, _ptr(words), x, y, iters, _ptr(out), threads),
           "life_rows")
    return out


def life_cells(cells: np.ndarray, iters: int, threads: int = 0) -> np.ndarray:
    """Bit-sliced oracle on a cell grid (x a multiple of 32), cells in and out."""
    y, x = cells.shape
    wb = 64 if x % 64 == 0 else 32
    return unpack_rows(life_rows(pack_rows(cells, wb), x, iters, wb, threads), x, wb)


def fnv1a64(a: np.ndarray) -> int:
    a = np.ascontiguousarray(a)
    return int(liboracle().gor_fnv1a64(_ptr(a), a.nbytes))


def max_threads() -> int:
    return int(liboracle().gor_max_threads())


# --------------------------------------------------------------------------
# the reference itself (oracle/_ref), when built
# --------------------------------------------------------------------------

def _need_ref():
    lib = libref()
    if lib is None:
        raise RuntimeError("reference build oracle/_ref/libgolref.so is not present")
    return lib


def ref_random_ones_zeros(x: int, y: int, seed: int) -> np.ndarray:
    out = np.empty((y, x), dtype=np.uint8)
    _check(_need_ref().ref_load_random_ones_zeros(x, y, seed, _ptr(out)), "ref_load_random")
    return out


def ref_cpu_naive(cells: np.ndarray, iters: int) -> np.ndarray:
    cells = np.ascontiguousarray(cells, dtype=np.uint8)
    y, x = cells.shape
    out = np.empty_like(cells)
    _check(_need_ref().ref_run_cpu_naive(_ptr(cells), x, y, iters, _ptr(out)), "ref_cpu_naive")
    return out


def ref_cpu_bitwise_adder(cells: np.ndarray, iters: int, word_bits: int = 64) -> np.ndarray:
    cells = np.ascontiguousarray(cells, dtype=np.uint8)
    y, x = cells.shape
    out = np.empty_like(cells)
    _check(_need_ref().ref_run_cpu_bitwise_adder(word_bits, _ptr(cells), x, y, iters, _ptr(out)),
           "ref_cpu_bitwise_adder")
    return out


def ref_pack_rows(cells: np.ndarray, word_bits: int = 64) -> np.ndarray:
    cells = np.ascontiguousarray(cells, dtype=np.uint8)
    y, x = cells.shape
    dt = np.uint64 if word_bits == 64 else np.uint32
    out = np.empty((y, x // word_bits), dtype=dt)
    _check(_need_ref().ref_pack_rows(word_bits, _ptr(cells), x, y, _ptr(out)), "ref_pack_rows")
    return out


def ref_unpack_rows(words: np.ndarray, x: int, word_bits: int = 64) -> np.ndarray:
    words = np.ascontiguousarray(words)
    y = words.shape[0]
    out = np.empty((y, x), dtype=np.uint8)
    _check(_need_ref().ref_unpack_rows(word_bits, _ptr(words), x, y, _ptr(out)), "ref_unpack_rows")
    return out


def ref_pack_layout(cells: np.ndarray, layout: int, word_bits: int) -> np.ndarray:
    cells = np.ascontiguousarray(cells, dtype=np.uint8)
    y, x = cells.shape
    xb, yb = layout_geom(layout, word_bits)
    out = np.empty((y // yb, x // xb), dtype=_WORD_DTYPES[word_bits])
    _check(_need_ref().ref_pack_layout(layout, word_bits, _ptr(cells), x, y, _ptr(out)),
           "ref_pack_layout")
    return out


def ref_unpack_layout(words: np.ndarray, x: int, y: int, layout: int, word_bits: int) -> np.ndarray:
    words = np.ascontiguousarray(words)
    out = np.empty((y, x), dtype=np.uint8)
    _check(_need_ref().ref_unpack_layout(layout, word_bits, _ptr(words), x, y, _ptr(out)),
           "ref_unpack_layout")
    return out


def ref_load_zeros(x: int, y: int) -> np.ndarray:
    out = np.full((y, x), 7, dtype=np.uint8)
    _check(_need_ref().ref_load_zeros(x, y, _ptr(out)), "ref_load_zeros")
    return out


def _need_lex():
    lib = liblexref()
    if lib is None:
        raise RuntimeError("reference pattern loaders oracle/_ref/libgollexref.so not present")
    return lib


def ref_load_always_changing(x: int, y: int) -> np.ndarray:
    out = np.empty((y, x), dtype=np.uint8)
    _check(_need_lex().ref_load_always_changing(x, y, _ptr(out)), "ref_load_always_changing")
    return out


def ref_load_lexicon(expr: str, x: int, y: int) -> np.ndarray:
    out = np.empty((y, x), dtype=np.uint8)
    _check(_need_lex().ref_load_lexicon(expr.encode(), x, y, _ptr(out)), "ref_load_lexicon")
    return out


def ref_lexicon_patterns() -> dict:
    """name -> uint8[h, w] (short rows padded dead) of the compiled dictionary."""
    lib = _need_lex()
    out = {}
    name = ctypes.create_string_buffer(4096)
    w, h = _u64(), _u64()
    for i in range(lib.ref_lexicon_count()):
        _check(lib.ref_lexicon_pattern(i, name, 4096, ctypes.byref(w), ctypes.byref(h), None),
               "ref_lexicon_pattern")
        cells = np.zeros((h.value, w.value), dtype=np.uint8)
        _check(lib.ref_lexicon_pattern(i, name, 4096, ctypes.byref(w), ctypes.byref(h),
                                       _ptr(cells)), "ref_lexicon_pattern")
        out[name.value.decode()] = cells
    return out


class RefBitwise:
    """The reference's GoLCpuBitwise<char,64,AdderOps> with its phases apart:
    construction packs and initialises, run(iters) advances, finish() returns
    the cell grid (and frees the instance)."""

    def __init__(self, cells: np.ndarray):
        cells = np.ascontiguousarray(cells, dtype=np.uint8)
        self.shape = cells.shape
        self._h = _need_ref().ref_bitwise_create(_ptr(cells), cells.shape[1], cells.shape[0])
        if not self._h:
            raise RuntimeError("ref_bitwise_create failed")

    def run(self, iters: int) -> None:
        _check(_need_ref().ref_bitwise_run(self._h, iters), "ref_bitwise_run")

    def finish(self) -> np.ndarray:
        out = np.empty(self.shape, dtype=np.uint8)
        h, self._h = self._h, None
        _check(_need_ref().ref_bitwise_finish(h, _ptr(out)), "ref_bitwise_finish")
        return out
