"""The reference's other input loaders (zeros, always-changing, lexicon
pattern expressions) and its column / tile word layouts, on the host:
against the oracle's restatement and, where it was built here, against the
reference's own loaders and GeneralBitGrid. CPU only."""
import os

import numpy as np
import pytest

import golb200
import oracle

# A dictionary in the reference's patterns.cpp format, written for these
# tests from the B3/S23 rule itself (still lifes, an oscillator, a glider).
OWN_DICTIONARY = """
    return {
        /* LEXICON_START */
{"block", {
{X, X},
{X, X}}},

{"tub", {
{_, X, _},
{X, _, X},
{_, X, _}}},

{"toad", {
{_, X, X, X},
{X, X, X, _}}},

{"glider", {
{_, X, _},
{_, _, X},
{X, X, X}}},

{"ragged", {
{X},
{_, _, X},
{}}},

{"block", {
{X}}},
        /* LEXICON_END */
    };
"""

REF_PATTERNS = os.path.join(oracle.REFERENCE_SRC, "infrastructure", "gol-lexicon", "patterns.cpp")


def test_zeros_loader():
    g = golb200.load_zeros(96, 17)
    assert g.shape == (17, 96) and not g.any()
    if oracle.ref_available():
        assert np.array_equal(g, oracle.ref_load_zeros(96, 17))


@pytest.mark.parametrize("x,y", [(64, 64), (96, 33), (30, 9), (7, 5), (4, 4), (1, 1)])
def test_always_changing_loader(x, y):
    g = golb200.load_always_changing(x, y)
    assert np.array_equal(g, oracle.load_always_changing(x, y)), (x, y)
    # The reference is only run where its last blinker stays inside the raster.
    if oracle.liblexref() is not None and (y - 1) // 4 * 4 * x + (x - 1) // 4 * 4 + 3 <= x * y:
        assert np.array_equal(g, oracle.ref_load_always_changing(x, y)), (x, y)


def test_always_changing_space_never_settles():
    """Every generation differs from the one before; after two generations
    the space oscillates with period two."""
    g = golb200.load_always_changing(64, 32)
    gens = [g] + [oracle.life_cells(g, n) for n in range(1, 7)]
    assert all(not np.array_equal(a, b) for a, b in zip(gens, gens[1:]))
    assert all(np.array_equal(gens[n], gens[n - 2]) for n in range(4, 7))


def test_dictionary_parsing_and_sizes():
    lx = golb200.Lexicon()
    assert len(lx) == 1 and lx.pattern_size("blinker") == (3, 1)
    assert lx.add_text(OWN_DICTIONARY) == 6           # entries read, repeated name included
    assert len(lx) == 6                               # blinker + 5 distinct names
    assert lx.pattern_size("block") == (2, 2)          # the first "block" wins
    assert lx.pattern_size("ragged") == (3, 3)
    with pytest.raises(ValueError):
        lx.pattern_size("nope")
    with pytest.raises(ValueError, match="unexpected"):
        lx.add_text('{"bad", {{X, Y}}}')
    with pytest.raises(ValueError, match="cannot open"):
        lx.add_file("/nonexistent/patterns.cpp")


@pytest.mark.parametrize("expr", [
    "glider[1,1]",
    "glider[ 1 , 1 ];  block[10,3]; tub[20,20]",
    "block[5,5]; glider[4,4]",                  # later patterns overwrite, dead cells too
    "toad[60,2]",                               # runs past the right edge onto the next row
    "ragged[0,0];unknown[3,3];toad[10,10]",     # unknown names place nothing
    "block[62,63]",                             # past the end of the raster: dropped
    "",
])
def test_lexicon_expressions_match_restatement(expr):
    lx = golb200.Lexicon(text=OWN_DICTIONARY)
    mine = lx.load(expr, 64, 64)
    ref = oracle.load_lexicon(oracle.parse_pattern_dictionary(OWN_DICTIONARY), expr, 64, 64)
    assert np.array_equal(mine, ref), expr


def test_lexicon_record_count_and_bad_coordinates():
    lx = golb200.Lexicon(text=OWN_DICTIONARY)
    g = np.zeros((32, 32), np.uint8)
    assert lx.insert("block[1,1]; nope[2,2]; tub[9,9]", g) == 2
    with pytest.raises(ValueError, match="bad coordinates"):
        lx.insert("block[a,1]", g)
    with pytest.raises(ValueError, match="bad coordinates"):
        lx.insert("block[-3,1]", g)
    h = np.zeros((16, 16), np.uint8)
    lx.insert_repeating("block", 5, 7, h)
    exp = np.zeros((16, 16), np.uint8)
    for ox in range(0, 16, 5):
        for oy in range(0, 16, 7):
            oracle.place_pattern(exp, [[1, 1], [1, 1]], ox, oy)
    assert np.array_equal(h, exp)


needs_lexref = pytest.mark.skipif(
    oracle.liblexref() is None or not os.path.exists(REF_PATTERNS),
    reason="reference pattern loaders (make -C oracle lexicon) not built here")


@needs_lexref
def test_reference_dictionary_parses_identically():
    """Every entry of the reference's dictionary, read from its source text,
    equals the compiled dictionary entry."""
    lx = golb200.Lexicon(path=REF_PATTERNS)
    ref = oracle.ref_lexicon_patterns()
    assert len(lx) == len(ref)
    for name, cells in ref.items():
        h, w = cells.shape
        assert lx.pattern_size(name) == (w, h), name
        g = np.zeros((max(h, 1), max(w, 1)), np.uint8)
        lx.insert(f"{name}[0,0]", g)
        assert np.array_equal(g[:h, :w], cells), name


@needs_lexref
@pytest.mark.parametrize("expr,x,y", [
    ("glider[10,10]; blinker[40,5]; block[3,50]", 128, 96),
    ("gosper-glider-gun[5,5];  pulsar[60,40]", 128, 128),
    ("101[0,0]; blinker-fuse[10,30]; no-such-pattern[1,1]", 256, 64),
])
def test_lexicon_loader_matches_reference(expr, x, y):
    lx = golb200.Lexicon(path=REF_PATTERNS)
    assert np.array_equal(lx.load(expr, x, y), oracle.ref_load_lexicon(expr, x, y)), expr


SHAPES = [(64, 64), (128, 32), (96, 16), (256, 128), (32, 64)]


@pytest.mark.parametrize("layout", ["columns", "tiles", "rows"])
@pytest.mark.parametrize("word_bits", [16, 32, 64])
def test_layout_pack_unpack_match_restatement_and_reference(layout, word_bits):
    lay = golb200.LAYOUTS[layout]
    for (x, y) in SHAPES:
        xb, yb = golb200.layout_block(layout, word_bits)
        if x % xb or y % yb:
            continue
        g = oracle.random_ones_zeros(x, y, x * 7 + y)
        w = golb200.pack_layout(g, layout, word_bits)
        if layout == "rows":
            assert w.tobytes() == oracle.pack_rows(g, 32).tobytes()
        else:
            assert np.array_equal(w, oracle.pack_layout(g, lay, word_bits)), (x, y)
            if oracle.ref_available():
                assert np.array_equal(w, oracle.ref_pack_layout(g, lay, word_bits)), (x, y)
        assert np.array_equal(golb200.unpack_layout(w, x, y, layout, word_bits), g)


def test_layout_rejects_partial_blocks():
    g = np.zeros((12, 64), np.uint8)
    with pytest.raises(ValueError):
        golb200.pack_layout(g, "columns", 16)     # 12 rows is not a whole 16-row word
    with pytest.raises(ValueError):
        golb200.pack_layout(np.zeros((8, 36), np.uint8), "tiles", 64)


@pytest.mark.parametrize("layout,word_bits", [("columns", 64), ("columns", 16), ("tiles", 64),
                                              ("tiles", 32), ("tiles", 16), ("rows", 16)])
def test_engine_layout_input_and_output_on_host(layout, word_bits):
    """set_input_layout then fetch_layout / fetch_result with no device work:
    the conversions to and from the engine's rows on the host."""
    x, y = 192, 64
    g = oracle.random_ones_zeros(x, y, 5)
    alg = golb200.GolB200(grid_dimensions=(x, y), state_bits_count=64)
    alg.set_input_layout(golb200.pack_layout(g, layout, word_bits), layout, word_bits)
    assert np.array_equal(alg.fetch_result(), g)
    assert np.array_equal(alg.fetch_words(64), oracle.pack_rows(g, 64))
    for lay2, wb2 in (("columns", 32), ("tiles", 64), ("rows", 64), (layout, word_bits)):
        assert np.array_equal(alg.fetch_layout(lay2, wb2), golb200.pack_layout(g, lay2, wb2))
    alg.close()
