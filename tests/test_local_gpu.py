"""Change-tracking engine (GOL_ALG_LOCAL) on a GPU: bit-exact against the
oracle and the golden fixtures, with the skip rule exercised by sparse,
settling and moving patterns, and the census reporting skipped tiles."""
import numpy as np
import pytest

import golb200
import oracle
from golden_inputs import case_input, case_output

pytestmark = pytest.mark.gpu


def run_local(cells, iters, k=4, tile_rows=0, word_bits=None, stats=False, **kw):
    y, x = cells.shape
    if word_bits is None:
        word_bits = 64 if x % 64 == 0 else 32
    with golb200.GolB200(grid_dimensions=(x, y), state_bits_count=word_bits, temporal_steps=k,
                         algorithm="local", **({"tile_rows": tile_rows} if tile_rows else {}),
                         **kw) as alg:
        alg.set_and_format_input_data(cells)
        alg.initialize_data_structures()
        alg.run(iters)
        alg.finalize_data_structures()
        out = alg.fetch_result()
        return (out, alg.local_stats()) if stats else out


@pytest.mark.parametrize("k,tile_rows", [(1, 0), (2, 8), (4, 0), (4, 4), (8, 16), (5, 0)])
def test_local_golden_fixtures(golden_cases, k, tile_rows):
    for case in golden_cases:
        g = case_input(case)
        out = run_local(g, case["iters"], k=k, tile_rows=tile_rows)
        assert f"{oracle.fnv1a64(out):016x}" == case["output_fnv1a64"], (case["name"], k)
        stored = case_output(case)
        if stored is not None:
            assert np.array_equal(out, stored), (case["name"], k)


@pytest.mark.parametrize("x,y,iters,k", [(1024, 1024, 600, 4), (2048, 512, 333, 8),
                                         (3072, 640, 257, 2), (4096, 256, 100, 1),
                                         (960, 192, 151, 3)])
def test_sparse_patches_vs_oracle(x, y, iters, k):
    g = golb200.load_sparse_patches(x, y, seed=x + iters, patch=64, fraction=0.05, density=0.35)
    ref = oracle.life_cells(g, iters)
    out, st = run_local(g, iters, k=k, stats=True)
    assert np.array_equal(out, ref)
    assert st["passes"] == iters // k
    assert st["computed_tiles"] <= st["passes"] * st["tiles_per_pass"]


@pytest.mark.parametrize("wpl,k,tile_rows", [(2, 4, 0), (4, 4, 8), (2, 8, 12), (1, 3, 0)])
def test_wider_lanes_and_tile_heights(wpl, k, tile_rows):
    """Change tracking with 2 and 4 words per lane (wider tiles and halos)
    and explicit tile heights, on a sparse input that settles and moves."""
    g = golb200.load_sparse_patches(2048, 768, seed=wpl * 10 + k, patch=64, fraction=0.05,
                                    density=0.35)
    n = 6 * k + 1
    assert np.array_equal(run_local(g, n, k=k, tile_rows=tile_rows, lane_words=wpl),
                          oracle.life_cells(g, n)), (wpl, k, tile_rows)


def test_sparse_input_skips_most_tiles():
    g = golb200.load_sparse_patches(8192, 4096, seed=11, patch=64, fraction=0.002, density=0.35)
    out, st = run_local(g, 1000, k=8, stats=True)
    assert np.array_equal(out, oracle.life_cells(g, 1000))
    assert st["computed_tiles"] < 0.5 * st["passes"] * st["tiles_per_pass"]


def test_still_life_retires_all_tiles():
    g = np.zeros((256, 2048), np.uint8)
    for (cx, cy) in ((100, 100), (1000, 30), (1500, 200)):   # 2x2 blocks
        g[cy:cy + 2, cx:cx + 2] = 1
    with golb200.GolB200(grid_dimensions=(2048, 256), temporal_steps=4, algorithm="local") as alg:
        alg.set_and_format_input_data(g)
        alg.initialize_data_structures()
        alg.run(400)
        st = alg.local_stats(max_entries=100)
        alg.finalize_data_structures()
        assert np.array_equal(alg.fetch_result(), g)
    per = st["per_pass"]
    # The first pass computes every tile (dense), and so does the next: a pass
    # after one with that many active tiles is planned without a tile list.
    assert st["passes"] == 100 and list(per[:2]) == [st["tiles_per_pass"]] * 2
    assert int(per[2:].sum()) == 0          # nothing changed: nothing recomputed after


def test_oscillators_with_even_depth_and_odd_remainder():
    """Blinkers look stable to 4-generation passes; the 3-generation
    remainder pass must still flip them."""
    g = np.zeros((128, 1024), np.uint8)
    for cx in range(10, 1000, 97):
        g[60, cx:cx + 3] = 1
    for iters in (4 * 50, 4 * 50 + 3, 4 * 50 + 1):
        assert np.array_equal(run_local(g, iters, k=4), oracle.life_cells(g, iters)), iters


def test_gliders_cross_tiles():
    g = np.zeros((512, 2048), np.uint8)
    glider = [(1, 0), (2, 1), (0, 2), (1, 2), (2, 2)]
    for ox, oy in ((20, 20), (900, 100), (1700, 300), (31, 250)):
        for cx, cy in glider:
            g[oy + cy, ox + cx] = 1
    for k in (1, 4, 7):
        assert np.array_equal(run_local(g, 777, k=k), oracle.life_cells(g, 777)), k


def test_local_rounds_and_repeated_runs():
    g = golb200.load_sparse_patches(1024, 512, seed=3, patch=64, fraction=0.1, density=0.35)
    with golb200.GolB200(grid_dimensions=(1024, 512), temporal_steps=4, algorithm="local") as alg:
        for _ in range(2):
            alg.set_and_format_input_data(g)
            alg.initialize_data_structures()
            alg.run(101)
            alg.run(64)          # runs continue from the current state
            alg.finalize_data_structures()
            assert np.array_equal(alg.fetch_result(), oracle.life_cells(g, 165))


@pytest.mark.slow
def test_sparse_benchmark_size_local_equals_dense():
    """16384^2 sparse/settling input: change tracking and the dense engine
    give the same grid (size-independent cross-check), and the oracle agrees
    on the first 256 generations."""
    g = golb200.load_sparse_patches(16384, 16384, seed=42)
    dense = golb200.run_generations(g, 2048, temporal_steps=4)
    local = run_local(g, 2048, k=8)
    assert np.array_equal(dense, local)
    ref = oracle.life_cells(g, 256)
    assert np.array_equal(run_local(g, 256, k=8), ref)


@pytest.mark.parametrize("k", [5, 6])
def test_published_loaders(k):
    """The reference's change-tracking benchmark inputs: the blinker lattice
    (period 2) and the all-dead grid. At an odd depth every tile of the
    lattice changes every pass; at an even one every tile returns to its
    input, so after the first two passes (dense: all tiles active, then
    the pass planned without a list) only the top two tile rows are
    computed again (the lattice's row-0 blinkers die against the dead
    outside)."""
    n = 4 * k + 1
    blink = golb200.load_always_changing(1024, 512)
    out, st = run_local(blink, n, k=k, stats=True)
    assert np.array_equal(out, oracle.life_cells(blink, n))
    full = st["passes"] * st["tiles_per_pass"]
    if k % 2:
        assert st["computed_tiles"] == full
    else:
        assert st["computed_tiles"] < 2.1 * st["tiles_per_pass"]
    zeros = golb200.load_zeros(1024, 512)
    out, st = run_local(zeros, n, k=k, stats=True)
    assert not out.any()
    assert st["computed_tiles"] <= 2 * st["tiles_per_pass"]


@pytest.mark.parametrize("x,y,k,wpl,dense_pct", [
    (1024, 512, 6, 0, 1), (1024, 512, 6, 0, 30), (1024, 512, 6, 0, 101),
    (2048, 384, 4, 4, 20), (2048, 384, 5, 2, 20), (1152, 200, 3, 0, 15),
    (32768, 192, 6, 0, 10),     # the dense form cut into x-slices
    (64, 130, 5, 0, 50),        # one tile column
])
def test_dense_passes_hand_over(x, y, k, wpl, dense_pct):
    """A settling random grid crosses the dense threshold: passes run dense
    while many tiles are active and as tiles later, each mode planning from
    the other's change bits. Results against the oracle for thresholds from
    "almost always dense" (1 %) to "never" (above 100 %)."""
    g = golb200.load_bernoulli(x, y, seed=x + y + k, density=0.3)
    n = 40 * k + (k - 1)
    out, st = run_local(g, n, k=k, stats=True, lane_words=wpl, dense_pct=dense_pct)
    assert np.array_equal(out, oracle.life_cells(g, n)), (x, y, k, wpl, dense_pct)
    full = st["passes"] * st["tiles_per_pass"]
    assert st["computed_tiles"] <= full
    if dense_pct == 1:      # a soup keeps more than 1 % of its tiles active
        assert st["computed_tiles"] == full


def test_dense_pass_census_counts_every_tile():
    """A pass that runs dense computes, and records, every tile."""
    g = golb200.load_bernoulli(1024, 512, seed=3, density=0.5)
    out, st = run_local(g, 5 * 6, k=6, stats=True, dense_pct=1)
    assert np.array_equal(out, oracle.life_cells(g, 30))
    per = None
    with golb200.GolB200(grid_dimensions=(1024, 512), temporal_steps=6, algorithm="local",
                         dense_pct=1) as alg:
        alg.set_and_format_input_data(g)
        alg.initialize_data_structures()
        alg.run(30)
        per = alg.local_stats(max_entries=8)["per_pass"]
    assert list(per) == [st["tiles_per_pass"]] * 5
