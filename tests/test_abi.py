"""The C-ABI library without compute on a GPU: it loads, exports every
symbol include/gol_b200.h declares, validates arguments, enforces the
contract's phase order, and packs/unpacks on the host. CPU only."""
import ctypes

import numpy as np
import pytest

import golb200
import oracle


def test_library_exports_every_declared_symbol():
    L = golb200.lib()
    names = golb200.declared_symbols()
    assert "gol_create" in names and "gol_run" in names
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    assert L.gol_abi_version() == 1
    assert b"sm_100a" in L.gol_build_info()


def test_config_struct_size_matches_library():
    cfg = golb200.GolConfig()
    golb200.lib().gol_config_init(ctypes.byref(cfg), 64, 64)
    assert cfg.struct_size == ctypes.sizeof(golb200.GolConfig)
    assert cfg.word_bits == 64


@pytest.mark.parametrize("kw,needle", [
    (dict(grid_dimensions=(96, 8), state_bits_count=64), "multiple of word_bits"),
    (dict(grid_dimensions=(64, 8), state_bits_count=16), "32 or 64"),
    (dict(grid_dimensions=(64, 8), temporal_steps=17), "at most 16"),
])
def test_create_rejects_bad_config(kw, needle):
    with pytest.raises(RuntimeError, match=needle):
        golb200.GolB200(**kw)


def test_phase_order_is_enforced():
    alg = golb200.GolB200(grid_dimensions=(64, 4))
    with pytest.raises(RuntimeError, match="before set_input"):
        alg.initialize_data_structures()
    with pytest.raises(RuntimeError, match="before initialize"):
        alg.run(1)
    with pytest.raises(RuntimeError, match="before initialize"):
        alg.finalize_data_structures()
    with pytest.raises(RuntimeError, match="shape"):
        alg.set_and_format_input_data(np.zeros((4, 32), np.uint8))
    alg.close()


def test_host_pack_round_trip_matches_reference_layout():
    """set_and_format_input_data then fetch_result (no device work) packs and
    unpacks exactly as GeneralBitGrid<..., FullyPackedRows> does."""
    g = oracle.random_ones_zeros(256, 37, 5)
    g[3, 7] = 200          # any nonzero byte is alive when packing
    alive = (g != 0).astype(np.uint8)
    alg = golb200.GolB200(grid_dimensions=(256, 37))
    alg.set_and_format_input_data(g)
    assert np.array_equal(alg.fetch_result(), alive)
    assert np.array_equal(alg.fetch_words(64), oracle.pack_rows(alive, 64))
    assert np.array_equal(alg.fetch_words(32), oracle.pack_rows(alive, 32))
    gi = alive.astype(np.int32)
    alg.set_and_format_input_data(gi)
    out = alg.fetch_result()
    assert out.dtype == np.int32 and np.array_equal(out, gi)
    alg.set_input_words(oracle.pack_rows(alive, 32), 32)
    assert np.array_equal(alg.fetch_result(np.empty((37, 256), np.uint8)), alive)
    alg.close()


def test_large_host_pack_threads():
    g = oracle.random_ones_zeros(4096, 1100, 3)
    alg = golb200.GolB200(grid_dimensions=(4096, 1100))
    alg.set_and_format_input_data(g)
    assert np.array_equal(alg.fetch_words(64), oracle.pack_rows(g, 64))
    assert np.array_equal(alg.fetch_result(), g)
    alg.close()


def test_stateless_entry_points_validate_arguments():
    L = golb200.lib()
    assert L.gol_rows_pass(None, None, 64, 64, 1, 0, None) == golb200.GOL_E_INVALID
    assert L.gol_rows_pass(1, 2, 40, 64, 1, 0, None) == golb200.GOL_E_INVALID
    assert L.gol_rows_pass(1, 2, 64, 64, 0, 0, None) == golb200.GOL_E_INVALID
    assert L.gol_rows_pass(1, 2, 64, 64, 17, 0, None) == golb200.GOL_E_INVALID
    assert L.gol_pack_cells_device(1, 2, 33, 1, None) == golb200.GOL_E_INVALID
    assert L.gol_rows_pass(16 + 8, 64, 64, 64, 1, 0, None) == golb200.GOL_E_INVALID   # misaligned
    assert L.gol_pack_cells_device(24, 64, 64, 1, None) == golb200.GOL_E_INVALID


def test_product_loader_matches_reference_generator(golden_cases):
    """gol_load_random_ones_zeros draws the reference's RandomOnesZerosDataLoader grid."""
    for case in golden_cases:
        if case["input"] != "random_ones_zeros" or case["x"] * case["y"] > 5_000_000:
            continue
        g = golb200.load_random_ones_zeros(case["x"], case["y"], case["seed"])
        assert f"{oracle.fnv1a64(g):016x}" == case["input_fnv1a64"], case["name"]


@pytest.mark.parametrize("x,y", [(32, 1), (2048, 600), (4096, 1024), (16384, 700), (96, 3)])
def test_host_pack_round_trip_without_a_device(x, y):
    """set_and_format_input_data packs on the host (worker threads for
    grids of more than 256 KiB of cells) and fetch_result unpacks: the
    packed words are the reference's row layout and the round trip returns
    the grid, all without a GPU."""
    g = oracle.random_ones_zeros(x, y, x + y)
    e = golb200.GolB200(grid_dimensions=(x, y), state_bits_count=32)
    try:
        e.set_and_format_input_data(g)
        assert np.array_equal(e.fetch_words(32), oracle.pack_rows(g, 32))
        assert np.array_equal(e.fetch_result(), g)
    finally:
        e.close()
