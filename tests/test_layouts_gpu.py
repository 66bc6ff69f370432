"""Column and tile layouts and the pattern loaders on a GPU: the device
conversions between the engine's rows and the reference's BitColumns /
BitTile words against the oracle, and engine runs fed through the layout
input and the loaders, bit-exact against the oracle."""
import numpy as np
import pytest

import golb200
import oracle

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

CASES = [("columns", 16), ("columns", 32), ("columns", 64),
         ("tiles", 16), ("tiles", 32), ("tiles", 64)]


@pytest.mark.parametrize("layout,word_bits", CASES)
@pytest.mark.parametrize("x,y", [(32, 64), (96, 80), (1024, 192), (4096, 512), (160, 16)])
def test_device_conversions_match_oracle(layout, word_bits, x, y):
    xb, yb = golb200.layout_block(layout, word_bits)
    if y % yb:
        pytest.skip("grid is not a whole number of layout words")
    lay = golb200.LAYOUTS[layout]
    g = oracle.random_ones_zeros(x, y, x + 3 * y)
    want = oracle.pack_layout(g, lay, word_bits)
    rows = torch.from_numpy(oracle.pack_rows(g, 32).view(np.int32)).cuda()
    dt = {16: torch.int16, 32: torch.int32, 64: torch.int64}[word_bits]
    lw = torch.empty(want.shape, dtype=dt, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    golb200.rows_to_layout_device(rows.data_ptr(), lw.data_ptr(), x, y, layout, word_bits, s)
    back = torch.full_like(rows, -1)
    golb200.layout_to_rows_device(lw.data_ptr(), back.data_ptr(), x, y, layout, word_bits, s)
    torch.cuda.synchronize()
    assert lw.cpu().numpy().view(want.dtype).tobytes() == want.tobytes()
    assert torch.equal(back, rows)


@pytest.mark.parametrize("layout,word_bits,algorithm", [("tiles", 64, "auto"), ("columns", 32, "auto"),
                                                        ("tiles", 16, "auto"), ("tiles", 64, "resident"),
                                                        ("columns", 64, "resident")])
def test_engine_run_through_layout_io(layout, word_bits, algorithm):
    x, y, n = 512, 256, 77
    g = oracle.random_ones_zeros(x, y, 21)
    with golb200.GolB200(grid_dimensions=(x, y), state_bits_count=64, temporal_steps=4,
                         algorithm=algorithm) as alg:
        alg.set_input_layout(golb200.pack_layout(g, layout, word_bits), layout, word_bits)
        alg.initialize_data_structures()
        alg.run(n)
        alg.finalize_data_structures()
        out = alg.fetch_layout(layout, word_bits)
    ref = oracle.life_cells(g, n)
    assert np.array_equal(out, oracle.pack_layout(ref, golb200.LAYOUTS[layout], word_bits))


def test_device_tiled_pipeline_with_stateless_passes():
    """A device grid kept in 8x8 tiles: convert to rows, run passes, convert back."""
    x, y = 2048, 512
    g = oracle.random_ones_zeros(x, y, 8)
    tiles = torch.from_numpy(oracle.pack_layout(g, 2, 64).view(np.int64)).cuda()
    a = torch.empty((y, x // 32), dtype=torch.int32, device="cuda")
    b = torch.empty_like(a)
    s = torch.cuda.current_stream().cuda_stream
    golb200.layout_to_rows_device(tiles.data_ptr(), a.data_ptr(), x, y, "tiles", 64, s)
    for k in (4, 4, 3):
        golb200.rows_pass(a.data_ptr(), b.data_ptr(), x, y, k, 0, s)
        a, b = b, a
    golb200.rows_to_layout_device(a.data_ptr(), tiles.data_ptr(), x, y, "tiles", 64, s)
    torch.cuda.synchronize()
    got = tiles.cpu().numpy().view(np.uint64)
    assert np.array_equal(got, oracle.pack_layout(oracle.life_cells(g, 11), 2, 64))


def test_always_changing_and_zeros_inputs():
    for loader in (golb200.load_always_changing, golb200.load_zeros):
        g = loader(1024, 256)
        for k, n in ((1, 9), (4, 64), (8, 101)):
            out = golb200.run_generations(g, n, temporal_steps=k)
            assert np.array_equal(out, oracle.life_cells(g, n)), (loader.__name__, k, n)


def test_lexicon_input_on_dense_and_change_tracking_engines():
    from test_loaders_layouts import OWN_DICTIONARY
    lx = golb200.Lexicon(text=OWN_DICTIONARY)
    g = lx.load("glider[10,10]; toad[300,40]; glider[900,200]; block[500,100]; tub[64,64]",
                1024, 256)
    ref = oracle.life_cells(g, 333)
    assert np.array_equal(golb200.run_generations(g, 333, temporal_steps=4), ref)
    with golb200.GolB200(grid_dimensions=(1024, 256), temporal_steps=4, algorithm="local") as alg:
        alg.set_and_format_input_data(g)
        alg.initialize_data_structures()
        alg.run(333)
        alg.finalize_data_structures()
        assert np.array_equal(alg.fetch_result(), ref)
