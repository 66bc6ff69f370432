"""Parity of the CUDA engine with the oracle, through the C ABI, on a GPU.

Bit-exact comparison (integer work: no tolerance) against
  * the golden fixtures made by the reference's own GoLCpuNaive,
  * the oracle restatement on seeded grids of many shapes and depths,
  * at the benchmark sizes (16384^2 / 64-bit, 8192^2 / 32-bit) against the
    multi-threaded bit-sliced oracle, and through size-independent
    properties (different depths and band heights agree; N=0 is identity;
    a time-budgeted run equals the oracle at the generations it reports).
"""
import numpy as np
import pytest

import golb200
import oracle
from golden_inputs import case_input, case_output

pytestmark = pytest.mark.gpu


def run_engine(cells, iters, k=0, word_bits=None, band=0, **kw):
    y, x = cells.shape
    if word_bits is None:
        word_bits = 64 if x % 64 == 0 else 32
    return golb200.run_generations(cells, iters, state_bits_count=word_bits, temporal_steps=k,
                                   thread_block_size=band, **kw)


@pytest.mark.parametrize("k", [0, 1, 2, 3, 4, 7, 8, 16])
def test_golden_fixtures(golden_cases, k):
    for case in golden_cases:
        g = case_input(case)
        out = run_engine(g, case["iters"], k=k)
        assert f"{oracle.fnv1a64(out):016x}" == case["output_fnv1a64"], (case["name"], k)
        stored = case_output(case)
        if stored is not None:
            assert np.array_equal(out, stored), (case["name"], k)


@pytest.mark.parametrize("band", [1, 2, 3, 5, 16, 1000])
def test_band_heights(golden_cases, band):
    for case in golden_cases:
        if case["x"] * case["y"] > 600_000:
            continue
        g = case_input(case)
        for k in (1, 4, 6):
            out = run_engine(g, case["iters"], k=k, band=band)
            assert f"{oracle.fnv1a64(out):016x}" == case["output_fnv1a64"], (case["name"], k, band)


SHAPES = [(32, 1), (32, 2), (32, 3), (64, 17), (96, 33), (160, 5), (256, 64), (1024, 40),
          (4064, 9), (4096, 24), (4128, 11), (8192, 8), (16384, 6), (32768, 4)]


@pytest.mark.parametrize("x,y", SHAPES)
def test_shapes_vs_oracle(x, y):
    g = oracle.random_ones_zeros(x, y, x + y)
    for iters in (1, 5, 23):
        ref = oracle.life_cells(g, iters)
        for k in (1, 2, 4, 8, 16):
            out = run_engine(g, iters, k=k)
            assert np.array_equal(out, ref), (x, y, iters, k)


@pytest.mark.parametrize("wpl,ks", [(1, (1, 5, 16)), (2, (1, 3, 8)), (4, (1, 2, 4))])
def test_forced_lane_widths(wpl, ks):
    """Every words-per-lane width at its depths, on narrow, one-CTA and
    x-sliced widths (32 * 1025 words at one word per lane needs 5 slices)."""
    for x, y in ((128, 40), (4096, 37), (32 * 1025, 7)):
        if (x // 32) % wpl:
            continue
        g = oracle.random_ones_zeros(x, y, x + wpl)
        for k in ks:
            n = 2 * k + 1
            assert np.array_equal(run_engine(g, n, k=k, word_bits=32, lane_words=wpl),
                                  oracle.life_cells(g, n)), (x, y, wpl, k)


@pytest.mark.parametrize("wpl", [1, 2, 4])
def test_one_generation_streaming_kernel(wpl):
    """k = 1 runs the streaming kernel (gol_rows_stream.cuh): any rows per
    thread (band), rows across several CTAs (lanes 0 and 31 of each warp read
    their outer words from memory), bands cut by the grid's last row."""
    for x, y in ((128, 1), (96, 7), (4096 + 128, 45), (32 * 1025, 5), (16384, 33)):
        if (x // 32) % wpl:
            continue
        g = oracle.random_ones_zeros(x, y, 3 * x + y + wpl)
        for band in (1, 2, 3, 4, 7, 64):
            for n in (1, 2, 5):
                out = run_engine(g, n, k=1, word_bits=32, band=band, lane_words=wpl)
                assert np.array_equal(out, oracle.life_cells(g, n)), (x, y, wpl, band, n)


def test_streaming_kernel_stateless_pass():
    """gol_rows_pass_ex with k = 1 (the streaming kernel) between two device
    grids, chained, against the oracle."""
    torch = pytest.importorskip("torch")
    s = torch.cuda.current_stream().cuda_stream
    for x, y, wpl in ((8192, 70, 0), (4096 + 64, 19, 2), (32 * 257, 11, 1)):
        g = oracle.random_ones_zeros(x, y, x ^ y)
        a = torch.from_numpy(oracle.pack_rows(g, 32).view(np.int32)).cuda()
        b = torch.empty_like(a)
        for _ in range(9):
            golb200.rows_pass(a.data_ptr(), b.data_ptr(), x, y, 1, 0, s, wpl)
            a, b = b, a
        torch.cuda.synchronize()
        got = a.cpu().numpy().view(np.uint32)
        assert np.array_equal(got, oracle.pack_rows(oracle.life_cells(g, 9), 32)), (x, y, wpl)


@pytest.mark.parametrize("x,y,gens,k", [(8192, 8192, 300, 0), (4096, 1000, 77, 8), (96, 40, 33, 4),
                                         (32 * 37, 300, 100, 5), (2048, 64, 0, 8), (1024, 500, 1, 8),
                                         (64, 148 * 9 + 5, 50, 3), (32 * 255, 700, 64, 16),
                                         (64, 5, 40, 8), (96, 1, 9, 4), (128, 12, 30, 8),
                                         (32768, 1000, 30, 8)])
def test_resident_run(x, y, gens, k):
    """GOL_ALG_RESIDENT: the whole run in one cooperative launch, each CTA's
    band in shared memory, halos exchanged every k generations; odd widths
    (one word per lane), bands of unequal height, generation counts that k
    does not divide, zero and one generation, grids of fewer rows than k
    (one band) and of one row, and 32768-cell rows (512 lanes, one row group
    doing both edges)."""
    g = oracle.random_ones_zeros(x, y, x + y + gens)
    out = run_engine(g, gens, k=k, word_bits=32, algorithm="resident")
    assert np.array_equal(out, oracle.life_cells(g, gens)), (x, y, gens, k)


def test_resident_run_reused_and_rejected_when_too_large():
    g = oracle.random_ones_zeros(2048, 2048, 5)
    ref = oracle.life_cells(g, 40)
    with golb200.GolB200(grid_dimensions=(2048, 2048), algorithm="resident") as alg:
        for _ in range(2):
            alg.set_and_format_input_data(g)
            alg.initialize_data_structures()
            alg.run(40)
            alg.finalize_data_structures()
            assert np.array_equal(alg.fetch_result(), ref)
    # 16384^2 is 32 MiB of cells: more than the SMs' shared memory holds
    with golb200.GolB200(grid_dimensions=(16384, 16384), algorithm="resident") as alg:
        alg.set_and_format_input_data(np.zeros((16384, 16384), np.uint8))
        with pytest.raises(RuntimeError, match="shared memory"):
            alg.initialize_data_structures()


def test_word_bits_32_and_64_agree():
    g = oracle.random_ones_zeros(512, 100, 77)
    a = run_engine(g, 37, word_bits=32)
    b = run_engine(g, 37, word_bits=64)
    assert np.array_equal(a, b)
    assert np.array_equal(a, oracle.life_cells(g, 37))


def test_zero_generations_is_identity():
    g = oracle.random_ones_zeros(128, 64, 3)
    assert np.array_equal(run_engine(g, 0), g)


@pytest.mark.parametrize("alg", ["auto", "resident"])
def test_int32_encoding(alg):
    g = oracle.random_ones_zeros(192, 50, 8).astype(np.int32)
    out = run_engine(g, 19, algorithm=alg)
    assert out.dtype == np.int32
    assert np.array_equal(out, oracle.life_cells(g.astype(np.uint8), 19).astype(np.int32))


def test_instance_reused_across_rounds():
    """ExperimentManager reuses one instance for warm-up and measured rounds
    (experiment_manager.hpp:322-394): every round redoes the phases."""
    g = oracle.random_ones_zeros(256, 128, 4)
    ref = oracle.life_cells(g, 50)
    with golb200.GolB200(grid_dimensions=(256, 128), temporal_steps=4) as alg:
        for _ in range(3):
            alg.set_and_format_input_data(g)
            alg.initialize_data_structures()
            alg.run(50)
            assert alg.actually_performed_iterations() == 50
            alg.finalize_data_structures()
            assert np.array_equal(alg.fetch_result(), ref)


def test_graph_chunked_long_run():
    """Long runs go through captured CUDA graphs of 16 passes each."""
    g = oracle.random_ones_zeros(1024, 256, 12)
    for k, n in ((1, 101), (4, 4 * 40 + 3), (8, 8 * 33)):
        assert np.array_equal(run_engine(g, n, k=k), oracle.life_cells(g, n)), (k, n)


@pytest.mark.parametrize("alg", ["auto", "resident"])
def test_runtime_budget_stops_early_and_reports_generations(alg):
    g = oracle.random_ones_zeros(64, 64, 1)
    with golb200.GolB200(grid_dimensions=(64, 64), temporal_steps=1 if alg == "auto" else 0,
                         max_runtime_seconds=1, algorithm=alg) as alg:
        alg.set_and_format_input_data(g)
        alg.initialize_data_structures()
        alg.run(10**12)
        alg.finalize_data_structures()
        done = alg.actually_performed_iterations()
        out = alg.fetch_result()
    assert 0 < done < 10**12
    assert np.array_equal(out, oracle.life_cells(g, done))


def test_wide_and_odd_width_grids_are_sliced():
    """Rows wider than one CTA are cut into x-slices with a one-lane halo."""
    for x, y in ((32 * 1025, 9), (65536, 5), (32 * 771, 13)):
        g = oracle.random_ones_zeros(x, y, 5)
        for k in (1, 4, 8, 16):
            iters = 2 * k + 1
            assert np.array_equal(run_engine(g, iters, k=k, word_bits=32),
                                  oracle.life_cells(g, iters)), (x, y, k)


def test_stateless_rows_pass_and_device_packing():
    torch = pytest.importorskip("torch")
    x, y = 2048, 300
    g = oracle.random_ones_zeros(x, y, 99)
    cells = torch.from_numpy(g).cuda()
    words = torch.empty((y, x // 32), dtype=torch.int32, device="cuda")
    other = torch.empty_like(words)
    s = torch.cuda.current_stream().cuda_stream
    golb200.pack_cells_device(cells.data_ptr(), words.data_ptr(), x, y, s)
    torch.cuda.synchronize()
    assert words.cpu().numpy().view(np.uint32).tobytes() == oracle.pack_rows(g, 32).tobytes()
    for k in (1, 3, 8):
        golb200.rows_pass(words.data_ptr(), other.data_ptr(), x, y, k, 0, s)
        words, other = other, words
    back = torch.empty_like(cells)
    golb200.unpack_cells_device(words.data_ptr(), back.data_ptr(), x, y, s)
    torch.cuda.synchronize()
    assert np.array_equal(back.cpu().numpy(), oracle.life_cells(g, 12))


@pytest.mark.slow
@pytest.mark.parametrize("x,word_bits,k", [(16384, 64, 4), (16384, 64, 8), (8192, 32, 4)])
def test_benchmark_sizes_vs_oracle(x, word_bits, k):
    """Full benchmark grid sizes, Bernoulli(0.5) seed 42, checked bit-exactly
    against the threaded bit-sliced oracle for 256 generations."""
    g = oracle.random_ones_zeros(x, x, 42)
    iters = 256
    ref = oracle.life_rows(oracle.pack_rows(g, word_bits), x, iters, word_bits)
    with golb200.GolB200(grid_dimensions=(x, x), state_bits_count=word_bits,
                         temporal_steps=k) as alg:
        alg.set_and_format_input_data(g)
        alg.initialize_data_structures()
        alg.run(iters)
        alg.finalize_data_structures()
        assert np.array_equal(alg.fetch_words(word_bits), ref)


@pytest.mark.slow
def test_depths_agree_at_full_size():
    """Size-independent property at 16384^2: every depth gives the same grid."""
    g = oracle.random_ones_zeros(16384, 16384, 42)
    outs = []
    for k in (1, 2, 3, 4, 5, 8):
        with golb200.GolB200(grid_dimensions=(16384, 16384), temporal_steps=k) as alg:
            alg.set_and_format_input_data(g)
            alg.initialize_data_structures()
            alg.run(120)
            alg.finalize_data_structures()
            outs.append(alg.fetch_words(64))
    for o in outs[1:]:
        assert np.array_equal(o, outs[0])
