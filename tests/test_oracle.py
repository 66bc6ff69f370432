"""Pins the oracle: the C restatement (oracle/gol_oracle.c) against the
golden fixtures produced by the reference's own CPU code, and against the
reference build itself (oracle/_ref) where that build exists. CPU only."""
import numpy as np
import pytest

import oracle
from golden_inputs import case_input, case_output


def test_generator_matches_fixture(golden_cases):
    for case in golden_cases:
        if case["input"] != "random_ones_zeros":
            continue
        g = case_input(case)
        assert f"{oracle.fnv1a64(g):016x}" == case["input_fnv1a64"], case["name"]


def test_restatement_matches_golden(golden_cases):
    for case in golden_cases:
        g = case_input(case)
        x = case["x"]
        if x % 32 == 0 and x * case["y"] * case["iters"] > 2_000_000:
            out = oracle.life_cells(g, case["iters"])
        else:
            out = oracle.life_naive(g, case["iters"])
        assert f"{oracle.fnv1a64(out):016x}" == case["output_fnv1a64"], case["name"]
        assert int(out.sum()) == case["output_alive"], case["name"]
        stored = case_output(case)
        if stored is not None:
            assert np.array_equal(out, stored), case["name"]


def test_naive_and_bitwise_restatements_agree():
    for (x, y, seed, iters) in [(64, 48, 3, 25), (96, 17, 4, 40), (32, 5, 5, 7), (128, 1, 6, 3)]:
        g = oracle.random_ones_zeros(x, y, seed)
        a = oracle.life_naive(g, iters)
        for wb in (32, 64):
            if x % wb:
                continue
            b = oracle.unpack_rows(oracle.life_rows(oracle.pack_rows(g, wb), x, iters, wb), x, wb)
            assert np.array_equal(a, b), (x, y, wb)


def test_pack_unpack_round_trip():
    g = oracle.random_ones_zeros(192, 7, 9)
    for wb in (32, 64):
        w = oracle.pack_rows(g, wb)
        assert np.array_equal(oracle.unpack_rows(w, 192, wb), g)
    # 32- and 64-bit rows are the same bytes (little-endian, LSB = smallest x)
    assert oracle.pack_rows(g, 32).tobytes() == oracle.pack_rows(g, 64).tobytes()


def test_threaded_rows_oracle_is_deterministic():
    g = oracle.random_ones_zeros(256, 300, 17)
    w = oracle.pack_rows(g, 64)
    a = oracle.life_rows(w, 256, 30, 64, threads=1)
    b = oracle.life_rows(w, 256, 30, 64, threads=7)
    assert np.array_equal(a, b)


needs_ref = pytest.mark.skipif(not oracle.ref_available(),
                               reason="reference build oracle/_ref not present")


@needs_ref
def test_restatement_vs_reference_build():
    for (x, y, seed, iters) in [(64, 64, 1, 10), (96, 40, 2, 33), (256, 33, 3, 50),
                                (32, 3, 4, 5), (320, 64, 5, 64)]:
        g = oracle.ref_random_ones_zeros(x, y, seed)
        assert np.array_equal(g, oracle.random_ones_zeros(x, y, seed))
        ref = oracle.ref_cpu_naive(g, iters)
        assert np.array_equal(ref, oracle.life_naive(g, iters))
        assert np.array_equal(ref, oracle.life_cells(g, iters))
        for wb in (32, 64):
            if x % wb:
                continue
            assert np.array_equal(ref, oracle.ref_cpu_bitwise_adder(g, iters, wb))
            assert np.array_equal(oracle.ref_pack_rows(g, wb), oracle.pack_rows(g, wb))
            w = oracle.pack_rows(g, wb)
            assert np.array_equal(oracle.ref_unpack_rows(w, x, wb), g)


@needs_ref
def test_reference_bitwise_matches_naive_at_c1():
    """The fast reference path (GoLCpuBitwise<AdderOps>) equals the oracle of
    record (GoLCpuNaive) on the 2048^2 / 128-generation benchmark case."""
    g = oracle.ref_random_ones_zeros(2048, 2048, 42)
    a = oracle.ref_cpu_bitwise_adder(g, 128, 64)
    b = oracle.life_cells(g, 128)
    assert np.array_equal(a, b)
    assert int(a.sum()) == 362221
