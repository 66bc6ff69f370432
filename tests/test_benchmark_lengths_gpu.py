"""Bit-exact parity at the lengths the benchmark times, for every benchmark
configuration, against the threaded bit-sliced oracle (the reference's
GoLCpuBitwise<AdderOps> restated, itself pinned to the reference's own CPU
build by tests/test_oracle.py). The reference validates the final grid after
the full run the same way (experiment_manager.hpp:272-307).

  dense 16384^2, 64-bit rows, Bernoulli(0.5) seed 42, 4096 generations, k = 4 and 8
  dense 8192^2, 32-bit rows, 4096 generations
  sparse 16384^2 (1 % of 64x64 slots Bernoulli(0.35)), 20000 generations, change tracking
  the 512 uneven grids of the batched workload after one batched launch
  every 64th request of the serving stream
"""
import os
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

import golb200
import oracle

pytestmark = [pytest.mark.gpu, pytest.mark.slow, pytest.mark.timeout(900)]

GENS = 4096


def usable_cpus() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except (AttributeError, OSError):
        return os.cpu_count() or 1


def engine_words(cells, gens, word_bits, **kw):
    y, x = cells.shape
    with golb200.GolB200(grid_dimensions=(x, y), state_bits_count=word_bits, **kw) as alg:
        alg.set_and_format_input_data(cells)
        alg.initialize_data_structures()
        alg.run(gens)
        alg.finalize_data_structures()
        assert alg.actually_performed_iterations() == gens
        return alg.fetch_words(word_bits)


@pytest.mark.parametrize("size,word_bits,k,alg", [(16384, 64, 4, "auto"), (16384, 64, 8, "auto"),
                                                  (8192, 32, 0, "auto"), (8192, 32, 8, "auto"),
                                                  (8192, 32, 0, "resident")])
def test_dense_configs_at_full_length(size, word_bits, k, alg):
    cells = oracle.random_ones_zeros(size, size, 42)
    got = engine_words(cells, GENS, word_bits, temporal_steps=k, algorithm=alg)
    want = oracle.life_rows(oracle.pack_rows(cells, word_bits), size, GENS, word_bits)
    assert np.array_equal(got, want), (size, word_bits, k, alg)


def test_sparse_change_tracking_at_full_length():
    size, gens = 16384, 20000
    cells = golb200.load_sparse_patches(size, size, 42, 64, 0.01, 0.35)
    got = engine_words(cells, gens, 64, algorithm="local")
    want = oracle.life_rows(oracle.pack_rows(cells, 64), size, gens, 64)
    assert np.array_equal(got, want)


def oracle_grid(words: np.ndarray, x: int, gens: int) -> np.ndarray:
    """The oracle on one grid: one thread for small grids (many run at once)."""
    threads = 1 if words.size < (1 << 16) else 4
    return oracle.life_rows(words, x, gens, 64, threads=threads)


@pytest.mark.parametrize("mode", ["passes", "resident"])
def test_batched_workload_every_grid(mode):
    work = golb200.workload_uneven(42, 512, 256, 4096, 64, (0.2, 0.5), (64, 4096))
    inputs = []
    with golb200.GolBatch() as b:
        for d in work:
            cells = golb200.load_bernoulli(d["x"], d["y"], d["cell_seed"], d["density"])
            inputs.append(oracle.pack_rows(cells, 64))
            b.add(cells, d["gens"])
        b.upload()
        if mode == "resident":
            b.run_resident()
        else:
            b.run()
        b.sync()
        got = [oracle.pack_rows(b.fetch(i), 64) for i in range(len(work))]
    workers = max(1, (usable_cpus() or 1) // 2)
    with ThreadPoolExecutor(max_workers=workers) as pool:
        want = list(pool.map(lambda i: oracle_grid(inputs[i], work[i]["x"], work[i]["gens"]),
                             range(len(work))))
    bad = [i for i in range(len(work)) if not np.array_equal(got[i], want[i])]
    assert not bad, bad[:10]


def test_serving_stream_sampled_requests():
    """The benchmark's serving stream (Poisson 2000 req/s for 2 s, sides
    128..8192, 16..8192 generations, change tracking on long requests):
    every 64th request's result, fetched as cells, equals the oracle on the
    same input made on the host."""
    import serve
    r = serve.run_stream(rate=2000.0, seconds=2.0, seed=42, fetch="cells", check_every=64)
    assert r["requests"] > 3000
    samples = r["samples"]
    assert len(samples) > 40

    def one(item):
        d, out = item
        cells = golb200.load_hash_bernoulli(d["x"], d["y"], d["cell_seed"], d["density"])
        want = oracle.life_rows(oracle.pack_rows(cells, 32), d["x"], d["gens"], 32,
                                threads=1 if d["x"] * d["y"] < (1 << 21) else 8)
        return bool(np.array_equal(oracle.pack_rows(out, 32), want))
    workers = max(1, (usable_cpus() or 2) // 2)
    with ThreadPoolExecutor(max_workers=workers) as pool:
        ok = list(pool.map(one, samples))
    assert all(ok), [i for i, v in enumerate(ok) if not v][:10]
