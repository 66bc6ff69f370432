"""The continuous-batching server on a GPU: requests admitted while others
run give the same grids as when each runs alone (and as the oracle);
admission waits for arena memory; device-generated inputs equal their host
restatement."""
import numpy as np
import pytest

import golb200
import oracle

pytestmark = [pytest.mark.gpu, pytest.mark.timeout(600)]


def run_alone(cells, gens, quantum=64):
    with golb200.GolServer(arena_bytes=64 << 20, quantum=quantum) as s:
        rid = s.submit(cells, gens)
        while True:
            s.step()
            if rid in s.finished():
                return s.fetch(rid)


def test_results_same_alone_and_in_the_mix():
    work = golb200.workload_uneven(5, 24, 64, 1536, 64, (0.1, 0.5), (1, 700))
    cells = [golb200.load_bernoulli(d["x"], d["y"], d["cell_seed"], d["density"]) for d in work]
    results = {}
    with golb200.GolServer(arena_bytes=256 << 20, quantum=64) as s:
        ids = {}
        # staggered arrivals: a few requests join after rounds are already queued
        for i, (c, d) in enumerate(zip(cells, work)):
            ids[s.submit(c, d["gens"])] = i
            if i % 4 == 3:
                s.step()
        while len(results) < len(ids):
            s.step()
            for rid in s.finished():
                results[ids[rid]] = s.fetch(rid)
    for i, (c, d) in enumerate(zip(cells, work)):
        alone = run_alone(c, d["gens"])
        assert np.array_equal(results[i], alone), i
        if d["x"] * d["y"] * d["gens"] < 3e8:
            assert np.array_equal(alone, oracle.life_cells(c, d["gens"])), i


def test_admission_waits_for_memory():
    # room for about two 1024 x 1024 requests at a time (2 x 2 x 128 KiB)
    cells = [oracle.random_ones_zeros(1024, 1024, seed) for seed in range(6)]
    with golb200.GolServer(arena_bytes=600 << 10, quantum=32) as s:
        ids = {s.submit(c, 100 + 10 * i): i for i, c in enumerate(cells)}
        s.step()
        assert s.stats()["queued"] > 0
        got = {}
        while len(got) < len(ids):
            s.step()
            for rid in s.finished():
                got[ids[rid]] = s.fetch(rid)
    for i, c in enumerate(cells):
        assert np.array_equal(got[i], oracle.life_cells(c, 100 + 10 * i)), i


def test_device_generated_inputs_and_zero_generations():
    with golb200.GolServer(arena_bytes=64 << 20) as s:
        a = s.submit_random(640, 96, 0, seed=123, density=0.3)
        b = s.submit_random(640, 96, 77, seed=123, density=0.3)
        got = {}
        while len(got) < 2:
            s.step()
            for rid in s.finished():
                got[rid] = s.fetch(rid)
    host = golb200.load_hash_bernoulli(640, 96, 123, 0.3)
    assert abs(host.mean() - 0.3) < 0.02
    assert np.array_equal(got[a], host)
    assert np.array_equal(got[b], oracle.life_cells(host, 77))


def test_poisson_stream_small():
    import serve
    r = serve.run_stream(rate=200.0, seconds=0.5, seed=3, min_side=64, max_side=1024,
                         gens=(16, 512), quantum=64, arena_bytes=512 << 20)
    assert r["requests"] > 50
    assert r["latency_p99_ms"] >= r["latency_p50_ms"] > 0
