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


def test_resident_rounds_vs_oracle():
    """GOL_SERVE_RESIDENT: rounds with every running request's bands in
    shared memory; staggered arrivals, quanta that split a request's
    generations unevenly, odd word counts, one row; every result equals the
    oracle. The mode cannot change while requests are queued."""
    work = golb200.workload_uneven(9, 20, 64, 1536, 64, (0.1, 0.5), (1, 500))
    cells = [golb200.load_bernoulli(d["x"], d["y"], d["cell_seed"], d["density"]) for d in work]
    gens = [d["gens"] for d in work]
    cells += [oracle.random_ones_zeros(32 * 37, 200, 1), oracle.random_ones_zeros(64, 1, 2),
              oracle.random_ones_zeros(2048, 3, 3)]
    gens += [77, 33, 0]
    with golb200.GolServer(arena_bytes=256 << 20, quantum=48) as s:
        s.set_mode("resident")
        with pytest.raises(RuntimeError, match="resident round"):   # rows wider than 32768 cells
            s.submit(np.zeros((2, 32768 + 64), np.uint8), 5)
        ids = {}
        got = {}
        for i, (c, n) in enumerate(zip(cells, gens)):
            ids[s.submit(c, n)] = i
            if i == 0:
                with pytest.raises(RuntimeError, match="mode"):
                    s.set_mode("passes")
            if i % 3 == 2:
                s.step()
        while len(got) < len(ids):
            s.step()
            for rid in s.finished():
                got[ids[rid]] = s.fetch(rid)
    for i, (c, n) in enumerate(zip(cells, gens)):
        assert np.array_equal(got[i], oracle.life_cells(c, n)), (i, c.shape, n)


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


def settling_requests():
    """Inputs that settle: sparse soup patches in dead grids, a lone blinker
    (period 2, so a 4-generation pass leaves it as it was and its tiles look
    still), an all-dead grid and a block (a still life from the start), plus
    one dense soup."""
    reqs = []
    for i, (x, y) in enumerate([(1024, 512), (512, 768), (2048, 256)]):
        reqs.append((golb200.load_sparse_patches(x, y, 70 + i, 64, 0.05, 0.35), 600 + 131 * i))
    g = np.zeros((128, 256), np.uint8)
    g[60, 100:103] = 1
    reqs.append((g, 257))
    reqs.append((np.zeros((96, 640), np.uint8), 900))
    g = np.zeros((64, 128), np.uint8)
    g[10:12, 20:22] = 1
    reqs.append((g, 1000))
    reqs.append((oracle.random_ones_zeros(320, 200, 17), 450))
    return reqs


@pytest.mark.parametrize("tracking,policy", [("on", "fifo"), ("on", "srpt"), ("off", "srpt"),
                                             ("auto", "fifo")])
def test_tracking_and_policies_same_alone_and_in_the_mix(tracking, policy):
    reqs = settling_requests()
    mixed = {}
    with golb200.GolServer(arena_bytes=256 << 20, quantum=64) as s:
        s.set_tracking(tracking)
        s.set_policy(policy)
        ids = {}
        for i, (c, n) in enumerate(reqs):
            ids[s.submit(c, n)] = i
            if i % 3 == 2:
                s.step()
        while len(mixed) < len(ids):
            s.step()
            for rid in s.finished():
                mixed[ids[rid]] = s.fetch(rid)
        t = s.tiles()
    for i, (c, n) in enumerate(reqs):
        want = oracle.life_cells(c, n)
        assert np.array_equal(mixed[i], want), (i, tracking, policy)
        with golb200.GolServer(arena_bytes=64 << 20, quantum=64) as a:
            a.set_tracking(tracking)
            a.set_policy(policy)
            rid = a.submit(c, n)
            while True:
                a.step()
                if rid in a.finished():
                    assert np.array_equal(a.fetch(rid), want), (i, "alone", tracking, policy)
                    break
    if tracking == "on":
        # tiles of the dead grid, the block and the settled patches are
        # skipped; the dead grid and the block are found still in their first
        # 64-generation round and finish early
        assert t["skipped"] > 0
        assert t["early_finished"] >= 2
    if tracking == "off":
        assert t["skipped"] == 0 and t["early_finished"] == 0


def test_still_request_finishes_before_its_generations():
    """A still life asked for 10^6 generations finishes after its first
    round: the first pass changes nothing, so nothing later can."""
    g = np.zeros((64, 256), np.uint8)
    g[10:12, 20:22] = 1                      # block
    g[40:43, 50:53] = np.array([[0, 1, 0], [1, 0, 1], [0, 1, 0]], np.uint8)   # tub
    with golb200.GolServer(arena_bytes=64 << 20, quantum=64) as s:
        s.set_tracking("on")
        rid = s.submit(g, 10**6)
        rounds = 0
        while True:
            s.step()
            rounds += 1
            if rid in s.finished():
                break
            assert rounds < 200
        assert np.array_equal(s.fetch(rid), g)
        assert s.tiles()["early_finished"] == 1
