"""Batched uneven grids in one persistent launch, on a GPU: every grid's
result is bit-exact against the oracle (and against the one-launch-per-pass
baseline), for autotuned and forced plans, narrow (segmented warps) and
wide (x-sliced) grids, and uneven generation counts."""
import numpy as np
import pytest

import golb200
import oracle

pytestmark = [pytest.mark.gpu, pytest.mark.timeout(600)]


def small_workload(seed, n, lo=64, hi=1024, gens=(1, 300)):
    w = golb200.workload_uneven(seed, n, lo, hi, 32, (0.1, 0.5), gens)
    return [(golb200.load_bernoulli(d["x"], d["y"], d["cell_seed"], d["density"]), d["gens"])
            for d in w]


def test_batch_uneven_vs_oracle():
    work = small_workload(1, 40)
    with golb200.GolBatch() as b:
        ids = [b.add(c, n) for c, n in work]
        b.run()
        b.sync()
        for gid, (c, n) in zip(ids, work):
            assert np.array_equal(b.fetch(gid), oracle.life_cells(c, n)), (gid, c.shape, n)


@pytest.mark.parametrize("wpl,k,band", [(1, 1, 16), (1, 3, 24), (2, 2, 16), (2, 4, 64),
                                        (4, 4, 32), (4, 1, 48), (1, 4, 8)])
def test_batch_forced_plans(wpl, k, band):
    work = small_workload(2 + wpl * 10 + k, 12, lo=128, hi=768, gens=(1, 97))
    with golb200.GolBatch() as b:
        ids = []
        for c, n in work:                # rows padded to whole lanes where W % wpl != 0
            gid = b.add(c, n)
            b.set_plan(gid, wpl, k, band)
            ids.append((gid, c, n))
        b.run()
        b.sync()
        for gid, c, n in ids:
            assert np.array_equal(b.fetch(gid), oracle.life_cells(c, n)), (gid, c.shape, n)


def test_batch_resident_vs_oracle():
    """gol_batch_run_resident: every grid cut into bands held in shared memory
    for all its generations; uneven sizes (odd word counts, one row, fewer
    rows than an epoch), zero, one and few generations, twice in a row and
    after a pass-by-pass run of the same batch."""
    work = small_workload(11, 40, lo=32, hi=2048, gens=(1, 300))
    work += [(oracle.random_ones_zeros(32 * 37, 90, 3), 41),     # odd word count
             (oracle.random_ones_zeros(32, 1, 5), 9),            # one word, one row
             (oracle.random_ones_zeros(64, 3, 6), 0),            # zero generations
             (oracle.random_ones_zeros(128, 5, 7), 20),          # fewer rows than an epoch
             (oracle.random_ones_zeros(4096, 700, 8), 3),        # fewer generations than an epoch
             (oracle.random_ones_zeros(8192, 1000, 9), 64),      # many bands
             (oracle.random_ones_zeros(32768, 300, 10), 20)]     # 512 lanes, one row group
    with golb200.GolBatch() as b:
        ids = [b.add(c, n) for c, n in work]
        want = [oracle.life_cells(c, n) for c, n in work]
        for run in ("resident", "passes", "resident"):
            if run == "resident":
                b.run_resident()
            else:
                b.run()
            b.sync()
            for gid, w in zip(ids, want):
                assert np.array_equal(b.fetch(gid), w), (run, gid, work[gid][0].shape, work[gid][1])
        info = b.resident_info()
        assert info["bands"] > len(work) and info["ctas"] >= 148


def test_batch_wide_sliced_and_tiny_grids():
    work = [(oracle.random_ones_zeros(5120, 40, 3), 37),        # 160 words: x-sliced
            (oracle.random_ones_zeros(8192, 24, 4), 21),
            (oracle.random_ones_zeros(32, 1, 5), 9),             # one word, one row
            (oracle.random_ones_zeros(64, 3, 6), 0),             # zero generations
            (oracle.random_ones_zeros(4096, 70, 7), 64),
            (oracle.random_ones_zeros(96, 500, 8), 130)]
    with golb200.GolBatch() as b:
        ids = [b.add(c, n) for c, n in work]
        b.run()
        b.sync()
        for gid, (c, n) in zip(ids, work):
            assert np.array_equal(b.fetch(gid), oracle.life_cells(c, n)), (c.shape, n)


@pytest.mark.parametrize("wpl", [4, 2])
def test_batch_padded_rows(wpl):
    """Word counts that are not a multiple of the lane width: rows are padded
    on the device and the padding stays dead (narrow, single-lane-tail and
    x-sliced widths)."""
    shapes = [(96, 50, 33), (160, 17, 20), (32 * 7, 64, 41), (32 * 130, 30, 12),
              (32 * 131, 21, 9), (32 * 66, 40, 25), (32 * 127, 33, 17), (32 * 250, 12, 7)]
    work = [(oracle.random_ones_zeros(x, y, x + y), n) for x, y, n in shapes]
    with golb200.GolBatch() as b:
        ids = []
        for c, n in work:
            gid = b.add(c, n)
            b.set_plan(gid, wpl, 4, 16)
            ids.append(gid)
        b.run()
        b.sync()
        got = [b.fetch(g) for g in ids]
        b.run_plain(4)
        b.sync()
        plain = [b.fetch(g) for g in ids]
    for (c, n), g, p in zip(work, got, plain):
        ref = oracle.life_cells(c, n)
        assert np.array_equal(g, ref), (c.shape, n)
        assert np.array_equal(p, ref), (c.shape, n)


def test_batch_matches_plain_and_reruns():
    work = small_workload(9, 24, lo=256, hi=2048, gens=(10, 400))
    with golb200.GolBatch() as b:
        ids = [b.add(c, n) for c, n in work]
        b.run_plain(4)
        b.sync()
        plain = [b.fetch(g) for g in ids]
        for _ in range(2):                       # re-running restarts from the inputs
            b.run()
            b.sync()
            for g, p in zip(ids, plain):
                assert np.array_equal(b.fetch(g), p)
    for (c, n), p in list(zip(work, plain))[:6]:
        assert np.array_equal(p, oracle.life_cells(c, n))


def test_autotuner_uses_segments_for_narrow_grids():
    with golb200.GolBatch() as b:
        gid = b.add(np.zeros((2048, 256), np.uint8), 1000)
        p = b.plan(gid)
        assert p["segments"] > 1 and p["lane_words"] * (256 // 32 // p["lane_words"]) == 8
        gid2 = b.add(np.zeros((64, 8192), np.uint8), 10)
        assert b.plan(gid2)["segments"] == 1


def test_dependency_wait_gives_up_with_a_status():
    """The bounded dependency wait ends with GOL_E_TIMEOUT (no trap, no hang)
    when a dependency never completes, and the context stays usable."""
    import time
    t0 = time.perf_counter()
    assert golb200.probe_batch_timeout(1 << 12) == golb200.GOL_E_TIMEOUT
    assert time.perf_counter() - t0 < 30
    c = oracle.random_ones_zeros(256, 64, 1)
    with golb200.GolBatch() as b:
        gid = b.add(c, 17)
        b.run()
        b.sync()
        assert np.array_equal(b.fetch(gid), oracle.life_cells(c, 17))


# --- change tracking inside the batch -------------------------------------

GLIDER = np.array([[0, 1, 0], [0, 0, 1], [1, 1, 1]], dtype=np.uint8)


def settling_workload():
    """Grids that settle or stay sparse: dead grids with a few patches of
    Bernoulli(0.35) soup, a lone glider crossing item boundaries (also in an
    x-sliced grid), blinkers, an all-dead grid and one dense soup."""
    work = []
    for i, (x, y) in enumerate([(1024, 512), (2048, 256), (512, 1024), (4096, 128)]):
        work.append((golb200.load_sparse_patches(x, y, 50 + i, 64, 0.05, 0.35), 300 + 97 * i))
    g = np.zeros((256, 5120), np.uint8)             # 160 words: x-sliced
    g[10:13, 900:903] = GLIDER
    g[100:103, 2000:2003] = GLIDER
    work.append((g, 400))
    g = np.zeros((300, 96), np.uint8)               # narrow: segmented warps
    g[5:8, 40:43] = GLIDER
    work.append((g, 257))
    g = np.zeros((128, 256), np.uint8)
    g[60, 100:103] = 1                              # a blinker (period 2)
    work.append((g, 101))
    work.append((np.zeros((64, 640), np.uint8), 50))
    work.append((oracle.random_ones_zeros(768, 96, 9), 333))
    return work


@pytest.mark.parametrize("k", [1, 2, 3, 4])
def test_batch_tracking_settling_vs_oracle(k):
    work = settling_workload()
    with golb200.GolBatch() as b:
        ids = []
        for c, n in work:
            gid = b.add(c, n)
            b.set_plan(gid, 0, k, 0)
            b.set_tracking(gid, "on")
            ids.append(gid)
        b.run()
        b.sync()
        for gid, (c, n) in zip(ids, work):
            assert np.array_equal(b.fetch(gid), oracle.life_cells(c, n)), (gid, c.shape, n, k)
        t = b.tiles()
        assert t["skipped"] > 0 and t["computed"] > 0
        stats = [b.grid_stats(g) for g in ids]
        assert all(s["tracked"] for s in stats)
        # all dead: pass 0 computes every item and changes nothing, so the
        # grid is still from pass 1 and every later full pass is skipped; a
        # last pass shorter than k computes every item again
        assert stats[7]["still_pass"] == 1
        kk = b.plan(ids[7])["temporal_steps"]
        passes, short = -(-50 // kk), 50 % kk != 0
        nper = stats[7]["computed"] // (2 if short else 1)
        assert stats[7]["computed"] == nper * (2 if short else 1)
        assert stats[7]["skipped"] == nper * (passes - (2 if short else 1))
        # a run again from the same inputs gives the same grids
        b.run()
        b.sync()
        for gid, (c, n) in zip(ids, work):
            assert np.array_equal(b.fetch(gid), oracle.life_cells(c, n)), (gid, "rerun", k)


def test_batch_tracked_and_dense_grids_in_one_launch():
    work = settling_workload()
    with golb200.GolBatch() as b:
        ids = []
        for i, (c, n) in enumerate(work):
            gid = b.add(c, n)
            b.set_tracking(gid, "on" if i % 2 else "off")
            ids.append(gid)
        b.run()
        b.sync()
        for gid, (c, n) in zip(ids, work):
            assert np.array_equal(b.fetch(gid), oracle.life_cells(c, n)), (gid, c.shape, n)
            assert b.grid_stats(gid)["tracked"] == bool(gid % 2)
            if not gid % 2:
                assert b.grid_stats(gid)["skipped"] == 0


def test_batch_retune_keeps_results():
    """The autotuner's second look (per-grid tracking and tile rows from the
    first run's census) re-plans the batch; results stay bit-exact."""
    work = settling_workload()
    with golb200.GolBatch() as b:
        ids = [b.add(c, n) for c, n in work]
        b.run()
        b.sync()
        first = [b.fetch(g) for g in ids]
        b.retune()
        b.run()
        b.sync()
        for gid, (c, n) in zip(ids, work):
            got = b.fetch(gid)
            assert np.array_equal(got, first[gid])
            assert np.array_equal(got, oracle.life_cells(c, n)), (gid, c.shape, n)
        # the dense soup keeps computing most items; the dead grid is still at once
        assert b.grid_stats(7)["still_pass"] in (1, None)
