"""Runs one of the engine's kernels on a small, fixed workload, for
profiling (ncu) and quick timing.

    python stencil-optimalizations_b200/profile_pass.py --size 16384 --k 5 --passes 8
    python stencil-optimalizations_b200/profile_pass.py --mode local --size 4096 --gens 400
    python stencil-optimalizations_b200/profile_pass.py --mode batch --grids 32
    python stencil-optimalizations_b200/profile_pass.py --mode resident --size 8192 --gens 240 --k 0

dense (default): k-generation passes of the row-band kernel on the dense
benchmark input (Bernoulli(0.5), seed 42, from the reference's
RandomOnesZerosDataLoader); each pass reads one device buffer and writes the
other through gol_rows_pass; prints the mean per-launch time (CUDA events).
local: the change-tracking engine, --gens generations, on the sparse input
(1 % of 64x64 slots Bernoulli(0.35), seed 42), the blinker lattice of the
reference's always-changing loader (--input blinkers) or the dense benchmark
input (--input random); prints the run time and the fraction of tiles
computed. --dense-pct sets the active-tile share from which passes run dense.
batch: the first --grids grids of the uneven batched workload (seed 42), one
persistent launch after a warm-up launch (--batch-mode passes: gol_batch_run;
resident: gol_batch_run_resident); prints the launch time.
resident: the shared-memory-resident run (GOL_ALG_RESIDENT) on the dense
benchmark input, --gens generations in one cooperative launch after a
warm-up run, --k generations per epoch (0 = the engine's default); prints
the launch time.
"""
from __future__ import annotations

import argparse
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

import golb200  # noqa: E402


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--size", type=int, default=16384)
    ap.add_argument("--height", type=int, default=0)
    ap.add_argument("--k", type=int, default=5)
    ap.add_argument("--passes", type=int, default=8)
    ap.add_argument("--band", type=int, default=0)
    ap.add_argument("--wpl", type=int, default=0)
    ap.add_argument("--mode", choices=["dense", "local", "batch", "resident"], default="dense")
    ap.add_argument("--gens", type=int, default=400)
    ap.add_argument("--grids", type=int, default=32)
    ap.add_argument("--tile-rows", type=int, default=0, help="change-tracking tile height (0 = auto)")
    ap.add_argument("--input", choices=["sparse", "blinkers", "random"], default="sparse")
    ap.add_argument("--dense-pct", type=int, default=0)
    ap.add_argument("--batch-mode", choices=["passes", "resident"], default="passes")
    a = ap.parse_args()
    if a.mode == "local":
        return run_local(a)
    if a.mode == "batch":
        return run_batch(a)
    if a.mode == "resident":
        return run_resident(a)

    import torch
    x, y = a.size, a.height or a.size
    cells = torch.from_numpy(golb200.load_random_ones_zeros(x, y, 42)).cuda()
    words = torch.empty((y, x // 32), dtype=torch.int32, device="cuda")
    other = torch.empty_like(words)
    s = torch.cuda.current_stream().cuda_stream
    golb200.pack_cells_device(cells.data_ptr(), words.data_ptr(), x, y, s)
    evs = []
    for _ in range(a.passes):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        golb200.rows_pass(words.data_ptr(), other.data_ptr(), x, y, a.k, a.band, s, a.wpl)
        e1.record()
        evs.append((e0, e1))
        words, other = other, words
    torch.cuda.synchronize()
    ms = [e0.elapsed_time(e1) for e0, e1 in evs]
    warm = ms[min(2, len(ms) - 1):]
    mean = sum(warm) / len(warm)
    print(f"{x}x{y} k={a.k} wpl={a.wpl or 'auto'} band={a.band or 'auto'}: "
          f"{mean * 1e3:.1f} us per pass, "
          f"{x * y * a.k / (mean * 1e-3) / 1e12:.2f} Tcell-updates/s")


def run_local(a) -> None:
    import time
    x, y = a.size, a.height or a.size
    if a.input == "blinkers":
        g = golb200.load_always_changing(x, y)
    elif a.input == "random":
        g = golb200.load_random_ones_zeros(x, y, 42)
    else:
        g = golb200.load_sparse_patches(x, y, seed=42)
    with golb200.GolB200(grid_dimensions=(x, y), temporal_steps=a.k if a.k <= 16 else 8,
                         algorithm="local", tile_rows=a.tile_rows, dense_pct=a.dense_pct) as alg:
        alg.set_and_format_input_data(g)
        alg.initialize_data_structures()
        t0 = time.perf_counter()
        alg.run(a.gens)
        alg.sync()
        dt = time.perf_counter() - t0
        st = alg.local_stats()
        alg.finalize_data_structures()
    frac = st["computed_tiles"] / max(1, st["passes"] * st["tiles_per_pass"])
    print(f"local {x}x{y}, {a.gens} generations, k={a.k}: {dt * 1e3:.2f} ms (wall), "
          f"{frac:.3f} of tile-passes computed")


def run_resident(a) -> None:
    import torch
    x, y = a.size, a.height or a.size
    g = golb200.load_random_ones_zeros(x, y, 42)
    s = torch.cuda.Stream()
    with golb200.GolB200(grid_dimensions=(x, y), state_bits_count=32, temporal_steps=a.k,
                         algorithm="resident", stream=s.cuda_stream) as alg:
        alg.set_and_format_input_data(g)
        alg.initialize_data_structures()
        alg.run(min(a.gens, 16))   # warm-up (module load, attributes)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(s)
        alg.run(a.gens)
        e1.record(s)
        plan = alg.plan()
        alg.finalize_data_structures()
        ms = e0.elapsed_time(e1)
    print(f"resident {x}x{y}, {a.gens} generations, epochs of {plan['temporal_steps']}, "
          f"bands of {plan['band_rows']} rows, {plan['words_per_lane']} words per lane: {ms:.3f} ms, "
          f"{x * y * a.gens / (ms * 1e-3) / 1e12:.2f} Tcell-updates/s")


def run_batch(a) -> None:
    import torch
    work = golb200.workload_uneven(42, 512, 256, 4096, 64, (0.2, 0.5), (64, 4096))[:a.grids]
    s = torch.cuda.Stream()
    b = golb200.GolBatch(stream=s.cuda_stream)
    cu = 0
    for d in work:
        b.add(golb200.load_bernoulli(d["x"], d["y"], d["cell_seed"], d["density"]), d["gens"])
        cu += d["x"] * d["y"] * d["gens"]
    b.upload()
    run = b.run_resident if a.batch_mode == "resident" else b.run
    run()
    b.sync()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(s)
    run()
    e1.record(s)
    b.sync()
    ms = e0.elapsed_time(e1)
    units = (f"{b.resident_info()['bands']} bands" if a.batch_mode == "resident"
             else f"{b.info()['items']} items")
    print(f"batch of {len(work)} grids ({a.batch_mode}), {units}: {ms:.2f} ms, "
          f"{cu / (ms * 1e-3) / 1e12:.2f} Tcell-updates/s")
    b.close()


if __name__ == "__main__":
    main()
