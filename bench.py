#!/usr/bin/env python
"""Benchmark of the B200 Game of Life engine (one JSON line on rank 0).

Workload (the dense bit-packed configuration): a 16384 x 16384 grid of
i.i.d. Bernoulli(0.5) cells from the reference's RandomOnesZerosDataLoader
(seed 42), packed into 64-bit rows, advanced 4096 generations per step,
cells outside the grid dead. The temporal depth k is swept over 1..16
first and the fastest k runs the headline.

  value  cell-updates/s with the grid resident in HBM (CUDA events on the
         engine's stream, L2 flushed between steps by a 256 MiB write);
  e2e    the same metric through the public C ABI with host buffers: per
         step set_input_u8 (host pack) -> init (H2D) -> run -> finalize
         (D2H) -> fetch_u8 (host unpack), wall clock;
  roofline  the pass kernel against measured HBM bandwidth (algorithmic
         bytes: the grid read once and written once per launch), plus the
         integer-pipe view against a live LOP3 peak probe;
  cpu_baseline  the reference's own CPU path (oracle/_ref, GoLCpuBitwise
         <char,64,AdderOps>) on a bounded sample on this host, one thread,
         its run phase timed (its pack/unpack phases outside).

Beside the headline (N = 1 only): the 8192^2 32-bit variant, timed in this
process, and, each in a fresh `bench.py --only …` process, `sparse` (change
tracking vs the dense engine on a settling 16384^2 input), `batched` (512
uneven grids in one persistent launch vs one launch per pass per grid) and
`serving` (a Poisson request stream; p50/p99 latency).

`--impl reference` times the reference's CPU implementation instead, on all
host threads (its run phase, row bands of the grid, one instance per
thread). Multi-GPU (torchrun): every rank advances its own replica (the
path has no exchange step); value = all ranks' cell-updates / the slowest
rank's time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "stencil-optimalizations_b200")
for _p in (PKG, os.path.join(ROOT, "oracle")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

METRIC = "Gcell-updates/s at 16384^2 bit-exact; batched vs plain on same GPU; p50/p99 lat"
UNIT = "Gcell-updates/s"
SIZE = 16384
GENS = 4096
SEED = 42
SWEEP_K = (1, 2, 3, 4, 5, 6, 8, 12, 16)
FLUSH_BYTES = 256 << 20
# sec. 8(d): the reference's full-adder formulation costs 33 word ops per
# 64-cell word (warp-exchange-full-adder-rows.cuh:50)
ALG_INT_OPS_PER_CELL = 33.0 / 64.0


def usable_cpus() -> int:
    """Host threads this process may run on (its CPU affinity), not the
    machine's total."""
    try:
        return len(os.sched_getaffinity(0))
    except (AttributeError, OSError):
        return os.cpu_count() or 1


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--size", type=int, default=SIZE)
    ap.add_argument("--gens", type=int, default=GENS)
    ap.add_argument("--k", type=int, default=0, help="temporal depth (0 = sweep)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-check", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the sparse, batched and serving measurements")
    ap.add_argument("--only", choices=["sparse", "published", "batched", "batched_settling",
                                       "serving", "hbm"],
                    help="measure just that configuration and print it")
    return ap.parse_args()


# ---------------------------------------------------------------------------
# distributed plumbing (one process per GPU, replicas)
# ---------------------------------------------------------------------------

class Dist:
    def __init__(self):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local_rank = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None

    def init(self, backend: str):
        if self.world > 1:
            import datetime

            import torch.distributed as dist
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
            self.pg = dist

    def barrier(self):
        if self.pg:
            self.pg.barrier()

    def max(self, v: float) -> float:
        if not self.pg:
            return v
        import torch
        dev = "cuda" if self.pg.get_backend() == "nccl" else "cpu"
        t = torch.tensor([v], dtype=torch.float64, device=dev)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


def replica_throughput(world: int, units_per_rank: float, slowest_seconds: float) -> float:
    """Whole-job rate of N independent replicas: every rank's units over the
    slowest rank's time (weak scaling)."""
    return world * units_per_rank / slowest_seconds


# ---------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------

class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines: list[str] = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def wait_first_sample(self, timeout_s: float = 5.0):
        t0 = time.time()
        while self.proc and not self.lines and time.time() - t0 < timeout_s:
            time.sleep(0.02)

    def reset(self):
        self.lines.clear()

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [v.strip() for v in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# reference CPU path (oracle/_ref when built here, else the oracle port)
# ---------------------------------------------------------------------------

class _PortEngine:
    """The oracle's restatement of GoLCpuBitwise<AdderOps> (used only when the
    reference build is absent), with the same run-only interface."""

    def __init__(self, cells):
        import oracle
        self.x = cells.shape[1]
        self.words = oracle.pack_rows(cells, 64)

    def run(self, gens):
        import oracle
        self.words = oracle.life_rows(self.words, self.x, gens, 64, threads=1)

    def finish(self):
        import oracle
        return oracle.unpack_rows(self.words, self.x, 64)


def reference_engine():
    """A factory for the reference's CPU path with its phases apart (the
    instance packs and initialises when made; run(gens) is the timed
    phase), and a description of it."""
    import oracle
    if oracle.ref_available():
        return (oracle.RefBitwise, "reference",
                "GoLCpuBitwise<char,64,AdderOps> built from the reference sources")
    return _PortEngine, "port", "oracle C restatement of GoLCpuBitwise<AdderOps> (reference build absent)"


def _timed(fn) -> float:
    t0 = time.perf_counter()
    fn()
    return time.perf_counter() - t0


def cpu_baseline(grid: np.ndarray, target_s: float = 10.0) -> dict:
    """The reference's CPU path, one core, on a bounded sample of the grid:
    its run phase timed alone (its pack/unpack phases are outside)."""
    make, kind, what = reference_engine()
    y, x = grid.shape
    eng = make(grid)
    per_gen = max(_timed(lambda: eng.run(2)), 1e-4) / 2.0
    gens = int(max(2, min(GENS, target_s / per_gen)))
    dt = _timed(lambda: eng.run(gens))
    eng.finish()
    return {"value": x * y * gens / dt / 1e9, "unit": UNIT, "cores": 1, "kind": kind,
            "sample": f"{x}x{y} seed {SEED}, {gens} generations ({dt:.1f} s of the run phase; the "
                      f"reference's pack/unpack phases outside), single thread ({what}); the "
                      "reference CPU path is single-threaded"}


def run_reference_arm(args, d: Dist) -> None:
    if d.rank != 0:
        return
    import oracle
    make, kind, what = reference_engine()
    cores = usable_cpus() or 1
    size = args.size
    grid = oracle.random_ones_zeros(size, size, SEED)
    bands = np.array_split(np.arange(size), cores)
    pieces = [np.ascontiguousarray(grid[b[0]:b[-1] + 1]) for b in bands if len(b)]

    def on_all(fn):
        ts = [threading.Thread(target=fn, args=(i,)) for i in range(len(pieces))]
        for t in ts:
            t.start()
        for t in ts:
            t.join()

    engines = [None] * len(pieces)

    def make_one(i):
        engines[i] = make(pieces[i])
    on_all(make_one)                       # pack + initialise, outside the timed steps

    def step(gens):
        return _timed(lambda: on_all(lambda i: engines[i].run(gens)))

    dt = max(step(2), 1e-4)
    gens = int(max(2, min(args.gens, 2 * 2.0 / dt)))   # ~2 s per step
    for _ in range(max(args.warmup, 0)):
        step(gens)
    times = [step(gens) for _ in range(args.steps)]
    on_all(lambda i: engines[i].finish())
    total = sum(times)
    value = size * size * gens * args.steps / total / 1e9
    sample = (f"{size}x{size} Bernoulli(0.5) seed {SEED} cut into {len(pieces)} row bands, one "
              f"{what} instance per host thread, {gens} generations per step, the run phase "
              f"timed (the reference's pack/unpack phases outside)")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": total / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
        "data": "synthetic",
        "config": {"workload": f"dense {size}x{size} Bernoulli(0.5) seed {SEED}, 64-bit rows, "
                               f"{gens} generations per step (bounded CPU sample)"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": len(pieces), "kind": kind,
                         "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------

def measured_peaks() -> dict:
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except OSError:
        return {}


def ncu_traffic(kernel: str, size: int = SIZE) -> float | None:
    """DRAM bytes per launch of a pass kernel from a committed ncu summary
    (profiles/ncu_traffic.json, keyed "kernel@size")."""
    try:
        with open(os.path.join(ROOT, "profiles", "ncu_traffic.json")) as f:
            d = json.load(f)
    except (OSError, ValueError):
        return None
    ent = d.get(f"{kernel}@{size}")
    return None if ent is None else float(ent["dram_bytes_per_launch"])


# ---------------------------------------------------------------------------
# the other configurations (reported beside the dense headline, N = 1)
# ---------------------------------------------------------------------------

def _events_ms(stream, fn, sync):
    import torch
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record(stream)
    fn()
    b.record(stream)
    sync()
    b.synchronize()
    return a.elapsed_time(b)


def _engine_rate(stream, device, cells, gens: int, **kw):
    """Times `gens` generations of one engine on `cells` after a warm-up run
    of the same length (which captures its graphs), restarting from the same
    input. Returns (Gcell-updates/s, change-tracking census or None, result
    as 64-bit row words)."""
    import golb200
    y, x = cells.shape
    e = golb200.GolB200(grid_dimensions=(x, y), device=device, stream=stream.cuda_stream, **kw)
    e.set_and_format_input_data(cells)
    e.initialize_data_structures()
    e.run(gens)
    e.sync()
    e.finalize_data_structures()
    e.set_and_format_input_data(cells)
    e.initialize_data_structures()
    ms = _events_ms(stream, lambda: e.run(gens), e.sync)
    st = e.local_stats() if kw.get("algorithm") == "local" else None
    e.finalize_data_structures()
    words = e.fetch_words(64)
    e.close()
    return x * y * gens / (ms * 1e-3) / 1e9, st, words


def _tile_fraction(st) -> float:
    return st["computed_tiles"] / max(1, st["passes"] * st["tiles_per_pass"])


def bench_sparse(stream, device) -> dict:
    """16384^2 all-dead grid, 1% of 64x64 slots Bernoulli(0.35), 20000
    generations: change-tracking tiles vs the dense engine, same input."""
    import golb200
    size, gens, seed = SIZE, 20000, SEED
    g = golb200.load_sparse_patches(size, size, seed, 64, 0.01, 0.35)
    out = {"workload": f"{size}x{size} dead grid, 1% of 64x64 slots Bernoulli(0.35) seed {seed}, "
                       f"{gens} generations", "unit": UNIT}
    out["value_local"], st, local = _engine_rate(stream, device, g, gens, algorithm="local",
                                                 temporal_steps=6)
    out["local_temporal_steps"] = 6
    out["computed_tile_fraction"] = _tile_fraction(st)
    out["value_dense"], _, dense = _engine_rate(stream, device, g, gens, temporal_steps=4)
    out["local_equals_dense"] = bool(np.array_equal(local, dense))
    import oracle
    want = oracle.life_rows(oracle.pack_rows(g, 64), size, gens, 64)
    out["bit_exact_vs_oracle_full_length"] = bool(np.array_equal(local, want))
    return out


def bench_published(stream, device) -> dict:
    """The reference's published change-tracking workloads at 16384^2: the
    all-dead grid (`zeros`, no work) and the blinker lattice
    (`always-changing`, every tile changes every generation), 4096
    generations, change tracking beside the dense engine. The blinker
    lattice has period 2, so at an even pass depth every tile is back to its
    input after each pass and change tracking skips it; an odd depth (5)
    keeps every tile changing and measures the full-work case. Then change
    tracking on the dense benchmark's own random grid."""
    import golb200
    size, gens = SIZE, 4096
    out = {"workload": f"{size}x{size}, {gens} generations: zeros and always-changing loaders",
           "unit": UNIT}
    zeros = golb200.load_zeros(size, size)
    out["zeros_value_local"], st, w = _engine_rate(stream, device, zeros, gens, algorithm="local",
                                                   temporal_steps=6)
    out["zeros_computed_tile_fraction"] = _tile_fraction(st)
    out["zeros_result_dead"] = not bool(w.any())
    blink = golb200.load_always_changing(size, size)
    ref = None
    for k in (5, 6):
        v, st, w = _engine_rate(stream, device, blink, gens, algorithm="local", temporal_steps=k)
        out[f"always_changing_value_local_k{k}"] = v
        out[f"always_changing_computed_tile_fraction_k{k}"] = _tile_fraction(st)
        ref = w if ref is None else ref
        out[f"always_changing_k{k}_equals_k5"] = bool(np.array_equal(w, ref))
    for k in (4, 5):
        out[f"always_changing_value_dense_k{k}"], _, w = _engine_rate(stream, device, blink, gens,
                                                                      temporal_steps=k)
        out[f"always_changing_dense_k{k}_equals_local"] = bool(np.array_equal(w, ref))
    # The dense benchmark's own input (Bernoulli(0.5) seed 42) with change
    # tracking: every tile active at first, about half of them by the end.
    soup = golb200.load_random_ones_zeros(size, size, SEED)
    out["random_value_local_k6"], st, w = _engine_rate(stream, device, soup, gens, algorithm="local",
                                                       temporal_steps=6)
    out["random_computed_tile_fraction_k6"] = _tile_fraction(st)
    _, _, wd = _engine_rate(stream, device, soup, gens, temporal_steps=4)
    out["random_local_equals_dense"] = bool(np.array_equal(w, wd))
    return out


HBM_SIZE = 32768
HBM_SWEEP_K = (1, 2, 3, 4, 5, 6, 8)


def bench_hbm(stream, device) -> dict:
    """The dense engine on a grid larger than L2: 32768^2 Bernoulli(0.5) seed
    42 (128 MiB per buffer; the two buffers are 268 MB against the 126 MB
    L2), depth swept 1..8. Per depth: cell-updates/s, the algorithmic HBM
    rate (grid read and written once per pass) against the measured HBM
    peak, and the integer view against the live LOP3 probe. Depths agree
    with each other and k = 1 with the oracle."""
    import torch

    import golb200
    import oracle
    size, gens = HBM_SIZE, 384
    cells = golb200.load_random_ones_zeros(size, size, SEED)
    peaks = measured_peaks()
    hbm_peak = peaks.get("hbm_gbs") or 6650.0
    int_peak = golb200.probe_int_peak(stream.cuda_stream)
    grid_bytes = size * size // 8
    rows = {}
    results = {}
    for k in HBM_SWEEP_K:
        e = golb200.GolB200(grid_dimensions=(size, size), state_bits_count=64, temporal_steps=k,
                            device=device, stream=stream.cuda_stream)
        e.set_and_format_input_data(cells)
        e.initialize_data_structures()
        e.run(gens)           # warm-up (graph capture)
        e.sync()
        ms = min(_events_ms(stream, lambda: e.run(gens), e.sync) for _ in range(3))
        passes = gens // k + (1 if gens % k else 0)
        pass_ms = ms / passes
        plan = e.plan()
        e.close()
        cu = size * size * gens / (ms * 1e-3)
        gbs = 2 * grid_bytes / (pass_ms * 1e-3) / 1e9
        rows[str(k)] = {"value": cu / 1e9, "pass_us": pass_ms * 1e3, "hbm_gbs": gbs,
                        "hbm_frac": gbs / hbm_peak,
                        "int_frac": cu * ALG_INT_OPS_PER_CELL / int_peak,
                        "words_per_lane": plan["words_per_lane"], "band_rows": plan["band_rows"],
                        "kernel": "rows_stream_kernel" if k == 1 else "rows_temporal_kernel"}
    # parity: every depth gives the k = 1 grid after 96 generations, and
    # k = 1 equals the oracle
    chk = 96
    for k in HBM_SWEEP_K:
        e = golb200.GolB200(grid_dimensions=(size, size), state_bits_count=64, temporal_steps=k,
                            device=device, stream=stream.cuda_stream)
        e.set_and_format_input_data(cells)
        e.initialize_data_structures()
        e.run(chk)
        e.finalize_data_structures()
        results[k] = e.fetch_words(64)
        e.close()
    want = oracle.life_rows(oracle.pack_rows(cells, 64), size, chk, 64)
    del cells
    torch.cuda.synchronize()
    return {"workload": f"dense {size}x{size} Bernoulli(0.5) seed {SEED}, 64-bit rows, {gens} "
                        f"generations per timing (min of 3)", "unit": UNIT,
            "hbm_peak_gbs": hbm_peak, "int_peak_lane_ops": int_peak, "per_k": rows,
            "k1_bit_exact_vs_oracle_96_gens": bool(np.array_equal(results[1], want)),
            "all_depths_equal_96_gens": all(np.array_equal(results[k], results[1]) for k in results)}


def _plain_graphs_multistream(work, inputs, device, nstreams: int = 8) -> tuple:
    """The fair plain baseline: every grid through the one-grid engine
    (gol_run: its own plan, CUDA graphs of 16 passes), grids dealt round-robin
    to `nstreams` streams so independent grids overlap on the device. Returns
    (ms of the timed run, the engines' results as 64-bit row words)."""
    import torch

    import golb200
    streams = [torch.cuda.Stream(device=device) for _ in range(nstreams)]
    master = torch.cuda.Stream(device=device)
    engines = []
    for i, (d, w) in enumerate(zip(work, inputs)):
        e = golb200.GolB200(grid_dimensions=(d["x"], d["y"]), state_bits_count=64, temporal_steps=4,
                            device=device, stream=streams[i % nstreams].cuda_stream)
        engines.append(e)

    def load():
        for e, w in zip(engines, inputs):
            e.set_input_words(w, 64)
            e.initialize_data_structures()
        torch.cuda.synchronize()

    def run_all() -> float:
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(master)
        for st in streams:
            st.wait_event(a)
        for e, d in zip(engines, work):
            e.run(d["gens"])
        for st in streams:
            ev = torch.cuda.Event()
            ev.record(st)
            master.wait_event(ev)
        b.record(master)
        b.synchronize()
        return a.elapsed_time(b)

    load()
    run_all()                                   # warm-up: captures every engine's graphs
    for e in engines:
        e.finalize_data_structures()
    load()
    ms = run_all()
    out = []
    for e in engines:
        e.finalize_data_structures()
        out.append(e.fetch_words(64))
        e.close()
    return ms, out


def bench_batched(stream, device, n: int = 512, seed: int = SEED) -> dict:
    """512 grids, sides log-uniform [256, 4096] (multiples of 64), density
    U[0.2, 0.5], generations log-uniform [64, 4096]: one persistent launch
    (both batched modes: dependent pass items, and bands resident in shared
    memory; value_batched is the faster), against (1) one launch per pass per
    grid on one stream and (2) every grid through the one-grid engine's
    graph-chunked gol_run over 8 streams; every grid's result of both batched
    modes checked against the oracle."""
    import concurrent.futures as cf

    import golb200
    import oracle
    work = golb200.workload_uneven(seed, n, 256, 4096, 64, (0.2, 0.5), (64, 4096))
    b = golb200.GolBatch(device=device, stream=stream.cuda_stream)
    inputs = []
    with cf.ThreadPoolExecutor(max_workers=min(32, usable_cpus() or 1)) as pool:
        for i in range(0, n, 32):
            chunk = work[i:i + 32]
            grids = list(pool.map(lambda d: golb200.load_bernoulli(d["x"], d["y"], d["cell_seed"],
                                                                   d["density"]), chunk))
            for d, c in zip(chunk, grids):
                b.add(c, d["gens"])
                inputs.append(oracle.pack_rows(c, 64))
    b.upload()
    info = b.info()
    b.run()
    b.sync()                                        # first run: the census the autotuner reads
    first_tiles = b.tiles()
    b.retune()                                      # per-grid tracking / tile choice
    b.run()
    b.sync()                                        # warm-up (and graph capture)
    batched = [_events_ms(stream, b.run, b.sync) for _ in range(3)]
    tiles = b.tiles()
    tracked = sum(1 for i in range(n) if b.grid_stats(i)["tracked"])
    results = [oracle.pack_rows(b.fetch(i), 64) for i in range(n)]
    # the resident batch: every grid's bands in shared memory for all their
    # generations (first run plans the bands)
    b.run_resident()
    b.sync()
    resident = [_events_ms(stream, b.run_resident, b.sync) for _ in range(3)]
    rinfo = b.resident_info()
    results_res = [oracle.pack_rows(b.fetch(i), 64) for i in range(n)]
    b.run_plain(4)
    b.sync()
    plain = [_events_ms(stream, lambda: b.run_plain(4), b.sync) for _ in range(2)]
    same = all(np.array_equal(oracle.pack_rows(b.fetch(i), 64), results[i]) for i in range(0, n, 64))
    b.close()
    ms_graphs, graph_results = _plain_graphs_multistream(work, inputs, device)
    graphs_same = all(np.array_equal(graph_results[i], results[i]) for i in range(n))

    def check(i):
        d = work[i]
        want = oracle.life_rows(inputs[i], d["x"], d["gens"], 64,
                                threads=1 if inputs[i].size < (1 << 16) else 4)
        return bool(np.array_equal(results[i], want)), bool(np.array_equal(results_res[i], want))
    with cf.ThreadPoolExecutor(max_workers=max(1, (usable_cpus() or 2) // 2)) as pool:
        ok = list(pool.map(check, range(n)))
    cu = info["cell_updates"]
    v_passes = cu / (min(batched) * 1e-3) / 1e9
    v_res = cu / (min(resident) * 1e-3) / 1e9
    vb = max(v_passes, v_res)
    vp = cu / (min(plain) * 1e-3) / 1e9
    vg = cu / (ms_graphs * 1e-3) / 1e9
    return {"workload": f"{n} grids, sides log-uniform [256, 4096] x64, density U[0.2, 0.5], "
                        f"generations log-uniform [64, 4096], seed {seed}",
            "cell_updates": cu, "work_items": info["items"], "unit": UNIT,
            "value_batched": vb, "ms_batched": min(min(batched), min(resident)),
            "batched_mode": "resident" if v_res >= v_passes else "passes",
            "value_batched_passes": v_passes, "ms_batched_passes": min(batched),
            "value_batched_resident": v_res, "ms_batched_resident": min(resident),
            "resident_plan": rinfo,
            "modes": {"passes": "gol_batch_run: one persistent launch of dependent k-generation "
                                "work items (bands of passes), change tracking autotuned",
                      "resident": "gol_batch_run_resident: every grid cut into bands, each band "
                                  "in one CTA's shared memory for all its generations, halo "
                                  "rows exchanged every 8 generations"},
            "autotuner": {"first_run_items": first_tiles, "grids_tracked_after_retune": tracked,
                          "timed_run_items": tiles},
            "value_plain_per_grid": vp, "ms_plain": min(plain), "speedup": vb / vp,
            "value_plain_graphs_multistream": vg, "ms_plain_graphs_multistream": ms_graphs,
            "speedup_vs_graphs_multistream": vb / vg,
            "plain_graphs_multistream": "each grid through gol_run (its own plan, CUDA graphs "
                                        "of 16 passes), 8 streams, one engine per grid",
            "batched_equals_plain_on_sample": same,
            "batched_equals_graphs_multistream_all": graphs_same,
            "batched_all_equal_oracle": all(o[0] and o[1] for o in ok),
            "batched_passes_all_equal_oracle": all(o[0] for o in ok),
            "batched_resident_all_equal_oracle": all(o[1] for o in ok),
            "grids_checked_vs_oracle": len(ok)}


def _check_serving_samples(samples) -> dict:
    """Every sampled request's result against the oracle (its input remade
    on the host with the same hash as the device generator)."""
    import concurrent.futures as cf

    import golb200
    import oracle

    def one(item):
        d, out = item
        cells = golb200.load_hash_bernoulli(d["x"], d["y"], d["cell_seed"], d["density"])
        want = oracle.life_rows(oracle.pack_rows(cells, 32), d["x"], d["gens"], 32,
                                threads=1 if d["x"] * d["y"] < (1 << 21) else 8)
        got = out if out.dtype == np.uint32 else oracle.pack_rows(out, 32)
        return bool(np.array_equal(got.view(np.uint32), want))
    with cf.ThreadPoolExecutor(max_workers=max(1, (usable_cpus() or 2) // 2)) as pool:
        ok = list(pool.map(one, samples))
    return {"sampled": len(ok), "all_equal_oracle": all(ok)}


def bench_batched_settling(stream, device, n: int = 512, seed: int = SEED) -> dict:
    """The batched workload's grids (same sizes and generation counts) with
    settling inputs: dead grids with patches of Bernoulli(0.35) soup in 5 %
    of their 64 x 64 slots (at least one). Batched with change tracking
    (autotuned: a first run, gol_batch_retune, then timed runs) against the
    same batch with every grid tracked and with none, and the resident batch
    (every generation computed, bands in shared memory); every grid of every
    run checked against the oracle."""
    import concurrent.futures as cf

    import golb200
    import oracle
    work = golb200.workload_uneven(seed, n, 256, 4096, 64, (0.2, 0.5), (64, 4096))

    def cells_of(d):
        slots = (d["x"] // 64) * (d["y"] // 64)
        return golb200.load_sparse_patches(d["x"], d["y"], d["cell_seed"], 64,
                                           max(0.05, 1.0 / slots + 1e-9), 0.35)
    with cf.ThreadPoolExecutor(max_workers=min(32, usable_cpus() or 1)) as pool:
        inputs = list(pool.map(lambda d: oracle.pack_rows(cells_of(d), 64), work))
    out = {"workload": f"{n} grids as the batched workload (seed {seed}), dead with Bernoulli(0.35) "
                       "patches in 5 % of 64x64 slots (at least one)", "unit": UNIT}
    results = {}
    # on: every grid tracked; off: none; auto: the autotuner (a first run,
    # gol_batch_retune, then the timed runs)
    for mode in ("on", "off", "auto", "resident"):
        b = golb200.GolBatch(device=device, stream=stream.cuda_stream)
        for d, w in zip(work, inputs):
            gid = b.add(oracle.unpack_rows(w, d["x"], 64), d["gens"])
            b.set_tracking(gid, "off" if mode == "resident" else mode)
        b.upload()
        info = b.info()
        if mode == "resident":   # bands in shared memory, every generation computed
            b.run_resident()
            b.sync()
            ms = min(_events_ms(stream, b.run_resident, b.sync) for _ in range(3))
            out["value_resident"] = info["cell_updates"] / (ms * 1e-3) / 1e9
            out["ms_resident"] = ms
            results[mode] = [oracle.pack_rows(b.fetch(i), 64) for i in range(n)]
            b.close()
            continue
        b.run()
        b.sync()
        if mode == "auto":
            b.retune()
            b.run()
            b.sync()
        ms = min(_events_ms(stream, b.run, b.sync) for _ in range(3))
        out[f"value_tracking_{mode}"] = info["cell_updates"] / (ms * 1e-3) / 1e9
        out[f"ms_tracking_{mode}"] = ms
        out[f"items_tracking_{mode}"] = b.tiles()
        stats = [b.grid_stats(i) for i in range(n)]
        out[f"grids_tracked_{mode}"] = sum(1 for st in stats if st["tracked"])
        if mode == "on":
            out["grids_still_before_their_end"] = sum(1 for st in stats if st["still_pass"] is not None)
        results[mode] = [oracle.pack_rows(b.fetch(i), 64) for i in range(n)]
        b.close()
    out["speedup_tracking_on"] = out["value_tracking_on"] / out["value_tracking_off"]
    out["speedup_autotuned"] = out["value_tracking_auto"] / out["value_tracking_off"]
    out["cell_updates"] = info["cell_updates"]

    def check(i):
        d = work[i]
        want = oracle.life_rows(inputs[i], d["x"], d["gens"], 64,
                                threads=1 if inputs[i].size < (1 << 16) else 4)
        return all(bool(np.array_equal(results[m][i], want)) for m in results)
    with cf.ThreadPoolExecutor(max_workers=max(1, (usable_cpus() or 2) // 2)) as pool:
        ok = list(pool.map(check, range(n)))
    out["all_equal_oracle"] = all(ok)
    return out


def bench_serving(device) -> dict:
    """Poisson stream, mean 2000 requests/s, sides log-uniform [128, 8192]
    (multiples of 64), density U[0.1, 0.5], generations log-uniform
    [16, 8192]. Arrival-order (FIFO) and least-work-first (SRPT) scheduling
    on the 2-s stream with inputs generated on the device and packed results
    copied back, then both with host I/O (host cells, made before the stream
    starts, in through gol_serve_submit; cells out through gol_serve_fetch)
    on the stream's first 0.5 s. Change tracking is on for long requests
    (auto). The FIFO runs again with resident rounds (every request's bands
    in shared memory, no change tracking). Every 64th request of the FIFO
    runs is checked against the oracle."""
    import serve
    out = {"workload": "Poisson arrivals, mean 2000 req/s for 2 s, sides log-uniform [128, 8192] "
                       "x64, density U[0.1, 0.5], generations log-uniform [16, 8192], seed 42",
           "unit_throughput": "cell-updates/s"}
    runs = [("fifo", False, "passes"), ("fifo", True, "passes"), ("srpt", False, "passes"),
            ("srpt", True, "passes"), ("fifo", False, "resident"), ("fifo", True, "resident")]
    for policy, host_io, mode in runs:
        r = serve.run_stream(rate=2000.0, seconds=0.5 if host_io else 2.0, seed=SEED,
                             device=device, policy=policy, host_io=host_io, mode=mode,
                             check_every=64 if policy == "fifo" else 0)
        samples = r.pop("samples")
        if samples:
            r["check"] = _check_serving_samples(samples)
        r["p99_over_p50"] = r["latency_p99_ms"] / max(r["latency_p50_ms"], 1e-9)
        out[f"{policy}{'_host_io' if host_io else ''}{'_resident' if mode == 'resident' else ''}"] = r
    # the headline figures: the FIFO run with device-side inputs, in the
    # round mode with the lower p50
    best = min(("fifo", "fifo_resident"), key=lambda k: out[k]["latency_p50_ms"])
    out["headline_run"] = best
    for k in ("requests", "cell_updates_per_s", "latency_p50_ms", "latency_p99_ms"):
        out[k] = out[best][k]
    out["serving_sample_equal_oracle"] = all(
        out[k].get("check", {}).get("all_equal_oracle", True)
        for k in ("fifo", "fifo_host_io", "fifo_resident", "fifo_host_io_resident"))
    return out


def run_extra(name: str) -> dict:
    """Runs one extra workload (`bench.py --only name`) in a fresh process:
    its own CUDA context and allocator state, so what ran before it here
    (the dense steps, the other extras) cannot shape its numbers; the
    serving loop's latencies in particular depend on host scheduling."""
    try:
        r = subprocess.run([sys.executable, os.path.abspath(__file__), "--only", name],
                           capture_output=True, text=True, timeout=1200)
    except subprocess.TimeoutExpired:
        return {"error": "timed out"}
    for ln in reversed(r.stdout.splitlines()):
        if ln.startswith("{"):
            return json.loads(ln)[name]
    return {"error": f"exit {r.returncode}: {r.stderr.strip()[-300:]}"}


def run_ours(args, d: Dist) -> None:
    import torch

    import golb200
    torch.cuda.set_device(d.local_rank)
    dev = torch.device("cuda", d.local_rank)
    stream = torch.cuda.Stream(device=dev)
    size, gens = args.size, args.gens
    cells = golb200.load_random_ones_zeros(size, size, SEED)
    cell_updates = size * size * gens
    flush = torch.empty(FLUSH_BYTES // 4, dtype=torch.int32, device=dev)

    def make_engine(k):
        e = golb200.GolB200(grid_dimensions=(size, size), state_bits_count=64, temporal_steps=k,
                            device=d.local_rank, stream=stream.cuda_stream)
        e.set_and_format_input_data(cells)
        e.initialize_data_structures()
        return e

    def timed_run(e, n):
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        e.run(n)
        b.record(stream)
        b.synchronize()
        return a.elapsed_time(b)

    # -- depth sweep (short runs) -------------------------------------------
    sweep = {}
    ks = [args.k] if args.k else list(SWEEP_K)
    sweep_gens = min(gens, 1024)
    for k in ks:
        e = make_engine(k)
        timed_run(e, min(sweep_gens, 256))
        ms = timed_run(e, sweep_gens)
        sweep[k] = size * size * sweep_gens / (ms * 1e-3) / 1e9
        e.close()
    best_k = max(sweep, key=sweep.get)
    if d.world > 1:   # every rank uses rank 0's choice so all run the same work
        import torch.distributed as dist
        t = torch.tensor([best_k], device=dev)
        dist.broadcast(t, 0)
        best_k = int(t.item())

    # -- bit-exactness of the benchmark configuration at its full length ------
    bit_exact = None
    if not args.no_check and d.rank == 0:
        import oracle
        e = make_engine(best_k)
        e.run(gens)
        e.finalize_data_structures()
        got = e.fetch_words(64)
        e.close()
        want = oracle.life_rows(oracle.pack_rows(cells, 64), size, gens, 64)
        bit_exact = bool(np.array_equal(got, want))

    # -- headline: device-resident timed steps -------------------------------
    e = make_engine(best_k)
    plan = e.plan()
    clocks = ClockSampler(d.local_rank)
    clocks.start()
    for _ in range(args.warmup):
        e.run(gens)
        flush.zero_()
    torch.cuda.synchronize()
    clocks.wait_first_sample()
    clocks.reset()
    d.barrier()
    torch.cuda.synchronize()
    step_ms = []
    for _ in range(args.steps):
        step_ms.append(timed_run(e, gens))
        with torch.cuda.stream(stream):
            flush.zero_()          # outside the events: between timed steps
    torch.cuda.synchronize()
    d.barrier()
    torch.cuda.synchronize()
    clk = clocks.stop()
    total_ms = d.max(sum(step_ms))
    value = replica_throughput(d.world, cell_updates * args.steps, total_ms * 1e-3) / 1e9

    # -- dominant kernel: its in-step duration (one pass of k generations) ---
    # Every launch of the timed steps is this kernel (the step is one graph of
    # passes), so the per-pass time is the step's device time over its passes.
    passes = gens // best_k + (1 if gens % best_k else 0)
    launch_ms = total_ms / args.steps / passes
    grid_bytes = size * size // 8
    alg_bytes = 2 * grid_bytes                       # read once + write once per pass
    achieved_gbs = alg_bytes / (launch_ms * 1e-3) / 1e9
    peaks = measured_peaks()
    hbm_peak = peaks.get("hbm_gbs")
    peak_src = "measured" if hbm_peak else "fallback"
    hbm_peak = hbm_peak or 6650.0
    int_peak = golb200.probe_int_peak(stream.cuda_stream)
    pass_cell_updates = size * size * best_k
    int_achieved = pass_cell_updates * ALG_INT_OPS_PER_CELL / (launch_ms * 1e-3)
    e.close()
    kernel = (f"rows_stream_kernel<{plan['words_per_lane']}>" if best_k == 1 else
              f"rows_temporal_kernel<{plan['words_per_lane']},{best_k}>")
    hbm_view = {"bound": "hbm", "achieved": achieved_gbs, "peak": hbm_peak, "unit": "GB/s",
                "frac": achieved_gbs / hbm_peak, "peak_source": peak_src,
                "algorithmic_bytes_per_launch": alg_bytes,
                "note": "bytes = grid read once + written once per k-generation pass "
                        "(0.25/k B per cell-update)"}
    int_view = {"bound": "alu", "achieved": int_achieved / 1e12, "peak": int_peak / 1e12,
                "unit": "Tlane-ops/s", "frac": int_achieved / int_peak,
                "peak_source": "live LOP3 probe (gol_probe_int_peak): 64 lanes/clk/SM",
                "ops_per_cell_update": ALG_INT_OPS_PER_CELL,
                "note": "algorithmic ops = the reference full adder's 33 word-ops per 64 cells"}
    # One generation per pass is HBM-bound; deeper passes are bound by the
    # integer (ALU) pipe (ncu: ALU 84 %, DRAM 12 % at k = 4).
    primary, secondary = (hbm_view, int_view) if best_k == 1 else (int_view, hbm_view)
    roofline = dict(primary)
    roofline.update({"traffic": ncu_traffic(kernel, size), "kernel": kernel,
                     "launch_ms": launch_ms,
                     "launch_ms_source": "in-step: ms_per_step / passes per step (CUDA events "
                                         "around the captured graphs of the timed steps)",
                     "other_view": secondary})

    # -- 32-bit variant at 8192^2 (reported beside the headline) -------------
    var = None
    if d.rank == 0:
        vsize = 8192
        vcells = golb200.load_random_ones_zeros(vsize, vsize, SEED)
        # The pass engine over the depth sweep, and the shared-memory-resident
        # run (the 8 MiB grid fits in the SMs' shared memory) over its epoch
        # lengths.
        best = None
        by_algorithm = {}
        for alg, k in [("rows", k) for k in SWEEP_K] + [("resident", k) for k in (4, 6, 8)]:
            ve = golb200.GolB200(grid_dimensions=(vsize, vsize), state_bits_count=32,
                                 temporal_steps=k, algorithm=alg, device=d.local_rank,
                                 stream=stream.cuda_stream)
            ve.set_and_format_input_data(vcells)
            ve.initialize_data_structures()
            timed_run(ve, 256)
            ms = timed_run(ve, gens)
            ve_plan = ve.plan()
            ve.close()
            r = vsize * vsize * gens / (ms * 1e-3) / 1e9
            if r > by_algorithm.get(alg, (0, 0))[1]:
                by_algorithm[alg] = (k, r)
            if best is None or r > best[1]:
                best = (k, r, ve_plan, alg)
        var = {"workload": f"dense {vsize}x{vsize} Bernoulli(0.5) seed {SEED}, 32-bit rows, "
                           f"{gens} generations", "value": best[1], "unit": UNIT,
               "algorithm": best[3], "temporal_steps": best[0], "plan": best[2],
               "by_algorithm": {a: {"temporal_steps": v[0], "value": v[1]}
                                for a, v in by_algorithm.items()}}
        if not args.no_check:
            import oracle
            ve = golb200.GolB200(grid_dimensions=(vsize, vsize), state_bits_count=32,
                                 temporal_steps=best[0], algorithm=best[3], device=d.local_rank,
                                 stream=stream.cuda_stream)
            ve.set_and_format_input_data(vcells)
            ve.initialize_data_structures()
            ve.run(gens)
            ve.finalize_data_structures()
            got = ve.fetch_words(32)
            ve.close()
            want = oracle.life_rows(oracle.pack_rows(vcells, 32), vsize, gens, 32)
            var["bit_exact_vs_oracle_full_length"] = bool(np.array_equal(got, want))

    # -- e2e through the public API with host buffers -------------------------
    e2e_times, phases = [], {"set_input": [], "init": [], "run": [], "finalize": [], "fetch": []}
    out = np.empty_like(cells)
    eng = golb200.GolB200(grid_dimensions=(size, size), state_bits_count=64,
                          temporal_steps=best_k, device=d.local_rank, stream=stream.cuda_stream)
    for it in range(args.warmup + args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        eng.set_and_format_input_data(cells)
        t1 = time.perf_counter()
        eng.initialize_data_structures()
        t2 = time.perf_counter()
        eng.run(gens)
        t3 = time.perf_counter()
        eng.finalize_data_structures()
        t4 = time.perf_counter()
        eng.fetch_result(out)
        t5 = time.perf_counter()
        if it >= args.warmup:
            e2e_times.append(t5 - t0)
            for kname, v in zip(phases, (t1 - t0, t2 - t1, t3 - t2, t4 - t3, t5 - t4)):
                phases[kname].append(v * 1e3)
        with torch.cuda.stream(stream):
            flush.zero_()
    eng.close()
    e2e_total = d.max(sum(e2e_times))
    e2e_value = replica_throughput(d.world, cell_updates * args.steps, e2e_total) / 1e9

    cpu = None
    if d.rank == 0 and d.world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(cells)

    sparse = published = batched = batched_settling = serving = hbm = None
    if d.rank == 0 and d.world == 1 and not args.no_extras:
        hbm = run_extra("hbm")
        sparse = run_extra("sparse")
        published = run_extra("published")
        batched = run_extra("batched")
        batched_settling = run_extra("batched_settling")
        serving = run_extra("serving")

    if d.rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": d.world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
            "dtype_note": "the kernels compute on 32-bit words; the 64-bit-row layout is the same "
                          "bytes on the device",
            "data": "synthetic",
            "config": {
                "workload": f"dense {size}x{size} Bernoulli(0.5) seed {SEED}, 64-bit rows, "
                            f"{gens} generations per step, cells outside dead",
                "x": size, "y": size, "generations": gens, "word_bits": 64,
                "temporal_steps": best_k, "band_rows": plan["band_rows"],
                "words_per_lane": plan["words_per_lane"],
                "l2": "flushed between timed steps (256 MiB write, outside the events)",
                "parallelism": f"replicas x{d.world}" if d.world > 1 else "single GPU",
            },
            "bit_exact_vs_oracle_full_length": bit_exact,
            "k_sweep": {str(k): round(v, 1) for k, v in sweep.items()},
            "roofline": roofline,
            "variant_8192_32bit": var,
            "larger_than_l2_32768": hbm,
            "sparse_settling": sparse,
            "published_workloads": published,
            "batched_uneven": batched,
            "batched_uneven_settling": batched_settling,
            "serving": serving,
            "e2e": {"value": e2e_value, "unit": UNIT,
                    "h2d_bytes_per_step": grid_bytes, "d2h_bytes_per_step": grid_bytes,
                    "phases_ms_median": {k: statistics.median(v) for k, v in phases.items()},
                    "step_ms": [round(t * 1e3, 2) for t in e2e_times],
                    "path": "gol_set_input_u8 -> gol_init -> gol_run -> gol_finalize -> "
                            "gol_fetch_u8 (C ABI, host uint8 grid in and out)"},
            "gpu_launches": passes * args.steps,
            "clocks": clk,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)


def main():
    args = parse_args()
    d = Dist()
    if args.impl == "reference":
        run_reference_arm(args, d)      # rank 0 only; no process group needed
        return
    import torch
    if args.only:
        torch.cuda.set_device(d.local_rank)
        s = torch.cuda.Stream()
        fn = {"sparse": lambda: bench_sparse(s, d.local_rank),
              "published": lambda: bench_published(s, d.local_rank),
              "batched": lambda: bench_batched(s, d.local_rank),
              "serving": lambda: bench_serving(d.local_rank),
              "hbm": lambda: bench_hbm(s, d.local_rank),
              "batched_settling": lambda: bench_batched_settling(s, d.local_rank)}[args.only]
        print(json.dumps({args.only: fn()}), flush=True)
        return
    if d.world > 1:
        torch.cuda.set_device(d.local_rank)
    d.init("nccl")
    try:
        run_ours(args, d)
    finally:
        d.close()


if __name__ == "__main__":
    main()
