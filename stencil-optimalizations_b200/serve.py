"""Request loop for the serving configuration: a seeded Poisson stream of
Game of Life simulations fed to the continuous-batching server (GolServer).

    python stencil-optimalizations_b200/serve.py --rate 2000 --seconds 2

Each request draws its size, density, generation count and input seed from
gol_workload_uneven (sides log-uniform, multiples of 64; density uniform;
generations log-uniform) and its arrival time from gol_poisson_arrivals.
Requests are submitted when their arrival time has come (inputs generated on
the device at admission, or with --host-io made on the host and copied in,
results copied back and unpacked), the server is stepped continuously, and a
request completes when its last round has finished on the GPU (or earlier,
once change tracking finds it still). --policy picks arrival order or
least-work-first scheduling, --tracking the change-tracking mode. The loop
reports p50/p99 completion latency (arrival to completion, host clock) and
the aggregate cell-updates/s over the run.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
if HERE not in sys.path:
    sys.path.insert(0, HERE)

import numpy as np  # noqa: E402

import golb200  # noqa: E402


def usable_cpus() -> int:
    """Host threads this process may run on (its CPU affinity)."""
    try:
        return len(os.sched_getaffinity(0))
    except (AttributeError, OSError):
        return os.cpu_count() or 1


def run_stream(rate: float = 2000.0, seconds: float = 2.0, seed: int = 42, min_side: int = 128,
               max_side: int = 8192, density=(0.1, 0.5), gens=(16, 8192), quantum: int = 0,
               arena_bytes: int = 0, device: int = 0, fetch: str = "words",
               max_requests: int | None = None, server: golb200.GolServer | None = None,
               policy: str = "fifo", tracking: str = "auto", host_io: bool = False,
               check_every: int = 0, mode: str = "passes") -> dict:
    """Serves the seeded Poisson stream that arrives within `seconds`.

    host_io: every request's cells are made on the host before the stream
    starts (the same cells gol_serve_submit_random would make on the device,
    held as clients would hold them) and submitted through gol_serve_submit
    (host pack, copy to the device at admission); every result is fetched as
    cells (copy back, host unpack). Otherwise inputs are generated on the
    device and results fetched as packed words.
    check_every > 0 keeps the fetched result of every check_every-th request
    (submission order) in r["samples"] as (request, result).
    mode: "passes" (rounds of dependent pass items, change tracking as set)
    or "resident" (rounds with every request's bands in shared memory)."""
    from concurrent.futures import ThreadPoolExecutor
    n = int(rate * seconds * 1.2) + 16
    if max_requests:
        n = min(n, max_requests)
    work = golb200.workload_uneven(seed, n, min_side, max_side, 64, density, gens)
    arrivals = golb200.poisson_arrivals(seed + 1, n, rate)
    keep = [i for i in range(n) if arrivals[i] <= seconds] if not max_requests else list(range(n))
    own = server is None
    srv = server or golb200.GolServer(device=device, arena_bytes=arena_bytes, quantum=quantum)
    srv.set_policy(policy)
    srv.set_tracking(tracking)
    srv.set_mode(mode)
    host_cells = []
    if host_io:
        with ThreadPoolExecutor(max_workers=usable_cpus() or 1) as pool:
            host_cells = list(pool.map(
                lambda j: golb200.load_hash_bernoulli(work[j]["x"], work[j]["y"], work[j]["cell_seed"],
                                                      work[j]["density"]), keep))

    pending: dict[int, tuple[float, int, int]] = {}
    latencies: list[float] = []
    samples: list[tuple[dict, np.ndarray]] = []
    cell_updates = 0
    submitted = 0
    t0 = time.perf_counter()
    try:
        while submitted < len(keep) or pending:
            now = time.perf_counter() - t0
            while submitted < len(keep) and arrivals[keep[submitted]] <= now:
                d = work[keep[submitted]]
                if host_io:
                    rid = srv.submit(host_cells[submitted], d["gens"])
                    host_cells[submitted] = None
                else:
                    rid = srv.submit_random(d["x"], d["y"], d["gens"], d["cell_seed"], d["density"])
                pending[rid] = (float(arrivals[keep[submitted]]), d["x"] * d["y"] * d["gens"],
                                submitted)
                submitted += 1
            srv.step()
            done = srv.finished()
            t_done = time.perf_counter() - t0
            for rid in done:
                arr, cu, idx = pending.pop(rid)
                latencies.append(t_done - arr)
                cell_updates += cu
                keep_it = check_every > 0 and idx % check_every == 0
                if host_io or fetch == "cells":
                    out = srv.fetch(rid)
                elif fetch == "words" or keep_it:
                    out = srv.fetch_words(rid)
                else:
                    srv.release(rid)
                    out = None
                if keep_it:
                    samples.append((work[keep[idx]], out))
            if not done and submitted < len(keep) and not pending:
                wait = arrivals[keep[submitted]] - (time.perf_counter() - t0)
                if wait > 0:
                    time.sleep(min(wait, 0.001))
        wall = time.perf_counter() - t0
        stats = srv.stats()
        tiles = srv.tiles()
    finally:
        if own:
            srv.close()
    lat = np.array(latencies) if latencies else np.zeros(1)
    return {
        "policy": policy, "tracking": tracking, "host_io": host_io, "mode": mode,
        "tiles_computed": tiles["computed"],
        "tiles_skipped": tiles["skipped"], "finished_early_still": tiles["early_finished"],
        "samples": samples,
        "requests": len(latencies),
        "offered_rate_req_s": rate,
        "wall_s": wall,
        "cell_updates": cell_updates,
        "cell_updates_per_s": cell_updates / wall,
        "latency_p50_ms": float(np.percentile(lat, 50) * 1e3),
        "latency_p99_ms": float(np.percentile(lat, 99) * 1e3),
        "latency_max_ms": float(lat.max() * 1e3),
        "rounds": stats["rounds"],
        "quantum_generations": quantum or 64,
    }


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--rate", type=float, default=2000.0)
    ap.add_argument("--seconds", type=float, default=2.0)
    ap.add_argument("--seed", type=int, default=42)
    ap.add_argument("--quantum", type=int, default=0, help="generations per round (0 = the server default, 64)")
    ap.add_argument("--policy", choices=["fifo", "srpt"], default="fifo")
    ap.add_argument("--tracking", choices=["auto", "on", "off"], default="auto")
    ap.add_argument("--host-io", action="store_true")
    ap.add_argument("--mode", choices=["passes", "resident"], default="passes")
    a = ap.parse_args()
    r = run_stream(a.rate, a.seconds, a.seed, quantum=a.quantum, policy=a.policy,
                   tracking=a.tracking, host_io=a.host_io, mode=a.mode)
    r.pop("samples")
    print(json.dumps(r))


if __name__ == "__main__":
    main()
