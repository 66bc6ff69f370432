"""Request loop for the serving configuration: a seeded Poisson stream of
Game of Life simulations fed to the continuous-batching server (GolServer).

    python stencil-optimalizations_b200/serve.py --rate 2000 --seconds 2

Each request draws its size, density, generation count and input seed from
gol_workload_uneven (sides log-uniform, multiples of 64; density uniform;
generations log-uniform) and its arrival time from gol_poisson_arrivals.
Requests are submitted when their arrival time has come (inputs generated on
the device at admission), the server is stepped continuously, and a request
completes when its last round has finished on the GPU. The loop reports
p50/p99 completion latency (arrival to completion, host clock) and the
aggregate cell-updates/s over the run.
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


def run_stream(rate: float = 2000.0, seconds: float = 2.0, seed: int = 42, min_side: int = 128,
               max_side: int = 8192, density=(0.1, 0.5), gens=(16, 8192), quantum: int = 128,
               arena_bytes: int = 0, device: int = 0, fetch: str = "words",
               max_requests: int | None = None, server: golb200.GolServer | None = None) -> dict:
    """Serves the seeded Poisson stream that arrives within `seconds`."""
    n = int(rate * seconds * 1.2) + 16
    if max_requests:
        n = min(n, max_requests)
    work = golb200.workload_uneven(seed, n, min_side, max_side, 64, density, gens)
    arrivals = golb200.poisson_arrivals(seed + 1, n, rate)
    keep = [i for i in range(n) if arrivals[i] <= seconds] if not max_requests else list(range(n))
    own = server is None
    srv = server or golb200.GolServer(device=device, arena_bytes=arena_bytes, quantum=quantum)
    pending: dict[int, tuple[float, int]] = {}
    latencies: list[float] = []
    cell_updates = 0
    submitted = 0
    t0 = time.perf_counter()
    try:
        while submitted < len(keep) or pending:
            now = time.perf_counter() - t0
            while submitted < len(keep) and arrivals[keep[submitted]] <= now:
                d = work[keep[submitted]]
                rid = srv.submit_random(d["x"], d["y"], d["gens"], d["cell_seed"], d["density"])
                pending[rid] = (float(arrivals[keep[submitted]]), d["x"] * d["y"] * d["gens"])
                submitted += 1
            srv.step()
            done = srv.finished()
            t_done = time.perf_counter() - t0
            for rid in done:
                arr, cu = pending.pop(rid)
                latencies.append(t_done - arr)
                cell_updates += cu
                if fetch == "words":
                    srv.fetch_words(rid)
                elif fetch == "cells":
                    srv.fetch(rid)
                else:
                    srv.release(rid)
            if not done and submitted < len(keep) and not pending:
                wait = arrivals[keep[submitted]] - (time.perf_counter() - t0)
                if wait > 0:
                    time.sleep(min(wait, 0.001))
        wall = time.perf_counter() - t0
        stats = srv.stats()
    finally:
        if own:
            srv.close()
    lat = np.array(latencies) if latencies else np.zeros(1)
    return {
        "requests": len(latencies),
        "offered_rate_req_s": rate,
        "wall_s": wall,
        "cell_updates": cell_updates,
        "cell_updates_per_s": cell_updates / wall,
        "latency_p50_ms": float(np.percentile(lat, 50) * 1e3),
        "latency_p99_ms": float(np.percentile(lat, 99) * 1e3),
        "latency_max_ms": float(lat.max() * 1e3),
        "rounds": stats["rounds"],
        "quantum_generations": quantum,
    }


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--rate", type=float, default=2000.0)
    ap.add_argument("--seconds", type=float, default=2.0)
    ap.add_argument("--seed", type=int, default=42)
    ap.add_argument("--quantum", type=int, default=128)
    a = ap.parse_args()
    print(json.dumps(run_stream(a.rate, a.seconds, a.seed, quantum=a.quantum)))


if __name__ == "__main__":
    main()
