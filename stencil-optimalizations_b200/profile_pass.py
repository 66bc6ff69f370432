"""Runs a few k-generation passes of the row-band kernel on one grid, for
profiling (ncu) and quick timing.

    python stencil-optimalizations_b200/profile_pass.py --size 16384 --k 5 --passes 8

The grid is the dense benchmark input (Bernoulli(0.5), seed 42, from the
reference's RandomOnesZerosDataLoader). Each pass reads one device buffer
and writes the other through gol_rows_pass; the script prints the mean
per-launch time measured with CUDA events.
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
    a = ap.parse_args()

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


if __name__ == "__main__":
    main()
