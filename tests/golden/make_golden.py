"""Generates tests/golden/golden.json from the REFERENCE's own CPU code.

Every output recorded here comes from oracle/_ref/libgolref.so — the
reference's GoLCpuNaive<char> (its default validator,
src/infrastructure/experiment_params.hpp:43) or GoLCpuBitwise<char,64,AdderOps>,
compiled from the reference sources by oracle/Makefile — never from code of
this repository. Inputs come from the reference's RandomOnesZerosDataLoader
(src/infrastructure/data_loader.hpp:57-75) or from small patterns written
here from the B3/S23 rule (blinker, block, glider, single cell).

Run in a container that has the reference sources:
    make -C oracle all ref && python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden.json")


def pattern(x: int, y: int, cells: list[tuple[int, int]]) -> np.ndarray:
    g = np.zeros((y, x), dtype=np.uint8)
    for cx, cy in cells:
        g[cy, cx] = 1
    return g


# Small shapes drawn from the rule itself, not from any pattern collection.
BLINKER = [(0, 1), (1, 1), (2, 1)]
BLOCK = [(0, 0), (1, 0), (0, 1), (1, 1)]
GLIDER = [(1, 0), (2, 1), (0, 2), (1, 2), (2, 2)]


def shift(cells, dx, dy):
    return [(cx + dx, cy + dy) for cx, cy in cells]


def main() -> None:
    if not oracle.ref_available():
        raise SystemExit("oracle/_ref/libgolref.so missing: run `make -C oracle ref` first")

    cases = []

    def add(name, grid, iters, kind, store_grids, seed=None, spec=None, use_naive=True):
        y, x = grid.shape
        if use_naive:
            out = oracle.ref_cpu_naive(grid, iters)
            via = "GoLCpuNaive<char>"
        else:
            out = oracle.ref_cpu_bitwise_adder(grid, iters, 64)
            via = "GoLCpuBitwise<char,64,AdderOps>"
        case = {
            "name": name,
            "x": x,
            "y": y,
            "iters": iters,
            "input": kind,
            "reference_path": via,
            "input_fnv1a64": f"{oracle.fnv1a64(grid):016x}",
            "output_fnv1a64": f"{oracle.fnv1a64(out):016x}",
            "output_alive": int(out.sum()),
        }
        if seed is not None:
            case["seed"] = seed
        if spec is not None:
            case["cells"] = spec
        if store_grids:
            # cells packed LSB-first along x (the rows layout, any x)
            case["output_bits_hex"] = np.packbits(out, axis=1, bitorder="little").tobytes().hex()
        cases.append(case)

    # C1: the reference's CPU-runnable benchmark case (2048^2, seed 42, 128 gens).
    c1 = oracle.ref_random_ones_zeros(2048, 2048, 42)
    add("c1_2048x2048_seed42_128", c1, 128, "random_ones_zeros", False, seed=42)

    # Seeded random grids, odd and non-square shapes, several generation counts.
    for (x, y, seed, iters) in [
        (64, 64, 1, 1), (64, 64, 2, 37), (96, 40, 7, 33), (128, 320, 3, 20),
        (256, 128, 4, 64), (32, 1, 5, 3), (32, 32, 6, 11), (32, 200, 8, 50),
        (320, 17, 9, 40), (64, 3, 10, 9), (1024, 64, 11, 100), (512, 512, 12, 0),
        (512, 512, 13, 1), (160, 96, 14, 129), (2048, 16, 15, 31), (32, 2, 16, 4),
    ]:
        g = oracle.ref_random_ones_zeros(x, y, seed)
        add(f"random_{x}x{y}_seed{seed}_{iters}", g, iters, "random_ones_zeros", True, seed=seed)

    # Known-answer patterns from the rule.
    pats = [
        ("blinker_mid", 32, 8, shift(BLINKER, 14, 3), 1),
        ("blinker_mid_even", 32, 8, shift(BLINKER, 14, 3), 2),
        ("blinker_word_edge", 64, 8, shift(BLINKER, 30, 3), 3),   # straddles bits 31|32
        ("blinker_left_edge", 32, 8, shift(BLINKER, 0, 3), 1),    # half outside -> dies
        ("block_still", 64, 8, shift(BLOCK, 31, 3), 10),
        ("block_corner", 32, 4, shift(BLOCK, 0, 0), 5),
        ("glider_4gens", 64, 32, shift(GLIDER, 5, 5), 4),
        ("glider_cross_word", 128, 64, shift(GLIDER, 58, 2), 80),
        ("glider_into_wall", 64, 64, shift(GLIDER, 40, 40), 200),
        ("single_cell_dies", 32, 4, [(10, 2)], 1),
        ("all_dead", 64, 16, [], 7),
    ]
    for name, x, y, cells, iters in pats:
        add(name, pattern(x, y, cells), iters, "cells", True, spec=cells)
    full = np.ones((16, 64), dtype=np.uint8)
    add("all_alive", full, 3, "all_ones", True)

    # A larger case through the reference's fast bitwise path (checked against
    # GoLCpuNaive at 2048^2 by tests/test_oracle.py).
    g = oracle.ref_random_ones_zeros(4096, 1024, 21)
    add("random_4096x1024_seed21_256_adder64", g, 256, "random_ones_zeros", False, seed=21,
        use_naive=False)

    with open(OUT, "w") as f:
        json.dump({"generator": "tests/golden/make_golden.py", "cases": cases}, f, indent=1)
    print(f"wrote {len(cases)} cases to {OUT}")


if __name__ == "__main__":
    main()
