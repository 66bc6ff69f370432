"""Rebuilds the input grid of a golden case (tests/golden/golden.json)."""
import numpy as np

import oracle


def case_input(case) -> np.ndarray:
    x, y = case["x"], case["y"]
    kind = case["input"]
    if kind == "random_ones_zeros":
        return oracle.random_ones_zeros(x, y, case["seed"])
    if kind == "cells":
        g = np.zeros((y, x), dtype=np.uint8)
        for cx, cy in case["cells"]:
            g[cy, cx] = 1
        return g
    if kind == "all_ones":
        return np.ones((y, x), dtype=np.uint8)
    raise ValueError(kind)


def case_output(case) -> np.ndarray | None:
    """The stored output grid, when the fixture keeps it."""
    if "output_bits_hex" not in case:
        return None
    x, y = case["x"], case["y"]
    bits = np.frombuffer(bytes.fromhex(case["output_bits_hex"]), dtype=np.uint8)
    return np.unpackbits(bits.reshape(y, -1), axis=1, bitorder="little")[:, :x]
