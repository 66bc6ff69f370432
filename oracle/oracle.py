"""ORACLE — test infrastructure, not product code.

ctypes front end for the two checkers of bit-packed Game of Life:

* ``liboracle`` — oracle/libgoloracle.so, the plain-C restatement of the
  reference's CPU path (oracle/gol_oracle.c; each function there cites the
  reference file:line it follows);
* ``libref`` — oracle/_ref/libgolref.so, the reference's own CPU code
  (GoLCpuNaive, GoLCpuBitwise<AdderOps>, RandomOnesZerosDataLoader,
  GeneralBitGrid) compiled from the reference sources by oracle/Makefile.
  It exists only where the reference sources were present at build time;
  ``ref_available()`` says whether it loaded.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module, and only as the checker or the timed CPU baseline.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "libgoloracle.so")
REF_SO = os.path.join(HERE, "_ref", "libgolref.so")

_u8p = ctypes.POINTER(ctypes.c_uint8)
_vp = ctypes.c_void_p
_u64 = ctypes.c_uint64

_oracle = None
_ref = None
_ref_tried = False


def build(with_ref: bool | None = None) -> None:
    """Compiles the oracle (and the reference harness when its sources exist)."""
    targets = ["all"]
    if with_ref is None:
        with_ref = os.path.isdir("/root/reference/src")
    if with_ref:
        targets.append("ref")
    subprocess.run(["make", "-s", "-C", HERE, *targets], check=True)


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_vp)


def liboracle():
    global _oracle
    if _oracle is None:
        if not os.path.exists(ORACLE_SO):
            build(with_ref=False)
        lib = ctypes.CDLL(ORACLE_SO)
        lib.gor_random_ones_zeros.argtypes = [_u64, _u64, _u64, _vp]
        lib.gor_life_naive.argtypes = [_vp, _u64, _u64, _u64, _vp]
        lib.gor_pack_rows.argtypes = [ctypes.c_int, _vp, _u64, _u64, _vp]
        lib.gor_unpack_rows.argtypes = [ctypes.c_int, _vp, _u64, _u64, _vp]
        lib.gor_life_rows.argtypes = [ctypes.c_int, _vp, _u64, _u64, _u64, _vp, ctypes.c_int]
        lib.gor_fnv1a64.argtypes = [_vp, _u64]
        lib.gor_fnv1a64.restype = _u64
        lib.gor_max_threads.restype = ctypes.c_int
        _oracle = lib
    return _oracle


def libref():
    """The reference's own CPU path, or None when it was not built here."""
    global _ref, _ref_tried
    if not _ref_tried:
        _ref_tried = True
        if os.path.exists(REF_SO):
            lib = ctypes.CDLL(REF_SO)
            lib.ref_load_random_ones_zeros.argtypes = [_u64, _u64, _u64, _vp]
            lib.ref_run_cpu_naive.argtypes = [_vp, _u64, _u64, _u64, _vp]
            lib.ref_run_cpu_bitwise_adder.argtypes = [ctypes.c_int, _vp, _u64, _u64, _u64, _vp]
            lib.ref_pack_rows.argtypes = [ctypes.c_int, _vp, _u64, _u64, _vp]
            lib.ref_unpack_rows.argtypes = [ctypes.c_int, _vp, _u64, _u64, _vp]
            _ref = lib
    return _ref


def ref_available() -> bool:
    return libref() is not None


def _check(rc: int, what: str) -> None:
    if rc != 0:
        raise RuntimeError(f"oracle call {what} failed with status {rc}")


# --------------------------------------------------------------------------
# restatement (oracle/gol_oracle.c)
# --------------------------------------------------------------------------

def random_ones_zeros(x: int, y: int, seed: int) -> np.ndarray:
    """uint8[y, x] of 0/1 cells as RandomOnesZerosDataLoader draws them."""
    out = np.empty((y, x), dtype=np.uint8)
    _check(liboracle().gor_random_ones_zeros(x, y, seed, _ptr(out)), "random_ones_zeros")
    return out


def life_naive(cells: np.ndarray, iters: int) -> np.ndarray:
    """GoLCpuNaive restated: uint8[y, x] in, uint8[y, x] out."""
    cells = np.ascontiguousarray(cells, dtype=np.uint8)
    y, x = cells.shape
    out = np.empty_like(cells)
    _check(liboracle().gor_life_naive(_ptr(cells), x, y, iters, _ptr(out)), "life_naive")
    return out


def pack_rows(cells: np.ndarray, word_bits: int = 64) -> np.ndarray:
    cells = np.ascontiguousarray(cells, dtype=np.uint8)
    y, x = cells.shape
    dt = np.uint64 if word_bits == 64 else np.uint32
    out = np.empty((y, x // word_bits), dtype=dt)
    _check(liboracle().gor_pack_rows(word_bits, _ptr(cells), x, y, _ptr(out)), "pack_rows")
    return out


def unpack_rows(words: np.ndarray, x: int, word_bits: int = 64) -> np.ndarray:
    words = np.ascontiguousarray(words)
    y = words.shape[0]
    out = np.empty((y, x), dtype=np.uint8)
    _check(liboracle().gor_unpack_rows(word_bits, _ptr(words), x, y, _ptr(out)), "unpack_rows")
    return out


def life_rows(words: np.ndarray, x: int, iters: int, word_bits: int = 64,
              threads: int = 0) -> np.ndarray:
    """GoLCpuBitwise<AdderOps> restated on row-packed words (multi-threaded)."""
    words = np.ascontiguousarray(words)
    y = words.shape[0]
    out = np.empty_like(words)
    _check(liboracle().gor_life_rows(word_bits, _ptr(words), x, y, iters, _ptr(out), threads),
           "life_rows")
    return out


def life_cells(cells: np.ndarray, iters: int, threads: int = 0) -> np.ndarray:
    """Bit-sliced oracle on a cell grid (x a multiple of 32), cells in and out."""
    y, x = cells.shape
    wb = 64 if x % 64 == 0 else 32
    return unpack_rows(life_rows(pack_rows(cells, wb), x, iters, wb, threads), x, wb)


def fnv1a64(a: np.ndarray) -> int:
    a = np.ascontiguousarray(a)
    return int(liboracle().gor_fnv1a64(_ptr(a), a.nbytes))


def max_threads() -> int:
    return int(liboracle().gor_max_threads())


# --------------------------------------------------------------------------
# the reference itself (oracle/_ref), when built
# --------------------------------------------------------------------------

def _need_ref():
    lib = libref()
    if lib is None:
        raise RuntimeError("reference build oracle/_ref/libgolref.so is not present")
    return lib


def ref_random_ones_zeros(x: int, y: int, seed: int) -> np.ndarray:
    out = np.empty((y, x), dtype=np.uint8)
    _check(_need_ref().ref_load_random_ones_zeros(x, y, seed, _ptr(out)), "ref_load_random")
    return out


def ref_cpu_naive(cells: np.ndarray, iters: int) -> np.ndarray:
    cells = np.ascontiguousarray(cells, dtype=np.uint8)
    y, x = cells.shape
    out = np.empty_like(cells)
    _check(_need_ref().ref_run_cpu_naive(_ptr(cells), x, y, iters, _ptr(out)), "ref_cpu_naive")
    return out


def ref_cpu_bitwise_adder(cells: np.ndarray, iters: int, word_bits: int = 64) -> np.ndarray:
    cells = np.ascontiguousarray(cells, dtype=np.uint8)
    y, x = cells.shape
    out = np.empty_like(cells)
    _check(_need_ref().ref_run_cpu_bitwise_adder(word_bits, _ptr(cells), x, y, iters, _ptr(out)),
           "ref_cpu_bitwise_adder")
    return out


def ref_pack_rows(cells: np.ndarray, word_bits: int = 64) -> np.ndarray:
    cells = np.ascontiguousarray(cells, dtype=np.uint8)
    y, x = cells.shape
    dt = np.uint64 if word_bits == 64 else np.uint32
    out = np.empty((y, x // word_bits), dtype=dt)
    _check(_need_ref().ref_pack_rows(word_bits, _ptr(cells), x, y, _ptr(out)), "ref_pack_rows")
    return out


def ref_unpack_rows(words: np.ndarray, x: int, word_bits: int = 64) -> np.ndarray:
    words = np.ascontiguousarray(words)
    y = words.shape[0]
    out = np.empty((y, x), dtype=np.uint8)
    _check(_need_ref().ref_unpack_rows(word_bits, _ptr(words), x, y, _ptr(out)), "ref_unpack_rows")
    return out
