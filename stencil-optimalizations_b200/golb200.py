"""Python front end of the B200 Game of Life engine (libgolb200.so, C ABI
in include/gol_b200.h).

``GolB200`` mirrors the reference's algorithm contract
``infrastructure::Algorithm<2, cell_t>`` (src/infrastructure/algorithm.hpp:17-87)
method for method — set_and_format_input_data, initialize_data_structures,
run, finalize_data_structures, fetch_result, actually_performed_iterations,
set_params — and raises RuntimeError where the reference throws
(std::runtime_error / CudaError, cuch.hpp:42-52).

There is no CPU fallback: if libgolb200.so is missing this module raises on
first use, and every computation runs on the GPU through the C ABI.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("GOLB200_LIB") or os.path.join(HERE, "libgolb200.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "gol_b200.h")

GOL_OK = 0
GOL_E_INVALID = -1
GOL_E_STATE = -2
GOL_E_CUDA = -3
GOL_E_NOMEM = -4
GOL_E_UNSUPPORTED = -5
GOL_E_TIMEOUT = -6

LAYOUTS = {"rows": 0, "columns": 1, "tiles": 2}
_WORD_DTYPES = {16: np.uint16, 32: np.uint32, 64: np.uint64}


def layout_block(layout: str, word_bits: int) -> tuple:
    """(cells per word in x, in y) of a layout (bit_modes.hpp:10-177)."""
    if word_bits not in _WORD_DTYPES:
        raise ValueError("word_bits must be 16, 32 or 64")
    if layout == "rows":
        return word_bits, 1
    if layout == "columns":
        return 1, word_bits
    if layout == "tiles":
        return {16: (4, 4), 32: (8, 4), 64: (8, 8)}[word_bits]
    raise ValueError(f"unknown layout {layout!r}")

ALGORITHMS = {"auto": 0, "rows": 1, "local": 2, "resident": 3}


class GolConfig(ctypes.Structure):
    _fields_ = [
        ("struct_size", ctypes.c_uint32),
        ("algorithm", ctypes.c_uint32),
        ("x", ctypes.c_uint64),
        ("y", ctypes.c_uint64),
        ("word_bits", ctypes.c_uint32),
        ("temporal_steps", ctypes.c_uint32),
        ("thread_block_size", ctypes.c_uint32),
        ("tile_rows", ctypes.c_uint32),
        ("max_runtime_seconds", ctypes.c_uint64),
        ("device", ctypes.c_int32),
        ("lane_words", ctypes.c_uint32),
        ("stream", ctypes.c_void_p),
        ("dense_pct", ctypes.c_uint32),
        ("reserved", ctypes.c_uint32),
    ]


_lib = None
_vp = ctypes.c_void_p
_u64 = ctypes.c_uint64
_u32 = ctypes.c_uint32


def lib():
    """Loads libgolb200.so (building it first if this tree has nvcc)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            f"{LIB_PATH} is not built; run `python stencil-optimalizations_b200/build.py` "
            "(the engine has no CPU fallback)")
    L = ctypes.CDLL(LIB_PATH)
    L.gol_config_init.argtypes = [ctypes.POINTER(GolConfig), _u64, _u64]
    L.gol_config_init.restype = None
    L.gol_create.argtypes = [ctypes.POINTER(_vp), ctypes.POINTER(GolConfig)]
    L.gol_set_input_u8.argtypes = [_vp, _vp, _u64, _u64]
    L.gol_set_input_i32.argtypes = [_vp, _vp, _u64, _u64]
    L.gol_set_input_words.argtypes = [_vp, _vp, _u64, _u64, _u32]
    L.gol_init.argtypes = [_vp]
    L.gol_run.argtypes = [_vp, _u64]
    L.gol_sync.argtypes = [_vp]
    L.gol_finalize.argtypes = [_vp]
    L.gol_fetch_u8.argtypes = [_vp, _vp]
    L.gol_fetch_i32.argtypes = [_vp, _vp]
    L.gol_fetch_words.argtypes = [_vp, _vp, _u32]
    L.gol_set_input_layout.argtypes = [_vp, _vp, ctypes.c_int, _u32]
    L.gol_fetch_layout.argtypes = [_vp, _vp, ctypes.c_int, _u32]
    L.gol_pack_layout.argtypes = [_vp, _u64, _u64, ctypes.c_int, _u32, _vp]
    L.gol_unpack_layout.argtypes = [_vp, _u64, _u64, ctypes.c_int, _u32, _vp]
    L.gol_layout_to_rows_device.argtypes = [_vp, _vp, _u64, _u64, ctypes.c_int, _u32, _vp]
    L.gol_rows_to_layout_device.argtypes = [_vp, _vp, _u64, _u64, ctypes.c_int, _u32, _vp]
    L.gol_performed.argtypes = [_vp]
    L.gol_performed.restype = _u64
    L.gol_destroy.argtypes = [_vp]
    L.gol_destroy.restype = None
    L.gol_last_error.argtypes = [_vp]
    L.gol_last_error.restype = ctypes.c_char_p
    L.gol_device_grid.argtypes = [_vp]
    L.gol_device_grid.restype = _vp
    L.gol_stream.argtypes = [_vp]
    L.gol_stream.restype = _vp
    L.gol_plan.argtypes = [_vp, ctypes.POINTER(_u32), ctypes.POINTER(_u32), ctypes.POINTER(_u32)]
    L.gol_rows_pass.argtypes = [_vp, _vp, _u64, _u64, _u32, _u32, _vp]
    L.gol_rows_pass_ex.argtypes = [_vp, _vp, _u64, _u64, _u32, _u32, _u32, _vp]
    L.gol_pack_cells_device.argtypes = [_vp, _vp, _u64, _u64, _vp]
    L.gol_unpack_cells_device.argtypes = [_vp, _vp, _u64, _u64, _vp]
    L.gol_load_random_ones_zeros.argtypes = [_vp, _u64, _u64, _u64]
    L.gol_local_stats.argtypes = [_vp, ctypes.POINTER(_u64), ctypes.POINTER(_u64),
                                  ctypes.POINTER(_u64), _vp, _u64]
    L.gol_load_sparse_patches.argtypes = [_vp, _u64, _u64, _u64, _u32, ctypes.c_double,
                                          ctypes.c_double]
    L.gol_workload_uneven.argtypes = [_u64, _u32, _u32, _u32, _u32, ctypes.c_double,
                                      ctypes.c_double, _u64, _u64, _vp, _vp, _vp, _vp, _vp]
    L.gol_load_bernoulli.argtypes = [_vp, _u64, _u64, _u64, ctypes.c_double]
    L.gol_load_zeros.argtypes = [_vp, _u64, _u64]
    L.gol_batch_probe_timeout.argtypes = [ctypes.c_int32, _u64, ctypes.POINTER(ctypes.c_int32)]
    L.gol_load_always_changing.argtypes = [_vp, _u64, _u64]
    L.gol_lexicon_create.argtypes = [ctypes.POINTER(_vp)]
    L.gol_lexicon_add_text.argtypes = [_vp, ctypes.c_char_p]
    L.gol_lexicon_add_file.argtypes = [_vp, ctypes.c_char_p]
    L.gol_lexicon_count.argtypes = [_vp]
    L.gol_lexicon_pattern_size.argtypes = [_vp, ctypes.c_char_p, ctypes.POINTER(_u64),
                                           ctypes.POINTER(_u64)]
    L.gol_lexicon_insert.argtypes = [_vp, ctypes.c_char_p, _vp, _u64, _u64]
    L.gol_lexicon_insert_repeating.argtypes = [_vp, ctypes.c_char_p, _u64, _u64, _vp, _u64, _u64]
    L.gol_lexicon_last_error.argtypes = [_vp]
    L.gol_lexicon_last_error.restype = ctypes.c_char_p
    L.gol_lexicon_destroy.argtypes = [_vp]
    L.gol_lexicon_destroy.restype = None
    L.gol_poisson_arrivals.argtypes = [_u64, _u32, ctypes.c_double, _vp]
    L.gol_batch_create.argtypes = [ctypes.POINTER(_vp), ctypes.c_int32, _vp]
    L.gol_batch_add.argtypes = [_vp, _vp, _u64, _u64, _u64, ctypes.POINTER(ctypes.c_int32)]
    L.gol_batch_set_plan.argtypes = [_vp, ctypes.c_int32, _u32, _u32, _u32]
    L.gol_batch_plan.argtypes = [_vp, ctypes.c_int32, ctypes.POINTER(_u32), ctypes.POINTER(_u32),
                                 ctypes.POINTER(_u32), ctypes.POINTER(_u32)]
    L.gol_batch_upload.argtypes = [_vp]
    L.gol_batch_run.argtypes = [_vp]
    L.gol_batch_run_plain.argtypes = [_vp, _u32]
    L.gol_batch_run_resident.argtypes = [_vp]
    L.gol_batch_resident_info.argtypes = [_vp, ctypes.POINTER(_u64), ctypes.POINTER(_u32),
                                          ctypes.POINTER(_u64)]
    L.gol_batch_sync.argtypes = [_vp]
    L.gol_batch_fetch.argtypes = [_vp, ctypes.c_int32, _vp]
    L.gol_batch_info.argtypes = [_vp, ctypes.POINTER(_u64), ctypes.POINTER(_u64), ctypes.POINTER(_u64)]
    L.gol_batch_census.argtypes = [_vp, ctypes.POINTER(_u64), ctypes.POINTER(_u64)]
    L.gol_batch_set_tracking.argtypes = [_vp, ctypes.c_int32, ctypes.c_int32]
    L.gol_batch_retune.argtypes = [_vp]
    L.gol_batch_tiles.argtypes = [_vp, ctypes.POINTER(_u64), ctypes.POINTER(_u64)]
    L.gol_batch_grid_stats.argtypes = [_vp, ctypes.c_int32] + [ctypes.POINTER(_u32)] * 4
    L.gol_batch_stream.argtypes = [_vp]
    L.gol_batch_stream.restype = _vp
    L.gol_batch_last_error.argtypes = [_vp]
    L.gol_batch_last_error.restype = ctypes.c_char_p
    L.gol_batch_destroy.argtypes = [_vp]
    L.gol_batch_destroy.restype = None
    L.gol_rows_run_noalloc.argtypes = [_vp, _vp, _u64, _u64, _u64, _u32, _vp]
    L.gol_load_hash_bernoulli.argtypes = [_vp, _u64, _u64, _u64, ctypes.c_double]
    L.gol_serve_create.argtypes = [ctypes.POINTER(_vp), ctypes.c_int32, _u64, _u32, _vp]
    L.gol_serve_submit.argtypes = [_vp, _vp, _u64, _u64, _u64, ctypes.POINTER(_u64)]
    L.gol_serve_submit_random.argtypes = [_vp, _u64, _u64, _u64, _u64, ctypes.c_double,
                                          ctypes.POINTER(_u64)]
    L.gol_serve_step.argtypes = [_vp]
    L.gol_serve_finished.argtypes = [_vp, _vp, _u32, ctypes.POINTER(_u32)]
    L.gol_serve_fetch.argtypes = [_vp, _u64, _vp]
    L.gol_serve_fetch_words.argtypes = [_vp, _u64, _vp]
    L.gol_serve_release.argtypes = [_vp, _u64]
    L.gol_serve_stats.argtypes = [_vp] + [ctypes.POINTER(_u64)] * 5
    L.gol_serve_drain.argtypes = [_vp]
    L.gol_serve_set_policy.argtypes = [_vp, ctypes.c_int32]
    L.gol_serve_set_mode.argtypes = [_vp, ctypes.c_int32]
    L.gol_serve_set_tracking.argtypes = [_vp, ctypes.c_int32]
    L.gol_serve_tiles.argtypes = [_vp] + [ctypes.POINTER(_u64)] * 3
    L.gol_serve_last_error.argtypes = [_vp]
    L.gol_serve_last_error.restype = ctypes.c_char_p
    L.gol_serve_stream.argtypes = [_vp]
    L.gol_serve_stream.restype = _vp
    L.gol_serve_destroy.argtypes = [_vp]
    L.gol_serve_destroy.restype = None
    L.gol_probe_int_peak.argtypes = [ctypes.POINTER(ctypes.c_double), _vp]
    L.gol_abi_version.restype = ctypes.c_int
    L.gol_build_info.restype = ctypes.c_char_p
    _lib = L
    return L


def declared_symbols() -> list[str]:
    """Function names declared in include/gol_b200.h."""
    import re
    text = open(HEADER).read()
    return sorted(set(re.findall(r"\b(gol_[a-z0-9_]+)\s*\(", text)))


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_vp)


@dataclass
class ExperimentParams:
    """The ExperimentParams fields the hot path reads
    (src/infrastructure/experiment_params.hpp:21-116)."""
    grid_dimensions: tuple = (0, 0)
    iterations: int = 0
    max_runtime_seconds: int = 0          # 0 = unlimited
    state_bits_count: int = 64            # word width of the packed layout
    thread_block_size: int = 0            # rows per CTA band (0 = auto)
    temporal_steps: int = 0               # k (0 = auto)
    lane_words: int = 0                   # 32-bit words per lane (0 = auto)
    tile_rows: int = 0                    # change-tracking tile height (0 = auto)
    dense_pct: int = 0                    # change tracking: active-tile percentage from
                                          # which a pass runs dense (0 = auto, > 100 never)
    algorithm: str = "auto"
    device: int = 0
    stream: int | None = None             # cudaStream_t as an integer
    extra: dict = field(default_factory=dict)


class GolB200:
    """One grid advanced on the GPU, behind the reference's phase contract."""

    def __init__(self, params: ExperimentParams | None = None, **kw):
        self._e = _vp()
        self._cells_dtype = np.uint8
        self.params = params or ExperimentParams(**kw)
        self._create()

    # -- Algorithm::set_params (algorithm.hpp:76-78) -----------------------
    def set_params(self, params: ExperimentParams) -> None:
        self.close()
        self.params = params
        self._create()

    def _create(self) -> None:
        p = self.params
        x, y = (int(v) for v in p.grid_dimensions)
        cfg = GolConfig()
        lib().gol_config_init(ctypes.byref(cfg), x, y)
        cfg.algorithm = ALGORITHMS[p.algorithm]
        cfg.word_bits = int(p.state_bits_count)
        cfg.temporal_steps = int(p.temporal_steps)
        cfg.lane_words = int(p.lane_words)
        cfg.tile_rows = int(p.tile_rows)
        cfg.dense_pct = int(p.dense_pct)
        cfg.thread_block_size = int(p.thread_block_size)
        cfg.max_runtime_seconds = int(p.max_runtime_seconds)
        cfg.device = int(p.device)
        cfg.stream = p.stream
        rc = lib().gol_create(ctypes.byref(self._e), ctypes.byref(cfg))
        if rc != GOL_OK:
            raise RuntimeError(f"gol_create: {lib().gol_last_error(None).decode()} ({rc})")
        self.x, self.y = x, y

    def _check(self, rc: int, what: str) -> None:
        if rc != GOL_OK:
            msg = lib().gol_last_error(self._e).decode()
            raise RuntimeError(f"{what}: {msg} (status {rc})")

    # -- the contract --------------------------------------------------------
    def set_and_format_input_data(self, grid: np.ndarray) -> None:
        g = np.ascontiguousarray(grid)
        if g.shape != (self.y, self.x):
            raise RuntimeError(f"grid shape {g.shape} != ({self.y}, {self.x})")
        if g.dtype == np.int32:
            self._cells_dtype = np.int32
            self._check(lib().gol_set_input_i32(self._e, _ptr(g), self.x, self.y), "set_input")
        else:
            self._cells_dtype = np.uint8
            g = g.astype(np.uint8, copy=False)
            self._check(lib().gol_set_input_u8(self._e, _ptr(g), self.x, self.y), "set_input")

    def set_input_words(self, words: np.ndarray, word_bits: int = 64) -> None:
        w = np.ascontiguousarray(words)
        self._check(lib().gol_set_input_words(self._e, _ptr(w), self.x, self.y, word_bits),
                    "set_input_words")

    def set_input_layout(self, words: np.ndarray, layout: str, word_bits: int) -> None:
        """Input as words of the column / tile / rows layout."""
        xb, yb = layout_block(layout, word_bits)
        w = np.ascontiguousarray(words, dtype=_WORD_DTYPES[word_bits])
        if w.size * xb * yb != self.x * self.y:
            raise ValueError("words do not cover the grid")
        self._check(lib().gol_set_input_layout(self._e, _ptr(w), LAYOUTS[layout], word_bits),
                    "set_input_layout")

    def initialize_data_structures(self) -> None:
        self._check(lib().gol_init(self._e), "initialize")

    def run(self, iterations: int) -> None:
        self._check(lib().gol_run(self._e, int(iterations)), "run")

    def sync(self) -> None:
        self._check(lib().gol_sync(self._e), "sync")

    def finalize_data_structures(self) -> None:
        self._check(lib().gol_finalize(self._e), "finalize")

    def fetch_result(self, out: np.ndarray | None = None) -> np.ndarray:
        if out is None:
            out = np.empty((self.y, self.x), dtype=self._cells_dtype)
        if out.dtype == np.int32:
            self._check(lib().gol_fetch_i32(self._e, _ptr(out)), "fetch")
        else:
            self._check(lib().gol_fetch_u8(self._e, _ptr(out)), "fetch")
        return out

    def fetch_words(self, word_bits: int = 64) -> np.ndarray:
        dt = np.uint64 if word_bits == 64 else np.uint32
        out = np.empty((self.y, self.x // word_bits), dtype=dt)
        self._check(lib().gol_fetch_words(self._e, _ptr(out), word_bits), "fetch_words")
        return out

    def fetch_layout(self, layout: str, word_bits: int) -> np.ndarray:
        xb, yb = layout_block(layout, word_bits)
        out = np.empty((self.y // yb, self.x // xb), dtype=_WORD_DTYPES[word_bits])
        self._check(lib().gol_fetch_layout(self._e, _ptr(out), LAYOUTS[layout], word_bits),
                    "fetch_layout")
        return out

    def actually_performed_iterations(self) -> int:
        return int(lib().gol_performed(self._e))

    # -- device-resident access ---------------------------------------------
    def device_grid_ptr(self) -> int:
        return int(lib().gol_device_grid(self._e) or 0)

    def stream_ptr(self) -> int:
        return int(lib().gol_stream(self._e) or 0)

    def plan(self) -> dict:
        k, b, w = _u32(), _u32(), _u32()
        self._check(lib().gol_plan(self._e, ctypes.byref(k), ctypes.byref(b), ctypes.byref(w)),
                    "plan")
        return {"temporal_steps": k.value, "band_rows": b.value, "words_per_lane": w.value}

    def local_stats(self, max_entries: int = 0) -> dict:
        """Change-tracking census (GOL_ALG_LOCAL): passes, tiles, computed tiles."""
        p, t, c = _u64(), _u64(), _u64()
        per = np.zeros(max_entries, dtype=np.uint32)
        self._check(lib().gol_local_stats(self._e, ctypes.byref(p), ctypes.byref(t), ctypes.byref(c),
                                          _ptr(per) if max_entries else None, max_entries),
                    "local_stats")
        out = {"passes": p.value, "tiles_per_pass": t.value, "computed_tiles": c.value}
        if max_entries:
            out["per_pass"] = per[:min(p.value, max_entries)]
        return out

    def close(self) -> None:
        if self._e:
            lib().gol_destroy(self._e)
            self._e = _vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def run_generations(cells: np.ndarray, iterations: int, **kw) -> np.ndarray:
    """Whole contract in one call: cells (uint8/int32 [y, x]) in, cells out."""
    y, x = cells.shape
    with GolB200(grid_dimensions=(x, y), **kw) as alg:
        alg.set_and_format_input_data(cells)
        alg.initialize_data_structures()
        alg.run(iterations)
        alg.finalize_data_structures()
        return alg.fetch_result()


def load_random_ones_zeros(x: int, y: int, seed: int) -> np.ndarray:
    """RandomOnesZerosDataLoader: uint8[y, x] of 0/1 from std::mt19937(seed)."""
    out = np.empty((y, x), dtype=np.uint8)
    rc = lib().gol_load_random_ones_zeros(_ptr(out), x, y, seed)
    if rc != GOL_OK:
        raise RuntimeError(f"gol_load_random_ones_zeros failed with status {rc}")
    return out


def load_sparse_patches(x: int, y: int, seed: int, patch: int = 64, fraction: float = 0.01,
                        density: float = 0.35) -> np.ndarray:
    """All-dead grid with a seeded `fraction` of patch x patch slots filled
    with Bernoulli(density) cells (the sparse/settling workload)."""
    out = np.empty((y, x), dtype=np.uint8)
    rc = lib().gol_load_sparse_patches(_ptr(out), x, y, seed, patch, fraction, density)
    if rc < 0:
        raise RuntimeError(f"gol_load_sparse_patches failed with status {rc}")
    return out


def load_zeros(x: int, y: int) -> np.ndarray:
    """ZerosLoader (src/infrastructure/data_loader.hpp:128-146): every cell dead."""
    out = np.empty((y, x), dtype=np.uint8)
    rc = lib().gol_load_zeros(_ptr(out), x, y)
    if rc < 0:
        raise RuntimeError(f"gol_load_zeros failed with status {rc}")
    return out


def load_always_changing(x: int, y: int) -> np.ndarray:
    """AlwaysChangingSpaceLoader (data_loader.hpp:102-125): a blinker every
    4 cells in x and y on a dead grid."""
    out = np.empty((y, x), dtype=np.uint8)
    rc = lib().gol_load_always_changing(_ptr(out), x, y)
    if rc < 0:
        raise RuntimeError(f"gol_load_always_changing failed with status {rc}")
    return out


class Lexicon:
    """Pattern dictionary and expression loader (LexiconLoader,
    data_loader.hpp:77-99; lexicon::Lexicon, gol-lexicon/lexicon.hpp).

    Entries come from text in the format of the reference's generated
    dictionary (gol-lexicon/patterns.cpp); "blinker" is built in."""

    def __init__(self, path: str | None = None, text: str | None = None):
        h = _vp()
        rc = lib().gol_lexicon_create(ctypes.byref(h))
        if rc != GOL_OK:
            raise RuntimeError(f"gol_lexicon_create failed with status {rc}")
        self._h = h
        if path is not None:
            self.add_file(path)
        if text is not None:
            self.add_text(text)

    def _check(self, rc: int, what: str) -> int:
        if rc < 0:
            msg = lib().gol_lexicon_last_error(self._h).decode()
            raise ValueError(f"{what}: {msg} (status {rc})")
        return rc

    def add_text(self, text: str) -> int:
        return self._check(lib().gol_lexicon_add_text(self._h, text.encode()), "add_text")

    def add_file(self, path: str) -> int:
        return self._check(lib().gol_lexicon_add_file(self._h, os.fsencode(path)), "add_file")

    def __len__(self) -> int:
        return lib().gol_lexicon_count(self._h)

    def pattern_size(self, name: str) -> tuple:
        w, h = _u64(), _u64()
        self._check(lib().gol_lexicon_pattern_size(self._h, name.encode(), ctypes.byref(w),
                                                   ctypes.byref(h)), f"pattern {name!r}")
        return w.value, h.value

    def insert(self, expression: str, cells: np.ndarray) -> int:
        """Place the patterns of `expression` ("name[x,y]; ...") into the
        (y, x) uint8 grid in place; returns the records placed."""
        if cells.dtype != np.uint8 or not cells.flags.c_contiguous or cells.ndim != 2:
            raise ValueError("cells must be a C-contiguous (y, x) uint8 array")
        y, x = cells.shape
        return self._check(lib().gol_lexicon_insert(self._h, expression.encode(), _ptr(cells),
                                                    x, y), "insert")

    def insert_repeating(self, name: str, x_jump: int, y_jump: int, cells: np.ndarray) -> None:
        if cells.dtype != np.uint8 or not cells.flags.c_contiguous or cells.ndim != 2:
            raise ValueError("cells must be a C-contiguous (y, x) uint8 array")
        y, x = cells.shape
        self._check(lib().gol_lexicon_insert_repeating(self._h, name.encode(), x_jump, y_jump,
                                                       _ptr(cells), x, y), "insert_repeating")

    def load(self, expression: str, x: int, y: int) -> np.ndarray:
        """LexiconLoader::load_data: a dead (y, x) grid with the expression's patterns."""
        out = np.zeros((y, x), dtype=np.uint8)
        self.insert(expression, out)
        return out

    def close(self) -> None:
        if self._h:
            lib().gol_lexicon_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def probe_batch_timeout(spin_limit: int = 1 << 14, device: int = 0) -> int:
    """Runs the batch kernel on a work list whose only item waits forever on
    its dependency; returns the status word (GOL_E_TIMEOUT expected)."""
    st = ctypes.c_int32()
    rc = lib().gol_batch_probe_timeout(device, spin_limit, ctypes.byref(st))
    if rc != GOL_OK:
        raise RuntimeError(f"gol_batch_probe_timeout failed with status {rc}")
    return st.value


def probe_int_peak(stream: int = 0) -> float:
    """Measured 32-bit LOP3 lane-ops/s of the current device."""
    v = ctypes.c_double()
    rc = lib().gol_probe_int_peak(ctypes.byref(v), stream)
    if rc != GOL_OK:
        raise RuntimeError(f"gol_probe_int_peak failed with status {rc}")
    return v.value


def rows_pass(d_src: int, d_dst: int, x: int, y: int, k: int, band_rows: int = 0,
              stream: int = 0, lane_words: int = 0) -> None:
    rc = lib().gol_rows_pass_ex(d_src, d_dst, x, y, k, band_rows, lane_words, stream)
    if rc != GOL_OK:
        raise RuntimeError(f"gol_rows_pass failed with status {rc}")


def pack_cells_device(d_cells: int, d_words: int, x: int, y: int, stream: int = 0) -> None:
    rc = lib().gol_pack_cells_device(d_cells, d_words, x, y, stream)
    if rc != GOL_OK:
        raise RuntimeError(f"gol_pack_cells_device failed with status {rc}")


def unpack_cells_device(d_words: int, d_cells: int, x: int, y: int, stream: int = 0) -> None:
    rc = lib().gol_unpack_cells_device(d_words, d_cells, x, y, stream)
    if rc != GOL_OK:
        raise RuntimeError(f"gol_unpack_cells_device failed with status {rc}")


def pack_layout(cells: np.ndarray, layout: str, word_bits: int) -> np.ndarray:
    """Host cells -> words of a layout (GeneralBitGrid::fill_grid)."""
    cells = np.ascontiguousarray(cells, dtype=np.uint8)
    y, x = cells.shape
    xb, yb = layout_block(layout, word_bits)
    out = np.empty((y // yb, x // xb), dtype=_WORD_DTYPES[word_bits])
    rc = lib().gol_pack_layout(_ptr(cells), x, y, LAYOUTS[layout], word_bits, _ptr(out))
    if rc != GOL_OK:
        raise ValueError(f"gol_pack_layout failed with status {rc}")
    return out


def unpack_layout(words: np.ndarray, x: int, y: int, layout: str, word_bits: int) -> np.ndarray:
    """Words of a layout -> host cells (GeneralBitGrid::to_grid)."""
    w = np.ascontiguousarray(words, dtype=_WORD_DTYPES[word_bits])
    out = np.empty((y, x), dtype=np.uint8)
    rc = lib().gol_unpack_layout(_ptr(w), x, y, LAYOUTS[layout], word_bits, _ptr(out))
    if rc != GOL_OK:
        raise ValueError(f"gol_unpack_layout failed with status {rc}")
    return out


def layout_to_rows_device(d_src: int, d_rows: int, x: int, y: int, layout: str, word_bits: int,
                          stream: int = 0) -> None:
    rc = lib().gol_layout_to_rows_device(d_src, d_rows, x, y, LAYOUTS[layout], word_bits, stream)
    if rc != GOL_OK:
        raise RuntimeError(f"gol_layout_to_rows_device failed with status {rc}")


def rows_to_layout_device(d_rows: int, d_dst: int, x: int, y: int, layout: str, word_bits: int,
                          stream: int = 0) -> None:
    rc = lib().gol_rows_to_layout_device(d_rows, d_dst, x, y, LAYOUTS[layout], word_bits, stream)
    if rc != GOL_OK:
        raise RuntimeError(f"gol_rows_to_layout_device failed with status {rc}")


# ---------------------------------------------------------------------------
# multi-grid workloads and the batched engine
# ---------------------------------------------------------------------------

def workload_uneven(seed: int, n: int, min_side: int, max_side: int, multiple: int = 64,
                    density=(0.2, 0.5), gens=(64, 4096)) -> list[dict]:
    """The documented uneven workload draw (gol_workload_uneven)."""
    xs = np.empty(n, np.uint64)
    ys = np.empty(n, np.uint64)
    ds = np.empty(n, np.float64)
    gs = np.empty(n, np.uint64)
    cs = np.empty(n, np.uint64)
    rc = lib().gol_workload_uneven(seed, n, min_side, max_side, multiple, density[0], density[1],
                                   gens[0], gens[1], _ptr(xs), _ptr(ys), _ptr(ds), _ptr(gs),
                                   _ptr(cs))
    if rc != GOL_OK:
        raise RuntimeError(f"gol_workload_uneven failed with status {rc}")
    return [{"x": int(xs[i]), "y": int(ys[i]), "density": float(ds[i]), "gens": int(gs[i]),
             "cell_seed": int(cs[i])} for i in range(n)]


def load_bernoulli(x: int, y: int, seed: int, density: float) -> np.ndarray:
    out = np.empty((y, x), dtype=np.uint8)
    rc = lib().gol_load_bernoulli(_ptr(out), x, y, seed, density)
    if rc != GOL_OK:
        raise RuntimeError(f"gol_load_bernoulli failed with status {rc}")
    return out


def poisson_arrivals(seed: int, n: int, rate: float) -> np.ndarray:
    out = np.empty(n, np.float64)
    rc = lib().gol_poisson_arrivals(seed, n, rate, _ptr(out))
    if rc != GOL_OK:
        raise RuntimeError(f"gol_poisson_arrivals failed with status {rc}")
    return out


class GolBatch:
    """Many grids advanced together by one persistent launch (gol_batch_*)."""

    def __init__(self, device: int = 0, stream: int | None = None):
        self._b = _vp()
        rc = lib().gol_batch_create(ctypes.byref(self._b), device, stream)
        if rc != GOL_OK:
            raise RuntimeError(f"gol_batch_create failed with status {rc}")
        self.shapes: list[tuple[int, int]] = []

    def _check(self, rc: int, what: str) -> None:
        if rc != GOL_OK:
            raise RuntimeError(f"{what}: {lib().gol_batch_last_error(self._b).decode()} "
                               f"(status {rc})")

    def add(self, cells: np.ndarray, generations: int) -> int:
        g = np.ascontiguousarray(cells, dtype=np.uint8)
        y, x = g.shape
        gid = ctypes.c_int32()
        self._check(lib().gol_batch_add(self._b, _ptr(g), x, y, int(generations),
                                        ctypes.byref(gid)), "batch_add")
        self.shapes.append((y, x))
        return gid.value

    def set_plan(self, gid: int, lane_words: int = 0, temporal_steps: int = 0,
                 band_rows: int = 0) -> None:
        self._check(lib().gol_batch_set_plan(self._b, gid, lane_words, temporal_steps, band_rows),
                    "batch_set_plan")

    def plan(self, gid: int) -> dict:
        w, k, b, s = _u32(), _u32(), _u32(), _u32()
        self._check(lib().gol_batch_plan(self._b, gid, ctypes.byref(w), ctypes.byref(k),
                                         ctypes.byref(b), ctypes.byref(s)), "batch_plan")
        return {"lane_words": w.value, "temporal_steps": k.value, "band_rows": b.value,
                "segments": s.value}

    def upload(self) -> None:
        self._check(lib().gol_batch_upload(self._b), "batch_upload")

    def run(self) -> None:
        self._check(lib().gol_batch_run(self._b), "batch_run")

    def run_plain(self, temporal_steps: int = 4) -> None:
        self._check(lib().gol_batch_run_plain(self._b, temporal_steps), "batch_run_plain")

    def run_resident(self) -> None:
        """Every grid's bands in shared memory for all their generations, one
        persistent cooperative launch (gol_batch_run_resident)."""
        self._check(lib().gol_batch_run_resident(self._b), "batch_run_resident")

    def resident_info(self) -> dict:
        n, c, m = ctypes.c_uint64(), ctypes.c_uint32(), ctypes.c_uint64()
        self._check(lib().gol_batch_resident_info(self._b, ctypes.byref(n), ctypes.byref(c),
                                                  ctypes.byref(m)), "batch_resident_info")
        return {"bands": n.value, "ctas": c.value, "smem_bytes": m.value}

    def sync(self) -> None:
        self._check(lib().gol_batch_sync(self._b), "batch_sync")

    def fetch(self, gid: int) -> np.ndarray:
        y, x = self.shapes[gid]
        out = np.empty((y, x), np.uint8)
        self._check(lib().gol_batch_fetch(self._b, gid, _ptr(out)), "batch_fetch")
        return out

    def info(self) -> dict:
        g, i, c = _u64(), _u64(), _u64()
        self._check(lib().gol_batch_info(self._b, ctypes.byref(g), ctypes.byref(i), ctypes.byref(c)),
                    "batch_info")
        return {"grids": g.value, "items": i.value, "cell_updates": c.value}

    def census(self) -> dict:
        """SM cycles the last run's items spent waiting / computing."""
        w, c = _u64(), _u64()
        self._check(lib().gol_batch_census(self._b, ctypes.byref(w), ctypes.byref(c)), "batch_census")
        return {"wait_cycles": w.value, "work_cycles": c.value}

    TRACK = {"auto": 0, "off": 1, "on": 2}

    def set_tracking(self, gid: int, mode: str = "auto") -> None:
        """Change tracking of one grid: "auto" (the autotuner's choice),
        "off" (every item computed) or "on"."""
        self._check(lib().gol_batch_set_tracking(self._b, gid, self.TRACK[mode]),
                    "batch_set_tracking")

    def retune(self) -> None:
        """Per-grid tracking and tile choice from the last run's census."""
        self._check(lib().gol_batch_retune(self._b), "batch_retune")

    def tiles(self) -> dict:
        """Work items of the last run computed and skipped."""
        c, k = _u64(), _u64()
        self._check(lib().gol_batch_tiles(self._b, ctypes.byref(c), ctypes.byref(k)), "batch_tiles")
        return {"computed": c.value, "skipped": k.value}

    def grid_stats(self, gid: int) -> dict:
        t, c, k, st = _u32(), _u32(), _u32(), _u32()
        self._check(lib().gol_batch_grid_stats(self._b, gid, ctypes.byref(t), ctypes.byref(c),
                                               ctypes.byref(k), ctypes.byref(st)), "batch_grid_stats")
        return {"tracked": bool(t.value), "computed": c.value, "skipped": k.value,
                "still_pass": None if st.value == 0xFFFFFFFF else st.value}

    def stream_ptr(self) -> int:
        return int(lib().gol_batch_stream(self._b) or 0)

    def close(self) -> None:
        if self._b:
            lib().gol_batch_destroy(self._b)
            self._b = _vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def load_hash_bernoulli(x: int, y: int, seed: int, density: float) -> np.ndarray:
    """The cells gol_serve_submit_random generates on the device."""
    out = np.empty((y, x), dtype=np.uint8)
    rc = lib().gol_load_hash_bernoulli(_ptr(out), x, y, seed, density)
    if rc != GOL_OK:
        raise RuntimeError(f"gol_load_hash_bernoulli failed with status {rc}")
    return out


class GolServer:
    """Continuous-batching server (gol_serve_*): requests stay resident on the
    device and advance together, one persistent launch per round."""

    def __init__(self, device: int = 0, arena_bytes: int = 0, quantum: int = 0,
                 stream: int | None = None):
        self._s = _vp()
        rc = lib().gol_serve_create(ctypes.byref(self._s), device, arena_bytes, quantum, stream)
        if rc != GOL_OK:
            raise RuntimeError(f"gol_serve_create failed with status {rc}")
        self.shapes: dict[int, tuple[int, int]] = {}
        self._ids = np.zeros(4096, np.uint64)

    def _check(self, rc: int, what: str) -> None:
        if rc != GOL_OK:
            raise RuntimeError(f"{what}: {lib().gol_serve_last_error(self._s).decode()} "
                               f"(status {rc})")

    def submit(self, cells: np.ndarray, generations: int) -> int:
        g = np.ascontiguousarray(cells, dtype=np.uint8)
        y, x = g.shape
        rid = _u64()
        self._check(lib().gol_serve_submit(self._s, _ptr(g), x, y, int(generations),
                                           ctypes.byref(rid)), "serve_submit")
        self.shapes[rid.value] = (y, x)
        return rid.value

    def submit_random(self, x: int, y: int, generations: int, seed: int, density: float) -> int:
        rid = _u64()
        self._check(lib().gol_serve_submit_random(self._s, x, y, int(generations), seed, density,
                                                  ctypes.byref(rid)), "serve_submit_random")
        self.shapes[rid.value] = (y, x)
        return rid.value

    def step(self) -> None:
        self._check(lib().gol_serve_step(self._s), "serve_step")

    def finished(self) -> list[int]:
        n = _u32()
        self._check(lib().gol_serve_finished(self._s, _ptr(self._ids), self._ids.size,
                                             ctypes.byref(n)), "serve_finished")
        return [int(v) for v in self._ids[:n.value]]

    def fetch(self, rid: int) -> np.ndarray:
        y, x = self.shapes.pop(rid)
        out = np.empty((y, x), np.uint8)
        self._check(lib().gol_serve_fetch(self._s, rid, _ptr(out)), "serve_fetch")
        return out

    def fetch_words(self, rid: int) -> np.ndarray:
        y, x = self.shapes.pop(rid)
        out = np.empty((y, x // 32), np.uint32)
        self._check(lib().gol_serve_fetch_words(self._s, rid, _ptr(out)), "serve_fetch_words")
        return out

    def release(self, rid: int) -> None:
        self.shapes.pop(rid, None)
        self._check(lib().gol_serve_release(self._s, rid), "serve_release")

    def stats(self) -> dict:
        v = [_u64() for _ in range(5)]
        self._check(lib().gol_serve_stats(self._s, *[ctypes.byref(a) for a in v]), "serve_stats")
        return dict(zip(["queued", "running", "rounds", "cell_updates", "arena_free_bytes"],
                        [a.value for a in v]))

    def drain(self) -> None:
        self._check(lib().gol_serve_drain(self._s), "serve_drain")

    POLICIES = {"fifo": 0, "srpt": 1}

    def set_policy(self, policy: str) -> None:
        """"fifo" (arrival order) or "srpt" (least work first) admission; every
        running request advances the quantum per round either way."""
        self._check(lib().gol_serve_set_policy(self._s, self.POLICIES[policy]), "serve_set_policy")

    def set_tracking(self, mode: str) -> None:
        self._check(lib().gol_serve_set_tracking(self._s, GolBatch.TRACK[mode]), "serve_set_tracking")

    MODES = {"passes": 0, "resident": 1}

    def set_mode(self, mode: str) -> None:
        """"passes" (dependent pass items, change tracking) or "resident"
        (bands in shared memory for the round's generations); only while no
        request is queued or running."""
        self._check(lib().gol_serve_set_mode(self._s, self.MODES[mode]), "serve_set_mode")

    def tiles(self) -> dict:
        c, k, e = _u64(), _u64(), _u64()
        self._check(lib().gol_serve_tiles(self._s, ctypes.byref(c), ctypes.byref(k), ctypes.byref(e)),
                    "serve_tiles")
        return {"computed": c.value, "skipped": k.value, "early_finished": e.value}

    def close(self) -> None:
        if self._s:
            lib().gol_serve_destroy(self._s)
            self._s = _vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
