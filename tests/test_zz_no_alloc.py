"""gol_rows_run_noalloc — the entry point for callers that cannot allocate
device memory (their framework owns every allocation, or they cannot afford
the synchronisation cudaMalloc/cudaFree may cause). It must give the same
grids as the allocating path (gol_rows_pass chained over caller buffers),
call after call, although every call reuses the one scratch array compiled
into the library.

Collected last on purpose: if it fails, a run that stops at the first
failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest

import golb200
import oracle

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def reference_path(words: "torch.Tensor", x: int, y: int, n: int, k: int, stream: int):
    """The existing allocating path: k-generation passes with gol_rows_pass."""
    a = words.clone()
    b = torch.empty_like(a)
    left = n
    while left > 0:
        kk = min(k, left)
        golb200.rows_pass(a.data_ptr(), b.data_ptr(), x, y, kk, 0, stream)
        a, b = b, a
        left -= kk
    return a


def device_words(cells: np.ndarray) -> "torch.Tensor":
    packed = oracle.pack_rows(cells, 32)
    return torch.from_numpy(packed.view(np.int32)).cuda()


def test_noalloc_matches_allocating_path_twice_in_a_row():
    L = golb200.lib()
    s = torch.cuda.current_stream().cuda_stream
    cases = [(2048, 600, 37, 4, 5), (16384, 512, 50, 3, 6)]   # two calls, different shapes
    for x, y, n, k, seed in cases:
        cells = oracle.random_ones_zeros(x, y, seed)
        src = device_words(cells)
        out = torch.empty_like(src)
        rc = L.gol_rows_run_noalloc(src.data_ptr(), out.data_ptr(), x, y, n, k, s)
        assert rc == golb200.GOL_OK
        want = reference_path(src, x, y, n, k, s)
        torch.cuda.synchronize()
        assert torch.equal(out, want), (x, y, n, k)
        # the oracle agrees, and the input grid is left as it was
        got = out.cpu().numpy().view(np.uint32)
        assert np.array_equal(got, oracle.pack_rows(oracle.life_cells(cells, n), 32)), (x, y, n, k)
        assert np.array_equal(src.cpu().numpy().view(np.uint32), oracle.pack_rows(cells, 32))


def test_noalloc_at_its_size_limit_against_the_oracle():
    """16384 x 16384 is exactly GOL_NOALLOC_MAX_BYTES (32 MiB of words): the
    largest grid the scratch array holds, twice in a row (k = 1 and k = 4,
    both ending with a shorter pass)."""
    L = golb200.lib()
    s = torch.cuda.current_stream().cuda_stream
    x = y = 16384
    assert x * y // 8 == 32 << 20
    cells = oracle.random_ones_zeros(x, y, 11)
    src = device_words(cells)
    out = torch.empty_like(src)
    for n, k in ((3, 1), (6, 4)):
        assert L.gol_rows_run_noalloc(src.data_ptr(), out.data_ptr(), x, y, n, k, s) == golb200.GOL_OK
        torch.cuda.synchronize()
        want = oracle.life_rows(oracle.pack_rows(cells, 32), x, n, 32)
        assert np.array_equal(out.cpu().numpy().view(np.uint32), want), (n, k)


def test_noalloc_rejects_grids_beyond_its_scratch():
    L = golb200.lib()
    s = torch.cuda.current_stream().cuda_stream
    a = torch.empty(16, dtype=torch.int32, device="cuda")
    b = torch.empty(16, dtype=torch.int32, device="cuda")
    # 32768 x 16384 cells = 64 MiB of words: more than GOL_NOALLOC_MAX_BYTES (32 MiB)
    rc = L.gol_rows_run_noalloc(a.data_ptr(), b.data_ptr(), 32768, 16384, 1, 1, s)
    assert rc == golb200.GOL_E_UNSUPPORTED
    # one row more than the largest grid that fits
    rc = L.gol_rows_run_noalloc(a.data_ptr(), b.data_ptr(), 16384, 16385, 1, 1, s)
    assert rc == golb200.GOL_E_UNSUPPORTED
    # sizes whose byte count would wrap are invalid, not truncated
    rc = L.gol_rows_run_noalloc(a.data_ptr(), b.data_ptr(), 1 << 40, 1 << 40, 1, 1, s)
    assert rc == golb200.GOL_E_INVALID
    assert L.gol_rows_run_noalloc(a.data_ptr(), a.data_ptr(), 64, 1, 1, 1, s) == golb200.GOL_E_INVALID
