"""The tile-index division of the spreading kernels, checked on the CPU.

`TileDiv` (cugridder_b200/csrc/cg_tiles.cuh) divides a cell index n by a tile
extent d with one multiply-high: m = floor((2^32 - 1) / d) + 1 and
n / d = (n * m) >> 32, exact while n * d < 2^32 (d = 1 answered directly).
The gridding flush, the empty-tile fill and the tiled degridding's staging
turn a cell index into (x, y, plane) this way. These tests restate that
arithmetic in numpy and check it against integer division over the extents the
kernels use (tiles of at most 226 KB of complex64 cells: n and d below 2^15) and beyond.
"""
import numpy as np

TWO32 = 1 << 32


def tile_div(n, d):
    """(n * m) >> 32 with m the rounded-up reciprocal of d, as the kernels compute it."""
    n = np.asarray(n, dtype=np.uint64)
    if d == 1:
        return n.astype(np.int64)
    m = np.uint64((TWO32 - 1) // d + 1)
    return ((n * m) >> np.uint64(32)).astype(np.int64)


def test_exact_for_every_divisor_up_to_4096():
    rng = np.random.default_rng(7)
    for d in range(1, 4097):
        nmax = min((TWO32 - 1) // d, 1 << 18)
        ks = np.arange(0, nmax // d + 2, dtype=np.int64)
        edges = np.concatenate([ks * d, ks * d - 1, ks * d + 1, [nmax - 1]])
        edges = edges[(edges >= 0) & (edges < nmax)]
        rand = rng.integers(0, nmax, size=64)
        n = np.concatenate([edges, rand])
        assert np.array_equal(tile_div(n, d), n // d), d


def test_exact_for_large_tile_extents():
    rng = np.random.default_rng(11)
    ds = np.concatenate([rng.integers(4097, 29_000, size=300), [8192, 16384, 28_928, 28_999]])
    for d in ds.tolist():
        nmax = min((TWO32 - 1) // d, 29_000)
        n = np.concatenate([np.arange(0, nmax, max(1, nmax // 4096)), [nmax - 1, d - 1, d]])
        n = n[n < nmax]
        assert np.array_equal(tile_div(n, d), n // d), d


def test_cell_decomposition_matches_modulo():
    """The flush's (x, y, plane) of every cell, single cells and 16-byte pairs."""
    for wx, wy, wz in [(16, 8, 14), (16, 16, 5), (32, 8, 26), (14, 8, 3), (6, 2, 1), (48, 24, 7)]:
        i = np.arange(wx * wy * wz)
        z = tile_div(i, wx * wy)
        r = i - z * wx * wy
        y = tile_div(r, wx)
        x = r - y * wx
        assert np.array_equal(x, i % wx)
        assert np.array_equal(y, (i // wx) % wy)
        assert np.array_equal(z, i // (wx * wy))
        if wx % 2 == 0:
            hx = wx // 2
            j = np.arange(hx * wy * wz)
            z2 = tile_div(j, hx * wy)
            r2 = j - z2 * hx * wy
            y2 = tile_div(r2, hx)
            x2 = 2 * (r2 - y2 * hx)
            cells = z2 * wx * wy + y2 * wx + x2
            both = np.sort(np.concatenate([cells, cells + 1]))
            assert np.array_equal(both, np.arange(wx * wy * wz))
