"""Dense-tile layout of the tensor-core kriging products, on the host (no GPU).

The layout is the tensor-core path's only host-side arithmetic: rows ordered
along a Z-order curve and cut into tiles of 128, each tile's column union cut
into chunks of 32, every nonzero placed at its (chunk, row, column) position of
the K-major core-matrix blocks, and the chunks split into per-CTA ranges and
per-tile segments.  Reading the blob back through the tile maps must give the
kriging matrix exactly (bit for bit), every chunk must be covered by exactly
one segment, every row must sit in exactly one tile, and the padding must stay
zero.
"""
import numpy as np
import pytest

from dualres_b200 import api, synth


def _w(oracle, dims, seed):
    vol = synth.make_volume(dims, 1.0, (0.806, 0.132, 1.0), 0.5, 0.3, 6.9, "ellipsoid", 0.6, seed)
    prep = oracle.prepare(vol.highres, vol.hmask, vol.omask)
    rp, col, val = oracle.kriging(prep["masked"], vol.qform_hr, vol.stdres, vol.qform_sr, vol.theta, vol.radius)
    return rp, col, val.astype(np.float32), prep["D"]


def _dense(rp, col, val, n_cols):
    W = np.zeros((len(rp) - 1, n_cols), np.float32)
    rows = np.repeat(np.arange(len(rp) - 1), np.diff(rp))
    W[rows, col] = val
    return W


def _transpose(rp, col, val, n_cols):
    rows = np.repeat(np.arange(len(rp) - 1), np.diff(rp))
    order = np.lexsort((rows, col))
    trp = np.zeros(n_cols + 1, np.int64)
    np.add.at(trp, col + 1, 1)
    return np.cumsum(trp), rows[order], val[order]


@pytest.mark.parametrize("g_max", [1, 7, 148])
def test_w_tiles_reproduce_the_matrix(oracle, g_max):
    rp, col, val, D = _w(oracle, (16, 16, 12), 3)
    n_h = len(D)
    # rows keyed by the centroid of their columns' voxels, as the library orders W
    rows = np.repeat(np.arange(len(rp) - 1), np.diff(rp))
    cnt = np.maximum(np.diff(rp), 1)[:, None]
    cen = np.zeros((len(rp) - 1, 3))
    np.add.at(cen, rows, D[col].astype(np.float64))
    keys = api.zorder_keys(np.rint(cen / cnt).astype(np.int64))
    dense, st = api.tc_layout(rp, col, val, n_h, keys, g_max)
    W = _dense(rp, col, val, n_h)
    assert np.array_equal(dense.view(np.uint32), W.view(np.uint32))
    assert st["chunks_once"] == st["chunks"] and st["rows_once"] == len(rp) - 1 and st["consistent"] == 1
    assert st["tiles"] == (len(rp) - 1 + 127) // 128 and st["ctas"] == min(g_max, st["chunks"])
    assert st["tiles"] <= st["segments"] <= st["tiles"] + st["ctas"]
    # the union of a tile's columns is a few times its nonzeros, not the whole column range
    assert st["chunks"] * 32 * 128 < 12 * len(col)


def test_wt_tiles_reproduce_the_transpose(oracle):
    rp, col, val, D = _w(oracle, (14, 15, 13), 5)
    n_h, n_s = len(D), len(rp) - 1
    trp, tcol, tval = _transpose(rp, col, val, n_h)
    dense, st = api.tc_layout(trp, tcol, tval, n_s, api.zorder_keys(D), 148)
    assert np.array_equal(dense, _dense(rp, col, val, n_h).T)
    assert st["rows_once"] == n_h and st["chunks_once"] == st["chunks"] and st["consistent"] == 1


def test_empty_rows_and_ragged_tiles():
    """Rows without nonzeros still get a tile row (their products are zero); a last tile of fewer than 128 rows
    and a chunk of fewer than 32 columns are padded with zeros."""
    rng = np.random.default_rng(0)
    n_rows, n_cols = 300, 77
    nnz_per_row = rng.integers(0, 9, n_rows)
    nnz_per_row[::17] = 0
    rp = np.concatenate([[0], np.cumsum(nnz_per_row)])
    col = np.concatenate([np.sort(rng.choice(n_cols, k, replace=False)) for k in nnz_per_row]).astype(np.int32)
    val = rng.standard_normal(len(col)).astype(np.float32) * np.float32(1e-3)
    keys = rng.integers(0, 2 ** 30, n_rows).astype(np.uint32)
    dense, st = api.tc_layout(rp, col, val, n_cols, keys, 5)
    assert np.array_equal(dense, _dense(rp, col, val, n_cols))
    assert st["tiles"] == 3 and st["rows_once"] == n_rows and st["chunks_once"] == st["chunks"]
    empty = np.zeros(n_rows + 1, np.int32)
    dense0, st0 = api.tc_layout(empty, np.zeros(0, np.int32), np.zeros(0, np.float32), n_cols, keys, 5)
    assert not dense0.any() and st0["chunks"] == 0 and st0["ctas"] == 0 and st0["segments"] == 0
