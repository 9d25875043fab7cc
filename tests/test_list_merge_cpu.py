"""Exactness arguments of the matching kernels, checked on the CPU with the lists' own rules.

The kernels keep each block's 8 best candidates with strict-less insertion in scan order
(top8_insert in csrc/zb3d_match.cuh, the reference's rule).  Two kernels rely on properties
of that rule rather than on running it once over the whole scan:

* zb_match_column (csrc/zb3d_kernels.cu) splits a block's candidate rows into 16 ordered
  ranges, builds one list per range, and merges them in range order by inserting a later
  range's entries into the earlier ranges' list (a tree over lane pairs: in round k, pair
  i, a multiple of 2k, takes the list of pair i + k);
* zb_match_temporal keeps per-frame lists of K = 2 entries when ps_num <= 2, because only
  the first ps_num entries of a per-frame list are read.

Both must give exactly the list of one sequential scan, ties and duplicate positions
included (overlapping search windows insert the same position more than once).

The finish kernel (zb_finish) sums the 8x8 boxes of origin weights from a 39 x 39 tile:
8-wide row sums, then an 8-row sum that each thread slides down 4 pixels.  The last test
restates its indexing and checks it against a direct box sum.
"""
import numpy as np
import pytest

FLT_MAX = np.float32(3.402823466e38)


def insert(e, q, err, pos):
    """top8_insert / topk_insert: strict-less insertion into a sorted list of len(e)."""
    n = len(e)
    for i in range(n - 1, 0, -1):
        ci = err < e[i]
        cp = err < e[i - 1]
        if cp:
            e[i], q[i] = e[i - 1], q[i - 1]
        elif ci:
            e[i], q[i] = err, pos
    if err < e[0]:
        e[0], q[0] = err, pos


def scan(items, k=8):
    e = [FLT_MAX] * k
    q = [0] * k
    for err, pos in items:
        if err < e[k - 1]:
            insert(e, q, err, pos)
    return e, q


def items_for(rng, n, tie_levels):
    errs = rng.integers(0, tie_levels, n).astype(np.float32)  # few levels: many ties
    pos = rng.integers(0, 40, n)                              # repeated positions too
    return list(zip(errs.tolist(), pos.tolist()))


@pytest.mark.parametrize("seed", range(40))
def test_range_split_tree_merge_equals_one_scan(seed):
    rng = np.random.default_rng(seed)
    nrows = int(rng.integers(1, 60))
    ncols = int(rng.integers(1, 30))
    rows = [items_for(rng, ncols, int(rng.integers(2, 12))) for _ in range(nrows)]
    want = scan([it for r in rows for it in r])
    per = (nrows + 15) // 16                                   # the kernel's ranges
    lists = []
    for pr in range(16):
        r0, r1 = pr * per, min(pr * per + per - 1, nrows - 1)
        lists.append(scan([it for r in rows[r0:r1 + 1] for it in r]) if r0 <= r1 else ([FLT_MAX] * 8, [0] * 8))
    k = 1
    while k < 16:                                              # the kernel's shuffle rounds
        for pr in range(0, 16, 2 * k):
            e, q = lists[pr]
            oe, oq = lists[pr + k]
            for i in range(8):
                if oe[i] < e[7]:
                    insert(e, q, oe[i], oq[i])
        k *= 2
    assert lists[0] == want


@pytest.mark.parametrize("seed", range(40))
def test_short_list_is_the_head_of_the_8_entry_list(seed):
    rng = np.random.default_rng(1000 + seed)
    items = items_for(rng, int(rng.integers(1, 300)), int(rng.integers(2, 20)))
    e8, q8 = scan(items, 8)
    for k in range(1, 9):
        ek, qk = scan(items, k)
        assert (ek, qk) == (e8[:k], q8[:k])


@pytest.mark.parametrize("w,h", [(32, 32), (70, 45), (1, 1), (33, 9), (96, 64)])
def test_finish_tile_box_sums(w, h):
    rng = np.random.default_rng(w * 131 + h)
    den = rng.integers(0, 1 << 40, (h, w), dtype=np.int64)
    # direct: pixel (y, x) sums origins (oy, ox) with y - 7 <= oy <= y, x - 7 <= ox <= x
    pad = np.zeros((h + 7, w + 7), np.int64)
    pad[7:, 7:] = den
    want = np.zeros((h, w), np.int64)
    for dy in range(8):
        for dx in range(8):
            want += pad[dy:dy + h, dx:dx + w]
    got = np.zeros((h, w), np.int64)
    rows_per_cta, per = 32, 4
    for y0 in range(0, h, rows_per_cta):
        for x0 in range(0, w, 32):
            t = np.zeros((rows_per_cta + 7, 40), np.int64)      # t[39][40]
            for r in range(rows_per_cta + 7):
                for c in range(39):
                    gy, gx = y0 - 7 + r, x0 - 7 + c
                    if 0 <= gy < h and 0 <= gx < w:
                        t[r, c] = den[gy, gx]
            hs = np.zeros((rows_per_cta + 7, 32), np.int64)     # hs[39][32]
            for r in range(rows_per_cta + 7):
                for c in range(32):
                    assert c + 7 < 39
                    hs[r, c] = t[r, c:c + 8].sum()
            for ty in range(8):
                for tx in range(32):
                    x, ry = x0 + tx, ty * per
                    if x >= w:
                        continue
                    ds = hs[ry:ry + 8, tx].sum()
                    for i in range(per):
                        y = y0 + ry + i
                        if y >= h:
                            break
                        if i > 0:
                            assert ry + i + 7 < rows_per_cta + 7 and ry + i - 1 >= 0
                            ds += hs[ry + i + 7, tx] - hs[ry + i - 1, tx]
                        got[y, x] = ds
    assert np.array_equal(got, want)
