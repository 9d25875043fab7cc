"""Shared-memory layouts of the kernels, checked on the CPU.

The index maps below restate the device code (csrc/zb3d_kernels.cu: split_off and
tile2_g of the packed matching tile, move_tr / move_bc / move_cd and the Wiener
coefficient buffer of zb_filter16; csrc/zb3d_dct_tc.cu: kmaj and the staging order).
For every map these tests check the properties that the kernels rely on:

* stores and loads stay inside their buffer, and a store map is a bijection, so that
  no two values collide;
* every warp-wide access touches distinct banks (or shares a word, which is a broadcast):
  4-byte accesses are checked over the 32 lanes, 16-byte accesses per 8-lane phase.

The parity tests on the GPU prove the values; these pin the layout design on any machine.
"""
import itertools

import pytest

BANKS = 32


def conflict_free_words(addrs):
    """4-byte accesses of 32 lanes (float offsets): distinct banks unless the same word"""
    by_bank = {}
    for a in addrs:
        by_bank.setdefault(a % BANKS, set()).add(a)
    return all(len(words) == 1 for words in by_bank.values())


# ---------------------------------------------------------------------------
# packed FP32x2 matching tile: pair rows of two half-planes of g 16-byte chunks
# ---------------------------------------------------------------------------
TILE2_G = 40


def tile2_g(tp, chunks):
    return TILE2_G if chunks <= (4 * TILE2_G - 128) // 4 else tp // 4


def split_off(col, g):
    return ((col >> 1) & 1) * 4 * g + 4 * (col >> 2) + 2 * (col & 1)


@pytest.mark.parametrize("bm_range", [1, 4, 9, 12, 15, 16, 24, 40])
@pytest.mark.parametrize("block_step", [4, 8])
def test_matching_tile_split_layout(bm_range, block_step):
    chunks = (2 * bm_range + 1 + 3) // 4
    tp = 128 + 4 * chunks
    g = tile2_g(tp, chunks)
    pp = 8 * g
    assert g >= tp // 4 and (pp * 4) % 16 == 0
    offs = [split_off(c, g) for c in range(tp)]
    assert len(set(offs)) == tp and max(offs) + 2 <= pp
    for c in range(0, tp, 2):  # a float4 holds columns c, c + 1 of a row pair
        assert split_off(c, g) % 4 == 0 and split_off(c + 1, g) == split_off(c, g) + 2
    # lane tile column at dx = -R: 4 b (shared halves, block_step 4) or 8 b + 4 hh (block_step 8)
    uo = [4 * l for l in range(32)] if block_step == 4 else [8 * (l >> 1) + 4 * (l & 1) for l in range(32)]
    assert all(u % 4 == 0 for u in uo)
    for m in range(chunks):
        for p in range(4):
            # the kernel's address: column uo + 4 m + 2 p, as (uo + 4 m) + (p & 1) 4 g + 4 (p >> 1)
            cols = [u + 4 * m + 2 * p for u in uo]
            assert all(c + 1 < tp for c in cols)
            got = [u + 4 * m + (p & 1) * 4 * g + 4 * (p >> 1) for u in uo]
            assert got == [split_off(c, g) for c in cols]
            for phase in range(4):  # 16-byte loads: 8 lanes per phase, distinct bank quads
                quads = {(got[l] // 4) % 8 for l in range(8 * phase, 8 * phase + 8)}
                assert len(quads) == 8


# ---------------------------------------------------------------------------
# zb_filter16: two 16-lane groups per warp, lane (j, h), group buffers 592 floats apart
# ---------------------------------------------------------------------------
GROUP = 592
LANES = [(g, h, j) for g in range(2) for h in range(2) for j in range(8)]


def move_tr(g, h, j, q, i):
    return g * GROUP + (2 * q + h) * 72 + i + 9 * j, g * GROUP + (2 * q + h) * 72 + j + 9 * i


def move_bc_store(g, h, j, q, i):
    return g * GROUP + (2 * q + h) * 72 + 9 * j + 2 * i


def move_bc_load(g, h, j, p, t):
    return g * GROUP + p * 72 + 9 * (2 * t + h) + 2 * j


def move_cd_store(g, h, j, p, t):
    return g * GROUP + p * 72 + 8 * (2 * t + h) + j


def move_cd_load(g, h, j, q, i):
    return g * GROUP + (2 * q + h) * 72 + 8 * i + j


def check_move(store, store_regs, load, load_regs):
    # per group: the store map is a bijection onto the addresses the loads read
    for g in range(2):
        st = [store(g, h, j, *r) for h in range(2) for j in range(8) for r in store_regs]
        ld = [load(g, h, j, *r) for h in range(2) for j in range(8) for r in load_regs]
        assert len(set(st)) == 512 and set(st) == set(ld)
        assert min(st) >= g * GROUP and max(st) < (g + 1) * GROUP
    for r in store_regs:
        assert conflict_free_words([store(g, h, j, *r) for g, h, j in LANES])
    for r in load_regs:
        assert conflict_free_words([load(g, h, j, *r) for g, h, j in LANES])


QI = [(q, i) for q in range(4) for i in range(8)]
PT = [(p, t) for p in range(8) for t in range(4)]


def test_filter_move_transpose():
    check_move(lambda g, h, j, q, i: move_tr(g, h, j, q, i)[0], QI,
               lambda g, h, j, q, i: move_tr(g, h, j, q, i)[1], QI)


def test_filter_move_to_all_patches():
    check_move(move_bc_store, QI, move_bc_load, PT)


def test_filter_move_to_spectra_halves():
    check_move(move_cd_store, PT, move_cd_load, QI)


def test_filter_moves_carry_the_right_elements():
    """each move puts element (patch, row, column) where the next layout expects it"""
    # A -> B: lane (j, h) has column j of patches 2q + h, row i; afterwards row j, column i
    for h, j, q, i in itertools.product(range(2), range(8), range(4), range(8)):
        st, _ = move_tr(0, h, j, q, i)
        # the lane (j' = i, h) that loads register (q, j) reads this address
        assert move_tr(0, h, i, q, j)[1] == st
    # B -> C: (patch 2q + h, row j, column i) -> lane (i, h') of the row's half, register (p, t)
    for h, j, q, i in itertools.product(range(2), range(8), range(4), range(8)):
        st = move_bc_store(0, h, j, q, i)
        p, row, col = 2 * q + h, j, i
        assert move_bc_load(0, row & 1, col, p, row >> 1) == st
    # C -> D: (spectrum p, row 2t + h, column j) -> lane (j, p & 1), register (p >> 1, row)
    for h, j, p, t in itertools.product(range(2), range(8), range(8), range(4)):
        st = move_cd_store(0, h, j, p, t)
        assert move_cd_load(0, p & 1, j, p >> 1, 2 * t + h) == st


def test_filter_wiener_coefficients():
    """[spectrum * 72 + row * 8 + column], groups 592 floats apart"""
    def cb(g, p, r, c):
        return g * GROUP + p * 72 + r * 8 + c
    addrs = {cb(0, p, r, c) for p in range(8) for r in range(8) for c in range(8)}
    assert len(addrs) == 512 and max(addrs) < GROUP
    for p, t in PT:  # written in layout C
        assert conflict_free_words([cb(g, p, 2 * t + h, j) for g, h, j in LANES])
    for q, i in QI:  # read in layout D
        assert conflict_free_words([cb(g, 2 * q + h, i, j) for g, h, j in LANES])
    for p, r in itertools.product(range(8), range(8)):  # the weight's chain: both halves of a column
        assert conflict_free_words([cb(g, p, r, j) for g, h, j in LANES])


# ---------------------------------------------------------------------------
# zb3d_dct2d_tf32: K-major core-matrix operands, staged in shared-memory order
# ---------------------------------------------------------------------------
def kmaj(row, k, rows):
    return (k >> 2) * rows * 16 + (row >> 3) * 128 + (row & 7) * 16 + (k & 3) * 4


@pytest.mark.parametrize("rows", [64, 128])
def test_tf32_operand_layout(rows):
    offs = {kmaj(r, k, rows) for r in range(rows) for k in range(64)}
    assert len(offs) == rows * 64 and max(offs) == rows * 64 * 4 - 4
    # core matrices: 8 rows x 16 bytes, 8-row groups 128 bytes apart (SBO), K chunks rows * 16 apart (LBO)
    assert kmaj(8, 0, rows) - kmaj(0, 0, rows) == 128
    assert kmaj(0, 4, rows) - kmaj(0, 0, rows) == rows * 16


def test_tf32_staging_order_is_the_operand_layout():
    for s in range(128 * 64):
        kk, row, kc = s & 3, (s >> 2) & 127, s >> 9
        assert kmaj(row, 4 * kc + kk, 128) == 4 * s
