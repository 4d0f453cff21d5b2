"""The tile-image layout of inner tables of width 65..320 and the generated lane table of the tile
product kernel (bpmax_b200/csrc/wide_tables.inc, bpmax_wide.cuh), checked on the CPU by restating the
kernels' index arithmetic in numpy:

* the finalize's write-back (every block, S1 piece and halo piece of every tile) and the table read
  used by every consumer (f_value) round-trip every entry of a table, and write inside the cell;
* the product kernel's items (A tile image, B tile image), lanes and k blocks give exactly the
  triangular max-plus product max_{k in [i2-1, j2]} A[i2][k] + B[k+1][j2] with the R3 term, and read
  only written floats of the two images;
* every micro-tile of an off-diagonal output tile has exactly two lanes (one per half), and the
  halves of every item kind cover each micro-tile's k blocks once.
"""
import os
import re

import numpy as np
import pytest

CSRC = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "bpmax_b200", "csrc")
NEG = -np.inf


def _load():
    inc = open(os.path.join(CSRC, "r0_tables.inc")).read()
    rows = re.findall(r"\{([0-9,]+)\}", re.search(r"constexpr int R0_TAB_COLBASE\[9\]\[9\] = \{(.*)\};", inc).group(1))
    cb8 = [int(x) for x in rows[8].split(",")]
    lane_rows = re.search(r"c_r0_lane\[8\]\[256\]\[4\] = \{\n(.*)\};", inc, re.S).group(1).split("\n")
    lane8 = [tuple(int(v) for v in t) for t in re.findall(r"\{(\d+),(\d+),(\d+),(\d+)\}", lane_rows[7])][:128]
    winc = open(os.path.join(CSRC, "wide_tables.inc")).read()
    cbd = [int(x) for x in re.search(r"WIDE_DENSE_COLBASE\[9\] = \{([0-9,]+)\}", winc).group(1).split(",")]
    lanew = [tuple(int(v) for v in t) for t in
             re.findall(r"\{(\d+),(\d+),(\d+)\}", re.search(r"c_tile_lane\[128\]\[3\] = \{(.*)\};", winc).group(1))]
    return cb8, lane8, cbd, lanew


CB8, LANE8, CBD, LANEW = _load()
SD, SQ = 4 * CB8[8], 4 * CBD[8]


def tile_off(NT, I, J):
    o = I * SD + SQ * (I * (NT - 1) - I * (I - 1) // 2)
    return o + (SD + (J - I - 1) * SQ if J > I else 0)


def cell_floats(NT):
    return NT * SD + NT * (NT - 1) // 2 * SQ


def wide_pos(NT, r, c):
    I, J, lr, lc = r >> 6, c >> 6, r & 63, c & 63
    cb = CB8[lc >> 3] if I == J else CBD[lc >> 3]
    return tile_off(NT, I, J) + 4 * (cb + 17 * (lr >> 3)) + 8 * (lr & 7) + (lc & 7)


def blk_decode(q):
    bi = 0
    while q >= 8 - bi:
        q -= 8 - bi
        bi += 1
    return bi, bi + q


def write_cell(NT, N, T, s1v):
    """finalize_wide_kernel's write-back of the logical table T (r <= c < N) into tile images."""
    img = np.full(cell_floats(NT), np.nan)

    def val(r, c):
        return T[r, c] if (r <= c < N) else (s1v if r == c + 1 else NEG)

    for I in range(NT):
        for J in range(I, NT):
            to, nblk = tile_off(NT, I, J), (36 if I == J else 64)
            for q4 in range(nblk * 16 + 16):
                if q4 >= nblk * 16:
                    bj, h = (q4 - nblk * 16) >> 1, q4 & 1
                    cb = CB8[bj] if I == J else CBD[bj]
                    v = [((s1v if (h == 1 and t == 3) else NEG) if I == J else
                          val(64 * I + 64, 64 * J + 8 * bj + 4 * h + t)) for t in range(4)]
                    o = to + 4 * (cb + 17 * (bj + 1 if I == J else 8)) + 4 * h
                else:
                    bi, bj = blk_decode(q4 >> 4) if I == J else ((q4 >> 4) & 7, q4 >> 7)
                    r, c0 = 64 * I + 8 * bi + ((q4 & 15) >> 1), 64 * J + 8 * bj + 4 * (q4 & 1)
                    o = to + 4 * ((CB8[bj] if I == J else CBD[bj]) + 17 * bi) + 4 * (q4 & 15)
                    v = [val(r, c0 + t) for t in range(4)]
                assert 0 <= o and o + 4 <= len(img) and np.isnan(img[o:o + 4]).all()  # inside, written once
                img[o:o + 4] = v
    return img


def logical(N, Np, s1v, rng):
    T = np.full((Np + 1, Np), NEG)
    for r in range(N):
        T[r, r:N] = rng.integers(0, 40, size=N - r)
    for r in range(1, Np + 1):
        T[r, r - 1] = s1v
    return T


@pytest.mark.parametrize("NT,N", [(2, 65), (2, 128), (3, 150), (4, 256), (5, 300)])
def test_layout_round_trip(NT, N):
    Np = 64 * NT
    T = logical(N, Np, 7.0, np.random.default_rng(NT))
    img = write_cell(NT, N, T[:Np], 7.0)
    for r in range(Np):
        for c in range(Np):
            got = (img[4 * 17 + 7] if r == c + 1 else NEG) if r > c else img[wide_pos(NT, r, c)]
            exp = T[r, c] if (r <= c < N or r == c + 1) else NEG
            assert got == exp, (r, c, got, exp)


def test_lane_table_covers_each_micro_tile_twice():
    assert sorted(LANEW) == sorted((bi, bj, h) for bi in range(8) for bj in range(8) for h in range(2))


def _kb_list(kind, bi, bj, h):
    if kind == "F":
        return list(range(4 * h, 4 * h + 4))
    lo, cnt = (bi, 8 - bi) if kind == "DA" else (0, bj + 1)
    half = (cnt + 1) >> 1
    return list(range(lo, lo + half)) if h == 0 else list(range(lo + half, lo + cnt))


def test_item_kinds_cover_the_k_blocks():
    for bi in range(8):
        for bj in range(8):
            assert _kb_list("F", bi, bj, 0) + _kb_list("F", bi, bj, 1) == list(range(8))
            assert _kb_list("DA", bi, bj, 0) + _kb_list("DA", bi, bj, 1) == list(range(bi, 8))
            assert _kb_list("DB", bi, bj, 0) + _kb_list("DB", bi, bj, 1) == list(range(bj + 1))
            assert _kb_list("DA", bi, bj, 0)[0] == bi  # the R3 step rides on the h = 0 lane


def _task(A, a_off, B, b_off, acc):
    Ab = np.array([A[a_off + 8 * i: a_off + 8 * i + 8] for i in range(8)])
    rows = [b_off + 8 * k + (4 if k == 7 else 0) for k in range(8)]
    Bb = np.array([B[o:o + 8] for o in rows])
    np.maximum(acc, (Ab[:, :, None] + Bb[None, :, :]).max(axis=1), out=acc)


@pytest.mark.parametrize("NT,N", [(2, 100), (3, 150), (2, 128)])
def test_tile_product_equals_the_triangular_product(NT, N):
    Np, rng = 64 * NT, np.random.default_rng(10 + NT)
    s1a, s1b = 5.0, 3.0
    TA, TB = logical(N, Np, s1a, rng), logical(N, Np, s1b, rng)
    imgA, imgB = write_cell(NT, N, TA[:Np], s1a), write_cell(NT, N, TB[:Np], s1b)
    C = np.full((Np, Np), NEG)
    for i in range(N):
        for j in range(i, N):
            C[i, j] = max([s1a + TB[i, j]] + [TA[i, k] + TB[k + 1, j] for k in range(i, j + 1)])
    out = np.full((Np, Np), NEG)
    slot = 4 * CBD[8]
    for BI in range(NT):
        for BJ in range(BI, NT):
            accs = [np.full((8, 8), NEG) for _ in range(128)]
            for KB in range(BI, BJ + 1):
                A, B = np.full(slot, np.nan), np.full(slot, np.nan)
                asz, bsz = (SD if KB == BI else SQ), (SD if KB == BJ else SQ)
                A[:asz] = imgA[tile_off(NT, BI, KB):tile_off(NT, BI, KB) + asz]
                B[:bsz] = imgB[tile_off(NT, KB, BJ):tile_off(NT, KB, BJ) + bsz]
                for t in range(128):
                    acc = accs[t]
                    if BI == BJ:
                        g, bi, bj, kb = LANE8[t]
                        if g == 255:
                            continue
                        _task(A, 4 * (CB8[kb] + 17 * bi), B, 4 * (CB8[bj] + 17 * kb + 2), acc)
                        if kb == bi:
                            o = 4 * (CB8[bj] + 17 * bi)
                            acc[0] = np.maximum(acc[0], A[8] + B[o:o + 8])
                    else:
                        bi, bj, h = LANEW[t]
                        kind = "DA" if KB == BI else ("DB" if KB == BJ else "F")
                        bcol = 4 * ((CB8[bj] if kind == "DB" else CBD[bj]) + 2)
                        for kb in _kb_list(kind, bi, bj, h):
                            _task(A, 4 * ((CB8[kb] if kind == "DA" else CBD[kb]) + 17 * bi), B, bcol + 4 * 17 * kb, acc)
                        if kind == "DA" and h == 0:
                            o = bcol + 4 * (17 * bi - 2)
                            acc[0] = np.maximum(acc[0], A[8] + B[o:o + 8])
                    assert not np.isnan(acc).any()  # only written floats of the two images are read
            for t in range(128):
                if BI == BJ:
                    g, bi, bj, _ = LANE8[t]
                    if g == 255:
                        continue
                else:
                    bi, bj, _ = LANEW[t]
                blk = out[64 * BI + 8 * bi:64 * BI + 8 * bi + 8, 64 * BJ + 8 * bj:64 * BJ + 8 * bj + 8]
                np.maximum(blk, accs[t], out=blk)
    iu = np.triu_indices(N)
    assert np.array_equal(out[:N, :N][iu], C[:N, :N][iu])
