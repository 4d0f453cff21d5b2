#!/usr/bin/env python
"""Generates wide_tables.inc: the dense tile-image layout and the lane -> micro-tile table of the
tile product kernel (bpmax_wide.cuh) for off-diagonal output tiles.

Inner tables wider than 64 (64 < Np <= 320, Np = 64*NT) are stored per outer cell as the upper
triangle of NT x NT tiles of 64 x 64. A diagonal tile is a width-64 cell image (the layout of
r0_tables.inc, NB = 8: block columns of the blocks (0..bj, bj), each closed by its S1 piece). An
off-diagonal ("dense") tile holds all 64 of its 8x8 blocks: block columns bj = 0..7 in turn, column
bj holding the blocks (0..7, bj) at a pitch of 17 chunks, then a 2-chunk halo piece (row 0 of block
(0, bj) of the tile below, i.e. the row after the tile's last row, so the row-shifted operand of a
tile is one image as in a cell image), then pad[bj] spare chunks.

A job of the product kernel takes one output tile (BI, BJ), BI < BJ, of one outer cell and loops
over k1 and the k tiles KB in [BI, BJ]; an item is the pair A = tile (BI, KB) of F(i1, k1), B =
tile (KB, BJ) of F(k1+1, j1), of three kinds: DA (KB = BI: A is a diagonal tile), F (both dense) and
DB (KB = BJ: B is a diagonal tile). Each of the 128 lanes owns one 8x8 micro-tile (bi, bj) of the
output tile for the whole job (two lanes per micro-tile, h = 0, 1) and takes, per item, a part of
the micro-tile's 8-wide k blocks kb:
  F:  kb = 4h .. 4h+3
  DA: the blocks kb = bi .. 7 (A is upper block-triangular), the first ceil(n/2) for h = 0
  DB: the blocks kb = 0 .. bj (B is upper block-triangular), the first ceil(n/2) for h = 0
Warp w holds the micro-tiles bi in [4(w>>1), +4), bj in [4(w&1), +4), both halves, so that the warp's
longest lane list stays short in DA and DB items. The search picks the dense column pads and the
lane order inside each warp that minimise the shared-memory wavefronts of every 128-bit load of the
product loop (a quarter-warp's load takes one wavefront when its distinct 16-byte addresses fall
in distinct bank groups, address mod 8 in chunks), weighting the kinds by their share of a 256-wide
table's items (DA 6 : F 4 : DB 6). It runs for a few minutes.

    python bpmax_b200/csrc/gen_wide_tables.py   # rewrites bpmax_b200/csrc/wide_tables.inc
"""
from __future__ import annotations

import os
import random
import re

HERE = os.path.dirname(os.path.abspath(__file__))
WEIGHT = {"DA": 6, "F": 4, "DB": 6}
ITERS, SEED = 12000, 5


def diag_colbase():
    """Column bases of the width-64 cell image, read from r0_tables.inc (NB = 8)."""
    with open(os.path.join(HERE, "r0_tables.inc")) as f:
        text = f.read()
    m = re.search(r"constexpr int R0_TAB_COLBASE\[9\]\[9\] = \{(.*)\};", text)
    rows = re.findall(r"\{([0-9,]+)\}", m.group(1))
    return [int(x) for x in rows[8].split(",")]


CB8 = diag_colbase()


def dense_colbase(pads):
    cb, o = [], 0
    for c in range(8):
        cb.append(o)
        o += 8 * 17 + 2 + pads[c]
    return cb + [o]


def kb_list(kind, bi, bj, h):
    if kind == "F":
        return list(range(4 * h, 4 * h + 4))
    ks = list(range(bi, 8)) if kind == "DA" else list(range(0, bj + 1))
    half = (len(ks) + 1) // 2
    return ks[:half] if h == 0 else ks[half:]


def a_addr(kind, cbd, bi, kb, i, q):
    base = CB8[kb] if kind == "DA" else cbd[kb]
    return base + 17 * bi + 2 * i + q


def b_addr(kind, cbd, kb, bj, k, hh):
    base = CB8[bj] if kind == "DB" else cbd[bj]
    return 4096 + base + 17 * kb + 2 + 2 * k + (1 if k == 7 else 0) + hh


def r3_addr(cbd, bi, bj, hh):  # DA items: row 0 of block (bi, bj) of the dense B tile
    return 4096 + cbd[bj] + 17 * bi + hh


def wavefronts(addrs):
    groups = {}
    for x in set(addrs):
        groups.setdefault(x % 8, set()).add(x)
    return max(len(v) for v in groups.values()) if groups else 0


def initial_lanes():
    lanes = []
    for w in range(4):
        rb, cb = w >> 1, w & 1
        for h in range(2):
            for bi in range(4 * rb, 4 * rb + 4):
                for bj in range(4 * cb, 4 * cb + 4):
                    lanes.append((bi, bj, h))
    return lanes


def quarter_cost(sel, cbd):
    c = 0
    for kind, wgt in WEIGHT.items():
        lists = [kb_list(kind, *x) for x in sel]
        for s in range(max(len(L) for L in lists)):
            act = [(x, L[s]) for x, L in zip(sel, lists) if len(L) > s]
            k = 0
            for i in range(8):
                for q in range(2):
                    k += wavefronts([a_addr(kind, cbd, x[0], kb, i, q) for x, kb in act])
            for kk in range(8):
                for hh in range(2):
                    k += wavefronts([b_addr(kind, cbd, kb, x[1], kk, hh) for x, kb in act])
            if kind == "DA" and s == 0:
                r3 = [x for x, kb in act if kb == x[0]]
                for hh in range(2):
                    k += wavefronts([r3_addr(cbd, x[0], x[1], hh) for x in r3])
            c += wgt * k
    return c


def cost(lanes, pads):
    cbd = dense_colbase(pads)
    return sum(quarter_cost(lanes[q * 8:q * 8 + 8], cbd) for q in range(16))


def warp_slots(lanes):
    """Per kind: sum over warps of the warp's longest lane list (task steps the warps issue)."""
    return {kind: sum(max(len(kb_list(kind, *x)) for x in lanes[32 * w:32 * w + 32]) for w in range(4))
            for kind in WEIGHT}


def search(iters=ITERS, seed=SEED):
    rnd = random.Random(seed)
    lanes, pads = initial_lanes(), [0] * 8
    cbd = dense_colbase(pads)
    qc = [quarter_cost(lanes[q * 8:q * 8 + 8], cbd) for q in range(16)]
    for _ in range(iters):
        if rnd.random() < 0.15:
            c = rnd.randrange(8)
            old = pads[c]
            pads[c] = rnd.randrange(8)
            cbd2 = dense_colbase(pads)
            qc2 = [quarter_cost(lanes[q * 8:q * 8 + 8], cbd2) for q in range(16)]
            if sum(qc2) <= sum(qc):
                qc, cbd = qc2, cbd2
            else:
                pads[c] = old
        else:
            w = rnd.randrange(4)
            x, y = 32 * w + rnd.randrange(32), 32 * w + rnd.randrange(32)
            if x // 8 == y // 8:
                continue
            lanes[x], lanes[y] = lanes[y], lanes[x]
            a, b = quarter_cost(lanes[x // 8 * 8:x // 8 * 8 + 8], cbd), quarter_cost(lanes[y // 8 * 8:y // 8 * 8 + 8], cbd)
            if a + b <= qc[x // 8] + qc[y // 8]:
                qc[x // 8], qc[y // 8] = a, b
            else:
                lanes[x], lanes[y] = lanes[y], lanes[x]
    return sum(qc), lanes, pads


def main():
    base = cost(initial_lanes(), [0] * 8)
    c, lanes, pads = search()
    cbd = dense_colbase(pads)
    slots = warp_slots(lanes)
    out = ["// wide_tables.inc -- generated by gen_wide_tables.py (seeded search); do not edit by hand.\n",
           "// Dense (off-diagonal) 64x64 tile image: block column bases in 16-byte chunks (index 8: the\n",
           "// image size), and the lane -> (bi, bj, h) table of off-diagonal output-tile jobs.\n",
           f"//   search cost {c} weighted wavefronts (unsearched order and no pads: {base}); warp task steps\n",
           f"//   per item kind {slots}\n",
           "constexpr int WIDE_DENSE_COLBASE[9] = {" + ",".join(map(str, cbd)) + "};\n",
           "__constant__ int c_wide_dense_colbase[9] = {" + ",".join(map(str, cbd)) + "};\n",
           "__constant__ unsigned char c_tile_lane[128][3] = {" +
           ",".join("{%d,%d,%d}" % x for x in lanes) + "};\n"]
    path = os.path.join(HERE, "wide_tables.inc")
    with open(path, "w") as f:
        f.write("".join(out))
    print(path, c, base, slots)


if __name__ == "__main__":
    main()
