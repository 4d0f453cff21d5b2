"""Structure of the generated product-kernel tables (bpmax_b200/csrc/r0_tables.inc): every task of
every item slot has exactly one lane, and each warp's program only skips candidates its tasks meet
below a diagonal (the skipped ones are -inf by the cell-image layout, so no maximum changes)."""
import os
import re

import numpy as np
import pytest

INC = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "bpmax_b200", "csrc", "r0_tables.inc")


def _arr(txt, name):
    m = re.search(name + r"\[[^=]*=\s*\{(.*?)\};", txt, re.S)
    return [int(x) for x in re.findall(r"\d+", m.group(1))]


@pytest.fixture(scope="module")
def tables():
    txt = open(INC).read()
    return {"threads": _arr(txt, "R0_TAB_THREADS"), "items": _arr(txt, "R0_TAB_ITEMS"),
            "colbase": np.array(_arr(txt, "R0_TAB_COLBASE")).reshape(9, 9),
            "lane": np.array(_arr(txt, "c_r0_lane")).reshape(8, 256, 4),
            "role": np.array(_arr(txt, "R0_TAB_ROLE")).reshape(9, 8)}


@pytest.mark.parametrize("nb", range(1, 9))
def test_every_task_once_per_item(tables, nb):
    threads, G = tables["threads"][nb], tables["items"][nb]
    want = sorted((g, bi, bj, kb) for g in range(G) for bi in range(nb) for bj in range(bi, nb)
                  for kb in range(bi, bj + 1))
    got = sorted(tuple(int(x) for x in t) for t in tables["lane"][nb - 1][:threads] if t[0] != 255)
    assert got == want
    assert all(t[0] == 255 for t in tables["lane"][nb - 1][threads:])


@pytest.mark.parametrize("nb", range(1, 9))
def test_warp_programs_fit_their_tasks(tables, nb):
    """Program 1 (rows i <= 2p+2 of k pair p) needs kb == bi, program 2 (column pairs jp >= p)
    needs kb == bj, program 3 both; program 0 takes any task."""
    threads = tables["threads"][nb]
    for w in range(threads // 32):
        role = tables["role"][nb][w]
        for t in tables["lane"][nb - 1][32 * w:32 * w + 32]:
            if t[0] == 255:
                continue
            bi, bj, kb = (int(x) for x in t[1:])
            if role & 1:
                assert kb == bi, (nb, w, t)
            if role & 2:
                assert kb == bj, (nb, w, t)


def test_skipped_candidates_lie_below_a_diagonal():
    """For every (row i, column pair jp, k pair p) a program skips, the A operand (program 1) or the
    shifted B operand (program 2) is below its diagonal in every column of the pair."""
    for p in range(4):
        for i in range(8):
            if not i <= 2 * p + 2:  # program 1 skips: A[i][k] with k in {2p, 2p+1} has k < i - 1
                assert all(k < i - 1 for k in (2 * p, 2 * p + 1))
        for jp in range(4):
            if not jp >= p:  # program 2 skips: Bs[k][j] = B[k+1][j] with k > j for both j of the pair
                assert all(k > j for k in (2 * p, 2 * p + 1) for j in (2 * jp, 2 * jp + 1))


def test_image_sizes_fix_the_allocation_free_capacity(tables):
    # cell image sizes in 16-byte chunks; the allocation-free entry point's documented limits
    # (include/bpmax_gpu.h) follow from these
    assert [int(tables["colbase"][nb][nb]) for nb in range(1, 9)] == [19, 59, 112, 179, 269, 379, 498, 630]
