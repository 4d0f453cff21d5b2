"""The blocked inner wavefront of the row-major tables (strand-2 lengths above 320;
large_tile_product_kernel and large_tile_local_kernel in bpmax_b200/csrc/bpmax_kernels_large.cuh),
checked on the CPU by restating the kernels' tile order and index arithmetic in numpy with small tiles:
after the start values, for every tile diagonal t the products over finished tiles (R1 slabs K = I..J-1
of F rows against ST1 rows, R2 slabs K = I+1..J of S2M rows shifted one column against FT rows), then
each tile's own wavefront over its diagonals b - a (R1 over b' < b, R2 over a' > a, SW2 from the tile or
a finished neighbour), must give exactly the plain inner wavefront (V3/bpmax_verify.c:614-667) on
every entry, also with padded widths and partial tiles. The GPU kernels use tiles of 64.
"""
import numpy as np
import pytest

NEG = -np.inf


def plain_wavefront(F0, S2, w, N):
    """R1, R2 and SW2 of one outer cell, inner diagonal by inner diagonal."""
    F = F0.copy()
    for dd in range(1, N):
        for i2 in range(N - dd):
            j2 = i2 + dd
            v = F[i2, j2]
            for k in range(i2, j2):
                v = max(v, F[i2, k] + S2[k + 1, j2], S2[i2, k] + F[k + 1, j2])
            if dd >= 4:
                v = max(v, F[i2 + 1, j2 - 1] + w[i2, j2])
            F[i2, j2] = v
    return F


def blocked_wavefront(F0, S2, w, N, Np, LT):
    """The kernels' tile order with tiles of LT (start values already in F0)."""
    NT = Np // LT
    S2M = np.full((Np, Np), NEG)
    ST1 = np.full((Np, Np), NEG)
    for i in range(N):
        S2M[i, i:N] = S2[i, i:N]  # S2M[i][k] = S2(i, k), i <= k < N
    for j in range(N):
        ST1[j, :j] = S2[1:j + 1, j]  # ST1[j][k] = S2(k+1, j), k+1 <= j < N
    F = np.full((Np, Np), NEG)
    for r in range(N):
        F[r, r:N] = F0[r, r:N]
    FT = F.T.copy()
    for t in range(NT):
        for I in range(NT - t):  # large_tile_product_kernel
            J = I + t
            if t == 0 or LT * I >= N or LT * J >= N:
                continue
            acc = np.full((LT, LT), NEG)
            for q in range(2 * t):
                r1 = q < t
                K = I + q if r1 else I + 1 + (q - t)
                A, B = (F, ST1) if r1 else (S2M, FT)
                ka, kb = (LT * K if r1 else LT * K - 1), LT * K
                As = A[LT * I:LT * I + LT, ka:ka + LT]
                Bs = B[LT * J:LT * J + LT, kb:kb + LT]
                acc = np.maximum(acc, (As[:, None, :] + Bs[None, :, :]).max(axis=2))
            for a in range(LT):
                for b in range(LT):
                    i2, j2 = LT * I + a, LT * J + b
                    if i2 <= j2 < N:
                        F[i2, j2] = max(F[i2, j2], acc[a, b])
        for I in range(NT - t):  # large_tile_local_kernel
            J = I + t
            if LT * I >= N or LT * J >= N:
                continue
            T = F[LT * I:LT * I + LT, LT * J:LT * J + LT].copy()
            Sj = ST1[LT * J:LT * J + LT, LT * J:LT * J + LT]
            Si = S2M[LT * I:LT * I + LT, LT * I:LT * I + LT]
            for l in range(1 if t == 0 else -(LT - 1), LT):
                new = []
                for slot in range(LT):
                    a = slot if l >= 0 else slot - l
                    b = a + l
                    i2, j2 = LT * I + a, LT * J + b
                    if not (a < LT and 0 <= b < LT and i2 <= j2 < N):
                        continue
                    red = NEG
                    for bp in range(b):
                        red = max(red, T[a, bp] + Sj[b, bp])
                    for ap in range(a + 1, LT):
                        red = max(red, Si[a, ap - 1] + T[ap, b])
                    v = max(T[a, b], red)
                    if j2 - i2 >= 4:
                        sw = T[a + 1, b - 1] if (a + 1 < LT and b >= 1) else F[i2 + 1, j2 - 1]
                        v = max(v, sw + w[i2, j2])
                    new.append((a, b, v))
                for a, b, v in new:  # one CTA barrier per tile diagonal
                    T[a, b] = v
            F[LT * I:LT * I + LT, LT * J:LT * J + LT] = T
            FT[LT * J:LT * J + LT, LT * I:LT * I + LT] = T.T
    return F


@pytest.mark.parametrize("N,Np,LT,seed", [(13, 16, 4, 1), (16, 16, 4, 2), (10, 12, 4, 3), (23, 24, 8, 4),
                                          (9, 16, 8, 5), (17, 24, 4, 6), (30, 32, 8, 7)])
def test_blocked_wavefront_equals_plain(N, Np, LT, seed):
    rng = np.random.default_rng(seed)
    S2 = np.triu(rng.integers(0, 6, (Np + 1, Np + 1)).astype(np.float32))
    F0 = np.triu(rng.integers(0, 20, (Np, Np)).astype(np.float32))
    w = rng.integers(0, 4, (Np, Np)).astype(np.float32)
    Fp = plain_wavefront(F0, S2, w, N)
    Fb = blocked_wavefront(F0, S2, w, N, Np, LT)
    iu = np.triu_indices(N)
    assert np.array_equal(Fp[:N, :N][iu], Fb[:N, :N][iu])
